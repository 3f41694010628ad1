"""The C++ host mirror (include/ursa_core.hpp) compiles against the C ABI
header (CPU), and its golden checks pass on the GPU."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "test_ursa_core.cpp")


def _build(tmp_path):
    from ursa_b200 import build

    build.build()
    exe = str(tmp_path / "test_ursa_core")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", os.path.dirname(build.GPU_SO), "-lursa_gpu", f"-Wl,-rpath,{os.path.dirname(build.GPU_SO)}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_mirror_compiles_and_links(tmp_path):
    exe = _build(tmp_path)
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_mirror_goldens_on_gpu(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr

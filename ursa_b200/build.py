"""Build recipe for the native libraries, written in-tree so they travel with
the repository snapshot:

  ursa_b200/libursa_gpu.so  -- the CUDA kernels + C ABI (nvcc, sm_100a)
  ursa_b200/libursa_gen.so  -- seeded synthetic graph generators (gcc)

Run `python -m ursa_b200.build` (or call build()).  Objects go to
ursa_b200/_build/, which is not committed.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
GPU_SO = os.path.join(PKG, "libursa_gpu.so")
GEN_SO = os.path.join(PKG, "libursa_gen.so")

NVCC_FLAGS = [
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-O3",
    "-std=c++17",
    "-fmad=false",  # no contraction: a*b+c rounds like the reference's Rust
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-Wall",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources() -> list[str]:
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers() -> list[str]:
    inc = os.path.join(os.path.dirname(PKG), "include")
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith((".h", ".hpp"))]
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_gpu(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    srcs = _sources()
    hdrs = _headers()
    objs = []
    jobs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs) or ptxas_info:
            cmd = [nvcc, *NVCC_FLAGS, "-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        return r.stdout + r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(run, jobs):
            if verbose and out.strip():
                print(out)
    # Link when the library is missing or any source/header is newer than it.
    # (Object mtimes are not used: a fresh checkout gives every file the same
    # timestamp, and a stale .so from an older tree must not survive.)
    if jobs or _stale(GPU_SO, srcs + hdrs):
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", GPU_SO, "-lcuda"]
        run(cmd)
    return GPU_SO


def build_gen() -> str:
    src = os.path.join(CSRC, "gen.c")
    if _stale(GEN_SO, [src]):
        cc = shutil.which("gcc") or "cc"
        cmd = [cc, "-O3", "-march=x86-64-v2", "-fPIC", "-shared", "-pthread", src, "-o", GEN_SO, "-lm"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("gcc failed:\n" + r.stdout + r.stderr)
    return GEN_SO


def build(verbose: bool = False) -> None:
    build_gen()
    build_gpu(verbose=verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    if "--ptxas" in sys.argv:
        build_gpu(verbose=True, ptxas_info=True)
    print(GPU_SO)
    print(GEN_SO)

"""CPU-side checks of the boundary: the C-ABI library builds, loads, and
exports every symbol include/ursa_gpu.h declares; the ctypes signature table
covers the header exactly.  No compute call is made (no GPU here)."""

import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ursa_gpu.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ursa_gpu_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from ursa_b200 import build

    build.build()
    return ctypes.CDLL(build.GPU_SO)


def test_header_declares_the_kernel_set():
    syms = declared_symbols()
    for name in [
        "ursa_gpu_topo_build",
        "ursa_gpu_degree",
        "ursa_gpu_pagerank",
        "ursa_gpu_pagerank_weighted",
        "ursa_gpu_bfs_distances",
        "ursa_gpu_shortest_path",
        "ursa_gpu_dijkstra_distances",
        "ursa_gpu_shortest_path_weighted_with_cost",
        "ursa_gpu_k_hop",
        "ursa_gpu_connected_components_weak",
        "ursa_gpu_triangle_count",
        "ursa_gpu_clustering_coefficient",
        "ursa_gpu_betweenness",
        "ursa_gpu_betweenness_weighted",
    ]:
        assert name in syms, name


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_dynamic_symbol_table_matches(lib):
    from ursa_b200 import build

    out = subprocess.run(["nm", "-D", "--defined-only", build.GPU_SO], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\b(ursa_gpu_[a-z0-9_]+)\b", out))
    assert set(declared_symbols()) <= exported


def test_ctypes_table_covers_header():
    from ursa_b200 import _lib

    assert set(_lib.SIGNATURES) == set(declared_symbols())


def test_version_and_error_string_without_gpu(lib):
    from ursa_b200 import _lib

    L = _lib.load()
    assert L.ursa_gpu_version() >= 100
    assert isinstance(L.ursa_gpu_last_error(), bytes)


def test_import_fails_loudly_without_library(tmp_path, monkeypatch):
    from ursa_b200 import _lib

    monkeypatch.setattr(_lib, "GPU_SO", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError, match="no CPU fallback"):
        _lib.load()

"""Seeded synthetic graph inputs (R-MAT, Poisson, f32 weights); see csrc/gen.c
for the exact definitions.  Host code, multi-threaded, thread-count
independent."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
GEN_SO = os.path.join(PKG, "libursa_gen.so")

RMAT_ABC = (0.57, 0.19, 0.19)
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(GEN_SO):
            from .build import build_gen

            build_gen()
        L = C.CDLL(GEN_SO)
        P, u64, i32, f64 = C.c_void_p, C.c_uint64, C.c_int, C.c_double
        L.ug_rmat.restype = u64
        L.ug_rmat.argtypes = [i32, u64, f64, f64, f64, u64, P, P, i32]
        L.ug_rmat_raw.restype = None
        L.ug_rmat_raw.argtypes = [i32, u64, f64, f64, f64, u64, P, P, i32]
        L.ug_dedup.restype = u64
        L.ug_dedup.argtypes = [P, P, u64, P, P, i32]
        L.ug_poisson_degrees.restype = u64
        L.ug_poisson_degrees.argtypes = [u64, f64, u64, P, i32]
        L.ug_poisson_fill.restype = None
        L.ug_poisson_fill.argtypes = [u64, u64, P, P, P, i32]
        L.ug_weights_f32.restype = None
        L.ug_weights_f32.argtypes = [u64, C.c_float, C.c_float, u64, P, i32]
        L.ug_draw.restype = u64
        L.ug_draw.argtypes = [u64, u64, u64]
        _lib = L
    return _lib


def _threads(threads: int | None) -> int:
    return threads or min(os.cpu_count() or 1, 64)


def rmat(scale: int, edge_factor: int = 16, seed: int = 1, abc=RMAT_ABC, threads: int | None = None):
    """R-MAT edges with self-loops and duplicates removed (first occurrence
    kept, generation order preserved).  Returns (n, src, dst)."""
    cap = edge_factor << scale
    src = np.empty(cap, np.uint32)
    dst = np.empty(cap, np.uint32)
    m = _load().ug_rmat(scale, edge_factor, abc[0], abc[1], abc[2], seed, src.ctypes.data, dst.ctypes.data,
                        _threads(threads))
    return 1 << scale, src[:m].copy(), dst[:m].copy()


def rmat_raw(scale: int, edge_factor: int = 16, seed: int = 1, abc=RMAT_ABC, threads: int | None = None):
    """R-MAT edges before cleaning (self-loops and duplicates kept)."""
    cap = edge_factor << scale
    src = np.empty(cap, np.uint32)
    dst = np.empty(cap, np.uint32)
    _load().ug_rmat_raw(scale, edge_factor, abc[0], abc[1], abc[2], seed, src.ctypes.data, dst.ctypes.data,
                        _threads(threads))
    return 1 << scale, src, dst


def poisson(n: int, mean: float = 16.0, seed: int = 3, threads: int | None = None):
    """Node-major Poisson(mean) out-degree graph with uniform targets;
    multiplicity and self-loops kept.  Returns (n, src, dst)."""
    L = _load()
    deg = np.empty(n, np.uint32)
    m = L.ug_poisson_degrees(n, mean, seed, deg.ctypes.data, _threads(threads))
    src = np.empty(m, np.uint32)
    dst = np.empty(m, np.uint32)
    L.ug_poisson_fill(n, seed, deg.ctypes.data, src.ctypes.data, dst.ctypes.data, _threads(threads))
    return n, src, dst


def weights_f32(m: int, lo: float = 1.0, hi: float = 10.0, seed: int = 3, threads: int | None = None) -> np.ndarray:
    """f32 weights uniform in [lo, hi) per edge row."""
    out = np.empty(m, np.float32)
    _load().ug_weights_f32(m, lo, hi, seed, out.ctypes.data, _threads(threads))
    return out


def batch_sizes(count: int, median: float = 2000.0, sigma: float = 1.0, lo: int = 100, hi: int = 50_000,
                ef_lo: int = 8, ef_hi: int = 32, seed: int = 100):
    """Node counts log-normal(median, sigma) clipped to [lo, hi] and integer
    edge factors uniform in [ef_lo, ef_hi], from numpy's seeded PCG64."""
    rng = np.random.default_rng(seed)
    n = np.clip(np.rint(median * np.exp(sigma * rng.standard_normal(count))), lo, hi).astype(np.uint64)
    ef = rng.integers(ef_lo, ef_hi + 1, count).astype(np.uint64)
    return n, ef


def rmat_batch(count: int, median: float = 2000.0, sigma: float = 1.0, lo: int = 100, hi: int = 50_000,
               ef_lo: int = 8, ef_hi: int = 32, seed0: int = 100, abc=RMAT_ABC, threads: int | None = None):
    """A batch of small R-MAT graphs: graph i has n_i nodes (batch_sizes),
    R-MAT on scale ceil(log2 n_i) with ef_i * n_i draws and seed seed0 + i,
    endpoints >= n_i rejected, self-loops and duplicates dropped.  Returns
    (n[count], edge_counts[count], src, dst) with local ids, graph after graph."""
    L = _load()
    n, ef = batch_sizes(count, median, sigma, lo, hi, ef_lo, ef_hi, seed0)
    cap = (n * ef).astype(np.uint64)
    off = np.zeros(count + 1, np.uint64)
    np.cumsum(cap, out=off[1:])
    src = np.empty(int(off[-1]), np.uint32)
    dst = np.empty(int(off[-1]), np.uint32)
    kept = np.empty(count, np.uint64)
    P = C.c_void_p
    L.ug_rmat_batch.restype = None
    L.ug_rmat_batch.argtypes = [C.c_uint64, P, P, C.c_uint64, C.c_double, C.c_double, C.c_double, P, P, P, P,
                                C.c_int]
    L.ug_rmat_batch(count, n.ctypes.data, ef.ctypes.data, seed0, abc[0], abc[1], abc[2], off.ctypes.data,
                    src.ctypes.data, dst.ctypes.data, kept.ctypes.data, _threads(threads))
    keep = np.zeros(src.size, bool)
    for g in range(count):
        keep[int(off[g]):int(off[g] + kept[g])] = True
    return n, kept, src[keep], dst[keep]


def draw(seed: int, index: int, lane: int = 0) -> int:
    """The generators' counter-based 64-bit draw."""
    return int(_load().ug_draw(seed, index, lane))


def dedup(src, dst, threads: int | None = None):
    """Drop self-loops and duplicate pairs, keeping first occurrences in order."""
    src = np.ascontiguousarray(src, np.uint32)
    dst = np.ascontiguousarray(dst, np.uint32)
    os_ = np.empty_like(src)
    od = np.empty_like(dst)
    k = _load().ug_dedup(src.ctypes.data, dst.ctypes.data, src.size, os_.ctypes.data, od.ctypes.data,
                         _threads(threads))
    return os_[:k].copy(), od[:k].copy()

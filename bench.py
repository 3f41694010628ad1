"""Benchmark: R-MAT-22 PageRank (GTEPS and achieved HBM GB/s) on one B200.

Workload (the reference's full plain-kernel configuration): R-MAT scale 22
(4,194,304 nodes, edge factor 16, a/b/c/d = .57/.19/.19/.05, seed 2, self-loops
and duplicate edges removed -> 65,243,929 directed edges), pull PageRank with
damping 0.85, tol 1e-6 (L1), max_iter 100.  A step is one pagerank() call to
convergence.  Inputs are synthetic (seeded generator; the reference publishes
no dataset at this scale) and larger than L2 (the in-CSR alone is 261 MB), so
no L2 flush is needed between steps.

  value  GTEPS = edges x iterations / device time, topology resident in HBM,
         through ursa_gpu_pagerank_device (events on the launch stream).
  e2e    the same metric through the C ABI a caller uses, from pinned host
         buffers: Topology::build (H2D of src/dst, CSR build, transpose) +
         pagerank (D2H of the n f64 ranks) per step.
  --impl reference
         the reference algorithm on the host cores: the CPU restatement of
         ursa-core (the Rust crate cannot be built here), same workload, all
         host threads, one full build + transpose + pagerank per step.

Multi-GPU (--gpus N under torchrun): replicas only (each rank runs the whole
workload on its own GPU, no collective on the data path); value sums ranks'
edges x iterations over the max time across ranks.

--workload batch: 10,000 uneven R-MAT graphs (node counts log-normal, median
2,000, clipped to [100, 50,000]; per-graph edge factor uniform in [8, 32];
seed 100 + i; see ursa_b200.gen.rmat_batch).  A step is pagerank (d 0.85,
tol 1e-6, max_iter 100), weak components and triangle counts for every graph
in one launch of the batch's captured CUDA graph (bucket and tile shapes
autotuned once before timing).  value = graphs/s of that launch (device
time); e2e = the public API from pinned host buffers per step (batch build
with the H2D of every edge row, the launch, the D2H of every result); beside
them the per-graph plain loop -- one topology and one pagerank /
connected_components_weak / triangle_count call per graph -- timed over the
whole batch with topologies resident, and with builds.

--workload serve: the serving loop on a resident R-MAT scale-24 graph
(16,777,216 nodes, edge factor 16, seed 4; out-CSR and transpose resident)
plus uploaded small graphs (sized as the batch workload) arriving as a
Poisson stream of 200/s, each kept for 2 s.  Queries arrive as a seeded
Poisson stream at each swept rate: 50% shortest_path between uniform random
nodes, 30% hop(k=2) from a uniform random seed, 20% pagerank (d 0.85, tol
1e-6, max_iter 100) on a live upload.  Per rate: completed queries/s and
p50/p99 latency (submit to completion, queueing included).  Beside it the
plain one-query-per-launch path (shortest_path / k_hop / pagerank C-ABI calls
from 4 host threads, closed loop) over the same queries.

--workload idmap: Int64 node-id interning of the R-MAT-22 edges, then the
topology from the dense device columns.

--workload closeness: all-source closeness on R-MAT-16 (65,536 nodes, edge
factor 16, seed 2); GTEPS = n sources x m edges / time.

--workload result: query_batch (id, degree, pagerank) on R-MAT-22 under
Int64 user ids to a pyarrow RecordBatch, beside the per-column plain path.

--workload suite: the per-kernel table (CSR build, transpose, degree,
pagerank, BFS, weak components, triangles, clustering, weighted paths,
betweenness) on C1 = R-MAT-16, C2 = R-MAT-22 and C3 = Poisson(16) n = 2^20
weighted, each beside the oracle on the host cores.
"""

from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import queue
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SCALE, EDGE_FACTOR, SEED = 22, 16, 2
DAMPING, TOL, MAX_ITER = 0.85, 1e-6, 100
WORKLOAD = "rmat22_pagerank"

# dram__bytes_read.sum + dram__bytes_write.sum of one PageRank kernel launch on
# this workload (prologue + NCU_TRAFFIC["iterations"] iterations), from an ncu
# --set full capture of pr_seg_k on this workload's own launch (converged in
# 18 iterations): 3.588198 GB read + 0.466520 GB written.
NCU_TRAFFIC = {"bytes_per_launch": 3_588_198_400 + 466_520_320, "iterations": 18}


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def combine_replicas(dist, device, t_dev_ms, t_e2e_s, edges, e2e_edges):
    """Replicas (one independent copy of the workload per rank): the job's
    times are the slowest rank's, its work the sum of every rank's.  dist is
    torch.distributed (any backend) or None for one process; returns
    (t_dev_ms, t_e2e_s, edges, e2e_edges) as floats."""
    if dist is None:
        return float(t_dev_ms), float(t_e2e_s), float(edges), float(e2e_edges)
    import torch

    tt = torch.tensor([float(t_dev_ms), float(t_e2e_s)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    ei = torch.tensor([float(edges), float(e2e_edges)], dtype=torch.float64, device=device)
    dist.all_reduce(ei, op=dist.ReduceOp.SUM)
    return float(tt[0]), float(tt[1]), float(ei[0]), float(ei[1])


def algorithmic_bytes(n: int, m: int, iters: int) -> int:
    """Compulsory HBM bytes of one pagerank launch.

    Per iteration: in-CSR sources 4m, in-CSR offsets 4(n+1), the f32 share of
    each node gathered at least once 4n, old rank 8n, out-degree 4n, new rank
    8n, new share 4n  ->  4m + 32n + 4.  Prologue: out-degree 4n, rank 8n,
    share 4n  ->  16n.
    """
    return iters * (4 * m + 32 * n + 4) + 16 * n


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=5)
        rows = [r for r in self.rows if self.uuid is None or self.uuid in r[0]]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def make_workload():
    from ursa_b200 import gen

    n, src, dst = gen.rmat(SCALE, EDGE_FACTOR, SEED)
    return n, src, dst


def rmat22_config(n, m, tol, max_iter, iters, world):
    """The workload's config dict, identical in both arms."""
    return {"workload": WORKLOAD, "n_nodes": n, "n_edges": m, "damping": DAMPING, "tol": tol,
            "max_iter": max_iter, "iterations": iters, "l2": "inputs larger than L2 (in-CSR 261 MB)",
            "parallelism": "replicas" if world > 1 else "single"}


REF_E2E_STEPS = 3


def run_reference(args, rank, world):
    """The reference algorithm on the host (CPU restatement of ursa-core).

    value: pagerank to tol with the CSR and its transpose already built (the
    warm kernel, as the device arm's value has its topology resident), one
    call per step.  e2e: Topology::build + transpose + pagerank per step, on
    REF_E2E_STEPS samples (the device arm's e2e also builds every step)."""
    if rank != 0:
        return
    from oracle import oracle as O

    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    n, src, dst = make_workload()
    m = int(src.size)
    topo = O.Topology(n, src, dst)
    topo.csr("in")  # the transpose, built once

    def warm_step():
        t0 = time.perf_counter()
        _, it = O.pagerank(topo, DAMPING, args.max_iter, args.tol, return_iters=True)
        return time.perf_counter() - t0, it

    def e2e_step():
        t0 = time.perf_counter()
        t = O.Topology(n, src, dst)
        t.csr("in")
        _, it = O.pagerank(t, DAMPING, args.max_iter, args.tol, return_iters=True)
        dt = time.perf_counter() - t0
        del t
        return dt, it

    for _ in range(args.warmup):
        warm_step()
    times, iters = [], []
    for _ in range(args.steps):
        dt, it = warm_step()
        times.append(dt)
        iters.append(it)
    del topo
    e2e = [e2e_step() for _ in range(REF_E2E_STEPS)]
    total = sum(times)
    value = m * sum(iters) / total / 1e9
    e2e_value = m * sum(it for _, it in e2e) / sum(dt for dt, _ in e2e) / 1e9
    line = {
        "impl": "reference",
        "metric": "pagerank_gteps",
        "value": value,
        "unit": "GTEPS",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": rmat22_config(n, m, args.tol, args.max_iter, iters[-1] if iters else 0, world),
        "cpu_baseline": {"value": value, "unit": "GTEPS", "cores": threads, "kind": "port",
                         "sample": "pagerank to tol per step with the CSR and transpose prebuilt (C restatement "
                                   "of ursa-core; the Rust crate cannot be built here)"},
        "e2e": {"value": e2e_value, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "ms_per_step": 1e3 * sum(dt for dt, _ in e2e) / len(e2e),
                "sample": f"{REF_E2E_STEPS} steps of Topology::build + transpose + pagerank to tol"},
    }
    print(json.dumps(line), flush=True)


def oracle_check(n, src, dst, got, gpu_iters, max_iter, tol, want_baseline):
    """PageRank of the oracle on the same graph and parameters: the device
    ranks' error against it (L1 and max relative error vs the f64 oracle,
    both iteration counts) and, when asked, the oracle's warm speed as the
    CPU baseline (that same call, timed, CSR and transpose prebuilt)."""
    from oracle import oracle as O

    O.build()
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    topo = O.Topology(n, src, dst)
    topo.csr("in")  # prebuild the transpose (warm kernel)
    t0 = time.perf_counter()
    ref, it = O.pagerank(topo, DAMPING, max_iter, tol, return_iters=True)
    dt = time.perf_counter() - t0
    deltas = O.pagerank_deltas()
    diff = np.abs(got - ref)
    error = {"l1": float(diff.sum()),
             "max_rel": float((diff / np.maximum(np.abs(ref), 1e-300)).max()) if ref.size else 0.0,
             "iters": int(gpu_iters), "iters_oracle": int(it),
             "oracle_last_delta": float(deltas[-1]) if deltas.size else None,
             "reference": "oracle (C restatement of ursa-core pagerank.rs, f64) on the same graph"}
    baseline = None
    if want_baseline:
        baseline = {"value": src.size * it / dt / 1e9, "unit": "GTEPS", "cores": threads, "kind": "port",
                    "sample": f"one warm pagerank to tol ({it} iterations) on the same R-MAT-22 graph, "
                              "CSR+transpose prebuilt"}
    return error, baseline


def e2e_phases(L, n, m, h_src, h_dst, h_out, params, reps=3):
    """Where an end-to-end step's time goes (medians over reps, each phase
    synchronised on its own): the H2D of the two endpoint columns from pinned
    memory, the out-CSR + transpose build from device columns, the first
    pagerank call on the new topology (its execution plan, the kernel, the
    rank unpermute and the D2H of the ranks), the kernel alone (device
    events), and the D2H of the n f64 ranks alone.  The e2e step itself
    overlaps the destinations' H2D with the first radix passes."""
    import torch

    from ursa_b200 import PageRankStats, _lib

    rec = {k: [] for k in ("h2d", "build", "pagerank_call", "kernel", "d2h")}
    d_src = torch.empty(m, dtype=torch.int32, device="cuda")
    d_dst = torch.empty(m, dtype=torch.int32, device="cuda")
    d_out = torch.empty(n, dtype=torch.float64, device="cuda")
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d_src.copy_(h_src.view(torch.int32), non_blocking=True)
        d_dst.copy_(h_dst.view(torch.int32), non_blocking=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        h = C.c_void_p()
        _lib.check(L.ursa_gpu_topo_build_device(n, d_src.data_ptr(), d_dst.data_ptr(), m, None, C.byref(h)))
        t2 = time.perf_counter()
        st = PageRankStats()
        try:
            _lib.check(L.ursa_gpu_pagerank(h, C.byref(params), h_out.data_ptr(), C.byref(st)))
        finally:
            t3 = time.perf_counter()
            L.ursa_gpu_topo_free(h)
        torch.cuda.synchronize()
        t4 = time.perf_counter()
        h_out.copy_(d_out, non_blocking=True)
        torch.cuda.synchronize()
        t5 = time.perf_counter()
        for k, v in (("h2d", t1 - t0), ("build", t2 - t1), ("pagerank_call", t3 - t2),
                     ("kernel", st.device_ms * 1e-3), ("d2h", t5 - t4)):
            rec[k].append(1e3 * v)
    out = {k: statistics.median(v) for k, v in rec.items()}
    out["h2d_gbs"] = 8 * m / (out["h2d"] * 1e-3) / 1e9
    out["plan_and_unpermute"] = out["pagerank_call"] - out["kernel"] - out["d2h"]
    return out


BATCH_COUNT = 10_000
BATCH_WORKLOAD = "rmat_batch10k_pr_cc_tc"


def batch_pagerank_bytes(n, m, iters) -> int:
    """Compulsory bytes of the batch's pagerank phase: per graph and
    iteration 4m (in-CSR sources) + 4(n+1) (offsets) + 4n (out-degree) + 8n
    (old rank) + 8n (new rank) + 4n (new share) = 4m + 28n + 4."""
    return int(np.sum(iters.astype(np.int64) * (4 * m + 28 * n + 4)))


def batch_graphs(count=BATCH_COUNT):
    from ursa_b200 import gen

    n, k, s, d = gen.rmat_batch(count)
    return n, k, s, d


def batch_cpu_sample(n, k, s, d, sample=64):
    """The oracle (CPU restatement of ursa-core) on a bounded, evenly spaced
    sample of the batch: topology build + pagerank + components + triangle
    count per graph, all host threads; returned as graphs/s."""
    from oracle import oracle as O

    O.build()
    O.set_threads(os.cpu_count() or 1)
    off = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
    idx = np.linspace(0, len(n) - 1, sample).astype(int)
    t0 = time.perf_counter()
    for i in idx:
        t = O.Topology(int(n[i]), s[off[i]:off[i + 1]], d[off[i]:off[i + 1]])
        O.pagerank(t, DAMPING, MAX_ITER, TOL)
        O.connected_components_weak(t)
        O.triangle_count(t)
    dt = time.perf_counter() - t0
    # scale by edges: the sample's share of the batch's edge rows
    frac = float(k[idx].sum()) / float(k.sum())
    per_batch_s = dt / frac
    return {"value": len(n) / per_batch_s, "unit": "graphs/s", "cores": O.get_threads(), "kind": "port",
            "sample": f"{sample} evenly spaced graphs of the batch (build + pagerank + components + triangles), "
                      f"scaled to the whole batch by edge rows ({100 * frac:.2f}% of them)"}


def run_reference_batch(args, rank, world):
    """The reference algorithm on the host for the batch workload: per step a
    bounded, evenly spaced sample of the batch through the oracle."""
    if rank != 0:
        return
    from oracle import oracle as O

    O.build()
    O.set_threads(os.cpu_count() or 1)
    n, k, s, d = batch_graphs()
    for _ in range(args.warmup):
        batch_cpu_sample(n, k, s, d, sample=16)
    vals = [batch_cpu_sample(n, k, s, d) for _ in range(args.steps)]
    value = statistics.median(v["value"] for v in vals)
    cb = dict(vals[-1])
    cb["value"] = value
    line = {
        "impl": "reference",
        "metric": "batch_graphs_per_s",
        "value": value,
        "unit": "graphs/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * len(n) / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": BATCH_WORKLOAD, "graphs": len(n), "n_nodes": int(n.sum()), "n_edges": int(k.sum()),
                   "damping": DAMPING, "tol": TOL, "max_iter": MAX_ITER},
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": "graphs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


IDMAP_WORKLOAD = "idmap_rmat22_int64"


def run_idmap(args, rank, world):
    """Node-id interning (IdMap::from_edge_batches) of the R-MAT-22 edges
    under seeded random 64-bit user ids, then Topology::build from the dense
    device columns.  A step: host Int64 columns in (pinned), dense ids and
    the topology out.  CPU baseline: the oracle's serial restatement."""
    import torch

    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    from ursa_b200 import _lib
    from ursa_b200.idmap import IdMap

    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(local_rank))
    n, s, d = make_workload()
    m = int(s.size)
    label = np.random.default_rng(SEED).integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64)
    h_src = torch.from_numpy(label[s]).pin_memory().numpy()
    h_dst = torch.from_numpy(label[d]).pin_memory().numpy()

    def step():
        t0 = time.perf_counter()
        mp = IdMap.from_edge_arrays(h_src, h_dst)
        t1 = time.perf_counter()
        topo = mp.topology()
        t2 = time.perf_counter()
        k = len(mp)
        del topo
        mp.close()
        return t1 - t0, t2 - t1, k

    for _ in range(max(args.warmup, 1)):
        step()
    launches0 = L.ursa_gpu_launch_count()
    res = [step() for _ in range(args.steps)]
    launches = L.ursa_gpu_launch_count() - launches0
    t_map = statistics.median(r[0] for r in res)
    t_topo = statistics.median(r[1] for r in res)
    distinct = res[-1][2]
    line = {
        "metric": "idmap_edges_per_s",
        "value": m / t_map,
        "unit": "edges/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * (t_map + t_topo),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int64 ids -> u32 dense ids",
        "data": "synthetic",
        "config": {"workload": IDMAP_WORKLOAD, "n_edges": m, "distinct_ids": distinct,
                   "ids": "seeded uniform random int64 per R-MAT-22 node"},
        "e2e": {"value": m / (t_map + t_topo), "unit": "edges/s", "h2d_bytes_per_step": 16 * m,
                "d2h_bytes_per_step": 0, "ms_per_step": 1e3 * (t_map + t_topo),
                "note": "host Int64 columns to a resident Topology (interning + CSR build + transpose)"},
        "idmap_ms": 1e3 * t_map, "topology_ms": 1e3 * t_topo,
        "gpu_launches": int(launches),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        O.build()
        k = min(m, 8_000_000)
        t0 = time.perf_counter()
        O.idmap_build(h_src[:k], h_dst[:k])
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": k / dt, "unit": "edges/s", "cores": 1, "kind": "port",
                                "sample": f"serial interning of the first {k:,} edges (the reference interns serially)"}
    if rank == 0:
        print(json.dumps(line), flush=True)


CLOSENESS_SCALE = 16
CLOSENESS_WORKLOAD = "rmat16_closeness"


def closeness_bytes(n: int, m: int, words: int) -> int:
    """Bytes one 64 x `words`-source batch must move at least once: the
    in-CSR (4m + 4(n+1)), the out-offsets for the frontier out-edge counts
    (4(n+1)), and the visited mask array written and read back once
    (2 x 8 words n)."""
    return 4 * m + 8 * (n + 1) + 16 * words * n


def run_closeness(args, rank, world):
    """All-source closeness (closeness.rs:69-135) on R-MAT-16 (edge factor 16,
    seed 2).  value: GTEPS = n sources x m edges / device time of
    ursa_gpu_closeness_device (events on the launch stream), topology
    resident, L2 flushed between steps (the graph fits in L2).  e2e: the
    host C ABI from pinned buffers -- Topology::build + closeness + D2H of
    the n f64 results.  CPU baseline: the oracle's closeness_one on a strided
    sample of sources, all host threads."""
    import torch

    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    from ursa_b200 import Topology, _lib, gen

    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(local_rank))
    n, src, dst = gen.rmat(CLOSENESS_SCALE, EDGE_FACTOR, SEED)
    m = int(src.size)
    topo = Topology.build(n, src, dst)
    topo.prepare(transpose=True)
    stream = torch.cuda.Stream()
    d_out = torch.empty(n, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # > L2 (126 MB)
    ms = C.c_float()

    def dev_step():
        _lib.check(L.ursa_gpu_closeness_device(topo.handle, d_out.data_ptr(), C.c_void_p(stream.cuda_stream),
                                               C.byref(ms)))
        return ms.value

    for _ in range(max(args.warmup, 3)):
        dev_step()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    launches0 = L.ursa_gpu_launch_count()
    step_ms, lib_ms = [], []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib_ms.append(dev_step())
        e1.record(stream)
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    launches = L.ursa_gpu_launch_count() - launches0
    clocks = sampler.stop() if sampler else None
    t_dev = sum(step_ms) / args.steps

    h_src = torch.from_numpy(src).pin_memory()
    h_dst = torch.from_numpy(dst).pin_memory()
    h_out = torch.empty(n, dtype=torch.float64).pin_memory()

    def e2e_step():
        h = C.c_void_p()
        _lib.check(L.ursa_gpu_topo_build(n, h_src.data_ptr(), h_dst.data_ptr(), m, C.byref(h)))
        try:
            _lib.check(L.ursa_gpu_closeness(h, h_out.data_ptr()))
        finally:
            L.ursa_gpu_topo_free(h)

    e2e_step()
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        e2e.append(time.perf_counter() - t0)
    t_e2e = sum(e2e) / args.steps
    words = 4 if n >= 256 and n <= (1 << 21) else 1
    batches = -(-n // (64 * words))
    alg = batches * closeness_bytes(n, m, words)
    peak, peak_kind = load_peaks()
    achieved = alg / (t_dev * 1e-3) / 1e9
    line = {
        "metric": "closeness_gteps",
        "value": n * m / (t_dev * 1e-3) / 1e9,
        "unit": "GTEPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_dev,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u64 source masks, integer distance folds, f64 quotient",
        "data": "synthetic",
        "config": {"workload": CLOSENESS_WORKLOAD, "n_nodes": n, "n_edges": m, "sources": n,
                   "teps": "n sources x m edges per source", "l2": "flushed between steps (256 MB write)",
                   "batch_sources": 64 * words},
        "e2e": {"value": n * m / t_e2e / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": 8 * m,
                "d2h_bytes_per_step": 8 * n, "ms_per_step": 1e3 * t_e2e},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": None, "kernel": "ms_persist_k",
                     "algorithmic_bytes_per_step": alg,
                     "note": "one pass over the in-CSR per batch; the graph is L2-resident, so the "
                             "level count and gather latency bound it, not HBM"},
        "clocks": clocks,
        "library_ms": statistics.median(lib_ms),
    }
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        O.build()
        threads = os.cpu_count() or 1
        O.set_threads(threads)
        ot = O.Topology(n, src, dst)
        k = 256
        while True:
            srcs = (np.arange(k, dtype=np.uint64) * n // k).astype(np.uint32)
            t0 = time.perf_counter()
            O.closeness_sources(ot, srcs)
            dt = time.perf_counter() - t0
            if dt >= 3.0 or k >= n:
                break
            k = min(n, k * 4)
        line["cpu_baseline"] = {"value": k * m / dt / 1e9, "unit": "GTEPS", "cores": threads, "kind": "port",
                                "sample": f"closeness_one from {k:,} strided sources of the same graph"}
    if rank == 0:
        print(json.dumps(line), flush=True)


RESULT_WORKLOAD = "rmat22_query_batch_id_degree_pagerank"


def run_result(args, rank, world):
    """Arrow result materialisation (result.rs:160-168): query_batch of
    (id, out-degree, pagerank d 0.85 tol 1e-6 max_iter 100) over R-MAT-22
    under seeded random Int64 user ids, topology and IdMap resident, to a
    pyarrow RecordBatch in host memory.  Beside it the plain path (the
    per-column C-ABI calls into numpy, the host user-id array, and
    RecordBatch.from_arrays) and an (id, degree) batch, whose time is nearly
    all the copy path (id gather on the device, one D2H into pinned memory,
    the zero-copy import)."""
    import pyarrow as pa
    import torch

    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    from ursa_b200 import _lib, algo
    from ursa_b200.idmap import IdMap
    from ursa_b200.result import OutputColumn, query_batch

    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(local_rank))
    n, s, d = make_workload()
    label = np.random.default_rng(SEED).integers(np.iinfo(np.int64).min, np.iinfo(np.int64).max, n, dtype=np.int64)
    ids = IdMap.from_edge_arrays(label[s], label[d])
    topo = ids.topology()
    topo.prepare(transpose=True)
    rows = len(ids)
    cols = [OutputColumn("deg", "degree", direction="out"),
            OutputColumn("pr", "pagerank", damping=DAMPING, max_iter=MAX_ITER, tol=TOL)]
    light = [OutputColumn("deg", "degree", direction="out")]

    def timed(fn, k):
        for _ in range(max(args.warmup, 1)):
            fn()
        ts = []
        for _ in range(k):
            t0 = time.perf_counter()
            fn()
            ts.append(time.perf_counter() - t0)
        return statistics.median(ts)

    def plain():
        deg = algo.degree(topo, "out")
        pr = algo.pagerank(topo, damping=DAMPING, max_iter=MAX_ITER, tol=TOL)
        return pa.RecordBatch.from_arrays([pa.array(ids.user_id_array()), pa.array(deg), pa.array(pr)],
                                          names=["id", "deg", "pr"])

    launches0 = L.ursa_gpu_launch_count()
    t_query = timed(lambda: query_batch(topo, ids, cols), args.steps)
    launches = (L.ursa_gpu_launch_count() - launches0) / (args.steps + max(args.warmup, 1))
    t_light = timed(lambda: query_batch(topo, ids, light), args.steps)
    t_plain = timed(plain, args.steps)
    bytes_full = rows * (8 + 4 + 8)
    bytes_light = rows * (8 + 4)
    # the host link's own D2H rate into pinned memory for the same bytes
    src_dev = torch.empty(bytes_light, dtype=torch.uint8, device="cuda")
    dst_host = torch.empty(bytes_light, dtype=torch.uint8).pin_memory()
    link = []
    for _ in range(max(args.steps, 3)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dst_host.copy_(src_dev)
        torch.cuda.synchronize()
        link.append(time.perf_counter() - t0)
    link_gbs = bytes_light / min(link) / 1e9
    line = {
        "metric": "query_batch_rows_per_s",
        "value": rows / t_query,
        "unit": "rows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * t_query,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int64 ids, u32 degree, f64 ranks",
        "data": "synthetic",
        "config": {"workload": RESULT_WORKLOAD, "rows": rows, "n_edges": int(s.size),
                   "columns": ["id", "deg", "pr"], "ids": "seeded uniform random int64 per R-MAT-22 node"},
        "e2e": {"value": rows / t_query, "unit": "rows/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": bytes_full, "ms_per_step": 1e3 * t_query,
                "note": "topology and IdMap resident; compute + id translation + one pinned D2H + import"},
        "plain": {"value": rows / t_plain, "unit": "rows/s", "ms_per_step": 1e3 * t_plain,
                  "note": "per-column C-ABI calls into numpy + host user ids + RecordBatch.from_arrays"},
        "id_degree_batch": {"ms": 1e3 * t_light, "bytes": bytes_light,
                            "gb_per_s": bytes_light / t_light / 1e9},
        "roofline": {"bound": "host_link", "achieved": bytes_light / t_light / 1e9, "peak": link_gbs,
                     "unit": "GB/s", "frac": link_gbs and (bytes_light / t_light / 1e9) / link_gbs,
                     "peak_kind": "measured here: torch device-to-pinned copy of the same bytes",
                     "traffic": None, "kernel": "(id, degree) query_batch end to end"},
        "gpu_launches": launches,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


SUITE = ("C1", "C2", "C3")


def run_suite(args, rank, world):
    """Per-kernel table of the hot-path scope on the single-graph
    configurations: C1 = R-MAT-16 (seed 1), C2 = R-MAT-22 (seed 2), C3 =
    n = 2^20 with Poisson(16) out-degrees, uniform targets, multi-edges and
    self-loops kept (seed 3), f32 weights U[1,10) widened to f64.  One JSON
    line per (config, kernel): the B200 device time (events on the library's
    launch stream around the C-ABI call, the n-sized result copied into
    pinned host memory inside it; median over --steps after one warm call),
    its rate, the oracle on all host cores and on one (bounded samples where
    the full run would take minutes), and the error vs the oracle."""
    if rank != 0:
        return
    import torch

    torch.cuda.set_device(0)
    from oracle import oracle as O
    from ursa_b200 import PageRankParams, PageRankStats, Topology, _lib, gen

    O.build()
    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(0))
    sp = C.c_void_p()
    _lib.check(L.ursa_gpu_thread_stream(0, C.byref(sp)))
    lib_stream = torch.cuda.ExternalStream(sp.value)
    cores = os.cpu_count() or 1
    peak, peak_kind = load_peaks()
    reps = max(args.steps, 1)
    only = set(args.suite.split(",")) if args.suite else set(SUITE)
    kern = set(args.suite_kernels.split(",")) if args.suite_kernels else None

    def want(name):  # --suite-kernels: run only these sections (profiling runs)
        return kern is None or name in kern

    def pinned(n, dtype):
        return torch.empty(max(n, 1), dtype=dtype).pin_memory().numpy()[:n]

    def gpu(fn):
        fn()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(lib_stream)
            fn()
            e1.record(lib_stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    def cpu(fn, threads):
        O.set_threads(threads)
        t0 = time.perf_counter()
        out = fn()
        return 1e3 * (time.perf_counter() - t0), out

    def emit(cfg, kernel, gpu_ms, rate, unit, cpu_ms=None, cpu_rate=None, cpu1_rate=None, error=None,
             alg_bytes=None, **extra):
        line = {"suite": cfg, "kernel": kernel, "gpu_ms": gpu_ms, "gpu_rate": rate, "rate_unit": unit,
                "cpu_ms": cpu_ms, "cpu_rate": cpu_rate, "cpu_cores": cores, "cpu1_rate": cpu1_rate,
                "speedup_vs_cpu": (rate / cpu_rate) if (rate and cpu_rate) else None, "error": error}
        if alg_bytes:
            gbs = alg_bytes / (gpu_ms * 1e-3) / 1e9
            line["roofline"] = {"bound": "hbm", "achieved_gbs": gbs, "peak_gbs": peak, "peak_kind": peak_kind,
                                "frac": gbs / peak, "frac_of_8tbs": gbs / 8000.0, "algorithmic_bytes": alg_bytes}
        line.update(extra)
        print(json.dumps(line), flush=True)

    def rel_err(got, ref):
        got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
        den = np.maximum(np.abs(ref), 1e-300)
        return {"l1": float(np.abs(got - ref).sum()), "max_rel": float((np.abs(got - ref) / den).max()) if ref.size else 0.0}

    def canon(labels):  # each node's label -> the smallest node id carrying it
        _, first, inv = np.unique(np.asarray(labels, np.int64), return_index=True, return_inverse=True)
        return first[inv]

    def graph(cfg):
        if cfg == "C1":
            n, s, d = gen.rmat(16, 16, 1)
            return n, s, d, None
        if cfg == "C2":
            n, s, d = gen.rmat(22, 16, 2)
            return n, s, d, None
        n, s, d = gen.poisson(1 << 20, 16.0, 3)
        w = pinned(s.size, torch.float64)  # weights cross to the device every call: keep them pinned
        w[:] = gen.weights_f32(s.size, 1.0, 10.0, 3)
        return n, s, d, w

    for cfg in [c for c in SUITE if c in only]:
        n, s, d, w = graph(cfg)
        m = int(s.size)
        # ---- CSR build and transpose (device arrays in; Topology::build + incoming)
        if want("build"):
            d_s = torch.from_numpy(s).cuda()
            d_d = torch.from_numpy(d).cuda()
            tb = []
            for r in range(reps + 1):  # each build freed before the next (outside the timed span)
                h = C.c_void_p()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(lib_stream)
                _lib.check(L.ursa_gpu_topo_build_device(n, d_s.data_ptr(), d_d.data_ptr(), m, C.c_void_p(sp.value),
                                                        C.byref(h)))
                e1.record(lib_stream)
                e1.synchronize()
                if r:
                    tb.append(e0.elapsed_time(e1))
                L.ursa_gpu_topo_free(h)
            t_build = statistics.median(tb)
            del d_s, d_d
        g = Topology.build(n, s, d)
        cb_ms, ot = cpu(lambda: O.Topology(n, s, d), cores)
        ct_ms, _ = cpu(lambda: ot.csr("in"), cores)
        if want("build"):
            go, oo = g.out(), ot.csr("out")
            gi, oi = g.incoming(), ot.csr("in")
            same = all(np.array_equal(a, b) for a, b in [(go.offsets, oo[0]), (go.targets, oo[1]),
                                                         (go.edge_ids, oo[2]), (gi.offsets, oi[0]),
                                                         (gi.targets, oi[1]), (gi.edge_ids, oi[2])])
            emit(cfg, "csr_build_and_transpose", t_build, m / (t_build * 1e-3), "edges/s", cb_ms + ct_ms,
                 m / ((cb_ms + ct_ms) * 1e-3), None, {"byte_identical": bool(same)}, 2 * (20 * m + 8 * (n + 1)),
                 input="device src/dst arrays",
                 note="the device build sorts the rows by source and by destination in one call (the endpoint "
                      "columns are already in row order on the device); the oracle builds, then transposes",
                 cpu_build_ms=cb_ms, cpu_transpose_ms=ct_ms)
        h = g.handle
        deg_out = pinned(n, torch.int32)

        # ---- degree
        if want("degree"):
            for dname, dval in (("out", 0), ("in", 1)):
                t = gpu(lambda: _lib.check(L.ursa_gpu_degree(h, dval, deg_out.ctypes.data)))
                c_ms, ref = cpu(lambda: O.degree(ot, dname), cores)
                emit(cfg, f"degree_{dname}", t, n / (t * 1e-3), "nodes/s", c_ms, n / (c_ms * 1e-3), None,
                     {"exact": bool(np.array_equal(deg_out.view(np.uint32), ref))}, 4 * (n + 1) + 4 * n)
        outdeg = O.degree(ot, "out")

        # ---- pagerank (plain; weighted on C3)
        if want("pagerank"):
            for weighted in ((False, True) if w is not None else (False,)):
                pr = pinned(n, torch.float64)
                stt = PageRankStats()
                par = PageRankParams(DAMPING, MAX_ITER, TOL)
                if weighted:
                    fn = lambda: _lib.check(L.ursa_gpu_pagerank_weighted(h, w.ctypes.data, m, C.byref(par),
                                                                         pr.ctypes.data, C.byref(stt)))
                else:
                    fn = lambda: _lib.check(L.ursa_gpu_pagerank(h, C.byref(par), pr.ctypes.data, C.byref(stt)))
                t = gpu(fn)
                iters = stt.iterations
                if weighted:
                    c_ms, (ref, oit) = cpu(lambda: O.pagerank_weighted(ot, w, DAMPING, MAX_ITER, TOL, True), cores)
                    c1_ms, _ = cpu(lambda: O.pagerank_weighted(ot, w, DAMPING, 1, 0.0), 1)
                else:
                    c_ms, (ref, oit) = cpu(lambda: O.pagerank(ot, DAMPING, MAX_ITER, TOL, True), cores)
                    c1_ms, _ = cpu(lambda: O.pagerank(ot, DAMPING, 1, 0.0), 1)
                err = rel_err(pr, ref)
                err.update({"iterations": iters, "oracle_iterations": int(oit)})
                alg = algorithmic_bytes(n, m, iters) + (4 * m * iters if weighted else 0)
                emit(cfg, "pagerank_weighted" if weighted else "pagerank", t, m * iters / (t * 1e-3) / 1e9, "GTEPS",
                     c_ms, m * oit / (c_ms * 1e-3) / 1e9, m / (c1_ms * 1e-3) / 1e9, err, alg)

        # ---- BFS from sampled sources with out-degree > 0
        have_out = np.flatnonzero(outdeg > 0)
        k_src = {"C1": 8, "C2": 64, "C3": 8}[cfg]
        srcs = [int(have_out[i]) for i in O.sample_indices(have_out.size, k_src, {"C1": 1, "C2": 2, "C3": 3}[cfg])]
        if want("bfs"):
            dist = [pinned(n, torch.int32) for _ in srcs]

            def bfs_all():
                for x, buf in zip(srcs, dist):
                    _lib.check(L.ursa_gpu_bfs_distances(h, x, 0, buf.ctypes.data))

            t = gpu(bfs_all)
            teps_edges = sum(int(outdeg[np.asarray(dd) >= 0].sum()) for dd in dist)
            k_cpu = min(len(srcs), 8)
            c_ms, refs = cpu(lambda: [O.bfs_distances(ot, x, "out") for x in srcs[:k_cpu]], cores)
            exact = all(np.array_equal(dist[i], refs[i]) for i in range(k_cpu))
            cpu_edges = sum(int(outdeg[r >= 0].sum()) for r in refs)
            touched = teps_edges / max(len(srcs), 1)
            emit(cfg, f"bfs_x{len(srcs)}", t, teps_edges / (t * 1e-3) / 1e9, "GTEPS", c_ms, cpu_edges / (c_ms * 1e-3) / 1e9,
                 cpu_edges / (c_ms * 1e-3) / 1e9, {"exact": bool(exact), "sources_checked": k_cpu},
                 int(len(srcs) * (4 * (n + 1) + 4 * touched + 4 * n)), sources=len(srcs),
                 cpu_note="the oracle's BFS is one serial walk per source (as bfs.rs)")
            # the same sources in one bit-parallel traversal (ursa_gpu_bfs_distances_multi)
            multi = pinned(len(srcs) * n, torch.int32)
            src_arr = np.asarray(srcs, np.uint32)
            t = gpu(lambda: _lib.check(L.ursa_gpu_bfs_distances_multi(h, src_arr.ctypes.data, len(srcs), 0,
                                                                      multi.ctypes.data)))
            mrows = multi.reshape(len(srcs), n)
            same = all(np.array_equal(mrows[i], dist[i]) for i in range(len(srcs)))
            emit(cfg, f"bfs_multi_x{len(srcs)}", t, teps_edges / (t * 1e-3) / 1e9, "GTEPS", c_ms,
                 cpu_edges / (c_ms * 1e-3) / 1e9, cpu_edges / (c_ms * 1e-3) / 1e9,
                 {"equal_to_single_source": bool(same), "sources": len(srcs)},
                 int(len(srcs) * (4 * (n + 1) + 4 * touched + 4 * n)), sources=len(srcs),
                 note="all sources in one traversal; the result rows cross the host link inside the timed span")

        # ---- weak components
        if want("cc"):
            cc = pinned(n, torch.int32)
            t = gpu(lambda: _lib.check(L.ursa_gpu_connected_components_weak(h, cc.ctypes.data)))
            c_ms, ref = cpu(lambda: O.connected_components_weak(ot), cores)
            exact = bool(np.array_equal(canon(cc.view(np.uint32)), canon(ref)))
            emit(cfg, "connected_components_weak", t, m / (t * 1e-3), "edges/s", c_ms, m / (c_ms * 1e-3),
                 m / (c_ms * 1e-3), {"same_partition": exact}, 4 * m + 4 * (n + 1) + 16 * n,
                 cpu_note="union-find is serial in the reference")

        # ---- triangles and clustering (C1, C2)
        if cfg in ("C1", "C2") and want("tc"):
            ms_len = C.c_uint64()
            _lib.check(L.ursa_gpu_topo_undirected_len(h, C.byref(ms_len)))
            m_s = int(ms_len.value)
            tri = pinned(n, torch.int32)
            t = gpu(lambda: _lib.check(L.ursa_gpu_triangle_count(h, tri.ctypes.data)))
            clu = pinned(n, torch.float64)
            tc_ = gpu(lambda: _lib.check(L.ursa_gpu_clustering_coefficient(h, clu.ctypes.data)))
            triangles = int(tri.view(np.uint32).astype(np.int64).sum()) // 3
            if cfg == "C1":
                c_ms, ref = cpu(lambda: O.triangle_count(ot), cores)
                cc_ms, cref = cpu(lambda: O.clustering_coefficient(ot), cores)
                e_t = {"exact": bool(np.array_equal(tri.view(np.uint32), ref))}
                e_c = {"bit_exact": bool(np.array_equal(clu.view(np.uint64), cref.view(np.uint64)))}
            else:
                c_ms = cc_ms = None
                e_t = e_c = {"checked": False,
                             "note": "the reference's merge counting is O(sum of squared degrees) on the host "
                                     "(hours at this scale); exact at C1 and in the GPU tests"}
            emit(cfg, "triangle_count", t, m_s / (t * 1e-3), "undirected entries/s", c_ms,
                 (m_s / (c_ms * 1e-3)) if c_ms else None, None, e_t, 4 * m_s + 8 * (n + 1),
                 triangles=triangles, triangles_per_s=triangles / (t * 1e-3))
            emit(cfg, "clustering_coefficient", tc_, m_s / (tc_ * 1e-3), "undirected entries/s", cc_ms,
                 (m_s / (cc_ms * 1e-3)) if cc_ms else None, None, e_c, 4 * m_s + 8 * (n + 1) + 16 * n)

        # ---- weighted shortest paths and betweenness (C3)
        if cfg == "C3" and want("sssp"):
            dd = pinned(n, torch.float64)
            s0 = srcs[0]
            t = gpu(lambda: _lib.check(L.ursa_gpu_dijkstra_distances(h, w.ctypes.data, m, s0, 0, dd.ctypes.data)))
            c_ms, ref = cpu(lambda: O.dijkstra_distances(ot, w, s0, "out"), 1)
            emit(cfg, "dijkstra_distances", t, m / (t * 1e-3) / 1e9, "GTEPS", c_ms, m / (c_ms * 1e-3) / 1e9,
                 m / (c_ms * 1e-3) / 1e9, {"bit_exact": bool(np.array_equal(dd.view(np.uint64), ref.view(np.uint64)))},
                 None, cpu_note="Dijkstra is serial per source")
            fin = np.flatnonzero(np.isfinite(ref))
            tgt = int(fin[np.argmax(ref[fin])])
            path = pinned(n, torch.int32)
            costs = pinned(n, torch.float64)
            ln = C.c_int64()
            t = gpu(lambda: _lib.check(L.ursa_gpu_shortest_path_weighted_with_cost(
                h, w.ctypes.data, m, s0, tgt, 0, path.ctypes.data, costs.ctypes.data, n, C.byref(ln))))
            c_ms, oref = cpu(lambda: O.shortest_path_weighted_with_cost(ot, w, s0, tgt, "out"), 1)
            k = int(ln.value)
            ok = oref is not None and k == len(oref[0]) and bool(np.array_equal(costs[:k], np.asarray(oref[1])))
            emit(cfg, "shortest_path_weighted_with_cost", t, None, None, c_ms, None, None,
                 {"cost_exact": ok, "path_len": k})
        if cfg == "C3" and want("bc"):
            frac = 2.0 ** -12  # 256 sources at n = 2^20
            for weighted in (False, True):
                bc = pinned(n, torch.float64)
                if weighted:
                    fn = lambda: _lib.check(L.ursa_gpu_betweenness_weighted(h, w.ctypes.data, m, 1, frac, 1, 3,
                                                                            bc.ctypes.data))
                    c_ms, ref = cpu(lambda: O.betweenness_weighted(ot, w, frac, 3), cores)
                else:
                    fn = lambda: _lib.check(L.ursa_gpu_betweenness(h, 1, frac, 1, 3, bc.ctypes.data))
                    c_ms, ref = cpu(lambda: O.betweenness(ot, frac, 3), cores)
                t = gpu(fn)
                k = 256
                emit(cfg, "betweenness_weighted" if weighted else "betweenness", t, k * m / (t * 1e-3) / 1e9, "GTEPS",
                     c_ms, k * m / (c_ms * 1e-3) / 1e9, None, rel_err(bc, ref), None, sources=k)
        del g, ot


SERVE_WORKLOAD = "serve_rmat24_uploads"
SERVE_RATES = (1000, 2000, 5000, 10000, 20000, 50000)


SERVE_MIX = {"shortest_path": 0.45, "bfs": 0.002, "hop2": 0.348, "pagerank": 0.20}


def serve_queries(n, rng, count):
    """(kind, a, b) with kind 0 = shortest_path(a, b), 1 = hop(a, k=2),
    2 = pagerank on the upload picked by b (a uniform draw), 3 = bfs from a
    (Out).  0.2% of the stream is bfs: a bfs answer is n i32 distances (67 MB
    at R-MAT-24), so bfs throughput is bound by the host link (~800/s) and
    by the client's copy of each answer (~10 ms) whatever the GPU does; at
    the sweep's top rate 0.2% is already 100 answers (6.7 GB) a second."""
    r = rng.random(count)
    kind = np.where(r < 0.45, 0, np.where(r < 0.452, 3, np.where(r < 0.80, 1, 2)))
    a = rng.integers(0, n, count)
    b = rng.integers(0, n, count)
    return kind, a, b


def run_serve(args, rank, world):
    import torch

    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    from ursa_b200 import PageRankParams, Topology, _lib, algo, gen
    from ursa_b200.serve import Server

    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(local_rank))
    n, src, dst = gen.rmat(24, 16, 4)
    m = int(src.size)
    topo = Topology.build(n, src, dst)
    topo.prepare(transpose=True)
    del src, dst
    un, uk, us, ud = gen.rmat_batch(600, seed0=5000)
    uoff = np.concatenate([[0], np.cumsum(uk)]).astype(np.int64)
    ups = [(int(un[i]), us[uoff[i]:uoff[i + 1]], ud[uoff[i]:uoff[i + 1]]) for i in range(len(un))]
    srv = Server(topo, path_lanes=4, path_slots=16, hop_lanes=4, hop_slots=16, pr_lanes=2, pr_slots=32,
                 pr_max_nodes=65536, hbm_reserve_bytes=16 << 30, bfs_lanes=2, bfs_slots=16)
    live, live_lock = [], threading.Lock()
    stop_up = threading.Event()

    def uploader():
        """Poisson(200/s) uploads, each released 2 s after it arrived."""
        r = np.random.default_rng(77)
        i = 0
        held = []
        t_next = time.perf_counter()
        while not stop_up.is_set():
            t_next += r.exponential(1 / 200.0)
            while time.perf_counter() < t_next and not stop_up.is_set():
                time.sleep(0.0005)
            g = ups[i % len(ups)]
            i += 1
            try:
                gid = srv.upload(*g)
            except Exception:
                continue  # not admitted: the stream moves on
            now = time.perf_counter()
            with live_lock:
                live.append(gid)
            held.append((now, gid))
            while held and now - held[0][0] > 2.0:
                _, old = held.pop(0)
                with live_lock:
                    live.remove(old)
                srv.release(old)
        for _, gid in held:
            with live_lock:
                if gid in live:
                    live.remove(gid)
            srv.release(gid)

    upt = threading.Thread(target=uploader, daemon=True)
    upt.start()
    while True:
        with live_lock:
            if len(live) >= 50:
                break
        time.sleep(0.01)

    def collector(tq, infos):
        """Fetches results as they complete, keeping only the timings and
        status (a bfs answer is n i32 values: holding thousands of them
        would fill host memory); bfs answers land in one reused buffer."""
        buf = torch.empty(n, dtype=torch.int32).pin_memory().numpy()
        while True:
            t = tq.get()
            if t is None:
                return
            info = srv.result(t, timeout_s=600, out=buf)
            info.result = None
            infos.append(info)

    def drive(rate, count, seed):
        """Open-loop Poisson arrivals at `rate`; returns per-query infos."""
        rng = np.random.default_rng(seed)
        kind, a, b = serve_queries(n, rng, count)
        gaps = rng.exponential(1.0 / rate, count)
        infos = []
        tq = queue.Queue()
        ct = threading.Thread(target=collector, args=(tq, infos), daemon=True)
        ct.start()
        t0 = time.perf_counter()
        t_next = t0
        try:
            for i in range(count):
                t_next += gaps[i]
                while time.perf_counter() < t_next:
                    pass
                if kind[i] == 0:
                    tq.put(srv.shortest_path(int(a[i]), int(b[i])))
                elif kind[i] == 1:
                    tq.put(srv.hop(int(a[i]), 2))
                elif kind[i] == 3:
                    tq.put(srv.bfs(int(a[i]), 0))
                else:
                    # pick and submit under the lock: the uploader removes an id
                    # from `live` (under it) before releasing the graph, and the
                    # submitted query keeps the graph until it finishes
                    with live_lock:
                        gid = live[int(b[i]) % len(live)]
                        tq.put(srv.pagerank(gid, max_iter=MAX_ITER, tol=TOL))
            offered = count / (time.perf_counter() - t0)
        finally:
            tq.put(None)
            ct.join()
        # infos come back in submission order (the collector waits on each
        # ticket in turn), so kind[i] still describes infos[i]
        return infos, offered, kind

    def summarize(infos, kind):
        lat = np.array([x.latency_us for x in infos]) / 1e3
        t_first = min(x.submit_us for x in infos)
        t_last = max(x.done_us for x in infos)
        out = {"completed_qps": len(infos) / ((t_last - t_first) * 1e-6),
               "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
               "errors": int(sum(1 for x in infos if x.status != 0))}
        for k, name in ((0, "shortest_path"), (1, "hop2"), (2, "pagerank"), (3, "bfs")):
            sel = lat[kind == k]
            if sel.size:
                out[name] = {"p50_ms": float(np.percentile(sel, 50)), "p99_ms": float(np.percentile(sel, 99))}
        return out

    def single_type(k, count, seed):
        """Closed loop of one query type on the server: its capacity."""
        rng = np.random.default_rng(seed)
        kind = np.full(count, k)
        a = rng.integers(0, n, count)
        b = rng.integers(0, n, count)
        # four collecting threads, as the plain path has four calling threads
        # (one query type, so the order of infos does not matter here)
        infos = []
        tq = queue.Queue()
        cts = [threading.Thread(target=collector, args=(tq, infos), daemon=True) for _ in range(4)]
        for ct in cts:
            ct.start()
        try:
            for i in range(count):
                if k == 0:
                    tq.put(srv.shortest_path(int(a[i]), int(b[i])))
                elif k == 1:
                    tq.put(srv.hop(int(a[i]), 2))
                elif k == 3:
                    tq.put(srv.bfs(int(a[i]), 0))
                else:
                    with live_lock:
                        gid = live[int(b[i]) % len(live)]
                        tq.put(srv.pagerank(gid, max_iter=MAX_ITER, tol=TOL))
        finally:
            for _ in cts:
                tq.put(None)
            for ct in cts:
                ct.join()
        return summarize(infos, kind)

    try:
        drive(2000, 2000, 1)  # warm-up
        launches0 = L.ursa_gpu_launch_count()
        uuid = None
        try:
            uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
        except Exception:
            pass
        sampler = ClockSampler(uuid) if rank == 0 else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        sweep = []
        total_q = 0
        for j, rate in enumerate(SERVE_RATES):
            count = int(min(max(rate * 3, 3000), 60000))
            infos, offered, kind = drive(rate, count, 100 + j)
            total_q += count
            row = {"rate_qps": rate, "offered_qps": offered, "queries": count}
            row.update(summarize(infos, kind))
            sweep.append(row)
        # closed loop: everything submitted at once (maximum sustained throughput)
        infos, offered, kind = drive(1e9, 60000, 999)
        total_q += 60000
        closed = summarize(infos, kind)
        per_type_server = {name: single_type(k, cnt, 700 + k) for k, name, cnt in
                           ((0, "shortest_path", 20000), (1, "hop2", 20000), (2, "pagerank", 5000), (3, "bfs", 400))}
        clocks = sampler.stop() if sampler else None
        launches = L.ursa_gpu_launch_count() - launches0
        stats = srv.stats()

    except BaseException:
        stop_up.set()
        upt.join(timeout=30)
        srv.close()
        raise
    # the server (and its uploads) go before the plain path is timed
    stop_up.set()
    upt.join(timeout=30)
    srv.close()

    # the plain path: one query per C-ABI call, 4 host threads, closed loop;
    # per type, and for shortest_path both the reference's algorithm
    # (unidirectional exact-order BFS) and the server's (bidirectional, one
    # launch per query)
    plain_topos = {}
    rng = np.random.default_rng(4242)
    kind, a, b = serve_queries(n, rng, 2000)
    pr_params = PageRankParams(DAMPING, MAX_ITER, TOL)
    for i in range(len(ups)):
        if len(plain_topos) >= 64:
            break
        plain_topos[i] = Topology.build(*ups[i])
    keys = list(plain_topos)
    lat = np.zeros(len(kind))

    tls = threading.local()

    def plain_call(k, x, y):
        if k == 0:
            algo.shortest_path(topo, x, y)
        elif k == 1:
            algo.k_hop(topo, [x], 2)
        elif k == 3:
            if not hasattr(tls, "buf"):
                tls.buf = np.empty(n, np.int32)
            _lib.check(L.ursa_gpu_bfs_distances(topo.handle, x, 0, tls.buf.ctypes.data))
        elif k == 4:
            algo.shortest_path_bidirectional(topo, x, y)
        else:
            algo.pagerank(plain_topos[keys[y % len(keys)]], pr_params)

    def plain_one(i):
        t0 = time.perf_counter()
        plain_call(int(kind[i]), int(a[i]), int(b[i]))
        lat[i] = time.perf_counter() - t0

    import concurrent.futures as cf

    with cf.ThreadPoolExecutor(4) as ex:
        list(ex.map(plain_one, range(200)))  # warm-up (plans, pools)
        t0 = time.perf_counter()
        list(ex.map(plain_one, range(len(kind))))
        plain_s = time.perf_counter() - t0
    plain = {"completed_qps": len(kind) / plain_s, "p50_ms": float(np.percentile(lat, 50) * 1e3),
             "p99_ms": float(np.percentile(lat, 99) * 1e3), "queries": int(len(kind)), "threads": 4,
             "note": "closed loop; latency is the per-call service time (no queueing)"}

    def plain_type(k, count, seed):
        r = np.random.default_rng(seed)
        xs, ys = r.integers(0, n, count), r.integers(0, n, count)
        lt = np.zeros(count)

        def one(i):
            t1 = time.perf_counter()
            plain_call(k, int(xs[i]), int(ys[i]))
            lt[i] = time.perf_counter() - t1

        with cf.ThreadPoolExecutor(4) as ex:
            list(ex.map(one, range(min(count, 20))))
            t1 = time.perf_counter()
            list(ex.map(one, range(count)))
            dt = time.perf_counter() - t1
        return {"completed_qps": count / dt, "p50_ms": float(np.percentile(lt, 50) * 1e3),
                "p99_ms": float(np.percentile(lt, 99) * 1e3), "queries": count}

    plain_types = {"shortest_path": plain_type(0, 400, 801), "shortest_path_same_algorithm": plain_type(4, 2000, 802),
                   "hop2": plain_type(1, 2000, 803), "pagerank": plain_type(2, 400, 804), "bfs": plain_type(3, 100, 805)}
    per_type = {}
    for name, srv_row in per_type_server.items():
        row = {"server": srv_row, "plain": plain_types[name],
               "speedup": srv_row["completed_qps"] / plain_types[name]["completed_qps"]}
        if name == "shortest_path":
            row["plain_same_algorithm"] = plain_types["shortest_path_same_algorithm"]
            row["speedup_same_algorithm"] = (srv_row["completed_qps"] /
                                             plain_types["shortest_path_same_algorithm"]["completed_qps"])
        per_type[name] = row

    if rank == 0:
        best = max(sweep, key=lambda r: r["completed_qps"])
        line = {
            "metric": "serve_queries_per_s",
            "value": closed["completed_qps"],
            "unit": "queries/s",
            "n_gpus": world,
            "steps": len(SERVE_RATES) + 1,
            "warmup": 1,
            "ms_per_step": None,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u32 ids; f32-compensated pagerank SpMV, f64 ranks",
            "data": "synthetic",
            "config": {"workload": SERVE_WORKLOAD, "resident_nodes": n, "resident_edges": m,
                       "uploads": "Poisson 200/s, 2 s lifetime, rmat_batch sizes",
                       "mix": SERVE_MIX,
                       "lanes": {"shortest_path": [4, 16], "hop": [4, 16], "pagerank": [2, 32], "bfs": [2, 16]}},
            "closed_loop": closed,
            "sweep": sweep,
            "best_open_loop": {"rate_qps": best["rate_qps"], "completed_qps": best["completed_qps"]},
            "plain_one_query_per_launch": plain,
            "speedup_vs_plain": closed["completed_qps"] / plain["completed_qps"],
            "per_type": per_type,
            "e2e": {"value": closed["completed_qps"], "unit": "queries/s", "h2d_bytes_per_step": None,
                    "d2h_bytes_per_step": None,
                    "note": "every query is submitted from and returned to host memory through the C ABI"},
            "server_stats": stats,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def run_batch(args, rank, world):
    import torch

    local_rank = env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local_rank)
    from ursa_b200 import PageRankParams, Topology, _lib, algo
    from ursa_b200.batch import GraphBatch

    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(local_rank))
    n, k, s, d = batch_graphs(args.batch_count)
    G, N, M = len(n), int(n.sum()), int(k.sum())
    params = PageRankParams(DAMPING, MAX_ITER, TOL)
    h_s = torch.from_numpy(s).pin_memory()
    h_d = torch.from_numpy(d).pin_memory()
    nn, kk = np.ascontiguousarray(n, np.uint64), np.ascontiguousarray(k, np.uint64)

    def build():
        h = C.c_void_p()
        _lib.check(L.ursa_gpu_batch_build(G, nn.ctypes.data, kk.ctypes.data, h_s.data_ptr(), h_d.data_ptr(),
                                          C.byref(h)))
        return h

    b = GraphBatch(n, k, s, d)
    if args.no_tune:
        cfg, tuned_ms = b.config(), None
    else:
        cfg, tuned_ms = b.tune(params)
    stream = torch.cuda.Stream()
    for _ in range(max(args.warmup, 3)):
        b.run(params, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    launches0 = L.ursa_gpu_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        ev[i][0].record(stream)
        b.run(params, stream=stream.cuda_stream)
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    launches = L.ursa_gpu_launch_count() - launches0
    clocks = sampler.stop() if sampler else None
    step_ms = [a.elapsed_time(c) for a, c in ev]
    res = b.results()
    iters = res.iterations
    # per-algorithm device time (one launch each, after the timed region)
    split = {}
    from ursa_b200.batch import BATCH_COMPONENTS, BATCH_PAGERANK, BATCH_TRIANGLES

    for name, what in (("pagerank", BATCH_PAGERANK), ("components", BATCH_COMPONENTS),
                       ("triangles", BATCH_TRIANGLES)):
        b.run(params, what=what)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(params, what=what, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        split[name] = e0.elapsed_time(e1)
    b.run(params)
    b_bytes = b.device_bytes()
    b.close()

    # e2e through the public API: build (H2D) + launch + results (D2H)
    h_pr = torch.empty(N, dtype=torch.float64).pin_memory()
    h_cc = torch.empty(N, dtype=torch.int32).pin_memory()
    h_tc = torch.empty(N, dtype=torch.int32).pin_memory()
    h_it = torch.empty(G, dtype=torch.int32).pin_memory()
    h_de = torch.empty(G, dtype=torch.float64).pin_memory()
    cfg_c = _lib.BatchConfig()
    cfg_c.n_buckets = cfg["n_buckets"]
    for i in range(cfg["n_buckets"]):
        cfg_c.cap[i], cfg_c.threads[i] = cfg["cap"][i], cfg["threads"][i]
    cfg_c.tc_tile, cfg_c.tc_threads = cfg["tc_tile"], cfg["tc_threads"]
    e2e = []
    for i in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        h = build()
        try:
            _lib.check(L.ursa_gpu_batch_set_config(h, C.byref(cfg_c)))
            _lib.check(L.ursa_gpu_batch_run(h, C.byref(params), 7, None))
            _lib.check(L.ursa_gpu_batch_results(h, h_pr.data_ptr(), h_cc.data_ptr(), h_tc.data_ptr(),
                                                h_it.data_ptr(), h_de.data_ptr()))
        finally:
            L.ursa_gpu_batch_free(h)
        if i:  # the first pass warms the pool
            e2e.append(time.perf_counter() - t0)

    # the per-graph plain loop over the same graphs
    plain_s = plain_build_s = float("nan")
    if not args.no_plain:
        off = np.concatenate([[0], np.cumsum(k)]).astype(np.int64)
        t0 = time.perf_counter()
        tops = [Topology.build(int(n[i]), s[off[i]:off[i + 1]], d[off[i]:off[i + 1]]) for i in range(G)]
        plain_build_s = time.perf_counter() - t0

        def plain_pass():
            for t in tops:
                algo.pagerank(t, params)
                algo.connected_components_weak(t)
                algo.triangle_count(t)

        plain_pass()  # plans, lazily built CSRs, pool
        t0 = time.perf_counter()
        plain_pass()
        plain_s = time.perf_counter() - t0
        del tops

    if rank == 0:
        ms = statistics.median(step_ms)
        pr_bytes = batch_pagerank_bytes(n.astype(np.int64), k.astype(np.int64), iters)
        pr_achieved = pr_bytes / (split["pagerank"] * 1e-3) / 1e9
        peak, peak_kind = load_peaks()
        line = {
            "metric": "batch_graphs_per_s",
            "value": G / (ms * 1e-3),
            "unit": "graphs/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32-compensated SpMV, f64 ranks/residual; u32 components and triangle counts",
            "data": "synthetic",
            "config": {"workload": BATCH_WORKLOAD if G == BATCH_COUNT else f"rmat_batch{G}_pr_cc_tc",
                       "graphs": G, "n_nodes": N, "n_edges": M,
                       "damping": DAMPING, "tol": TOL, "max_iter": MAX_ITER,
                       "pagerank_iterations": {"min": int(iters.min()), "median": float(np.median(iters)),
                                               "max": int(iters.max()), "sum": int(iters.sum())},
                       "tuned": cfg, "tuned_ms": tuned_ms, "device_bytes": b_bytes,
                       "l2": "inputs larger than L2 (in-CSR 1.9 GB)"},
            "split_ms": split,
            "e2e": {"value": G / statistics.median(e2e), "unit": "graphs/s",
                    "h2d_bytes_per_step": 8 * M + 16 * G, "d2h_bytes_per_step": 16 * N + 12 * G,
                    "ms_per_step": 1e3 * statistics.median(e2e)},
            "plain_loop": None if args.no_plain else {
                "graphs_per_s": G / plain_s, "s": plain_s, "build_s": plain_build_s,
                "e2e_graphs_per_s": G / (plain_s + plain_build_s),
                "calls": "Topology per graph; pagerank + connected_components_weak + triangle_count per graph, "
                         "host outputs"},
            "speedup_vs_plain": None if args.no_plain else {
                "device": (G / (ms * 1e-3)) / (G / plain_s),
                "e2e": (G / statistics.median(e2e)) / (G / (plain_s + plain_build_s))},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "batch_k (pagerank-only launch)", "achieved": pr_achieved,
                         "peak": peak, "unit": "GB/s", "frac": pr_achieved / peak, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_launch": pr_bytes,
                         "note": "triangle counting (most of the step) is intersection-bound, not HBM-bound"},
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = batch_cpu_sample(n, k, s, d)
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="rmat22_pagerank", choices=["rmat22_pagerank", "batch", "serve", "idmap", "closeness", "result", "suite"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    # profiling aids (defaults give the benchmark above)
    ap.add_argument("--max-iter", type=int, default=MAX_ITER, help="pagerank max_iter (rmat22 workload)")
    ap.add_argument("--tol", type=float, default=TOL, help="pagerank tol (rmat22 workload; 0 = fixed count)")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (rmat22 workload)")
    ap.add_argument("--batch-count", type=int, default=BATCH_COUNT, help="graphs in the batch workload")
    ap.add_argument("--no-tune", action="store_true", help="batch workload: keep the default launch shapes")
    ap.add_argument("--no-plain", action="store_true", help="batch workload: skip the per-graph plain loop")
    ap.add_argument("--suite", default="", help="suite workload: comma-separated configs (C1,C2,C3)")
    ap.add_argument("--suite-kernels", default="",
                    help="suite workload: only these sections (build,degree,pagerank,bfs,cc,tc,sssp,bc)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 0)

    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local_rank = env_int("LOCAL_RANK", 0)

    if args.impl == "reference":
        if args.workload == "batch":
            run_reference_batch(args, rank, world)
        else:
            run_reference(args, rank, world)
        return
    if args.workload == "batch":
        run_batch(args, rank, world)
        return
    if args.workload == "serve":
        run_serve(args, rank, world)
        return
    if args.workload == "idmap":
        run_idmap(args, rank, world)
        return
    if args.workload == "closeness":
        run_closeness(args, rank, world)
        return
    if args.workload == "result":
        run_result(args, rank, world)
        return
    if args.workload == "suite":
        run_suite(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    from ursa_b200 import PageRankParams, PageRankStats, Topology, _lib

    L = _lib.load()
    _lib.check(L.ursa_gpu_set_device(local_rank))
    n, src, dst = make_workload()
    m = int(src.size)
    params = PageRankParams(DAMPING, args.max_iter, args.tol)

    # ---- value: topology resident, device output
    topo = Topology.build(n, src, dst)
    topo.prepare(transpose=True)
    stream = torch.cuda.Stream()
    d_out = torch.empty(n, dtype=torch.float64, device="cuda")

    def dev_step(st):
        _lib.check(L.ursa_gpu_pagerank_device(topo.handle, C.byref(params), d_out.data_ptr(),
                                              C.c_void_p(stream.cuda_stream), C.byref(st)))

    for _ in range(max(args.warmup, 3)):
        dev_step(PageRankStats())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()

    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid) if rank == 0 else None
    if sampler:
        sampler.start()
        time.sleep(0.3)
    launches0 = L.ursa_gpu_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stats = []
    for i in range(args.steps):
        st = PageRankStats()
        ev[i][0].record(stream)
        dev_step(st)
        ev[i][1].record(stream)
        stats.append(st)
    torch.cuda.synchronize()
    launches = L.ursa_gpu_launch_count() - launches0
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    edges_iters = sum(m * s.iterations for s in stats)
    kernel_ms = [s.device_ms for s in stats]
    # clocks cover the kernel-timed region; the sampler's NVML polling is
    # stopped before the end-to-end loop so it cannot stall its driver calls
    clocks = sampler.stop() if sampler else None

    # ---- e2e: the C-ABI call from pinned host buffers (build + pagerank)
    h_src = torch.from_numpy(src).pin_memory()
    h_dst = torch.from_numpy(dst).pin_memory()
    h_out = torch.empty(n, dtype=torch.float64).pin_memory()
    ps, pd, po = h_src.data_ptr(), h_dst.data_ptr(), h_out.data_ptr()

    def e2e_step():
        h = C.c_void_p()
        st = PageRankStats()
        _lib.check(L.ursa_gpu_topo_build(n, ps, pd, m, C.byref(h)))
        try:
            _lib.check(L.ursa_gpu_pagerank(h, C.byref(params), po, C.byref(st)))
        finally:
            L.ursa_gpu_topo_free(h)
        return st.iterations

    e2e_times, e2e_iters = [], []
    if not args.no_e2e:
        for _ in range(max(min(args.warmup, 2), 1)):
            e2e_step()
        torch.cuda.synchronize()
        for _ in range(args.steps):
            t0 = time.perf_counter()
            it = e2e_step()
            e2e_times.append(time.perf_counter() - t0)
            e2e_iters.append(it)
    phases = e2e_phases(L, n, m, h_src, h_dst, h_out, params) if e2e_times else None
    got = d_out.cpu().numpy()

    # ---- max over ranks
    t_dev, t_e2e, edges_iters_all, e2e_edges_all = combine_replicas(
        dist, "cuda", total_ms, sum(e2e_times), edges_iters, m * sum(e2e_iters))

    if rank == 0:
        iters = stats[-1].iterations
        mean_kernel_ms = sum(kernel_ms) / len(kernel_ms)
        alg = algorithmic_bytes(n, m, iters)
        achieved = alg / (mean_kernel_ms * 1e-3) / 1e9
        peak, peak_kind = load_peaks()
        traffic = None
        if NCU_TRAFFIC:
            # scale the captured launch to this launch's iteration count (the
            # prologue moves 16n bytes once, the rest grows per iteration)
            per_iter = (NCU_TRAFFIC["bytes_per_launch"] - 16 * n) / max(NCU_TRAFFIC["iterations"], 1)
            traffic = 16 * n + per_iter * iters
        line = {
            "metric": "pagerank_gteps",
            "value": edges_iters_all / (t_dev * 1e-3) / 1e9,
            "unit": "GTEPS",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t_dev / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32-compensated SpMV, f64 ranks/residual",
            "data": "synthetic",
            "config": rmat22_config(n, m, args.tol, args.max_iter, iters, world),
            "e2e": None if not e2e_times else {"value": e2e_edges_all / t_e2e / 1e9, "unit": "GTEPS",
                    "h2d_bytes_per_step": 8 * m, "d2h_bytes_per_step": 8 * n,
                    "ms_per_step": 1e3 * t_e2e / args.steps,
                    "step_ms_min_median_max": [1e3 * min(e2e_times), 1e3 * statistics.median(e2e_times),
                                               1e3 * max(e2e_times)],
                    "phases_ms": phases},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                         "kernel": "pr_seg_k", "kernel_ms": mean_kernel_ms,
                         "algorithmic_bytes_per_launch": alg},
            "clocks": clocks,
        }
        error, baseline = oracle_check(n, src, dst, got, iters, args.max_iter, args.tol,
                                       world == 1 and not args.no_cpu_baseline)
        line["error"] = error
        if baseline:
            line["cpu_baseline"] = baseline
        print(json.dumps(line), flush=True)
    del topo
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

// serve.cu -- the serving loop: resident graphs, uploads admitted by free HBM,
// and continuous batching of shortest_path, hop and pagerank queries.
//
// The reference serves queries through its plan layer, one kernel call per
// query: ShortestPathExec -> path_batch -> shortest_path (ursa-plan/src/
// result.rs:216, ursa-core/src/algo/bfs.rs:48-102), hop_batch -> k_hop
// (result.rs:180, algo/hop.rs:52-130) and GraphAlgorithmExec -> pagerank
// (result.rs:82-140, algo/pagerank.rs:98-124).  Here a server owns:
//  * lanes: a CUDA stream with preallocated per-query slots, dedicated to one
//    query type.  A scheduler thread fills every free lane with up to
//    `slots` pending queries of its type and launches ONE kernel for them
//    (a CTA per query); lanes run concurrently, so queries that arrive while
//    others are on the GPU start as soon as a lane frees up and overlap with
//    the launches in flight.  Completions are detected with events, results
//    copied out, and the lane refilled at once.
//  * shortest_path: bidirectional BFS (out-CSR forward from the source,
//    in-CSR backward from the target), expanding the side whose frontier
//    has fewer edges; it stops after the first level on which the sides
//    meet and takes the shortest meeting (ties: smallest meeting id).
//    Parents are the smallest-id discoverer of each node at its level, so
//    the path is deterministic: the same alone and in any mix.  The path is
//    a valid shortest path (hop count equal to the reference's); its nodes
//    may differ from the reference's serial-order choice on ties.
//  * hop: k_hop from one seed in the reference's exact emission order
//    (level by level; within a level, candidates in the order of their
//    parents and of the CSR, first occurrence kept, the seed excluded).
//  * bfs: bfs_distances (algo/bfs.rs:18-42) for up to 64 queries of one
//    direction per launch, bit q of per-node masks belonging to query q; one
//    pull pass over the nodes per level (kernels that never wait on another
//    CTA, so they share the GPU with the persistent slot kernels).
//  * pagerank on uploaded graphs: the batch bucket kernel (batch.cu) over
//    the launch's graphs, whose results do not depend on the other graphs.
// Per-slot visit state is stamped (query base + level in the high word), so
// no array is cleared between queries.  No kernel waits on another CTA;
// cancellation is a per-query flag checked between BFS levels.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.cuh"
#include "primitives.cuh"

namespace ug {

namespace {

constexpr int kSvThreads = 512;
constexpr int kSvWarps = kSvThreads / 32;
constexpr uint32_t kStampStride = 1u << 16;  // levels per query
constexpr uint32_t kPathCap = 4096;          // nodes of a returned path
constexpr uint32_t kHubDegree = 4096;        // edges above which the whole CTA expands a node

__device__ __forceinline__ uint64_t pack_stamp(uint32_t stamp, uint32_t low) {
  return ((uint64_t)stamp << 32) | low;
}
__device__ __forceinline__ uint32_t stamp_of(uint64_t v) { return (uint32_t)(v >> 32); }
__device__ __forceinline__ uint64_t ld_volatile(const uint64_t* p) {
  return *(const volatile unsigned long long*)p;
}

// ------------------------------------------------------------ shortest path
struct PathSlot {
  uint64_t* fpar;  // n: (stamp, ~forward parent)
  uint64_t* bpar;  // n: (stamp, ~backward parent)
  uint32_t* q[4];  // frontier queues: forward cur/next, backward cur/next
};

struct PathQuery {
  uint32_t s, t, base;
};

struct PathOut {
  int32_t len;     // path nodes, -1 = no path
  int32_t status;  // URSA_GPU_OK / URSA_GPU_ECANCELED / URSA_GPU_ETRUNC
  uint64_t edges;  // edges scanned
};

struct PathArgs {
  const uint32_t* out_off;
  const uint32_t* out_tgt;
  const uint32_t* in_off;
  const uint32_t* in_tgt;
  uint64_t n;
};

struct PathShared {
  unsigned long long best;
  unsigned long long work;
  uint32_t next_size;
  uint32_t hubs[64];
  uint32_t n_hubs;
};

// Visits edge (u -> v) of the side being expanded at level L (stamp).
__device__ __forceinline__ void path_visit(uint32_t u, uint32_t v, uint32_t base, uint32_t stamp,
                                           uint32_t other_depth, uint64_t* par,
                                           const uint64_t* other, const uint32_t* off_next,
                                           uint32_t* nxt, PathShared& sh) {
  const uint32_t st = stamp_of(ld_volatile(par + v));
  if (st >= base && st < stamp) return;  // reached on an earlier level
  const uint64_t prev = atomicMax((unsigned long long*)(par + v), pack_stamp(stamp, ~u));
  if (stamp_of(prev) == stamp) return;  // already discovered on this level
  const uint32_t idx = atomicAdd(&sh.next_size, 1u);
  nxt[idx] = v;
  atomicAdd(&sh.work, (unsigned long long)(off_next[v + 1] - off_next[v]));
  const uint32_t os = stamp_of(other[v]);
  if (os >= base && os <= base + other_depth) {
    const uint32_t total = (stamp - base) + (os - base);
    atomicMin(&sh.best, ((unsigned long long)total << 32) | v);
  }
}

// Runs one shortest_path query with the whole CTA; thread 0 writes the path
// to `path` (kPathCap nodes) and returns the result.
__device__ PathOut path_query(const PathArgs& A, const PathQuery q, const PathSlot& S,
                              uint32_t* path, const volatile uint32_t* cancel, PathShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (q.s >= A.n || q.t >= A.n) return PathOut{-1, URSA_GPU_OK, 0};  // bfs.rs:55-57
  if (q.s == q.t) {
    if (threadIdx.x == 0) path[0] = q.s;
    return PathOut{1, URSA_GPU_OK, 0};
  }
  const uint32_t base = q.base;
  if (threadIdx.x == 0) {
    S.fpar[q.s] = pack_stamp(base, ~q.s);
    S.bpar[q.t] = pack_stamp(base, ~q.t);
    S.q[0][0] = q.s;
    S.q[2][0] = q.t;
  }
  uint32_t fsize = 1, bsize = 1, lf = 0, lb = 0;
  unsigned long long fwork = A.out_off[q.s + 1] - A.out_off[q.s];
  unsigned long long bwork = A.in_off[q.t + 1] - A.in_off[q.t];
  int fcur = 0, bcur = 2;
  uint64_t scanned = 0;
  int status = URSA_GPU_OK;
  int32_t len = -1;
  __syncthreads();
  while (true) {
    if (fsize == 0 || bsize == 0) break;  // one side is exhausted: no path
    if (*cancel) {
      status = URSA_GPU_ECANCELED;
      break;
    }
    const bool fwd = fwork <= bwork;
    const uint32_t* off = fwd ? A.out_off : A.in_off;
    const uint32_t* tgt = fwd ? A.out_tgt : A.in_tgt;
    const uint32_t* off_next = off;  // next frontier's work is measured on the same side
    uint64_t* par = fwd ? S.fpar : S.bpar;
    const uint64_t* other = fwd ? S.bpar : S.fpar;
    const uint32_t* cur = S.q[fwd ? fcur : bcur];
    uint32_t* nxt = S.q[fwd ? (fcur ^ 1) : (bcur ^ 1)];
    const uint32_t size = fwd ? fsize : bsize;
    const uint32_t stamp = base + (fwd ? lf : lb) + 1;
    const uint32_t other_depth = fwd ? lb : lf;
    if (stamp - base >= kStampStride - 1) {  // deeper than the stamp range
      status = URSA_GPU_ETRUNC;
      break;
    }
    if (threadIdx.x == 0) {
      sh.best = ~0ull;
      sh.work = 0;
      sh.next_size = 0;
      sh.n_hubs = 0;
    }
    __syncthreads();
    // warps take frontier nodes; nodes above kHubDegree edges are queued for
    // the whole CTA (or kept by their warp when the queue is full)
    for (uint32_t i = warp; i < size; i += kSvWarps) {
      const uint32_t u = cur[i];
      const uint32_t b = off[u], e = off[u + 1];
      if (e - b > kHubDegree) {
        uint32_t slot = 0;
        if (lane == 0) slot = atomicAdd(&sh.n_hubs, 1u);
        slot = __shfl_sync(0xffffffffu, slot, 0);
        if (slot < 64) {
          if (lane == 0) sh.hubs[slot] = u;
          continue;
        }
      }
      for (uint32_t k = b + lane; k < e; k += 32)
        path_visit(u, tgt[k], base, stamp, other_depth, par, other, off_next, nxt, sh);
    }
    __syncthreads();
    const uint32_t nh = sh.n_hubs < 64 ? sh.n_hubs : 64;
    for (uint32_t h = 0; h < nh; h++) {
      const uint32_t u = sh.hubs[h];
      const uint32_t b = off[u], e = off[u + 1];
      for (uint32_t k = b + threadIdx.x; k < e; k += kSvThreads)
        path_visit(u, tgt[k], base, stamp, other_depth, par, other, off_next, nxt, sh);
    }
    __syncthreads();
    const uint32_t ns = sh.next_size;
    const unsigned long long nwork = sh.work;
    const unsigned long long best = sh.best;
    if (fwd) {
      scanned += fwork;
      fcur ^= 1;
      fsize = ns;
      fwork = nwork;
      lf++;
    } else {
      scanned += bwork;
      bcur ^= 1;
      bsize = ns;
      bwork = nwork;
      lb++;
    }
    __syncthreads();  // sh is reset by thread 0 on the next level
    if (best != ~0ull) {
      const uint32_t v = (uint32_t)best;
      const uint32_t total = (uint32_t)(best >> 32);
      if (total + 1 > kPathCap) {
        status = URSA_GPU_ETRUNC;
        break;
      }
      if (threadIdx.x == 0) {
        const uint32_t df = stamp_of(S.fpar[v]) - base;
        uint32_t x = v;
        path[df] = v;
        for (int i = (int)df - 1; i >= 0; i--) {
          x = ~(uint32_t)S.fpar[x];
          path[i] = x;
        }
        x = v;
        for (uint32_t i = df + 1; i <= total; i++) {
          x = ~(uint32_t)S.bpar[x];
          path[i] = x;
        }
      }
      len = (int32_t)(total + 1);
      break;
    }
  }
  return PathOut{len, status, scanned};
}

// --------------------------------------------------------------------- hop
struct HopSlot {
  uint64_t* seen;  // n: (stamp, ~candidate position)
  uint32_t* out;   // n + 1: out[0] = seed, then levels 1..k in order
  uint32_t* pre;   // n: edge prefix of the previous level
  uint32_t* cnt;   // n: kept candidates per previous-level node (then prefix)
};

struct HopQuery {
  uint32_t s, k, base;
};

struct HopOut {
  uint32_t count;  // reached nodes (pairs)
  int32_t status;
  uint64_t edges;
};

struct HopArgs {
  const uint32_t* off;
  const uint32_t* tgt;
  uint64_t n;
};

struct HopShared {
  uint32_t warp_sum[kSvWarps];
  uint32_t carry;
};

// Exclusive scan of a[0..len) in place by the whole CTA (chunks of the CTA
// size, carried across chunks); returns the total.  a[i] = f(i) is read
// through the functor so the input need not be materialised.
template <class F>
__device__ uint32_t cta_exclusive_scan(uint32_t len, uint32_t* outp, F&& f, HopShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) sh.carry = 0;
  __syncthreads();
  for (uint32_t c = 0; c < len; c += kSvThreads) {
    const uint32_t i = c + threadIdx.x;
    const uint32_t v = i < len ? f(i) : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    if (lane == 31) sh.warp_sum[warp] = x;
    __syncthreads();
    uint32_t before = sh.carry;
    for (int w = 0; w < warp; w++) before += sh.warp_sum[w];
    if (i < len) outp[i] = before + x - v;
    __syncthreads();
    if (threadIdx.x == kSvThreads - 1) sh.carry = before + x;
    __syncthreads();
  }
  const uint32_t total = sh.carry;
  __syncthreads();
  return total;
}

// Runs one hop query with the whole CTA: the reached nodes are S.out[1..].
__device__ HopOut hop_query(const HopArgs& A, const HopQuery q, const HopSlot& S,
                            const volatile uint32_t* cancel, HopShared& sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (q.s >= A.n || q.k == 0) return HopOut{0, URSA_GPU_OK, 0};  // an out-of-range seed reaches nothing
  const uint32_t base = q.base;
  if (threadIdx.x == 0) {
    S.seen[q.s] = pack_stamp(base, ~0u);
    S.out[0] = q.s;
  }
  __syncthreads();
  uint32_t pa = 0, pb = 1;  // previous level = out[pa, pb)
  uint64_t scanned = 0;
  int status = URSA_GPU_OK;
  for (uint32_t lvl = 1; lvl <= q.k && pb > pa; lvl++) {
    if (*cancel) {
      status = URSA_GPU_ECANCELED;
      break;
    }
    if (lvl >= kStampStride - 1) {
      status = URSA_GPU_ETRUNC;
      break;
    }
    const uint32_t stamp = base + lvl;
    const uint32_t np = pb - pa;
    const uint32_t* prev = S.out + pa;
    // edge positions of the level's candidate stream
    const uint32_t total = cta_exclusive_scan(
        np, S.pre, [&](uint32_t i) { const uint32_t u = prev[i]; return A.off[u + 1] - A.off[u]; }, sh);
    scanned += total;
    // claim: the first position of each unseen node wins
    for (uint32_t i = warp; i < np; i += kSvWarps) {
      const uint32_t u = prev[i], b = A.off[u], e = A.off[u + 1], p0 = S.pre[i];
      for (uint32_t j = lane; j < e - b; j += 32) {
        const uint32_t w = A.tgt[b + j];
        const uint32_t st = stamp_of(ld_volatile(S.seen + w));
        if (st >= base && st < stamp) continue;
        atomicMax((unsigned long long*)(S.seen + w), pack_stamp(stamp, ~(p0 + j)));
      }
    }
    __syncthreads();
    // kept candidates per previous-level node
    for (uint32_t i = warp; i < np; i += kSvWarps) {
      const uint32_t u = prev[i], b = A.off[u], e = A.off[u + 1], p0 = S.pre[i];
      uint32_t c = 0;
      for (uint32_t j = lane; j < e - b; j += 32) {
        const uint32_t w = A.tgt[b + j];
        c += S.seen[w] == pack_stamp(stamp, ~(p0 + j)) ? 1u : 0u;
      }
      c = __reduce_add_sync(0xffffffffu, c);
      if (lane == 0) S.cnt[i] = c;
    }
    __syncthreads();
    const uint32_t kept = cta_exclusive_scan(np, S.cnt, [&](uint32_t i) { return S.cnt[i]; }, sh);
    // write the kept candidates in stream order
    for (uint32_t i = warp; i < np; i += kSvWarps) {
      const uint32_t u = prev[i], b = A.off[u], e = A.off[u + 1], p0 = S.pre[i];
      uint32_t at = pb + S.cnt[i];
      for (uint32_t j0 = 0; j0 < e - b; j0 += 32) {
        const uint32_t j = j0 + lane;
        bool keep = false;
        uint32_t w = 0;
        if (j < e - b) {
          w = A.tgt[b + j];
          keep = S.seen[w] == pack_stamp(stamp, ~(p0 + j));
        }
        const uint32_t m = __ballot_sync(0xffffffffu, keep);
        if (keep) S.out[at + __popc(m & ((1u << lane) - 1u))] = w;
        at += __popc(m);
      }
    }
    __syncthreads();
    pa = pb;
    pb += kept;
  }
  return HopOut{pb - 1, status, scanned};
}

// One shortest_path query as its own launch (the plain form of a server
// slot): the whole CTA runs path_query on fresh, zeroed visit arrays.
__global__ void __launch_bounds__(kSvThreads) path_once_k(PathArgs A, PathQuery q, PathSlot S,
                                                          uint32_t* path, PathOut* out,
                                                          const uint32_t* cancel) {
  __shared__ PathShared sh;
  const PathOut o = path_query(A, q, S, path, cancel, sh);
  if (threadIdx.x == 0) *out = o;
}

// --------------------------------------------------------------------- bfs
// Level L of a batch: a node v still missing some queries ORs the frontier
// masks of its pull neighbours (in-CSR for Out, out-CSR for In, undirected
// CSR for Both) until every missing query has found it; the new bits become
// v's next frontier mask and set its distance to L.  found[L & 1] records
// whether the level reached anything; every kernel of level L first reads
// found[(L + 1) & 1] (level L - 1) and returns at once when it is 0, so
// levels enqueued past the end cost a launch each.  Nodes with more than
// kBfsHub pull entries are done by a warp in bfs_level_hub_k.
constexpr uint32_t kBfsHub = 64;

struct BfsArgs {
  const uint32_t* off;
  const uint32_t* nbr;
  uint64_t n;
  const uint64_t* front;
  uint64_t* next;
  uint64_t* visited;
  int32_t* dist;  // queries x n
  uint64_t qmask;
  int32_t level;
  unsigned* found;  // [2]
  const uint32_t* hubs;
  uint32_t n_hubs;
};

__device__ __forceinline__ void bfs_settle(const BfsArgs& A, uint64_t v, uint64_t fresh) {
  A.visited[v] |= fresh;
  for (uint64_t bits = fresh; bits; bits &= bits - 1) {
    const uint64_t q = (uint64_t)(__ffsll((long long)bits) - 1);
    A.dist[q * A.n + v] = A.level;
  }
}

__global__ void bfs_level_k(BfsArgs A) {
  if (*(volatile unsigned*)&A.found[(A.level + 1) & 1] == 0) return;
  bool any = false;
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < A.n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t b = A.off[v], e = A.off[v + 1];
    if (e - b > kBfsHub) continue;  // the hub kernel's
    const uint64_t need = A.qmask & ~A.visited[v];
    uint64_t fresh = 0;
    if (need) {
      uint64_t acc = 0;
      for (uint32_t k = b; k < e; k++) {
        acc |= A.front[A.nbr[k]];
        if ((acc & need) == need) break;
      }
      fresh = acc & need;
      if (fresh) {
        bfs_settle(A, v, fresh);
        any = true;
      }
    }
    A.next[v] = fresh;
  }
  const unsigned m = __ballot_sync(0xffffffffu, any);  // every lane gets here
  if (m && (threadIdx.x & 31) == __ffs(m) - 1) atomicOr(&A.found[A.level & 1], 1u);
}

__global__ void bfs_level_hub_k(BfsArgs A) {
  if (*(volatile unsigned*)&A.found[(A.level + 1) & 1] == 0) return;
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = gw; i < A.n_hubs; i += nw) {
    const uint32_t v = A.hubs[i];
    const uint32_t b = A.off[v], e = A.off[v + 1];
    const uint64_t need = A.qmask & ~A.visited[v];
    uint64_t acc = 0;
    for (uint32_t k0 = b; k0 < e && need; k0 += 32) {
      const uint32_t k = k0 + lane;
      if (k < e) acc |= A.front[A.nbr[k]];
      const uint64_t all = ((uint64_t)__reduce_or_sync(0xffffffffu, (unsigned)(acc >> 32)) << 32) |
                           __reduce_or_sync(0xffffffffu, (unsigned)acc);
      acc = all;
      if ((acc & need) == need) break;
    }
    const uint64_t fresh = acc & need;
    if (lane == 0) {
      if (fresh) {
        bfs_settle(A, v, fresh);
        atomicOr(&A.found[A.level & 1], 1u);
      }
      A.next[v] = fresh;
    }
  }
}

// Sources of the batch: query q's bit at its source, distance 0.
__global__ void bfs_seed_k(const uint32_t* __restrict__ src, uint32_t nq, uint64_t n,
                           uint64_t* __restrict__ visited, uint64_t* __restrict__ front,
                           int32_t* __restrict__ dist) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  const uint32_t s = src[q];
  atomicOr((unsigned long long*)(visited + s), 1ull << q);
  atomicOr((unsigned long long*)(front + s), 1ull << q);
  dist[(uint64_t)q * n + s] = 0;
}

__global__ void bfs_hub_flag_k(const uint32_t* __restrict__ off, uint64_t n, uint32_t* __restrict__ flag) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    flag[v] = off[v + 1] - off[v] > kBfsHub ? 1u : 0u;
}

__global__ void bfs_hub_scatter_k(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                                  uint64_t n, uint32_t* __restrict__ hubs) {
  for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (uint64_t)gridDim.x * blockDim.x)
    if (flag[v]) hubs[pos[v]] = (uint32_t)v;
}

// ------------------------------------------------------- persistent lanes
// A slot's query lives in DEVICE memory (the CTA polls only its own GPU's
// memory): the host writes the fields with one async copy and then seq_in
// with a second copy on the same stream.  The CTA answers into pinned host
// memory mapped into the device (posted writes): the result fields, then
// seq_out = seq_in, which the host polls locally.
struct alignas(32) DevMail {
  uint32_t a, b, k, base;  // source / seed, target, hop depth, stamp base
  uint32_t cancel;
  uint32_t pad[2];
  uint32_t seq_in;
};

struct alignas(32) HostMail {
  uint32_t seq_out;
  int32_t len, status;
  uint32_t pad;
  uint64_t edges;
};

struct LaneCtl {
  uint32_t stop;       // host: the lane's CTAs return
  uint32_t heartbeat;  // host: bumped by the scheduler while it runs
};

struct LaneArgs {
  const DevMail* mail;  // slots (device memory)
  HostMail* res;        // slots (mapped host memory)
  const LaneCtl* ctl;   // device memory
  uint32_t* paths;      // shortest_path: slots * kPathCap (mapped host memory)
  PathArgs pa;
  const PathSlot* pslots;
  HopArgs ha;
  const HopSlot* hslots;
  uint64_t heartbeat_ns;  // return when the host's heartbeat stops this long
  uint64_t idle_ns;       // safety bound: return after this long without a query
  uint32_t* expired;      // mapped host word: set when a bounded wait ran out
};

template <class T>
__device__ __forceinline__ T vload(const T* p) {
  return *(const volatile T*)p;
}

// One CTA per slot.  Every wait is bounded: a CTA returns when the host asks
// (stop; the host stops a whole lane after it has been idle a while), when
// the host's heartbeat stalls for heartbeat_ns (the host is gone), or, as a
// last bound, after idle_ns without a query; the host relaunches the lane
// when it has work for it.
template <int KIND>
__global__ void __launch_bounds__(kSvThreads) lane_k(LaneArgs A) {
  __shared__ PathShared psh;
  __shared__ HopShared hsh;
  __shared__ uint32_t cmd[6];  // stop, seq, a, b, k, base
  const uint32_t slot = blockIdx.x;
  const DevMail* mb = A.mail + slot;
  HostMail* hr = A.res + slot;
  uint32_t done_seq = vload(&hr->seq_out);
  while (true) {
    if (threadIdx.x == 0) {
      uint32_t hb_last = vload(&A.ctl->heartbeat);
      uint64_t t_hb = global_ns(), t_idle = t_hb;
      uint32_t stop = 0, si = 0;
      while (true) {
        if (vload(&A.ctl->stop)) {
          stop = 1;
          break;
        }
        si = vload(&mb->seq_in);
        if (si != done_seq) break;
        const uint64_t now = global_ns();
        const uint32_t hb = vload(&A.ctl->heartbeat);
        if (hb != hb_last) {
          hb_last = hb;
          t_hb = now;
        }
        if (now - t_hb > A.heartbeat_ns || now - t_idle > A.idle_ns) {
          *(volatile uint32_t*)A.expired = 1u;  // the host counts the expiry
          __threadfence_system();
          stop = 1;
          break;
        }
        __nanosleep(500);
      }
      __threadfence();  // the query fields are read after seq_in
      cmd[0] = stop;
      cmd[1] = si;
      cmd[2] = vload(&mb->a);
      cmd[3] = vload(&mb->b);
      cmd[4] = vload(&mb->k);
      cmd[5] = vload(&mb->base);
    }
    __syncthreads();
    if (cmd[0]) return;
    const volatile uint32_t* cancel = &mb->cancel;
    int32_t len, status;
    uint64_t edges;
    if (KIND == 0) {
      const PathOut o = path_query(A.pa, PathQuery{cmd[2], cmd[3], cmd[5]}, A.pslots[slot],
                                   A.paths + (size_t)slot * kPathCap, cancel, psh);
      len = o.len;
      status = o.status;
      edges = o.edges;
    } else {
      const HopOut o = hop_query(A.ha, HopQuery{cmd[2], cmd[4], cmd[5]}, A.hslots[slot], cancel, hsh);
      len = (int32_t)o.count;
      status = o.status;
      edges = o.edges;
    }
    __syncthreads();
    done_seq = cmd[1];
    if (threadIdx.x == 0) {
      *(volatile int32_t*)&hr->len = len;
      *(volatile int32_t*)&hr->status = status;
      *(volatile uint64_t*)&hr->edges = edges;
      __threadfence_system();  // device buffers, results and the mapped path before seq_out
      *(volatile uint32_t*)&hr->seq_out = done_seq;
    }
    __syncthreads();
  }
}

double now_us() {
  return std::chrono::duration<double, std::micro>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

}  // namespace
}  // namespace ug

using namespace ug;

namespace {

struct Upload {
  uint32_t id = 0;
  ursa_gpu_batch* batch = nullptr;
  uint64_t n = 0, bytes = 0;
  int refs = 0;  // queries holding the upload
};

struct Request {
  uint64_t ticket = 0;
  ursa_gpu_query q{};
  ursa_gpu_query_info info{};
  std::vector<uint32_t> u32;  // path / reached nodes
  std::vector<double> f64;    // pagerank
  uint32_t* pinned = nullptr; // bfs: the n distances, in a buffer of the server's pool
  bool done = false;
  bool cancel = false;
  std::shared_ptr<Upload> up;
};

enum LaneKind { kLanePath = 0, kLaneHop = 1, kLanePr = 2, kLaneBfs = 3 };

struct Lane {
  LaneKind kind;
  uint32_t slots = 0;
  cudaStream_t stream = nullptr;  // kernels
  cudaStream_t copy = nullptr;    // result copies, slot clears
  cudaEvent_t done = nullptr;     // after the lane's current launch
  bool running = false;           // persistent kernel (path / hop) or launch (pagerank) in flight
  bool stopping = false;          // stop raised, kernel not yet returned
  double last_use = 0.0;          // host clock of the last post or harvest
  // path / hop: persistent slots
  DevArray<DevMail> d_mail;       // queries (device)
  DevMail* h_stage = nullptr;     // pinned staging of the queries
  DevArray<LaneCtl> d_ctl;        // stop / heartbeat (device)
  LaneCtl* h_ctl = nullptr;       // pinned staging of the control words
  HostMail* res = nullptr;        // mapped, host view
  HostMail* d_res = nullptr;      // device view
  uint32_t* paths = nullptr;      // mapped, host view
  uint32_t* d_paths = nullptr;
  uint32_t* h_expired = nullptr;  // mapped word the slot kernels set on a wait expiry
  uint32_t* d_expired = nullptr;
  std::vector<std::shared_ptr<Request>> slot_req;  // request in each slot (null = free)
  std::vector<uint32_t> seq;                       // last seq posted per slot
  std::vector<uint32_t> base;                      // next stamp base per slot
  std::vector<DevArray<uint64_t>> u64a, u64b;
  std::vector<DevArray<uint32_t>> a32[4];
  DevArray<PathSlot> d_pslots;
  DevArray<HopSlot> d_hslots;
  // pagerank: one launch per batch of queries
  std::vector<std::shared_ptr<Request>> reqs;
  DevArray<GraphDesc> d_desc;
  DevArray<uint32_t> d_work, d_iters;
  DevArray<double> d_delta, d_rank;
  DevArray<float> d_x;
  uint32_t* h_iters = nullptr;
  double* h_delta = nullptr;
  uint64_t pr_max_n = 0;
  // bfs: one batch of up to 64 queries of one direction per launch
  DevArray<uint64_t> b_vis, b_front[2];
  DevArray<int32_t> b_dist;
  DevArray<uint32_t> b_src;
  DevArray<unsigned> b_found;
  uint32_t* h_bsrc = nullptr;
  unsigned* h_found = nullptr;
  std::vector<int32_t> b_row;  // per queued request: its row in the batch, -1 = out of range
  int32_t b_level = 0;         // last level enqueued
  // a finished batch's n-sized answers are copied out by this thread (tens of
  // ms per batch), so that the scheduler keeps serving the other lanes; the
  // lane stays running until it is done (its device rows are reused)
  std::thread harvester;
  bool harvesting = false;
  int b_dir = 0;
  uint64_t b_qmask = 0;
};

}  // namespace

struct ursa_gpu_server {
  int device = 0;
  TopoImpl* topo = nullptr;
  ursa_gpu_server_config cfg{};
  std::vector<std::unique_ptr<Lane>> lanes;
  std::mutex mu;
  std::condition_variable cv_sched, cv_done;
  std::deque<std::shared_ptr<Request>> pending[4];
  // pull-entry hubs of the resident topology per bfs direction (built on first use)
  DevArray<uint32_t> bfs_hubs[3];
  uint32_t bfs_n_hubs[3] = {0, 0, 0};
  bool bfs_hubs_built[3] = {false, false, false};
  std::unordered_map<uint64_t, std::shared_ptr<Request>> reqs;
  std::deque<uint64_t> completed;  // tickets not yet returned by poll
  std::unordered_map<uint32_t, std::shared_ptr<Upload>> uploads;
  uint32_t next_upload = 1;
  uint64_t next_ticket = 1;
  uint64_t upload_bytes = 0;
  ursa_gpu_server_stats stats{};
  std::thread sched;
  std::atomic<bool> stop{false};
  double last_heartbeat = 0.0;
  std::string fatal;  // a CUDA failure in the scheduler ends the server
  // bfs answers (n i32 each) land in pinned host buffers at the host link's
  // full rate: two batches' worth per bfs lane, allocated with the server.  A
  // finished query holds one until its result is fetched; a batch waits for
  // free buffers when clients fall behind (back-pressure on the bfs lanes
  // only).
  std::vector<uint32_t*> bfs_bufs, bfs_free;
  std::condition_variable cv_bfs;
};

namespace ug {
namespace {

constexpr uint64_t kHeartbeatNs = 5000000000ull;  // 5 s without the scheduler
constexpr uint64_t kIdleNs = 600000000000ull;     // 10 min without a query (safety bound)
constexpr double kLaneIdleStopUs = 20e6;          // the host stops a lane idle for 20 s

void free_pinned(void* p) {
  if (p) cudaFreeHost(p);
}

// Raises the lane's stop word (its CTAs return within a poll).
void lane_raise_stop(Lane& L) {
  if (!L.h_ctl) return;
  L.h_ctl->stop = 1;
  cudaMemcpyAsync(&L.d_ctl.get()->stop, &L.h_ctl->stop, 4, cudaMemcpyHostToDevice, L.copy);
  cudaStreamSynchronize(L.copy);
}

// Frees a lane; every lane's stop must have been raised first (freeing
// pinned memory synchronises the whole device).
void lane_destroy(Lane& L) {
  if (L.stream) cudaStreamSynchronize(L.stream);
  if (L.copy) cudaStreamSynchronize(L.copy);
  L.d_mail.release();
  L.d_ctl.release();
  free_pinned(L.h_stage);
  free_pinned(L.h_ctl);
  free_pinned(L.res);
  free_pinned(L.paths);
  free_pinned(L.h_iters);
  free_pinned(L.h_delta);
  free_pinned(L.h_expired);
  free_pinned(L.h_bsrc);
  free_pinned(L.h_found);
  if (L.done) cudaEventDestroy(L.done);
  if (L.stream) cudaStreamDestroy(L.stream);
  if (L.copy) cudaStreamDestroy(L.copy);
}

template <class T>
T* mapped_alloc(size_t count, T** dev) {
  T* h = nullptr;
  UG_CUDA(cudaHostAlloc((void**)&h, count * sizeof(T), cudaHostAllocMapped));
  std::memset((void*)h, 0, count * sizeof(T));
  UG_CUDA(cudaHostGetDevicePointer((void**)dev, h, 0));
  return h;
}

void lane_create(ursa_gpu_server* S, Lane& L, LaneKind kind, uint32_t slots) {
  const uint64_t n = S->topo ? S->topo->n : 0;
  const uint64_t nn = n ? n : 1;
  L.kind = kind;
  L.slots = slots;
  UG_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
  UG_CUDA(cudaStreamCreateWithFlags(&L.copy, cudaStreamNonBlocking));
  UG_CUDA(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
  cudaStream_t s = L.stream;
  L.h_expired = mapped_alloc<uint32_t>(1, &L.d_expired);
  if (kind == kLanePath || kind == kLaneHop) {
    L.d_mail.alloc(slots, s);
    UG_CUDA(cudaMemsetAsync(L.d_mail.get(), 0, slots * sizeof(DevMail), s));
    UG_CUDA(cudaMallocHost((void**)&L.h_stage, slots * sizeof(DevMail)));
    std::memset((void*)L.h_stage, 0, slots * sizeof(DevMail));
    L.d_ctl.alloc(1, s);
    UG_CUDA(cudaMemsetAsync(L.d_ctl.get(), 0, sizeof(LaneCtl), s));
    UG_CUDA(cudaMallocHost((void**)&L.h_ctl, sizeof(LaneCtl)));
    std::memset((void*)L.h_ctl, 0, sizeof(LaneCtl));
    L.res = mapped_alloc<HostMail>(slots, &L.d_res);
    L.slot_req.assign(slots, nullptr);
    L.seq.assign(slots, 0);
    L.base.assign(slots, kStampStride);
  }
  if (kind == kLanePath) {
    L.paths = mapped_alloc<uint32_t>((size_t)slots * kPathCap, &L.d_paths);
    L.u64a.resize(slots);
    L.u64b.resize(slots);
    for (auto& v : L.a32) v.resize(slots);
    std::vector<PathSlot> ps(slots);
    for (uint32_t i = 0; i < slots; i++) {
      L.u64a[i].alloc(nn, s);
      L.u64b[i].alloc(nn, s);
      UG_CUDA(cudaMemsetAsync(L.u64a[i].get(), 0, nn * 8, s));
      UG_CUDA(cudaMemsetAsync(L.u64b[i].get(), 0, nn * 8, s));
      for (int j = 0; j < 4; j++) L.a32[j][i].alloc(nn, s);
      ps[i].fpar = L.u64a[i].get();
      ps[i].bpar = L.u64b[i].get();
      for (int j = 0; j < 4; j++) ps[i].q[j] = L.a32[j][i].get();
    }
    L.d_pslots.alloc(slots, s);
    UG_CUDA(cudaMemcpyAsync(L.d_pslots.get(), ps.data(), slots * sizeof(PathSlot),
                            cudaMemcpyHostToDevice, s));
  } else if (kind == kLaneHop) {
    L.u64a.resize(slots);
    for (int j = 0; j < 3; j++) L.a32[j].resize(slots);
    std::vector<HopSlot> hs(slots);
    for (uint32_t i = 0; i < slots; i++) {
      L.u64a[i].alloc(nn, s);
      UG_CUDA(cudaMemsetAsync(L.u64a[i].get(), 0, nn * 8, s));
      L.a32[0][i].alloc(n + 1, s);
      L.a32[1][i].alloc(nn, s);
      L.a32[2][i].alloc(nn, s);
      hs[i] = HopSlot{L.u64a[i].get(), L.a32[0][i].get(), L.a32[1][i].get(), L.a32[2][i].get()};
    }
    L.d_hslots.alloc(slots, s);
    UG_CUDA(cudaMemcpyAsync(L.d_hslots.get(), hs.data(), slots * sizeof(HopSlot),
                            cudaMemcpyHostToDevice, s));
  } else if (kind == kLaneBfs) {
    L.b_vis.alloc(nn, s);
    L.b_front[0].alloc(nn, s);
    L.b_front[1].alloc(nn, s);
    L.b_dist.alloc((size_t)slots * nn, s);
    L.b_src.alloc(slots, s);
    L.b_found.alloc(2, s);
    UG_CUDA(cudaMallocHost((void**)&L.h_bsrc, slots * 4));
    UG_CUDA(cudaMallocHost((void**)&L.h_found, 2 * sizeof(unsigned)));
    L.h_found[0] = L.h_found[1] = 0;
  } else {
    const uint64_t mx = S->cfg.pr_max_nodes;
    L.pr_max_n = mx;
    L.d_desc.alloc(slots, s);
    L.d_work.alloc(slots + 1, s);  // work list + counter
    L.d_iters.alloc(slots, s);
    L.d_delta.alloc(slots, s);
    L.d_rank.alloc((size_t)slots * mx, s);
    L.d_x.alloc((size_t)slots * 2 * mx, s);
    UG_CUDA(cudaMallocHost((void**)&L.h_iters, slots * 4));
    UG_CUDA(cudaMallocHost((void**)&L.h_delta, slots * 8));
  }
  UG_CUDA(cudaStreamSynchronize(s));
}

// (Re)launches a path / hop lane's persistent kernel.
void lane_start(ursa_gpu_server* S, Lane& L) {
  L.h_ctl->stop = 0;  // the previous kernel has returned
  UG_CUDA(cudaMemcpyAsync(&L.d_ctl.get()->stop, &L.h_ctl->stop, 4, cudaMemcpyHostToDevice, L.copy));
  UG_CUDA(cudaEventRecord(L.done, L.copy));
  UG_CUDA(cudaStreamWaitEvent(L.stream, L.done, 0));  // the launch sees stop = 0
  L.stopping = false;
  L.last_use = now_us();
  LaneArgs a{};
  a.mail = L.d_mail.get();
  a.res = L.d_res;
  a.ctl = L.d_ctl.get();
  a.paths = L.d_paths;
  const TopoImpl* t = S->topo;
  a.pa = PathArgs{t->out.off.get(), t->out.tgt.get(), t->in.off.get(), t->in.tgt.get(), t->n};
  a.pslots = L.d_pslots.get();
  a.ha = HopArgs{t->out.off.get(), t->out.tgt.get(), t->n};
  a.hslots = L.d_hslots.get();
  a.heartbeat_ns = S->cfg.heartbeat_limit_ns ? S->cfg.heartbeat_limit_ns : kHeartbeatNs;
  a.idle_ns = kIdleNs;
  a.expired = L.d_expired;
  if (L.kind == kLanePath)
    lane_k<0><<<L.slots, kSvThreads, 0, L.stream>>>(a);
  else
    lane_k<1><<<L.slots, kSvThreads, 0, L.stream>>>(a);
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaEventRecord(L.done, L.stream));
  L.running = true;
  S->stats.launches++;
}

// Next stamp base of a slot; when the range wraps, the slot's visit arrays
// are cleared first (the slot is idle: its CTA only reads them for a query).
uint32_t take_base(Lane& L, uint32_t slot, uint64_t n) {
  uint32_t b = L.base[slot];
  if (b > 0xFFFFFFFFu - 2 * kStampStride) {
    UG_CUDA(cudaMemsetAsync(L.u64a[slot].get(), 0, (n ? n : 1) * 8, L.copy));
    if (L.kind == kLanePath) UG_CUDA(cudaMemsetAsync(L.u64b[slot].get(), 0, (n ? n : 1) * 8, L.copy));
    UG_CUDA(cudaStreamSynchronize(L.copy));
    b = kStampStride;
  }
  L.base[slot] = b + kStampStride;
  return b;
}

void post(ursa_gpu_server* S, Lane& L, uint32_t slot, const std::shared_ptr<Request>& r) {
  DevMail* st = L.h_stage + slot;  // untouched until the slot completes
  st->a = r->q.source;
  st->b = r->q.target;
  st->k = r->q.k;
  st->base = take_base(L, slot, S->topo->n);
  st->cancel = r->cancel ? 1u : 0u;
  st->seq_in = ++L.seq[slot];
  DevMail* d = L.d_mail.get() + slot;
  // fields first, then the sequence number: copies on one stream run in order
  UG_CUDA(cudaMemcpyAsync(d, st, offsetof(DevMail, seq_in), cudaMemcpyHostToDevice, L.copy));
  UG_CUDA(cudaMemcpyAsync(&d->seq_in, &st->seq_in, 4, cudaMemcpyHostToDevice, L.copy));
  L.slot_req[slot] = r;
  r->info.launch_us = now_us();
  L.last_use = r->info.launch_us;
}

// A finished slot's result (the server lock is not held: the slot stays
// taken until this returns).
void slot_harvest(Lane& L, uint32_t slot, Request& r) {
  std::atomic_thread_fence(std::memory_order_acquire);
  const HostMail* mb = L.res + slot;
  r.info.status = *(const volatile int32_t*)&mb->status;
  r.info.edges = *(const volatile uint64_t*)&mb->edges;
  const int32_t len = *(const volatile int32_t*)&mb->len;
  if (L.kind == kLanePath) {
    r.info.result_len = len;
    if (r.info.status == URSA_GPU_OK && len > 0) {
      const uint32_t* p = L.paths + (size_t)slot * kPathCap;
      r.u32.assign(p, p + len);
    }
  } else {
    r.info.result_len = len;
    if (r.info.status == URSA_GPU_OK && len > 0) {
      r.u32.resize((size_t)len);
      UG_CUDA(cudaMemcpyAsync(r.u32.data(), L.a32[0][slot].get() + 1, (size_t)len * 4,
                              cudaMemcpyDeviceToHost, L.copy));
      UG_CUDA(cudaStreamSynchronize(L.copy));
    }
  }
}

// Launches a pagerank lane for its queued requests (server lock held).
void pr_launch(ursa_gpu_server* S, Lane& L) {
  const uint32_t nq = (uint32_t)L.reqs.size();
  cudaStream_t s = L.stream;
  const double t = now_us();
  std::vector<GraphDesc> desc(nq);
  std::vector<uint32_t> work(nq + 1, 0);
  uint32_t cap = 0;
  for (uint32_t i = 0; i < nq; i++) {
    auto& r = *L.reqs[i];
    r.info.launch_us = t;
    desc[i] = *batch_host_desc(r.up->batch, 0);
    desc[i].rank = L.d_rank.get() + (size_t)i * L.pr_max_n;
    desc[i].x0 = L.d_x.get() + (size_t)i * 2 * L.pr_max_n;
    desc[i].x1 = desc[i].x0 + L.pr_max_n;
    cap = std::max(cap, desc[i].n);
    work[i] = i;
  }
  std::stable_sort(work.begin(), work.begin() + nq,
                   [&](uint32_t x, uint32_t y) { return desc[x].n > desc[y].n; });
  work[nq] = 0;  // the work counter
  UG_CUDA(cudaMemcpyAsync(L.d_desc.get(), desc.data(), nq * sizeof(GraphDesc), cudaMemcpyHostToDevice, s));
  UG_CUDA(cudaMemcpyAsync(L.d_work.get(), work.data(), (nq + 1) * 4, cudaMemcpyHostToDevice, s));
  cap = std::min<uint32_t>(std::max<uint32_t>(cap, 1u), 57344u);
  const uint32_t threads = 256;
  const size_t smem = (size_t)cap * 4;
  const int resident = batch_kernel_resident(threads, smem, S->device);
  BucketArgs a;
  a.desc = L.d_desc.get();
  a.work = L.d_work.get();
  a.n_work = nq;
  a.next = L.d_work.get() + nq;
  a.cap = cap;
  a.what = kBkWhatPr;
  const auto& p = L.reqs[0]->q.pr;
  a.max_iter = p.max_iter;
  a.damping = p.damping;
  a.tol = p.tol;
  a.iters = L.d_iters.get();
  a.delta = L.d_delta.get();
  void* args[] = {&a};
  UG_CUDA(cudaLaunchKernel(batch_kernel_for(threads), dim3(std::min<int>(resident, (int)nq)),
                           dim3(threads), args, smem, s));
  count_launch();
  UG_CUDA(cudaMemcpyAsync(L.h_iters, L.d_iters.get(), nq * 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(L.h_delta, L.d_delta.get(), nq * 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaEventRecord(L.done, s));
  L.running = true;
  S->stats.launches++;
}

void pr_harvest(Lane& L) {
  const uint32_t nq = (uint32_t)L.reqs.size();
  for (uint32_t i = 0; i < nq; i++) {
    Request& r = *L.reqs[i];
    r.info.status = URSA_GPU_OK;
    r.info.iterations = L.h_iters[i];
    r.info.last_delta = L.h_delta[i];
    const uint64_t ng = r.up->n;
    r.info.result_len = (int64_t)ng;
    r.f64.resize(ng);
    if (ng)
      UG_CUDA(cudaMemcpyAsync(r.f64.data(), L.d_rank.get() + (size_t)i * L.pr_max_n, ng * 8,
                              cudaMemcpyDeviceToHost, L.copy));
  }
  UG_CUDA(cudaStreamSynchronize(L.copy));
}

// ---- bfs lanes
struct PullCsr {
  const uint32_t* off;
  const uint32_t* nbr;
};

// Pull CSR of a bfs direction on the resident topology: Out pulls over the
// in-CSR, In over the out-CSR, Both over the undirected CSR (built on first
// use).
PullCsr bfs_pull(ursa_gpu_server* S, int dir, cudaStream_t s) {
  TopoImpl* t = S->topo;
  if (dir == 2) {
    ensure_undirected(t, s);
    return PullCsr{t->und_off.get(), t->und_tgt.get()};
  }
  ensure_in(t, s);
  if (dir == 1) return PullCsr{t->out.off.get(), t->out.tgt.get()};
  return PullCsr{t->in.off.get(), t->in.tgt.get()};
}

// Nodes with more than kBfsHub pull entries, once per direction.
void bfs_build_hubs(ursa_gpu_server* S, int dir, const PullCsr& c, cudaStream_t s) {
  if (S->bfs_hubs_built[dir]) return;
  const uint64_t n = S->topo->n;
  Scratch<uint32_t> flag(n, s), pos(n, s), tot(1, s);
  bfs_hub_flag_k<<<grid_for(n), kBlock, 0, s>>>(c.off, n, flag.get());
  UG_LAUNCH_CHECK();
  exclusive_scan_u32(flag.get(), pos.get(), n, tot.get(), s);
  uint32_t nh = 0;
  UG_CUDA(cudaMemcpyAsync(&nh, tot.get(), 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  S->bfs_hubs[dir].alloc(nh ? nh : 1, s);
  if (nh) {
    bfs_hub_scatter_k<<<grid_for(n), kBlock, 0, s>>>(flag.get(), pos.get(), n, S->bfs_hubs[dir].get());
    UG_LAUNCH_CHECK();
  }
  UG_CUDA(cudaStreamSynchronize(s));
  S->bfs_n_hubs[dir] = nh;
  S->bfs_hubs_built[dir] = true;
}

constexpr int32_t kBfsLevelsPerStep = 8;

// Enqueues the batch's next kBfsLevelsPerStep levels, then the copy of the
// last level's found flag into h_found[0] and the lane's event.
void bfs_enqueue_levels(ursa_gpu_server* S, Lane& L) {
  const uint64_t n = S->topo->n;
  cudaStream_t s = L.stream;
  const PullCsr c = bfs_pull(S, L.b_dir, s);
  BfsArgs a;
  a.off = c.off;
  a.nbr = c.nbr;
  a.n = n;
  a.visited = L.b_vis.get();
  a.dist = L.b_dist.get();
  a.qmask = L.b_qmask;
  a.found = L.b_found.get();
  a.hubs = S->bfs_hubs[L.b_dir].get();
  a.n_hubs = S->bfs_n_hubs[L.b_dir];
  for (int k = 0; k < kBfsLevelsPerStep; k++) {
    const int32_t lvl = ++L.b_level;
    a.level = lvl;
    a.front = L.b_front[(lvl + 1) & 1].get();
    a.next = L.b_front[lvl & 1].get();
    UG_CUDA(cudaMemsetAsync(L.b_found.get() + (lvl & 1), 0, sizeof(unsigned), s));
    bfs_level_k<<<grid_for(n), kBlock, 0, s>>>(a);
    UG_LAUNCH_CHECK();
    if (a.n_hubs) {
      bfs_level_hub_k<<<grid_for((uint64_t)a.n_hubs * 32), kBlock, 0, s>>>(a);
      UG_LAUNCH_CHECK();
    }
  }
  UG_CUDA(cudaMemcpyAsync(L.h_found, L.b_found.get() + (L.b_level & 1), sizeof(unsigned),
                          cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaEventRecord(L.done, s));
}

// Starts a bfs batch for the lane's queued requests (server lock held):
// in-range sources get a row and a bit; the others answer all -1.
void bfs_launch(ursa_gpu_server* S, Lane& L) {
  const uint64_t n = S->topo->n;
  cudaStream_t s = L.stream;
  const double t = now_us();
  uint32_t nq = 0;
  L.b_row.assign(L.reqs.size(), -1);
  for (size_t i = 0; i < L.reqs.size(); i++) {
    L.reqs[i]->info.launch_us = t;
    const uint32_t src = L.reqs[i]->q.source;
    if (src < n) {  // bfs.rs:21-23: an out-of-range source reaches nothing
      L.h_bsrc[nq] = src;
      L.b_row[i] = (int32_t)nq;
      nq++;
    }
  }
  L.b_dir = (int)L.reqs[0]->q.direction;
  L.b_level = 0;
  L.b_qmask = nq >= 64 ? ~0ull : ((1ull << nq) - 1ull);
  L.running = true;
  S->stats.launches++;
  if (nq == 0) {
    L.h_found[0] = 0;
    UG_CUDA(cudaEventRecord(L.done, s));
    return;
  }
  const PullCsr c = bfs_pull(S, L.b_dir, s);
  bfs_build_hubs(S, L.b_dir, c, s);
  UG_CUDA(cudaMemcpyAsync(L.b_src.get(), L.h_bsrc, nq * 4, cudaMemcpyHostToDevice, s));
  UG_CUDA(cudaMemsetAsync(L.b_vis.get(), 0, n * 8, s));
  UG_CUDA(cudaMemsetAsync(L.b_front[0].get(), 0, n * 8, s));
  UG_CUDA(cudaMemsetAsync(L.b_dist.get(), 0xFF, (size_t)nq * n * 4, s));
  UG_CUDA(cudaMemsetAsync(L.b_found.get(), 0x01, sizeof(unsigned), s));  // level 0 reached the sources
  UG_CUDA(cudaMemsetAsync(L.b_found.get() + 1, 0, sizeof(unsigned), s));
  bfs_seed_k<<<(nq + 63) / 64, 64, 0, s>>>(L.b_src.get(), nq, n, L.b_vis.get(), L.b_front[0].get(),
                                           L.b_dist.get());
  UG_LAUNCH_CHECK();
  bfs_enqueue_levels(S, L);
}

// Copies each query's distance row out (the server lock is not held).
void bfs_harvest(ursa_gpu_server* S, Lane& L) {
  const uint64_t n = S->topo->n;
  {  // one pool buffer per answer (the server's close ends the wait)
    std::unique_lock<std::mutex> lk(S->mu);
    for (auto& rp : L.reqs) {
      while (S->bfs_free.empty() && !S->stop.load())
        S->cv_bfs.wait_for(lk, std::chrono::milliseconds(10));
      if (S->bfs_free.empty()) throw Error(URSA_GPU_ECANCELED, "bfs: the server is closing");
      rp->pinned = S->bfs_free.back();
      S->bfs_free.pop_back();
    }
  }
  for (size_t i = 0; i < L.reqs.size(); i++) {
    Request& r = *L.reqs[i];
    r.info.status = URSA_GPU_OK;
    r.info.result_len = (int64_t)n;
    r.info.iterations = (uint32_t)L.b_level;
    const int32_t row = L.b_row[i];
    if (row < 0) {
      std::fill(r.pinned, r.pinned + n, 0xFFFFFFFFu);
      continue;
    }
    if (n)
      UG_CUDA(cudaMemcpyAsync(r.pinned, L.b_dist.get() + (size_t)row * n, n * 4,
                              cudaMemcpyDeviceToHost, L.copy));
  }
  UG_CUDA(cudaStreamSynchronize(L.copy));
}

void complete(ursa_gpu_server* S, const std::shared_ptr<Request>& r, double t);

// The bfs lane's harvest thread: copies the finished batch's answers out,
// then completes its requests and frees the lane under the server's lock.  A
// CUDA failure fails the batch's requests and ends the server like a
// scheduler failure does.
void bfs_harvest_worker(ursa_gpu_server* S, Lane* L) {
  std::string err;
  try {
    UG_CUDA(cudaSetDevice(S->device));
    bfs_harvest(S, *L);
  } catch (const std::exception& ex) {
    err = ex.what();
  }
  {
    std::lock_guard<std::mutex> g(S->mu);
    const double t = now_us();
    for (auto& r : L->reqs) {
      if (!err.empty()) {
        r->info.status = S->stop.load() ? URSA_GPU_ECANCELED : URSA_GPU_ECUDA;
        r->info.result_len = 0;
        if (r->pinned) S->bfs_free.push_back(r->pinned);
        r->pinned = nullptr;
      }
      complete(S, r, t);
    }
    L->reqs.clear();
    L->running = false;
    L->harvesting = false;
    L->last_use = t;
    if (!err.empty() && !S->stop.load() && S->fatal.empty()) S->fatal = err;
  }
  S->cv_done.notify_all();
  S->cv_sched.notify_all();
}

void complete(ursa_gpu_server* S, const std::shared_ptr<Request>& r, double t) {
  r->info.done_us = t;
  r->done = true;
  if (r->up) {
    r->up->refs--;
    r->up.reset();
  }
  S->completed.push_back(r->ticket);
  S->stats.completed++;
}

void sched_loop(ursa_gpu_server* S) {
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  while (!S->stop.load()) {
    bool progressed = false;
    try {
      const double t_now = now_us();
      const double period = S->cfg.heartbeat_period_us ? (double)S->cfg.heartbeat_period_us : 1000.0;
      if (t_now - S->last_heartbeat > period) {  // about once a millisecond by default
        S->last_heartbeat = t_now;
        for (auto& lp : S->lanes)
          if (lp->h_ctl && lp->running) {
            lp->h_ctl->heartbeat++;
            UG_CUDA(cudaMemcpyAsync(&lp->d_ctl.get()->heartbeat, &lp->h_ctl->heartbeat, 4,
                                    cudaMemcpyHostToDevice, lp->copy));
          }
      }
      for (auto& lp : S->lanes) {
        Lane& L = *lp;
        if (L.kind == kLanePr) {
          // pagerank: harvest a finished launch, then refill the lane
          if (L.running) {
            const cudaError_t e = cudaEventQuery(L.done);
            if (e == cudaErrorNotReady) continue;
            UG_CUDA(e);
            lk.unlock();
            pr_harvest(L);
            lk.lock();
            const double t = now_us();
            for (auto& r : L.reqs) complete(S, r, t);
            L.reqs.clear();
            L.running = false;
            progressed = true;
          }
          auto& pq = S->pending[kLanePr];
          while (!pq.empty() && L.reqs.size() < L.slots) {
            auto r = pq.front();
            if (!L.reqs.empty() &&
                (r->q.pr.damping != L.reqs[0]->q.pr.damping || r->q.pr.tol != L.reqs[0]->q.pr.tol ||
                 r->q.pr.max_iter != L.reqs[0]->q.pr.max_iter))
              break;  // different parameters: next launch
            pq.pop_front();
            L.reqs.push_back(r);
          }
          if (!L.reqs.empty()) {
            pr_launch(S, L);
            progressed = true;
          }
          continue;
        }
        if (L.kind == kLaneBfs) {
          // bfs: more levels, or harvest a finished batch; then refill
          if (L.running) {
            if (L.harvesting) continue;  // its harvest thread frees the lane
            const cudaError_t e = cudaEventQuery(L.done);
            if (e == cudaErrorNotReady) continue;
            UG_CUDA(e);
            if (*(volatile unsigned*)L.h_found) {
              bfs_enqueue_levels(S, L);
              continue;
            }
            // the previous harvest thread has set harvesting = false and
            // released the lock, so this join returns at once
            if (L.harvester.joinable()) L.harvester.join();
            L.harvesting = true;
            L.harvester = std::thread(bfs_harvest_worker, S, &L);
            progressed = true;
            continue;
          }
          auto& bq = S->pending[kLaneBfs];
          while (!bq.empty() && L.reqs.size() < L.slots) {
            auto r = bq.front();
            if (!L.reqs.empty() && r->q.direction != L.reqs[0]->q.direction) break;  // next launch
            bq.pop_front();
            L.reqs.push_back(r);
          }
          if (!L.reqs.empty()) {
            bfs_launch(S, L);
            progressed = true;
          }
          continue;
        }
        // path / hop: finished slots out, pending queries into free slots
        if (L.running) {
          const cudaError_t e = cudaEventQuery(L.done);
          if (e == cudaSuccess) {
            L.running = false;  // every CTA returned
            if (*(volatile uint32_t*)L.h_expired) {  // ... because a bounded wait ran out
              *(volatile uint32_t*)L.h_expired = 0u;
              S->stats.wait_expiries++;
            }
          } else if (e != cudaErrorNotReady) {
            UG_CUDA(e);
          }
        }
        for (uint32_t i = 0; i < L.slots; i++) {
          auto r = L.slot_req[i];
          if (!r) continue;
          if (*(const volatile uint32_t*)&L.res[i].seq_out != L.seq[i]) continue;
          lk.unlock();
          slot_harvest(L, i, *r);
          lk.lock();
          L.slot_req[i] = nullptr;
          complete(S, r, now_us());
          progressed = true;
        }
        auto& pq = S->pending[L.kind];
        bool posted = false;
        for (uint32_t i = 0; i < L.slots && !pq.empty(); i++) {
          if (L.slot_req[i]) continue;
          post(S, L, i, pq.front());
          pq.pop_front();
          posted = true;
        }
        bool waiting = false;
        for (uint32_t i = 0; i < L.slots; i++) waiting |= L.slot_req[i] != nullptr;
        if (waiting && !L.running) lane_start(S, L);
        if (!waiting && L.running && !L.stopping && now_us() - L.last_use > kLaneIdleStopUs) {
          L.h_ctl->stop = 1;  // idle lane: give its SMs back
          UG_CUDA(cudaMemcpyAsync(&L.d_ctl.get()->stop, &L.h_ctl->stop, 4, cudaMemcpyHostToDevice, L.copy));
          L.stopping = true;
        }
        progressed |= posted;
      }
    } catch (const std::exception& ex) {
      S->fatal = ex.what();
      for (auto& kv : S->reqs)
        if (!kv.second->done) {
          kv.second->info.status = URSA_GPU_ECUDA;
          kv.second->done = true;
          S->completed.push_back(kv.first);
        }
      for (auto& q : S->pending) q.clear();
      S->cv_done.notify_all();
      break;
    }
    if (progressed) S->cv_done.notify_all();
    if (!progressed) {
      bool any_busy = false;
      for (auto& lp : S->lanes) {
        any_busy |= lp->running && (lp->kind == kLanePr || lp->kind == kLaneBfs);
        for (auto& r : lp->slot_req) any_busy |= r != nullptr;
      }
      if (any_busy) {
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(2));
        lk.lock();
      } else {
        S->cv_sched.wait_for(lk, std::chrono::milliseconds(1));
      }
    }
  }
}

}  // namespace
}  // namespace ug

extern "C" {

int ursa_gpu_server_create(ursa_gpu_topo* resident, const ursa_gpu_server_config* cfg,
                           ursa_gpu_server** out) {
  return guard([&] {
    UG_CHECK(out && cfg, URSA_GPU_EINVAL, "out / config is NULL");
    *out = nullptr;
    UG_CHECK(cfg->path_lanes + cfg->hop_lanes + cfg->pr_lanes + cfg->bfs_lanes > 0, URSA_GPU_EINVAL,
             "server: no lanes configured");
    UG_CHECK(!(cfg->path_lanes || cfg->hop_lanes || cfg->bfs_lanes) || resident, URSA_GPU_EINVAL,
             "server: path, hop and bfs lanes need a resident topology");
    UG_CHECK(cfg->bfs_lanes == 0 || (cfg->bfs_slots >= 1 && cfg->bfs_slots <= 64), URSA_GPU_EINVAL,
             "server: bfs lanes need 1..64 slots");
    for (uint32_t v : {cfg->path_slots, cfg->hop_slots, cfg->pr_slots})
      UG_CHECK(v <= 1024, URSA_GPU_EINVAL, "server: at most 1024 slots per lane");
    UG_CHECK((cfg->path_lanes == 0 || cfg->path_slots) && (cfg->hop_lanes == 0 || cfg->hop_slots),
             URSA_GPU_EINVAL, "server: lanes need slots");
    UG_CHECK(cfg->pr_lanes == 0 || (cfg->pr_slots && cfg->pr_max_nodes), URSA_GPU_EINVAL,
             "server: pagerank lanes need slots and pr_max_nodes");
    std::unique_ptr<ursa_gpu_server> S(new ursa_gpu_server());
    S->cfg = *cfg;
    if (resident) {
      S->topo = &resident->impl;
      S->device = S->topo->device;
      cudaStream_t ts = thread_stream(S->device);
      ensure_in(S->topo, ts);
    } else {
      UG_CUDA(cudaGetDevice(&S->device));
    }
    prepare_device(S->device);
    UG_CUDA(cudaSetDevice(S->device));
    // every persistent slot CTA must be resident at once (each waits for its
    // own queries only), with room left for other launches
    {
      int per_sm_p = 0, per_sm_h = 0;
      UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_p, lane_k<0>, kSvThreads, 0));
      UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_h, lane_k<1>, kSvThreads, 0));
      const uint64_t cap = (uint64_t)std::min(per_sm_p, per_sm_h) * sm_count(S->device);
      const uint64_t want = (uint64_t)cfg->path_lanes * cfg->path_slots +
                            (uint64_t)cfg->hop_lanes * cfg->hop_slots;
      UG_CHECK(want <= cap / 2, URSA_GPU_EINVAL,
               "server: more shortest-path and hop slots than half the GPU's resident CTAs");
    }
    auto add = [&](LaneKind k, uint32_t lanes, uint32_t slots) {
      for (uint32_t i = 0; i < lanes; i++) {
        S->lanes.emplace_back(new Lane());
        lane_create(S.get(), *S->lanes.back(), k, slots);
      }
    };
    try {
      add(kLanePath, cfg->path_lanes, cfg->path_slots);
      add(kLaneHop, cfg->hop_lanes, cfg->hop_slots);
      add(kLanePr, cfg->pr_lanes, cfg->pr_slots);
      add(kLaneBfs, cfg->bfs_lanes, cfg->bfs_slots);
      if (cfg->bfs_lanes && S->topo->n) {
        const uint64_t bufs = 2ull * cfg->bfs_lanes * cfg->bfs_slots;
        for (uint64_t i = 0; i < bufs; i++) {
          void* p = nullptr;
          UG_CUDA(cudaHostAlloc(&p, S->topo->n * 4, cudaHostAllocDefault));
          S->bfs_bufs.push_back(static_cast<uint32_t*>(p));
        }
        S->bfs_free = S->bfs_bufs;
      }
    } catch (...) {
      for (auto& l : S->lanes) lane_raise_stop(*l);
      for (auto& l : S->lanes) lane_destroy(*l);
      for (uint32_t* p : S->bfs_bufs) cudaFreeHost(p);
      throw;
    }
    ursa_gpu_server* raw = S.release();
    raw->sched = std::thread(sched_loop, raw);
    *out = raw;
  });
}

void ursa_gpu_server_destroy(ursa_gpu_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> g(S->mu);
    for (auto& kv : S->reqs) kv.second->cancel = true;
    S->stop.store(true);
  }
  S->cv_sched.notify_all();
  S->cv_bfs.notify_all();
  if (S->sched.joinable()) S->sched.join();
  for (auto& l : S->lanes)
    if (l->harvester.joinable()) l->harvester.join();
  for (uint32_t* p : S->bfs_bufs) cudaFreeHost(p);
  cudaSetDevice(S->device);
  for (auto& l : S->lanes) lane_raise_stop(*l);
  for (auto& l : S->lanes) lane_destroy(*l);
  for (auto& kv : S->uploads) ursa_gpu_batch_free(kv.second->batch);
  delete S;
}

int ursa_gpu_server_upload(ursa_gpu_server* S, uint64_t n_nodes, const uint32_t* src,
                           const uint32_t* dst, uint64_t n_edges, uint32_t* graph_id) {
  return guard([&] {
    UG_CHECK(S && graph_id, URSA_GPU_EINVAL, "server / graph_id is NULL");
    UG_CHECK(n_nodes <= S->cfg.pr_max_nodes, URSA_GPU_EINVAL,
             "upload: more nodes than the server's pr_max_nodes");
    // admission by free HBM: the estimate covers the build's peak (edge
    // columns, both CSRs, the undirected and oriented CSRs, per-node arrays)
    const uint64_t need = 48ull * n_edges + 96ull * n_nodes + (1ull << 20);
    size_t free_b = 0, total_b = 0;
    UG_CUDA(cudaSetDevice(S->device));
    UG_CUDA(cudaMemGetInfo(&free_b, &total_b));
    free_b += pool_cached_bytes(S->device);  // blocks the pool keeps are free for the build
    {
      std::lock_guard<std::mutex> g(S->mu);
      const bool fits = free_b > S->cfg.hbm_reserve_bytes && free_b - S->cfg.hbm_reserve_bytes >= need &&
                        (S->cfg.upload_budget_bytes == 0 ||
                         S->upload_bytes + need <= S->cfg.upload_budget_bytes);
      if (!fits) {
        S->stats.uploads_rejected++;
        throw Error(URSA_GPU_ENOMEM, "upload: not admitted (free HBM or the upload budget exhausted)");
      }
      S->upload_bytes += need;  // held until the build reports its real size
    }
    uint64_t nc = n_nodes, ec = n_edges;
    ursa_gpu_batch* b = nullptr;
    int st = ursa_gpu_batch_build(1, &nc, &ec, src, dst, &b);
    std::lock_guard<std::mutex> g(S->mu);
    S->upload_bytes -= need;
    if (st != URSA_GPU_OK) throw Error(st, std::string("upload: ") + ursa_gpu_last_error());
    auto up = std::make_shared<Upload>();
    up->id = S->next_upload++;
    up->batch = b;
    up->n = n_nodes;
    up->bytes = ursa_gpu_batch_device_bytes(b);
    S->upload_bytes += up->bytes;
    S->uploads[up->id] = up;
    S->stats.uploads_admitted++;
    *graph_id = up->id;
  });
}

int ursa_gpu_server_release(ursa_gpu_server* S, uint32_t graph_id) {
  return guard([&] {
    UG_CHECK(S, URSA_GPU_EINVAL, "server is NULL");
    std::shared_ptr<Upload> up;
    {
      std::lock_guard<std::mutex> g(S->mu);
      auto it = S->uploads.find(graph_id);
      UG_CHECK(it != S->uploads.end(), URSA_GPU_EINVAL, "release: unknown graph id");
      up = it->second;
      S->uploads.erase(it);
      S->upload_bytes -= up->bytes;
    }
    // queries in flight keep the graph; wait for them
    while (true) {
      {
        std::lock_guard<std::mutex> g(S->mu);
        if (up->refs == 0) break;
      }
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
    ursa_gpu_batch_free(up->batch);
  });
}

int ursa_gpu_server_submit(ursa_gpu_server* S, const ursa_gpu_query* q, uint64_t* ticket) {
  return guard([&] {
    UG_CHECK(S && q && ticket, URSA_GPU_EINVAL, "server / query / ticket is NULL");
    auto r = std::make_shared<Request>();
    r->q = *q;
    int kind = -1;
    std::lock_guard<std::mutex> g(S->mu);
    UG_CHECK(S->fatal.empty(), URSA_GPU_ECUDA, "server stopped: " + S->fatal);
    switch (q->type) {
      case URSA_GPU_QUERY_SHORTEST_PATH:
        UG_CHECK(S->cfg.path_lanes, URSA_GPU_EINVAL, "server has no shortest-path lanes");
        kind = kLanePath;
        break;
      case URSA_GPU_QUERY_HOP:
        UG_CHECK(S->cfg.hop_lanes, URSA_GPU_EINVAL, "server has no hop lanes");
        kind = kLaneHop;
        break;
      case URSA_GPU_QUERY_BFS:
        UG_CHECK(S->cfg.bfs_lanes, URSA_GPU_EINVAL, "server has no bfs lanes");
        UG_CHECK(q->direction <= 2, URSA_GPU_EINVAL, "bfs query: direction must be 0, 1 or 2");
        kind = kLaneBfs;
        break;
      case URSA_GPU_QUERY_PAGERANK: {
        UG_CHECK(S->cfg.pr_lanes, URSA_GPU_EINVAL, "server has no pagerank lanes");
        auto it = S->uploads.find(q->graph);
        UG_CHECK(it != S->uploads.end(), URSA_GPU_EINVAL, "pagerank query: unknown graph id");
        UG_CHECK(q->pr.damping >= 0.0 && q->pr.damping <= 1.0, URSA_GPU_EINVAL,
                 "damping must be in [0, 1]");
        r->up = it->second;
        r->up->refs++;
        kind = kLanePr;
        break;
      }
      default:
        throw Error(URSA_GPU_EINVAL, "unknown query type");
    }
    r->ticket = S->next_ticket++;
    r->info.type = q->type;
    r->info.status = URSA_GPU_OK;
    r->info.submit_us = now_us();
    S->reqs[r->ticket] = r;
    S->pending[kind].push_back(r);
    S->stats.submitted++;
    *ticket = r->ticket;
    S->cv_sched.notify_one();
  });
}

int ursa_gpu_server_cancel(ursa_gpu_server* S, uint64_t ticket) {
  return guard([&] {
    UG_CHECK(S, URSA_GPU_EINVAL, "server is NULL");
    std::lock_guard<std::mutex> g(S->mu);
    auto it = S->reqs.find(ticket);
    UG_CHECK(it != S->reqs.end(), URSA_GPU_EINVAL, "cancel: unknown ticket");
    auto r = it->second;
    if (r->done) return;
    r->cancel = true;
    // not started yet: drop it from its queue and complete it now
    for (auto& pq : S->pending) {
      auto pos = std::find(pq.begin(), pq.end(), r);
      if (pos != pq.end()) {
        pq.erase(pos);
        r->info.status = URSA_GPU_ECANCELED;
        complete(S, r, now_us());
        S->cv_done.notify_all();
        return;
      }
    }
    // in a slot: raise its mapped flag; the CTA reads it between BFS levels
    // (pagerank runs to the end)
    for (auto& lp : S->lanes) {
      Lane& L = *lp;
      for (size_t i = 0; i < L.slot_req.size(); i++)
        if (L.slot_req[i] == r) {
          L.h_stage[i].cancel = 1u;
          UG_CUDA(cudaMemcpyAsync(&L.d_mail.get()[i].cancel, &L.h_stage[i].cancel, 4,
                                  cudaMemcpyHostToDevice, L.copy));
        }
    }
  });
}

int ursa_gpu_server_wait(ursa_gpu_server* S, uint64_t ticket, uint64_t timeout_us,
                         ursa_gpu_query_info* info) {
  return guard([&] {
    UG_CHECK(S, URSA_GPU_EINVAL, "server is NULL");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    UG_CHECK(it != S->reqs.end(), URSA_GPU_EINVAL, "wait: unknown ticket");
    auto r = it->second;
    const auto until = std::chrono::steady_clock::now() + std::chrono::microseconds(timeout_us);
    while (!r->done) {
      if (timeout_us == 0 || S->cv_done.wait_until(lk, until) == std::cv_status::timeout) break;
    }
    if (info) *info = r->info;
    UG_CHECK(r->done, URSA_GPU_ETIMEOUT, "wait: the query has not completed");
  });
}

int ursa_gpu_server_poll(ursa_gpu_server* S, uint64_t* tickets, uint64_t cap, uint64_t* n_out) {
  return guard([&] {
    UG_CHECK(S && n_out && (tickets || cap == 0), URSA_GPU_EINVAL, "poll: NULL argument");
    std::lock_guard<std::mutex> g(S->mu);
    uint64_t k = 0;
    while (k < cap && !S->completed.empty()) {
      tickets[k++] = S->completed.front();
      S->completed.pop_front();
    }
    *n_out = k;
  });
}

int ursa_gpu_server_result(ursa_gpu_server* S, uint64_t ticket, ursa_gpu_query_info* info,
                           void* out, uint64_t cap_elems) {
  return guard([&] {
    UG_CHECK(S, URSA_GPU_EINVAL, "server is NULL");
    std::shared_ptr<Request> r;
    {
      std::lock_guard<std::mutex> g(S->mu);
      auto it = S->reqs.find(ticket);
      UG_CHECK(it != S->reqs.end(), URSA_GPU_EINVAL, "result: unknown ticket");
      r = it->second;
      UG_CHECK(r->done, URSA_GPU_ETIMEOUT, "result: the query has not completed");
      const uint64_t len = r->info.type == URSA_GPU_QUERY_PAGERANK ? r->f64.size()
                           : r->pinned                              ? (uint64_t)r->info.result_len
                                                                    : r->u32.size();
      if (len > cap_elems) throw Error(URSA_GPU_ETRUNC, "result: buffer too small");
      UG_CHECK(len == 0 || out, URSA_GPU_EINVAL, "result: out is NULL");
      S->reqs.erase(it);  // the result is handed over once
    }
    // the copy runs without the server's lock (a bfs answer is n values)
    if (info) *info = r->info;
    if (r->info.type == URSA_GPU_QUERY_PAGERANK) {
      if (!r->f64.empty()) std::memcpy(out, r->f64.data(), r->f64.size() * 8);
    } else if (r->pinned) {
      std::memcpy(out, r->pinned, (size_t)r->info.result_len * 4);
      {
        std::lock_guard<std::mutex> g(S->mu);
        S->bfs_free.push_back(r->pinned);
      }
      r->pinned = nullptr;
      S->cv_bfs.notify_all();
    } else if (!r->u32.empty()) {
      std::memcpy(out, r->u32.data(), r->u32.size() * 4);
    }
  });
}

int ursa_gpu_shortest_path_bidirectional(ursa_gpu_topo* t, uint32_t source, uint32_t target,
                                         uint32_t* path, uint64_t cap, int64_t* len) {
  return guard([&] {
    UG_CHECK(t && len, URSA_GPU_EINVAL, "topology / len is NULL");
    TopoImpl* ti = &t->impl;
    cudaStream_t s = thread_stream(ti->device);
    ensure_in(ti, s);
    const uint64_t n = ti->n, nn = n ? n : 1;
    Scratch<uint64_t> fpar(nn, s), bpar(nn, s);
    Scratch<uint32_t> q0(nn, s), q1(nn, s), q2(nn, s), q3(nn, s), d_path(kPathCap, s), cancel(1, s);
    Scratch<PathOut> d_out(1, s);
    UG_CUDA(cudaMemsetAsync(fpar.get(), 0, nn * 8, s));
    UG_CUDA(cudaMemsetAsync(bpar.get(), 0, nn * 8, s));
    UG_CUDA(cudaMemsetAsync(cancel.get(), 0, 4, s));
    PathSlot ps;
    ps.fpar = fpar.get();
    ps.bpar = bpar.get();
    ps.q[0] = q0.get();
    ps.q[1] = q1.get();
    ps.q[2] = q2.get();
    ps.q[3] = q3.get();
    const PathArgs pa{ti->out.off.get(), ti->out.tgt.get(), ti->in.off.get(), ti->in.tgt.get(), n};
    path_once_k<<<1, kSvThreads, 0, s>>>(pa, PathQuery{source, target, kStampStride}, ps, d_path.get(),
                                         d_out.get(), cancel.get());
    UG_LAUNCH_CHECK();
    PathOut o;
    UG_CUDA(cudaMemcpyAsync(&o, d_out.get(), sizeof(o), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
    *len = o.len;
    UG_CHECK(o.status == URSA_GPU_OK, o.status, "shortest_path_bidirectional: path too long");
    if (o.len > 0) {
      UG_CHECK((uint64_t)o.len <= cap, URSA_GPU_ETRUNC, "shortest_path_bidirectional: path longer than cap");
      UG_CHECK(path, URSA_GPU_EINVAL, "path is NULL");
      UG_CUDA(cudaMemcpyAsync(path, d_path.get(), (size_t)o.len * 4, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
    }
  });
}

int ursa_gpu_server_get_stats(ursa_gpu_server* S, ursa_gpu_server_stats* st) {
  return guard([&] {
    UG_CHECK(S && st, URSA_GPU_EINVAL, "server / stats is NULL");
    std::lock_guard<std::mutex> g(S->mu);
    *st = S->stats;
    st->upload_bytes = S->upload_bytes;
    st->uploads_live = S->uploads.size();
    uint64_t pend = 0;
    for (auto& q : S->pending) pend += q.size();
    st->pending = pend;
  });
}

}  // extern "C"

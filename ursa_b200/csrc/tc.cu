// tc.cu -- triangle_count and clustering_coefficient
// (ursa-core/src/algo/triangle.rs:23-62, clustering.rs:21-40).
//
// The reference counts, for every node u and neighbour a = N(u)[i], the
// common elements of N(u)[i+1..] and N(a): every triangle is counted once at
// each of its three vertices.  Here the vertices are ranked by (undirected
// degree, id) and each undirected edge is oriented from the lower to the
// higher rank, which bounds every oriented list N+ by O(sqrt(m)).  Each
// triangle u < v < w (in rank) is found exactly once, at its middle vertex
// v: w is in N+(v) and in N+(u) for an in-neighbour u of v, and only the
// elements of N+(u) ranked above v can be.  So a warp puts N+(v) in a hash
// table and probes, for each u with u -> v, the elements of N+(u) above v:
// sum over u of C(|N+(u)|, 2) probes (7.2 G at R-MAT-22, against 28.9 G for
// probing every N+(v), v in N+(u), into a table of N+(u)).  A hit credits u
// (one atomic per (u, v) pair), v (one per v) and w (a counter beside w's
// hash slot, flushed once per v).  Integer results are order-independent, so
// the counts are bit-identical to the reference.
#include "frontier.cuh"

namespace ug {

namespace {

__device__ __forceinline__ bool rank_less(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
  return du < dv || (du == dv && u < v);
}

__global__ void orient_flags_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                               uint64_t n, uint64_t ms, uint32_t* __restrict__ flag) {
  if (blockIdx.x == 0 && threadIdx.x == 0) flag[ms] = 0u;
  for_each_slot_owner(off, n, ms, [&](uint64_t k, uint32_t u) {
    uint32_t v = tgt[k];
    uint32_t du = off[u + 1] - off[u], dv = off[v + 1] - off[v];
    flag[k] = rank_less(du, u, dv, v) ? 1u : 0u;
  });
}

__global__ void orient_fill_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                              uint64_t n, uint64_t ms, const uint32_t* __restrict__ pos,
                              uint32_t* __restrict__ o_off, uint32_t* __restrict__ o_tgt) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < ms;
       k += (uint64_t)gridDim.x * blockDim.x) {
    if (pos[k + 1] != pos[k]) o_tgt[pos[k]] = tgt[k];
  }
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u <= n;
       u += (uint64_t)gridDim.x * blockDim.x)
    o_off[u] = pos[off[u]];
}

constexpr uint32_t kTcGrab = 16;
constexpr uint32_t kTcEmpty = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t tc_hash(uint32_t w, uint32_t bits) {
  return (w * 0x9E3779B1u) >> (32 - bits);
}

constexpr uint64_t kTcWork = 16384;  // probes per work item of a warp (one suffix may exceed it)
constexpr uint32_t kTcWarpMax = 256;  // larger N+(v): a block of kTcBlockWarps warps per item
constexpr uint32_t kTcBlockWarps = 8;

// One middle vertex v (original id) at a time: N+(v) = rank ids tgt[ob, oe)
// (all ranked above v, ascending) in a hash table T/C of 2^bits slots (load
// <= 1/2), shared by `threads` consecutive threads starting at `t0` (one warp,
// or a whole block); its in-neighbours' entries i in [ib, ie): u = in_src[i],
// the elements of N+(u) above v are tgt[in_pos[i] + 1, off[u + 1]).
__device__ __forceinline__ void tc_table_fill(uint32_t* T, uint32_t bits, uint32_t ob, uint32_t oe,
                                              const uint32_t* __restrict__ tgt, uint32_t t0,
                                              uint32_t threads) {
  const uint32_t bmask = (1u << (bits - 2)) - 1u;  // buckets of four slots
  for (uint32_t k = ob + t0; k < oe; k += threads) {
    const uint32_t x = tgt[k];
    for (uint32_t b = tc_hash(x, bits - 2);; b = (b + 1) & bmask) {
      uint32_t s = 0;
      while (s < 4 && atomicCAS(&T[4 * b + s], kTcEmpty, x) != kTcEmpty) s++;
      if (s < 4) break;
    }
  }
}

// Slot of w in the table (buckets of four keys, one 16-byte load each), or
// kTcEmpty if absent.
__device__ __forceinline__ uint32_t tc_find(const uint32_t* T, uint32_t bits, uint32_t w) {
  const uint32_t bmask = (1u << (bits - 2)) - 1u;
  for (uint32_t b = tc_hash(w, bits - 2);; b = (b + 1) & bmask) {
    const uint4 q = *reinterpret_cast<const uint4*>(T + 4 * b);
    if (q.x == w) return 4 * b;
    if (q.y == w) return 4 * b + 1;
    if (q.z == w) return 4 * b + 2;
    if (q.w == w) return 4 * b + 3;
    if (q.w == kTcEmpty) return kTcEmpty;  // slots fill in order: a bucket with room ends the chain
  }
}

// Credits the counts kept beside the table to their w and empties it.
__device__ __forceinline__ void tc_table_flush(uint32_t* T, uint32_t* C, uint32_t bits,
                                               const uint32_t* __restrict__ vertex_of,
                                               uint32_t* __restrict__ tri, uint32_t t0,
                                               uint32_t threads) {
  const uint32_t mask = (1u << bits) - 1u;
  for (uint32_t h = t0; h <= mask; h += threads) {
    const uint32_t t = T[h];
    if (t != kTcEmpty) {
      const uint32_t c = C[h];
      if (c) atomicAdd(&tri[vertex_of[t]], c);
      C[h] = 0;
      T[h] = kTcEmpty;
    }
  }
}

// One warp: the entries [i0, i0 + 32) of [.., ie), 32 pairs at a time with
// stride `stride`; credits each u and returns the warp's hit count (all lanes).
__device__ __forceinline__ uint32_t tc_pairs(uint32_t* T, uint32_t* C, uint32_t* P, uint32_t bits,
                                             uint32_t i0, uint32_t ie, uint32_t stride,
                                             const uint32_t* __restrict__ off,
                                             const uint32_t* __restrict__ tgt,
                                             const uint32_t* __restrict__ in_src,
                                             const uint32_t* __restrict__ in_pos,
                                             uint32_t* __restrict__ tri) {
  const uint32_t FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  uint32_t cv = 0;  // per lane; summed at the end
  for (; i0 < ie; i0 += stride) {
    // 32 (u, v) pairs, one per lane: u and the part of N+(u) above v
    uint32_t u = 0, b = 0, len = 0;
    if (i0 + lane < ie) {
      u = in_src[i0 + lane];
      b = in_pos[i0 + lane] + 1;
      len = off[u + 1] - b;
    }
    uint32_t incl = len;  // inclusive scan of the suffix lengths
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += t;
    }
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    const uint32_t start = b - (incl - len);  // element p of pair j is tgt[start_j + p]
    // the suffixes streamed back to back, lane l on element pb + l of pair
    // j (the first pair whose inclusive end exceeds it: a shuffle binary
    // search, since one round can span many short suffixes)
    for (uint32_t pb = 0; pb < total; pb += 32) {
      const uint32_t p = pb + lane;
      uint32_t j = 0;
#pragma unroll
      for (int step = 16; step >= 1; step >>= 1) {
        const uint32_t t = __shfl_sync(FULL, incl, j + step - 1);
        if (t <= p) j += step;
      }
      const uint32_t sj = __shfl_sync(FULL, start, j & 31);
      if (p < total) {
        const uint32_t h = tc_find(T, bits, tgt[sj + p]);
        if (h != kTcEmpty) {
          atomicAdd(&C[h], 1u);
          atomicAdd(&P[j], 1u);
        }
      }
    }
    __syncwarp();
    const uint32_t c = P[lane];
    P[lane] = 0;
    if (c) atomicAdd(&tri[u], c);
    cv += c;
    __syncwarp();
  }
  return __reduce_add_sync(FULL, cv);
}

struct TcArgs {
  const uint32_t* off;        // oriented CSR rows by original id
  const uint32_t* tgt;        // ... targets as rank ids, ascending in each row
  const uint32_t* in_off;     // in-lists of the oriented graph, by rank
  const uint32_t* in_src;     // ... holding original ids
  const uint32_t* in_pos;     // ... and the entry's slot in its row of tgt
  const uint32_t* vertex_of;  // rank -> original id
  const uint32_t* item_rank;   // work items, by rank ascending: middle vertex rank
  const uint32_t* item_begin;  // ... and their in-list entries [begin, end)
  const uint32_t* item_end;
  uint32_t n_items;
  uint32_t* tri;
  unsigned long long* next;   // item grab counter (from the end: hubs first)
  uint32_t lo, hi;            // this launch handles |N+(v)| in (lo, hi]
};

__device__ __forceinline__ bool tc_item(const TcArgs& a, uint32_t q, uint32_t& v, uint32_t& ob,
                                        uint32_t& oe, uint32_t& ib, uint32_t& ie,
                                        uint32_t& bits) {
  const uint32_t r = a.item_rank[q];
  v = a.vertex_of[r];
  ob = a.off[v];
  oe = a.off[v + 1];
  const uint32_t dv = oe - ob;
  if (dv <= a.lo || dv > a.hi) return false;
  ib = a.item_begin[q];
  ie = a.item_end[q];
  bits = 3;  // at least two buckets of four slots
  while ((1u << bits) < 2 * dv) bits++;
  return true;
}

// Items whose middle vertex has lo < |N+(v)| <= hi = kSlots / 2: one warp per
// item, a table per warp in shared memory (kWarps warps per block).
template <int kSlots, int kWarps>
__global__ void __launch_bounds__(kWarps * 32) tc_middle_warp_k(TcArgs a) {
  extern __shared__ uint32_t tc_sm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t* T = tc_sm + (size_t)wid * 2 * kSlots;
  uint32_t* C = T + kSlots;
  uint32_t* P = tc_sm + (size_t)kWarps * 2 * kSlots + wid * 32;
  for (int i = lane; i < kSlots; i += 32) {
    T[i] = kTcEmpty;
    C[i] = 0;
  }
  P[lane] = 0;
  __syncwarp();
  while (true) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(a.next, (unsigned long long)kTcGrab);
    g = __shfl_sync(0xffffffffu, g, 0);
    if (g >= a.n_items) break;
    const uint64_t g_end = g + kTcGrab < a.n_items ? g + kTcGrab : a.n_items;
    for (uint64_t q = g; q < g_end; q++) {
      uint32_t v, ob, oe, ib, ie, bits;
      if (!tc_item(a, (uint32_t)(a.n_items - 1 - q), v, ob, oe, ib, ie, bits)) continue;
      tc_table_fill(T, bits, ob, oe, a.tgt, lane, 32);
      __syncwarp();
      const uint32_t cv = tc_pairs(T, C, P, bits, ib, ie, 32, a.off, a.tgt, a.in_src, a.in_pos, a.tri);
      __syncwarp();
      tc_table_flush(T, C, bits, a.vertex_of, a.tri, lane, 32);
      if (cv && lane == 0) atomicAdd(&a.tri[v], cv);
      __syncwarp();
    }
  }
}

// Items whose middle vertex has |N+(v)| > lo (and <= hi): one block of
// kWarps warps per item sharing one table -- in shared memory of `slots`
// slots when `table` is null, else table[block * 2 * slots, +2 * slots) in
// global memory (keys, then counts; all empty on entry, left empty).
template <int kWarps>
__global__ void __launch_bounds__(kWarps * 32) tc_middle_block_k(TcArgs a, uint32_t* table,
                                                                 uint32_t slots) {
  extern __shared__ uint32_t tc_sm[];
  __shared__ uint32_t pair_cnt[kWarps][32];
  __shared__ unsigned long long s_g;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t* T = table ? table + (size_t)blockIdx.x * 2 * slots : tc_sm;
  uint32_t* C = T + slots;
  uint32_t* P = pair_cnt[wid];
  if (!table)
    for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x) {
      T[i] = kTcEmpty;
      C[i] = 0;
    }
  P[lane] = 0;
  __syncthreads();
  while (true) {
    if (threadIdx.x == 0) s_g = atomicAdd(a.next, 1ull);
    __syncthreads();
    const unsigned long long g = s_g;
    __syncthreads();  // read by all before thread 0 takes the next item
    if (g >= a.n_items) break;
    uint32_t v, ob, oe, ib, ie, bits;
    if (!tc_item(a, (uint32_t)(a.n_items - 1 - g), v, ob, oe, ib, ie, bits)) continue;
    tc_table_fill(T, bits, ob, oe, a.tgt, threadIdx.x, blockDim.x);
    __syncthreads();
    const uint32_t cv = tc_pairs(T, C, P, bits, ib + 32u * wid, ie, 32u * kWarps, a.off, a.tgt,
                                 a.in_src, a.in_pos, a.tri);
    if (cv && lane == 0) atomicAdd(&a.tri[v], cv);
    __syncthreads();
    tc_table_flush(T, C, bits, a.vertex_of, a.tri, threadIdx.x, blockDim.x);
    __syncthreads();
  }
}

// ---- small graphs (the per-graph calls of a batch's plain path): the
// rank relabelling, its two radix sorts and the host reads of the
// middle-vertex path are a fixed cost of about a millisecond, more than the
// whole count takes on a graph of a few tens of thousands of edges.  Below
// kSmallEntries undirected CSR entries one kernel over the (degree, id)
// orientation counts instead: a warp per vertex u puts N+(u) in a
// shared-memory hash set (open addressing, load <= 1/2; longer lists are
// searched by binary search in global memory) and streams the concatenation
// of N+(v), v in N+(u), 32 lists at a time with lane p taking element p (its
// list found by a warp scan of the lengths and a shuffle binary search); a
// hit w is the triangle (u, v, w), credited to w at once and to v and u
// through per-list counters in shared memory.
constexpr uint64_t kSmallEntries = 1u << 18;
constexpr int kSmThreads = 256;
constexpr int kSmWarps = kSmThreads / 32;
constexpr uint32_t kSmSlots = 2048;  // hash slots per warp
constexpr uint32_t kSmHashMax = kSmSlots / 2;

__global__ void __launch_bounds__(kSmThreads) count_small_k(const uint32_t* __restrict__ o_off,
                                                          const uint32_t* __restrict__ o_tgt,
                                                          uint64_t n, uint32_t* __restrict__ tri,
                                                          unsigned long long* __restrict__ next) {
  extern __shared__ uint32_t tc_sm[];
  const uint32_t FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t* T = tc_sm + (size_t)w * kSmSlots;
  uint32_t* cnt = tc_sm + (size_t)kSmWarps * kSmSlots + w * 32;
  for (uint32_t i = lane; i < kSmSlots; i += 32) T[i] = kTcEmpty;
  cnt[lane] = 0;
  __syncwarp();
  while (true) {
    unsigned long long g = 0;
    if (lane == 0) g = atomicAdd(next, (unsigned long long)kTcGrab);
    g = __shfl_sync(FULL, g, 0);
    if (g >= n) break;
    const uint64_t g_end = g + kTcGrab < n ? g + kTcGrab : n;
    for (uint64_t u = g; u < g_end; u++) {
      const uint32_t ob = o_off[u], oe = o_off[u + 1], du = oe - ob;
      if (du < 2) continue;  // u is the lowest vertex of no triangle
      const bool hashed = du <= kSmHashMax;
      uint32_t bits = 6;
      while ((1u << bits) < 2 * du) bits++;
      const uint32_t mask = (1u << bits) - 1;
      if (hashed) {
        for (uint32_t i = ob + lane; i < oe; i += 32) {
          const uint32_t x = o_tgt[i];
          uint32_t h = tc_hash(x, bits);
          while (atomicCAS(&T[h], kTcEmpty, x) != kTcEmpty) h = (h + 1) & mask;
        }
        __syncwarp();
      }
      uint32_t cu = 0;
      for (uint32_t vb = ob; vb < oe; vb += 32) {
        const uint32_t i = vb + lane;
        uint32_t v = 0, st = 0, len = 0;
        if (i < oe) {
          v = o_tgt[i];
          st = o_off[v];
          len = o_off[v + 1] - st;
        }
        uint32_t incl = len;  // inclusive scan of the list lengths
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint32_t t = __shfl_up_sync(FULL, incl, o);
          if (lane >= o) incl += t;
        }
        const uint32_t total = __shfl_sync(FULL, incl, 31);
        for (uint32_t pb = 0; pb < total; pb += 32) {
          const uint32_t p = pb + lane;
          uint32_t j = 0;  // first list whose inclusive end exceeds p
#pragma unroll
          for (int step = 16; step >= 1; step >>= 1) {
            const uint32_t t = __shfl_sync(FULL, incl, j + step - 1);
            if (t <= p) j += step;
          }
          const uint32_t sj = __shfl_sync(FULL, st, j & 31);
          const uint32_t ij = __shfl_sync(FULL, incl, j & 31);
          const uint32_t lj = __shfl_sync(FULL, len, j & 31);
          if (p < total) {
            const uint32_t x = o_tgt[sj + (p - (ij - lj))];
            bool hit = false;
            if (hashed) {
              uint32_t h = tc_hash(x, bits);
              while (true) {
                const uint32_t t = T[h];
                if (t == x) {
                  hit = true;
                  break;
                }
                if (t == kTcEmpty) break;
                h = (h + 1) & mask;
              }
            } else {
              uint32_t lo = ob, hi = oe;
              while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (o_tgt[mid] < x) lo = mid + 1; else hi = mid;
              }
              hit = lo < oe && o_tgt[lo] == x;
            }
            if (hit) {
              atomicAdd(&tri[x], 1u);
              atomicAdd(&cnt[j], 1u);
            }
          }
        }
        __syncwarp();
        const uint32_t c = cnt[lane];
        if (c) {
          atomicAdd(&tri[v], c);
          cu += c;
          cnt[lane] = 0;
        }
        __syncwarp();
      }
      cu = __reduce_add_sync(FULL, cu);
      if (lane == 0 && cu) atomicAdd(&tri[u], cu);
      if (hashed) {
        __syncwarp();
        for (uint32_t k = lane; k <= mask; k += 32) T[k] = kTcEmpty;
        __syncwarp();
      }
    }
  }
}


size_t small_smem_bytes() { return ((size_t)kSmWarps * kSmSlots + kSmWarps * 32) * sizeof(uint32_t); }

// ---- preparation: ranks, the rank-oriented CSR and its in-lists
__global__ void und_degree_k(const uint32_t* __restrict__ off, uint64_t n, uint32_t* __restrict__ deg) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    deg[u] = off[u + 1] - off[u];
}

__global__ void rank_scatter_k(const uint32_t* __restrict__ vertex_of, uint64_t n,
                               uint32_t* __restrict__ rank_of) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (uint64_t)gridDim.x * blockDim.x)
    rank_of[vertex_of[r]] = (uint32_t)r;
}

__global__ void rank_flags_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                             uint64_t n, uint64_t ms, const uint32_t* __restrict__ rank_of,
                             uint32_t* __restrict__ flag) {
  if (blockIdx.x == 0 && threadIdx.x == 0) flag[ms] = 0u;
  for_each_slot_owner(off, n, ms, [&](uint64_t k, uint32_t u) {
    flag[k] = rank_of[u] < rank_of[tgt[k]] ? 1u : 0u;
  });
}

__global__ void rank_fill_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                            uint64_t n, uint64_t ms, const uint32_t* __restrict__ rank_of,
                            const uint32_t* __restrict__ pos, uint32_t* __restrict__ o_off,
                            uint32_t* __restrict__ o_tgt, uint32_t* __restrict__ o_src) {
  for_each_slot_owner(off, n, ms, [&](uint64_t k, uint32_t u) {
    if (pos[k + 1] != pos[k]) {
      o_tgt[pos[k]] = rank_of[tgt[k]];
      o_src[pos[k]] = u;
    }
  });
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u <= n;
       u += (uint64_t)gridDim.x * blockDim.x)
    o_off[u] = pos[off[u]];
}

// in_pos[order[p]] = p: the final slot of each in-list entry in the sorted rows.
__global__ void pos_scatter_k(const uint32_t* __restrict__ order, uint64_t m,
                              uint32_t* __restrict__ in_pos) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < m;
       p += (uint64_t)gridDim.x * blockDim.x)
    in_pos[order[p]] = (uint32_t)p;
}

// Probes of in-list entry i: the elements of N+(u) above v.
__global__ void entry_work_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ in_src,
                             const uint32_t* __restrict__ in_pos, uint64_t m,
                             uint64_t* __restrict__ work) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    work[i] = off[in_src[i] + 1] - in_pos[i] - 1;
}

// Work items per rank: its in-list cut into pieces of about kTcWork probes
// (none when N+(v) is empty or the list has no probes: v is the middle of
// no triangle).  wp = exclusive prefix of the entries' probes.
__global__ void item_count_k(const uint32_t* __restrict__ in_off, const uint32_t* __restrict__ off,
                             const uint32_t* __restrict__ vertex_of,
                             const uint64_t* __restrict__ wp, uint64_t n,
                             uint32_t* __restrict__ cnt) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t v = vertex_of[r];
    const uint32_t dv = off[v + 1] - off[v];
    const uint64_t unit = dv > kTcWarpMax ? kTcWork * kTcBlockWarps : kTcWork;
    const uint64_t tot = wp[in_off[r + 1]] - wp[in_off[r]];
    cnt[r] = dv ? (uint32_t)((tot + unit - 1) / unit) : 0u;
  }
}

// Item k of rank r starts at the first entry whose probes begin at or after
// k * kTcWork (counted from the list's start) and ends where the next begins.
__global__ void item_fill_k(const uint32_t* __restrict__ first, const uint32_t* __restrict__ in_off,
                            const uint32_t* __restrict__ off, const uint32_t* __restrict__ vertex_of,
                            const uint64_t* __restrict__ wp, uint64_t n,
                            uint32_t* __restrict__ item_rank, uint32_t* __restrict__ item_begin,
                            uint32_t* __restrict__ item_end) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t q0 = first[r], q1 = first[r + 1];
    if (q0 == q1) continue;
    const uint32_t lo = in_off[r], hi = in_off[r + 1];
    const uint32_t v = vertex_of[r];
    const uint64_t unit = off[v + 1] - off[v] > kTcWarpMax ? kTcWork * kTcBlockWarps : kTcWork;
    const uint64_t base = wp[lo];
    uint32_t prev = lo;
    for (uint32_t q = q0; q < q1; q++) {
      uint32_t e = hi;
      if (q + 1 < q1) {  // first entry whose probes start at or after the next cut
        const uint64_t cut = base + (uint64_t)(q + 1 - q0) * unit;
        uint32_t a = prev, b = hi;
        while (a < b) {
          const uint32_t mid = (a + b) >> 1;
          if (wp[mid] < cut) a = mid + 1; else b = mid;
        }
        e = a;
      }
      item_rank[q] = (uint32_t)r;
      item_begin[q] = prev;
      item_end[q] = e;
      prev = e;
    }
  }
}

// Global tables, one per block: keys (empty) then counts (zero), slots each.
__global__ void fill_tables_k(uint32_t* __restrict__ table, uint64_t tables, uint32_t slots) {
  const uint64_t total = tables * 2 * slots;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x)
    table[i] = ((i / slots) & 1) ? 0u : kTcEmpty;
}

__global__ void max_outdeg_k(const uint32_t* __restrict__ off, uint64_t n, unsigned* __restrict__ mx) {
  uint32_t best = 0;
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    best = max(best, off[u + 1] - off[u]);
  best = __reduce_max_sync(0xffffffffu, best);
  if ((threadIdx.x & 31) == 0 && best) atomicMax(mx, best);
}

// clustering.rs:21-40: 2 T / (k (k - 1)), 0.0 for k < 2, in f64.
__global__ void clustering_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tri,
                             uint64_t n, double* __restrict__ out) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    double k = (double)(off[u + 1] - off[u]);
    out[u] = k < 2.0 ? 0.0 : __ddiv_rn(__dmul_rn(2.0, (double)tri[u]), __dmul_rn(k, __dsub_rn(k, 1.0)));
  }
}

}  // namespace

// Orientation of the undirected CSR by (degree, id), targets as original ids
// (the batched triangle kernel's input; host-synchronising, done once).
void orient_build(TopoImpl* t, OrientedCsr& o, cudaStream_t s) {
  const uint64_t n = t->n;
  ensure_undirected(t, s);
  const uint64_t ms = t->m_und;
  o.off.alloc(n + 1, s);
  o.mo = 0;
  if (ms == 0) {
    UG_CUDA(cudaMemsetAsync(o.off.get(), 0, (n + 1) * sizeof(uint32_t), s));
    o.tgt.alloc(1, s);
    return;
  }
  Scratch<uint32_t> pos(ms + 1, s);
  orient_flags_k<<<grid_for(ms), kBlock, 0, s>>>(t->und_off.get(), t->und_tgt.get(), n, ms,
                                                 pos.get());
  UG_LAUNCH_CHECK();
  Scratch<uint32_t> total(1, s);
  exclusive_scan_u32(pos.get(), pos.get(), ms + 1, total.get(), s);
  o.mo = read_u32(total.get(), s);
  o.tgt.alloc(o.mo ? o.mo : 1, s);
  orient_fill_k<<<grid_for(ms), kBlock, 0, s>>>(t->und_off.get(), t->und_tgt.get(), n, ms,
                                                pos.get(), o.off.get(), o.tgt.get());
  UG_LAUNCH_CHECK();
}

// Blocks per SM for a kernel and dynamic shared memory size, once per device
// (the shared-memory limit is raised on first use).
template <class K>
static int tc_blocks_per_sm(K kernel, int threads, size_t smem, int dev, int* cache,
                            std::mutex& mu) {
  std::lock_guard<std::mutex> g(mu);
  if (!cache[dev]) {
    UG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cache[dev], kernel, threads, smem));
    UG_CHECK(cache[dev] > 0, URSA_GPU_ECUDA, "triangle kernel cannot be resident");
  }
  return cache[dev];
}

void triangle_count_run(TopoImpl* t, uint32_t* d_tri, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n == 0) return;
  UG_CUDA(cudaMemsetAsync(d_tri, 0, n * sizeof(uint32_t), s));
  ensure_undirected(t, s);
  const uint64_t ms = t->m_und;
  if (ms == 0) return;
  int dev = 0;
  UG_CUDA(cudaGetDevice(&dev));
  UG_CHECK(dev >= 0 && dev < 64, URSA_GPU_EINVAL, "device index out of range");
  if (ms < kSmallEntries) {
    OrientedCsr o;
    orient_build(t, o, s);
    if (o.mo) {
      static std::mutex mu;
      static int cache[64] = {0};
      const int per_sm = tc_blocks_per_sm(count_small_k, kSmThreads, small_smem_bytes(), dev, cache, mu);
      Scratch<unsigned long long> next(1, s);
      UG_CUDA(cudaMemsetAsync(next.get(), 0, sizeof(unsigned long long), s));
      count_small_k<<<per_sm * sm_count(dev), kSmThreads, small_smem_bytes(), s>>>(
          o.off.get(), o.tgt.get(), n, d_tri, next.get());
      UG_LAUNCH_CHECK();
      count_launch();
    }
    UG_CUDA(cudaStreamSynchronize(s));  // o's buffers are released on return
    return;
  }
  // ranks by (undirected degree, id): a stable sort by degree
  Scratch<uint32_t> vertex_of(n, s), rank_of(n, s);
  {
    Scratch<uint32_t> deg(n, s), deg_sorted(n, s);
    und_degree_k<<<grid_for(n), kBlock, 0, s>>>(t->und_off.get(), n, deg.get());
    UG_LAUNCH_CHECK();
    radix_sort_pairs(deg.get(), nullptr, n, bits_for(ms), deg_sorted.get(), vertex_of.get(),
                     nullptr, nullptr, s);
    rank_scatter_k<<<grid_for(n), kBlock, 0, s>>>(vertex_of.get(), n, rank_of.get());
    UG_LAUNCH_CHECK();
  }
  // every undirected edge once, from the lower to the higher rank; targets
  // as rank ids, rows by original id
  Scratch<uint32_t> pos(ms + 1, s);
  rank_flags_k<<<grid_for(ms), kBlock, 0, s>>>(t->und_off.get(), t->und_tgt.get(), n, ms,
                                               rank_of.get(), pos.get());
  UG_LAUNCH_CHECK();
  Scratch<uint32_t> total(1, s);
  exclusive_scan_u32(pos.get(), pos.get(), ms + 1, total.get(), s);
  const uint64_t mo = read_u32(total.get(), s);
  Scratch<uint32_t> o_off(n + 1, s), o_tgt(mo ? mo : 1, s), o_src(mo ? mo : 1, s);
  rank_fill_k<<<grid_for(ms), kBlock, 0, s>>>(t->und_off.get(), t->und_tgt.get(), n, ms,
                                              rank_of.get(), pos.get(), o_off.get(), o_tgt.get(),
                                              o_src.get());
  UG_LAUNCH_CHECK();
  pos.release();
  rank_of.release();
  if (mo == 0) return;
  // in-lists: the oriented edges grouped by target rank (sources in row
  // order), then the rows re-sorted by target rank (a stable sort of the
  // in-list order by source), and each in-list entry's slot in its sorted row
  Scratch<uint32_t> in_off(n + 1, s), in_src(mo, s), in_pos(mo, s);
  {
    Scratch<uint32_t> keys(mo, s);
    radix_sort_pairs(o_tgt.get(), o_src.get(), mo, bits_for(n - 1), keys.get(), in_src.get(),
                     nullptr, nullptr, s);
    offsets_from_sorted(keys.get(), mo, n, in_off.get(), s);
    Scratch<uint32_t> rows(mo, s), order(mo, s);
    radix_sort_pairs(in_src.get(), nullptr, mo, bits_for(n - 1), rows.get(), order.get(),
                     keys.get(), o_tgt.get(), s);
    pos_scatter_k<<<grid_for(mo), kBlock, 0, s>>>(order.get(), mo, in_pos.get());
    UG_LAUNCH_CHECK();
  }
  o_src.release();
  // work items, by rank ascending, of about kTcWork probes each
  Scratch<uint64_t> wp(mo + 1, s);
  entry_work_k<<<grid_for(mo), kBlock, 0, s>>>(o_off.get(), in_src.get(), in_pos.get(), mo,
                                               wp.get());
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaMemsetAsync(wp.get() + mo, 0, sizeof(uint64_t), s));
  exclusive_scan_u64(wp.get(), wp.get(), mo + 1, nullptr, s);
  Scratch<uint32_t> item_first(n + 1, s);
  item_count_k<<<grid_for(n), kBlock, 0, s>>>(in_off.get(), o_off.get(), vertex_of.get(), wp.get(),
                                               n, item_first.get());
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaMemsetAsync(item_first.get() + n, 0, sizeof(uint32_t), s));
  exclusive_scan_u32(item_first.get(), item_first.get(), n + 1, nullptr, s);
  const uint32_t n_items = read_u32(item_first.get() + n, s);
  if (n_items == 0) return;
  Scratch<uint32_t> item_rank(n_items, s), item_begin(n_items, s), item_end(n_items, s);
  item_fill_k<<<grid_for(n), kBlock, 0, s>>>(item_first.get(), in_off.get(), o_off.get(),
                                              vertex_of.get(), wp.get(), n,
                                              item_rank.get(), item_begin.get(), item_end.get());
  UG_LAUNCH_CHECK();
  wp.release();
  uint32_t max_dv = 0;
  {
    Scratch<unsigned> mx(1, s);
    UG_CUDA(cudaMemsetAsync(mx.get(), 0, sizeof(unsigned), s));
    max_outdeg_k<<<grid_for(n), kBlock, 0, s>>>(o_off.get(), n, mx.get());
    UG_LAUNCH_CHECK();
    max_dv = read_u32(mx.get(), s);
  }
  Scratch<unsigned long long> next(1, s);
  TcArgs a;
  a.off = o_off.get();
  a.tgt = o_tgt.get();
  a.in_off = in_off.get();
  a.in_src = in_src.get();
  a.in_pos = in_pos.get();
  a.vertex_of = vertex_of.get();
  a.item_rank = item_rank.get();
  a.item_begin = item_begin.get();
  a.item_end = item_end.get();
  a.n_items = n_items;
  a.tri = d_tri;
  a.next = next.get();
  constexpr int kSmallSlots = 2 * kTcWarpMax, kMidSlots = 2048, kWarpsW = 8, kWarpsB = kTcBlockWarps;
  {  // |N+(v)| <= 256: a warp per item
    static std::mutex mu;
    static int cache[64] = {0};
    const size_t smem = ((size_t)kWarpsW * 2 * kSmallSlots + kWarpsW * 32) * sizeof(uint32_t);
    const int per_sm = tc_blocks_per_sm(tc_middle_warp_k<kSmallSlots, kWarpsW>, kWarpsW * 32, smem,
                                        dev, cache, mu);
    a.lo = 0;
    a.hi = kSmallSlots / 2;
    UG_CUDA(cudaMemsetAsync(a.next, 0, sizeof(unsigned long long), s));
    tc_middle_warp_k<kSmallSlots, kWarpsW><<<per_sm * sm_count(dev), kWarpsW * 32, smem, s>>>(a);
    UG_LAUNCH_CHECK();
    count_launch();
  }
  if (max_dv > (uint32_t)kSmallSlots / 2) {  // up to 1,024: a block per item, table in shared memory
    static std::mutex mu;
    static int cache[64] = {0};
    const size_t smem = (size_t)2 * kMidSlots * sizeof(uint32_t);
    const int per_sm = tc_blocks_per_sm(tc_middle_block_k<kWarpsB>, kWarpsB * 32, smem, dev, cache, mu);
    a.lo = kSmallSlots / 2;
    a.hi = kMidSlots / 2;
    UG_CUDA(cudaMemsetAsync(a.next, 0, sizeof(unsigned long long), s));
    tc_middle_block_k<kWarpsB><<<per_sm * sm_count(dev), kWarpsB * 32, smem, s>>>(a, nullptr, kMidSlots);
    UG_LAUNCH_CHECK();
    count_launch();
  }
  if (max_dv > (uint32_t)kMidSlots / 2) {  // above: a block per item, table in global memory
    uint32_t slots = 1;
    while (slots < 2ull * max_dv) slots <<= 1;
    const unsigned blocks = 2u * (unsigned)sm_count(dev);
    Scratch<uint32_t> table((size_t)blocks * 2 * slots, s);
    // keys empty (all ones), counts zero
    fill_tables_k<<<grid_for((uint64_t)blocks * 2 * slots), kBlock, 0, s>>>(table.get(), blocks,
                                                                              slots);
    UG_LAUNCH_CHECK();
    a.lo = kMidSlots / 2;
    a.hi = 0xFFFFFFFFu;
    UG_CUDA(cudaMemsetAsync(a.next, 0, sizeof(unsigned long long), s));
    tc_middle_block_k<kWarpsB><<<blocks, kWarpsB * 32, 0, s>>>(a, table.get(), slots);
    UG_LAUNCH_CHECK();
    count_launch();
  }
  UG_CUDA(cudaStreamSynchronize(s));  // the scratch above is released on return
}

void clustering_run(TopoImpl* t, double* d_out, cudaStream_t s) {
  const uint64_t n = t->n;
  if (n == 0) return;
  Scratch<uint32_t> tri(n, s);
  triangle_count_run(t, tri.get(), s);
  clustering_k<<<grid_for(n), kBlock, 0, s>>>(t->und_off.get(), tri.get(), n, d_out);
  UG_LAUNCH_CHECK();
}

}  // namespace ug

using namespace ug;

extern "C" {

int ursa_gpu_triangle_count(ursa_gpu_topo* t, uint32_t* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;  // triangle.rs:56-58
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<uint32_t> d(ti->n, s);
    triangle_count_run(ti, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_clustering_coefficient(ursa_gpu_topo* t, double* out) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;  // clustering.rs:23-25
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(ti->device);
    Scratch<double> d(ti->n, s);
    clustering_run(ti, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"

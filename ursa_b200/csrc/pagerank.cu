// pagerank.cu -- pull PageRank (unweighted and weighted) as ONE persistent
// cooperative kernel per call.
//
// Reference semantics (ursa-core/src/algo/pagerank.rs):
//   rank_0 = 1/n; per iteration
//     dangling_mass = sum of rank over dangling nodes           (:78)
//     base = (1-d)/n + d*dangling_mass/n                        (:79)
//     next[u] = base + d * sum_{v in in(u)} rank[v]/outdeg[v]   (:81-83, :113-123)
//               (weighted: w_e * rank[v] / out_strength[v], :159-166)
//     delta = L1(next, rank); swap; stop if delta < tol         (:85-91)
//   returns the last `next`, no renormalisation.
//
// B200 design.
//  * Arithmetic: the per-edge share x[v] = rank[v]/divisor[v] is stored as
//    f32 and each row sums its shares with Kahan-compensated f32 (pieces of a
//    row combined with TwoSum); the update, the L1 residual, the dangling mass
//    and the ranks are f64.  Residual and dangling sums are 128-bit fixed point
//    (fixedpoint.cuh): exact, so the result does not depend on which thread
//    summed which row.
//  * Execution layout (built once per topology, cached).  Nodes are relabelled
//    by in-degree, highest first; on skewed graphs the most-gathered shares
//    then have the smallest ids.  The relabelled source ids are cut into
//    segments of kSegW ids -- one shared-memory slice of shares (192 KB).
//      - Heavy rows (in-degree > kDirect): each row's in-edges are grouped by
//        source segment (stable, in-CSR order inside a segment) and cut into
//        pieces of at most kPiece edges.  The first S segments (chosen per
//        graph: the leading segments whose pieces average >= 5 edges) keep
//        16-bit ids local to their segment; the remaining "far" sources keep
//        32-bit ids.  Within a segment, pieces are sorted by length and packed
//        32 to a chunk in sliced-ELL order: lane l's ids sit in column blocks
//        of V ids, so each lane loads V ids with one vector load and a warp
//        reads 512 (or 128) contiguous bytes per instruction, with no
//        per-edge bounds test (short pieces are padded with an id whose share
//        is zero).
//      - Light rows (1..kDirect in-edges): 32 consecutive rows to a chunk,
//        one lane per row, 32-bit ids in the same order.
//  * One iteration:
//      phase A -- every chunk once.  A CTA owns a contiguous range of the
//        chunk list (split by a cost model); its warps take chunks from a
//        block counter.  Segment chunks gather from the slice in shared
//        memory, which the CTA loads with cp.async.bulk (completion on an
//        mbarrier, bounded wait) when it moves to another segment; far chunks
//        gather from L2; light chunks from the segment-0 slice or L2.  A light
//        row is finished by its lane; a piece writes its partial sum to its
//        slot.
//      grid barrier;
//      phase B -- each heavy row combines its slots in slot order (segment,
//        then piece) and is finished; rows with many slots take a warp.
//      grid barrier whose last block sums the residual and dangling mass.
//    Bounded waits everywhere (grid barriers and mbarrier waits give up after
//    5 s, set an error flag the host turns into URSA_GPU_ETIMEOUT).
#include <algorithm>
#include <cmath>
#include <vector>

#include "fixedpoint.cuh"
#include "primitives.cuh"
#include "topo.cuh"

namespace ug {

namespace {
constexpr int kPrBlock = 1024;
constexpr int kPrWarps = kPrBlock / 32;
constexpr uint32_t kSegW = 49152;    // source ids per shared-memory slice (192 KB of f32 shares)
constexpr uint32_t kSegMax = 16;     // segments considered; ids >= kSegMax*kSegW are far
constexpr uint32_t kBins = kSegMax + 1;
constexpr uint32_t kPiece = 128;     // max edges per piece of a heavy row
static_assert(kPiece <= 128, "kPiece - length (length >= 1) packs into 7 bits of a piece's sort key");
constexpr uint32_t kDirect = 64;     // rows with at most this many in-edges are light
constexpr uint32_t kTile = 1024;     // heavy-row edges per grouping tile (one warp)
constexpr uint32_t kWideSlots = 32;  // heavy rows with more slots are combined by a warp
constexpr int kMaxGroups = kSegMax + 3;
constexpr uint32_t kNoRow = 0xFFFFFFFFu;
constexpr uint32_t kPadEid = 0xFFFFFFFFu;
constexpr uint64_t kWaitLimitNs = 5000000000ull;  // 5 s per bounded wait
// chunk kinds
constexpr int kSeg8 = 0, kSeg2 = 1, kFar4 = 2, kFar1 = 3, kLight4 = 4, kLight1 = 5;
// Static share of the segment chunks per CTA: a chunk costs about one
// dependent index load per two column blocks (plus a fixed part), whatever
// its width (measured: a warp's time per chunk follows its chain of
// dependent loads, not its slot count).
constexpr uint32_t kCostSegBase = 10, kCostSegPerBlock = 4, kCostSegShort = 14;
}  // namespace

struct PrChunk {
  uint32_t base;   // first element in ids16 (segment kinds) or ids32 (others)
  uint16_t nblk;   // column blocks of V ids per lane
  uint8_t kind;
  uint8_t pad;
};

struct PrPlan {
  uint32_t H = 0;       // heavy rows [0, H)
  uint32_t zi_lo = 0;   // rows [zi_lo, n) have no in-edges: rank = base every iteration
  uint32_t iso_lo = 0;  // rows [iso_lo, n) are isolated
  uint32_t S = 0;       // segments with 16-bit ids
  uint32_t n_slots = 0, n_chunks = 0, n_groups = 0, n_wide = 0;
  uint32_t n_seg_chunks = 0;  // chunks [0, n_seg_chunks) are the segment groups
  uint32_t n16 = 0, n32 = 0;  // slots in ids16 / ids32
  bool with_eids = false;     // eid16 / eid32 built (weighted calls need them)
  uint32_t group_begin[kMaxGroups + 1] = {};
  int32_t group_slice[kMaxGroups] = {};
  DevArray<PrChunk> chunks;
  DevArray<uint32_t> chunk_slot;   // per chunk x lane: partial slot (pieces) or row (light)
  DevArray<uint32_t> cost_prefix;  // n_chunks + 1
  DevArray<uint16_t> ids16;
  DevArray<uint32_t> ids32, eid16, eid32;
  DevArray<uint32_t> first_slot;  // H + 1
  DevArray<uint32_t> wide_rows;
  DevArray<uint32_t> old_of_new, new_of_old, outdeg;
};

void pr_plan_free(PrPlan* p) { delete p; }
uint64_t pr_plan_bytes(const PrPlan* p) {
  if (!p) return 0;
  return (uint64_t)p->chunks.n * sizeof(PrChunk) + 2ull * p->ids16.n +
         4ull * (p->chunk_slot.n + p->cost_prefix.n + p->ids32.n + p->eid16.n + p->eid32.n +
                 p->first_slot.n + p->wide_rows.n + p->old_of_new.n + p->new_of_old.n +
                 p->outdeg.n);
}

namespace {

// ------------------------------------------------------------ plan kernels
// Relabel key, ascending = execution order: in-degree high to low; among
// in-degree-0 nodes, sources (out-degree > 0) before isolated nodes, which
// end the order (their ranks follow in closed form).
__global__ void exec_order_key_k(const uint32_t* __restrict__ in_off,
                                 const uint32_t* __restrict__ out_off, uint64_t n,
                                 uint32_t* __restrict__ key) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t din = in_off[u + 1] - in_off[u];
    const uint64_t dout = out_off[u + 1] - out_off[u];
    uint64_t r = din ? 2 * din : (dout ? 1 : 0);
    if (r > 0xFFFFFFFEull) r = 0xFFFFFFFEull;
    key[u] = ~(uint32_t)r;
  }
}

__global__ void relabel_maps_k(const uint32_t* __restrict__ old_of_new, uint64_t n,
                               const uint32_t* __restrict__ in_off,
                               const uint32_t* __restrict__ out_off,
                               uint32_t* __restrict__ new_of_old, uint32_t* __restrict__ deg_new,
                               uint32_t* __restrict__ outdeg_new) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u = old_of_new[i];
    new_of_old[u] = (uint32_t)i;
    deg_new[i] = in_off[u + 1] - in_off[u];
    outdeg_new[i] = out_off[u + 1] - out_off[u];
  }
}

// The in-CSR in the new labels (rows in execution order, sources relabelled).
// Heavy rows: one warp per tile of up to kTile in-edges (tile t of row r
// starts at edge t * kTile of the row), which also counts the tile's edges
// per source bin (bins 0..kSegMax-1 = kSegW-wide slices of the new ids, bin
// kSegMax = ids beyond).  *n_tiles is read on the device (tile_first[H]).
__global__ void relabel_heavy_k(const uint32_t* __restrict__ off_new,
                                const uint32_t* __restrict__ old_of_new,
                                const uint32_t* __restrict__ new_of_old,
                                const uint32_t* __restrict__ in_off,
                                const uint32_t* __restrict__ in_src,
                                const uint32_t* __restrict__ in_eid,
                                const uint32_t* __restrict__ tile_first,
                                const uint32_t* __restrict__ tile_row,
                                const uint32_t* __restrict__ n_tiles,
                                uint32_t* __restrict__ src_new, uint32_t* __restrict__ eid_new,
                                uint32_t* __restrict__ th) {
  __shared__ uint32_t hist[kBlock / 32][kBins];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * (blockDim.x / 32) + w, nw = gridDim.x * (blockDim.x / 32);
  const uint32_t T = *n_tiles;
  for (uint32_t t = gw; t < T; t += nw) {
    const uint32_t r = tile_row[t];
    const uint32_t first = (t - tile_first[r]) * kTile;
    const uint32_t k0 = off_new[r] + first;
    const uint32_t len = min(kTile, off_new[r + 1] - k0);
    const uint32_t s0 = in_off[old_of_new[r]] + first;
    if (lane < (int)kBins) hist[w][lane] = 0;
    __syncwarp();
    for (uint32_t x = lane; x < len; x += 4 * 32) {
      uint32_t v[4];  // four gathers in flight before the stores and counts
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t xq = x + 32u * q;
        v[q] = xq < len ? new_of_old[in_src[s0 + xq]] : 0u;
      }
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const uint32_t xq = x + 32u * q;
        if (xq < len) {
          src_new[k0 + xq] = v[q];
          if (eid_new) eid_new[k0 + xq] = in_eid[s0 + xq];
          atomicAdd(&hist[w][min(v[q] / kSegW, kSegMax)], 1u);
        }
      }
    }
    __syncwarp();
    if (lane < (int)kBins) th[(uint64_t)t * kBins + lane] = hist[w][lane];
    __syncwarp();
  }
}

// Light rows [lo, hi) (at most kDirect in-edges each): one thread per row.
__global__ void relabel_light_k(const uint32_t* __restrict__ off_new,
                                const uint32_t* __restrict__ old_of_new,
                                const uint32_t* __restrict__ new_of_old,
                                const uint32_t* __restrict__ in_off,
                                const uint32_t* __restrict__ in_src,
                                const uint32_t* __restrict__ in_eid, uint32_t lo, uint32_t hi,
                                uint32_t* __restrict__ src_new, uint32_t* __restrict__ eid_new) {
  for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi;
       i += gridDim.x * blockDim.x) {
    const uint32_t k0 = off_new[i], len = off_new[i + 1] - k0;
    const uint32_t s0 = in_off[old_of_new[i]];
#pragma unroll 4
    for (uint32_t x = 0; x < len; x++) {
      src_new[k0 + x] = new_of_old[in_src[s0 + x]];
      if (eid_new) eid_new[k0 + x] = in_eid[s0 + x];
    }
  }
}

// Over the non-increasing in-degree sequence: out[0] = rows with in-degree >
// kDirect (heavy), out[1] = rows with in-edges, out[2] = first isolated row.
__global__ void row_bounds_k(const uint32_t* __restrict__ deg, const uint32_t* __restrict__ outdeg,
                             uint64_t n, uint32_t* __restrict__ out) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (deg[mid] > kDirect) lo = mid + 1; else hi = mid;
  }
  out[0] = (uint32_t)lo;
  lo = 0;
  hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (deg[mid] != 0) lo = mid + 1; else hi = mid;
  }
  out[1] = (uint32_t)lo;
  lo = 0;
  hi = n;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (deg[mid] != 0 || outdeg[mid] != 0) lo = mid + 1; else hi = mid;
  }
  out[2] = (uint32_t)lo;
}

// Heavy rows' in-edges are grouped in tiles of up to kTile consecutive edges,
// one warp per tile, so that a row of 10^5 edges spreads over ~100 warps.
// tile_first[r] = row r's first tile (exclusive scan of these counts).
__global__ void tile_count_k(const uint32_t* __restrict__ off, uint32_t H,
                             uint32_t* __restrict__ tc) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x)
    tc[r] = (off[r + 1] - off[r] + kTile - 1) / kTile;
}

__global__ void tile_row_k(const uint32_t* __restrict__ tile_first, uint32_t H,
                           uint32_t* __restrict__ tile_row) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x)
    for (uint32_t t = tile_first[r]; t < tile_first[r + 1]; t++) tile_row[t] = r;
}

// Per heavy row (one warp, lane b = bin b): its per-bin totals cnt[r][b] and,
// in place, each tile's exclusive per-bin prefix within the row; per bin, the
// edge total and the number of rows with an edge there (for the choice of S).
__global__ void row_scan_k(const uint32_t* __restrict__ tile_first, uint32_t H,
                           uint32_t* __restrict__ th, uint32_t* __restrict__ cnt,
                           unsigned long long* __restrict__ tot) {
  __shared__ unsigned long long s_tot[2 * kBins];
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (int i = threadIdx.x; i < (int)(2 * kBins); i += blockDim.x) s_tot[i] = 0;
  __syncthreads();
  if (lane < (int)kBins) {
    unsigned long long my_edges = 0, my_pairs = 0;
    for (uint32_t r = gw; r < H; r += nw) {
      uint32_t run = 0;
      const uint32_t t1 = tile_first[r + 1];
      for (uint32_t t = tile_first[r]; t < t1; t += 8) {
        uint32_t c[8];  // eight tiles' counts in flight, then the running sum
#pragma unroll
        for (int q = 0; q < 8; q++) c[q] = t + q < t1 ? th[(uint64_t)(t + q) * kBins + lane] : 0u;
#pragma unroll
        for (int q = 0; q < 8; q++) {
          if (t + q < t1) th[(uint64_t)(t + q) * kBins + lane] = run;
          run += c[q];
        }
      }
      cnt[(uint64_t)r * kBins + lane] = run;
      my_edges += run;
      my_pairs += run ? 1 : 0;
    }
    if (my_edges) {  // the block's totals first: few global atomics per address
      atomicAdd(&s_tot[lane], my_edges);
      atomicAdd(&s_tot[kBins + lane], my_pairs);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < (int)(2 * kBins); i += blockDim.x)
    if (s_tot[i]) atomicAdd(&tot[i], s_tot[i]);
}

// Count of heavy row r's edges in merged bin b of S+1 (b == S: far).
__device__ __forceinline__ uint32_t merged_count(const uint32_t* __restrict__ cnt, uint32_t r,
                                                 uint32_t b, uint32_t S) {
  const uint32_t* c = cnt + (uint64_t)r * kBins;
  if (b < S) return c[b];
  uint32_t t = 0;
  for (uint32_t k = S; k < kBins; k++) t += c[k];
  return t;
}

__global__ void piece_count_k(const uint32_t* __restrict__ cnt, uint32_t H, uint32_t S,
                              uint32_t* __restrict__ pc) {
  const uint64_t total = (uint64_t)H * (S + 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(i / (S + 1)), b = (uint32_t)(i % (S + 1));
    pc[i] = (merged_count(cnt, r, b, S) + kPiece - 1) / kPiece;
  }
}

__global__ void first_slot_k(const uint32_t* __restrict__ slot_base, uint32_t H, uint32_t S,
                             const uint32_t* __restrict__ total, uint32_t* __restrict__ first) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r <= H; r += gridDim.x * blockDim.x)
    first[r] = r < H ? slot_base[(uint64_t)r * (S + 1)] : *total;
}

// segpre[r][b] = absolute start of row r's merged bin b (b in [0, S]) in the
// grouped arrays; bins in order, starting at the row's first edge.
__global__ void seg_prefix_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ cnt,
                             uint32_t H, uint32_t S, uint32_t* __restrict__ segpre) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x) {
    uint32_t run = off[r];
    for (uint32_t b = 0; b <= S; b++) {
      segpre[(uint64_t)r * (S + 1) + b] = run;
      run += merged_count(cnt, r, b, S);
    }
  }
}

// Stable grouping of each heavy row's in-edges by merged segment, one warp per
// tile: the tile's edges of bin b go after the row's earlier tiles' edges of
// bin b (th holds those per-tile exclusive prefixes).
__global__ void group_tiles_k(const uint32_t* __restrict__ off, const uint32_t* __restrict__ src,
                              const uint32_t* __restrict__ eid,
                              const uint32_t* __restrict__ tile_first,
                              const uint32_t* __restrict__ tile_row,
                              const uint32_t* __restrict__ n_tiles,
                              const uint32_t* __restrict__ th, const uint32_t* __restrict__ segpre,
                              uint32_t S, uint32_t* __restrict__ gsrc,
                              uint32_t* __restrict__ geid) {
  __shared__ uint32_t cursor[kBlock / 32][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * (blockDim.x / 32) + w, nw = gridDim.x * (blockDim.x / 32);
  const unsigned lt = (1u << lane) - 1u;
  const uint32_t T = *n_tiles;
  for (uint32_t t = gw; t < T; t += nw) {
    const uint32_t r = tile_row[t];
    const uint32_t rb = off[r] + (t - tile_first[r]) * kTile;
    const uint32_t re = min(rb + kTile, off[r + 1]);
    uint32_t c = 0;
    if (lane <= (int)S) {
      const uint32_t* p = th + (uint64_t)t * kBins;
      c = segpre[(uint64_t)r * (S + 1) + lane];
      if (lane < (int)S) {
        c += p[lane];
      } else {
        for (uint32_t b = S; b < kBins; b++) c += p[b];
      }
    }
    cursor[w][lane] = c;
    __syncwarp();
    for (uint32_t e0 = rb; e0 < re; e0 += 32) {
      const uint32_t e = e0 + lane;
      const bool valid = e < re;
      const uint32_t v = valid ? src[e] : 0u;
      const uint32_t b = valid ? min(v / kSegW, S) : 31u;
      const unsigned peers = __match_any_sync(0xffffffffu, b);
      const uint32_t pos = cursor[w][b] + __popc(peers & lt);
      __syncwarp();
      if (valid) {
        gsrc[pos] = v;
        if (geid) geid[pos] = eid[e];
        if (lane == __ffs(peers) - 1) cursor[w][b] += __popc(peers);
      }
      __syncwarp();
    }
  }
}

// One record per piece (slot order = row, bin, piece): sort key (bin, length
// descending) and (row << 5 | bin).
__global__ void piece_keys_k(const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ slot_base,
                             uint32_t H, uint32_t S, uint32_t* __restrict__ key,
                             uint32_t* __restrict__ prs) {
  const uint64_t total = (uint64_t)H * (S + 1);
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(i / (S + 1)), b = (uint32_t)(i % (S + 1));
    const uint32_t c = merged_count(cnt, r, b, S);
    const uint32_t sb = slot_base[i];
    for (uint32_t k = 0, left = c; left > 0; k++) {
      const uint32_t len = left < kPiece ? left : kPiece;
      key[sb + k] = (b << 7) | (kPiece - len);
      prs[sb + k] = (r << 5) | b;
      left -= len;
    }
  }
}

// bounds[b] = first sorted piece of bin b (b in [0, S+1]).
__global__ void bin_bounds_k(const uint32_t* __restrict__ skey, uint32_t n_pieces, uint32_t S,
                             uint32_t* __restrict__ bounds) {
  const uint32_t b = threadIdx.x;
  if (b > S + 1) return;
  uint32_t lo = 0, hi = n_pieces;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if ((skey[mid] >> 7) < b) lo = mid + 1; else hi = mid;
  }
  bounds[b] = lo;
}

struct GroupDesc {
  uint32_t chunk_begin, item_begin, item_end;
  int32_t type;  // 0 segment, 1 far, 2 light
  uint32_t bin;  // segment (type 0)
};

__device__ __forceinline__ int group_of(const GroupDesc* g, int ng, uint32_t c) {
  int k = 0;
  while (k + 1 < ng && c >= g[k + 1].chunk_begin) k++;
  return k;
}

// Chunk shapes: the first item of a chunk is its longest (pieces sorted by
// length, light rows by in-degree, both descending).
__global__ void chunk_shape_k(const GroupDesc* __restrict__ groups, int ng, uint32_t n_chunks,
                              const uint32_t* __restrict__ skey, const uint32_t* __restrict__ deg,
                              PrChunk* __restrict__ chunks, uint32_t* __restrict__ size16,
                              uint32_t* __restrict__ size32, uint32_t* __restrict__ cost) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_chunks;
       c += gridDim.x * blockDim.x) {
    const GroupDesc g = groups[group_of(groups, ng, c)];
    const uint32_t j0 = g.item_begin + 32u * (c - g.chunk_begin);
    const uint32_t len = g.type == 2 ? deg[j0] : kPiece - (skey[j0] & 127u);
    int kind;
    uint32_t V;
    if (g.type == 0) {
      kind = len >= 16 ? kSeg8 : kSeg2;
      V = len >= 16 ? 8 : 2;
    } else if (g.type == 1) {
      kind = len >= 8 ? kFar4 : kFar1;
      V = len >= 8 ? 4 : 1;
    } else {
      kind = len >= 8 ? kLight4 : kLight1;
      V = len >= 8 ? 4 : 1;
    }
    const uint32_t nblk = (len + V - 1) / V;
    const uint32_t size = 32u * nblk * V;
    PrChunk ch;
    ch.base = 0;
    ch.nblk = (uint16_t)nblk;
    ch.kind = (uint8_t)kind;
    ch.pad = 0;
    chunks[c] = ch;
    size16[c] = g.type == 0 ? size : 0u;
    size32[c] = g.type == 0 ? 0u : size;
    // only the segment chunks are split statically; far and light chunks
    // are taken dynamically (their cost entries are 0)
    cost[c] = g.type != 0 ? 0u : (kind == kSeg8 ? kCostSegBase + kCostSegPerBlock * nblk : kCostSegShort);
  }
}

__global__ void chunk_base_k(uint32_t n_chunks, const uint32_t* __restrict__ base16,
                             const uint32_t* __restrict__ base32, PrChunk* __restrict__ chunks) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n_chunks;
       c += gridDim.x * blockDim.x) {
    const int kind = chunks[c].kind;
    chunks[c].base = (kind == kSeg8 || kind == kSeg2) ? base16[c] : base32[c];
  }
}

// Fills the sliced-ELL ids (and original edge ids) of every chunk, one warp
// per chunk; lane l holds item l of the chunk.
__global__ void chunk_fill_k(const GroupDesc* __restrict__ groups, int ng, uint32_t n_chunks,
                             const PrChunk* __restrict__ chunks, const uint32_t* __restrict__ skey,
                             const uint32_t* __restrict__ order, const uint32_t* __restrict__ prs,
                             const uint32_t* __restrict__ slot_base,
                             const uint32_t* __restrict__ segpre, const uint32_t* __restrict__ gsrc,
                             const uint32_t* __restrict__ geid, const uint32_t* __restrict__ off,
                             const uint32_t* __restrict__ src, const uint32_t* __restrict__ eid,
                             const uint32_t* __restrict__ deg, uint32_t S, uint64_t n,
                             uint32_t n_slots, uint16_t* __restrict__ ids16,
                             uint32_t* __restrict__ eid16, uint32_t* __restrict__ ids32,
                             uint32_t* __restrict__ eid32, uint32_t* __restrict__ chunk_slot) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t c = gw; c < n_chunks; c += nw) {
    const GroupDesc g = groups[group_of(groups, ng, c)];
    const PrChunk ch = chunks[c];
    const uint32_t j = g.item_begin + 32u * (c - g.chunk_begin) + (uint32_t)lane;
    const bool valid = j < g.item_end;
    const uint32_t V = ch.kind == kSeg8 ? 8u
                       : ch.kind == kSeg2 ? 2u
                       : (ch.kind == kFar4 || ch.kind == kLight4) ? 4u : 1u;
    uint32_t len = 0, start = 0, sub = 0, slot_or_row = g.type == 2 ? kNoRow : n_slots;
    const uint32_t* ssrc = gsrc;
    const uint32_t* seid = geid;
    if (valid) {
      if (g.type == 2) {
        len = deg[j];
        start = off[j];
        ssrc = src;
        seid = eid;
        slot_or_row = j;
      } else {
        const uint32_t slot = order[j];
        const uint32_t pr = prs[slot];
        const uint32_t r = pr >> 5, b = pr & 31u;
        const uint64_t rb = (uint64_t)r * (S + 1) + b;
        len = kPiece - (skey[j] & 127u);
        start = segpre[rb] + (slot - slot_base[rb]) * kPiece;
        sub = g.type == 0 ? b * kSegW : 0u;
        slot_or_row = slot;
      }
    }
    chunk_slot[(uint64_t)c * 32 + lane] = slot_or_row;
    // a lane's V entries of a column block are contiguous (and V-aligned):
    // gather them, then write them with one or two vector stores
    const uint32_t pad = g.type == 0 ? kSegW : (uint32_t)n;
    const bool with_eids = eid16 != nullptr;  // eid16 and eid32 are given together
    for (uint32_t cb = 0; cb < ch.nblk; cb++) {
      const uint64_t el = (uint64_t)ch.base + ((uint64_t)cb * 32 + lane) * V;
      uint32_t vv[8], ee[8];
#pragma unroll
      for (uint32_t j = 0; j < 8; j++) {
        const uint32_t col = cb * V + j;
        const bool have = j < V && col < len;
        vv[j] = have ? ssrc[start + col] - sub : pad;
        ee[j] = have && with_eids ? seid[start + col] : kPadEid;
      }
      if (V == 8) {  // 16-bit ids
        *reinterpret_cast<uint4*>(ids16 + el) =
            make_uint4(vv[0] | vv[1] << 16, vv[2] | vv[3] << 16, vv[4] | vv[5] << 16,
                       vv[6] | vv[7] << 16);
        if (with_eids) {
          *reinterpret_cast<uint4*>(eid16 + el) = make_uint4(ee[0], ee[1], ee[2], ee[3]);
          *reinterpret_cast<uint4*>(eid16 + el + 4) = make_uint4(ee[4], ee[5], ee[6], ee[7]);
        }
      } else if (g.type == 0) {  // V == 2
        *reinterpret_cast<uint32_t*>(ids16 + el) = vv[0] | vv[1] << 16;
        if (with_eids) *reinterpret_cast<uint2*>(eid16 + el) = make_uint2(ee[0], ee[1]);
      } else if (V == 4) {
        *reinterpret_cast<uint4*>(ids32 + el) = make_uint4(vv[0], vv[1], vv[2], vv[3]);
        if (with_eids) *reinterpret_cast<uint4*>(eid32 + el) = make_uint4(ee[0], ee[1], ee[2], ee[3]);
      } else {
        ids32[el] = vv[0];
        if (with_eids) eid32[el] = ee[0];
      }
    }
  }
}

__global__ void wide_flag_k(const uint32_t* __restrict__ first, uint32_t H,
                            uint32_t* __restrict__ flag) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x)
    flag[r] = first[r + 1] - first[r] > kWideSlots ? 1u : 0u;
}

__global__ void wide_scatter_k(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                               uint32_t H, uint32_t* __restrict__ out) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < H; r += gridDim.x * blockDim.x)
    if (flag[r]) out[pos[r]] = r;
}

// ---------------------------------------------------------- iteration kernel
struct PrArgs {
  uint64_t n;
  uint32_t H, zi_lo, iso_lo;
  uint32_t n_chunks, n_groups, n_wide;
  uint32_t n_seg_chunks;    // [0, n_seg_chunks): segment chunks, split by cost;
                            // [n_seg_chunks, n_chunks): far / light, dealt round-robin
  uint32_t group_begin[kMaxGroups + 1];
  int32_t group_slice[kMaxGroups];
  const PrChunk* __restrict__ chunks;
  const uint32_t* __restrict__ chunk_slot;
  const uint32_t* __restrict__ cost_prefix;
  const uint16_t* __restrict__ ids16;
  const uint32_t* __restrict__ ids32;
  const float* __restrict__ w16;  // weighted: f32 weight per slot, else null
  const float* __restrict__ w32;
  const uint32_t* __restrict__ first_slot;
  const uint32_t* __restrict__ wide_rows;
  F2* partial;
  const uint32_t* __restrict__ outdeg;  // unweighted divisor (new ids)
  const double* __restrict__ out_str;   // weighted divisor (new ids), else null
  double* rank[2];
  float* x[2];
  FxPair* block_part[2];  // per block, fixed point
  double2* totals;        // [2]: (delta, dangling) published by the barrier
  unsigned* bar_count;
  unsigned* bar_gen;
  int* err;
  double damping;
  double tol;
  uint32_t max_iter;
  uint32_t* out_iters;
  double* out_delta;
  uint32_t* out_buf;
};

struct Fin {
  double delta, dang;
};

// Per-thread fixed-point accumulators of |next - rank| and of the dangling
// rows' next ranks: 128-bit integers in units of 2^-96 (fixedpoint.cuh), so
// the sums are exact and order-independent, and each term loses less than
// 2^-96 -- the L1 residual compared with tol is at least as precise as an
// f64 sum of the same terms.
struct Fx {
  u128 delta, dang;
};

struct PrSmem {
  float x[kSegW + 4];  // the loaded slice; [kSegW] is the zero share of padding ids
  FxPair red[kPrWarps];
  unsigned long long mbar;
  unsigned gen;
  int last;
  uint32_t n_sub;
  unsigned ctr[kMaxGroups];
  unsigned dctr;  // the block's position in its share of the far / light chunks
  uint32_t sub_begin[kMaxGroups], sub_end[kMaxGroups];
  int32_t sub_slice[kMaxGroups];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the mbarrier phase `parity`; false after kWaitLimitNs.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  if (mbar_try_wait(mbar, parity)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(mbar, parity))
    if (global_ns() - t0 > kWaitLimitNs) return false;
  return true;
}

// Loads x[seg * kSegW, +kSegW) into the slice with four bulk copies that
// complete on the block's mbarrier; every thread waits for the phase.  Called
// by the whole block after a block barrier.  A wait that runs out sets the
// error flag, then waits once more (bounded) for the copies still in flight.
__device__ __forceinline__ void load_slice(const PrArgs& a, PrSmem& sm, const float* x, int seg,
                                           uint32_t& phase) {
  const uint32_t mbar = smem_u32(&sm.mbar);
  constexpr uint32_t kPart = kSegW * 4 / 4;  // bytes per copy (a multiple of 16)
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar),
                 "r"(kSegW * 4)
                 : "memory");
    const char* src = reinterpret_cast<const char*>(x + (size_t)seg * kSegW);
    const uint32_t dst = smem_u32(sm.x);
#pragma unroll
    for (uint32_t k = 0; k < 4; k++)
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
          ::"r"(dst + k * kPart), "l"(src + (size_t)k * kPart), "r"(kPart), "r"(mbar)
          : "memory");
  }
  if (!mbar_wait(mbar, phase)) {
    atomicExch(a.err, 1);
    mbar_wait(mbar, phase);
  }
  phase ^= 1u;
}

__device__ __forceinline__ double row_divisor(const PrArgs& a, uint64_t u) {
  return a.out_str ? a.out_str[u] : (double)a.outdeg[u];
}

__device__ __forceinline__ void finish_row(const PrArgs& a, uint64_t u, double sum, double old,
                                           double div, double base, int cur, Fx& f) {
  // next[u] = base + d * contrib(u)   (pagerank.rs:81-83)
  double nx = __dadd_rn(base, __dmul_rn(a.damping, sum));
  f.delta += fx_of(fabs(__dsub_rn(nx, old)));
  a.rank[cur ^ 1][u] = nx;
  bool dangling = !(div > 0.0);
  a.x[cur ^ 1][u] = dangling ? 0.f : (float)(nx / div);
  if (dangling) f.dang += fx_of(nx);
}

__device__ __forceinline__ void init_row(const PrArgs& a, uint64_t u, double r0, Fx& f) {
  a.rank[0][u] = r0;
  double div = row_divisor(a, u);
  bool dangling = !(div > 0.0);
  a.x[0][u] = dangling ? 0.f : (float)(r0 / div);
  if (dangling) f.dang += fx_of(r0);
}

__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
  float y = __fsub_rn(v, c);
  float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}

// Share gathers.  far: global; light: the loaded slice when the id falls in
// it (slo = the slice's first id, have = a slice is loaded), else global.
__device__ __forceinline__ float g_far(const float* x, uint32_t v) { return x[v]; }
struct SliceView {
  uint32_t slo;
  bool have;
};
__device__ __forceinline__ float g_light(const PrSmem& sm, SliceView sv, const float* x, uint32_t v) {
  return (sv.have && v - sv.slo < kSegW) ? sm.x[v - sv.slo] : x[v];
}

__device__ __forceinline__ void add8(float& s, float& c, const float (&v)[8], int n) {
#pragma unroll
  for (int k = 0; k < 8; k++)
    if (k < n) kahan_add(s, c, v[k]);
}

// 16-bit local ids, eight per lane per block, gathered from the slice in
// shared memory (padding id kSegW reads the zero slot); two blocks ahead are
// in flight while a block is gathered and summed.
template <bool kW>
__device__ __forceinline__ F2 sum_seg8(const PrArgs& a, const PrSmem& sm, PrChunk ch, int lane) {
  const uint4* p = reinterpret_cast<const uint4*>(a.ids16 + ch.base) + lane;
  const uint4 pad = make_uint4(kSegW | (kSegW << 16), kSegW | (kSegW << 16), kSegW | (kSegW << 16),
                               kSegW | (kSegW << 16));
  const uint32_t nb = ch.nblk;
  float s = 0.f, c = 0.f;
  uint4 q0 = __ldcs(p);
  uint4 q1 = nb > 1 ? __ldcs(p + 32) : pad;
  for (uint32_t b = 0; b < nb; b++) {
    const uint4 q2 = b + 2 < nb ? __ldcs(p + (b + 2) * 32) : pad;
    const uint32_t w4[4] = {q0.x, q0.y, q0.z, q0.w};
    float v[8];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v[2 * k] = sm.x[w4[k] & 0xFFFFu];
      v[2 * k + 1] = sm.x[w4[k] >> 16];
    }
    if (kW) {
      const float4* wp =
          reinterpret_cast<const float4*>(a.w16 + ch.base) + ((size_t)b * 32 + lane) * 2;
      const float4 w0 = __ldcs(wp), w1 = __ldcs(wp + 1);
      v[0] = __fmul_rn(v[0], w0.x);
      v[1] = __fmul_rn(v[1], w0.y);
      v[2] = __fmul_rn(v[2], w0.z);
      v[3] = __fmul_rn(v[3], w0.w);
      v[4] = __fmul_rn(v[4], w1.x);
      v[5] = __fmul_rn(v[5], w1.y);
      v[6] = __fmul_rn(v[6], w1.z);
      v[7] = __fmul_rn(v[7], w1.w);
    }
    add8(s, c, v, 8);
    q0 = q1;
    q1 = q2;
  }
  return F2{s, -c};
}

// 16-bit local ids, two per lane per block, at most 8 blocks: every block's
// ids are loaded at once, then gathered.
template <bool kW>
__device__ __forceinline__ F2 sum_seg2(const PrArgs& a, const PrSmem& sm, PrChunk ch, int lane) {
  const uint32_t* p = reinterpret_cast<const uint32_t*>(a.ids16 + ch.base) + lane;
  const uint32_t nb = ch.nblk;
  uint32_t q[8];
#pragma unroll
  for (int k = 0; k < 8; k++) q[k] = (uint32_t)k < nb ? __ldcs(p + k * 32) : (kSegW | (kSegW << 16));
  float s = 0.f, c = 0.f;
#pragma unroll
  for (int h = 0; h < 2; h++) {  // two halves of four blocks: eight gathers each
    float v[8];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      v[2 * k] = sm.x[q[4 * h + k] & 0xFFFFu];
      v[2 * k + 1] = sm.x[q[4 * h + k] >> 16];
    }
    if (kW) {
      const float2* wp = reinterpret_cast<const float2*>(a.w16 + ch.base) + lane;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const float2 w = (uint32_t)(4 * h + k) < nb ? __ldcs(wp + (4 * h + k) * 32) : make_float2(0.f, 0.f);
        v[2 * k] = __fmul_rn(v[2 * k], w.x);
        v[2 * k + 1] = __fmul_rn(v[2 * k + 1], w.y);
      }
    }
    const int left = (int)nb - 4 * h;
    add8(s, c, v, left <= 0 ? 0 : (left >= 4 ? 8 : 2 * left));
  }
  return F2{s, -c};
}

// 32-bit ids, four per lane per block, two blocks per step (eight gathers in
// flight) while the next two blocks' ids load; kLight uses the loaded slice
// as a cache.
template <bool kW, bool kLight>
__device__ __forceinline__ F2 sum_u32x4(const PrArgs& a, const PrSmem& sm, SliceView sv,
                                        const float* x, PrChunk ch, int lane) {
  const uint4* p = reinterpret_cast<const uint4*>(a.ids32 + ch.base) + lane;
  const uint32_t pad = (uint32_t)a.n;
  const uint4 pq = make_uint4(pad, pad, pad, pad);
  const uint32_t nb = ch.nblk;
  float s = 0.f, c = 0.f;
  uint4 a0 = __ldcs(p);
  uint4 a1 = nb > 1 ? __ldcs(p + 32) : pq;
  for (uint32_t b = 0; b < nb; b += 2) {
    const uint4 n0 = b + 2 < nb ? __ldcs(p + (b + 2) * 32) : pq;
    const uint4 n1 = b + 3 < nb ? __ldcs(p + (b + 3) * 32) : pq;
    const uint32_t id[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
    float v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = kLight ? g_light(sm, sv, x, id[k]) : g_far(x, id[k]);
    if (kW) {
      const float4* wp = reinterpret_cast<const float4*>(a.w32 + ch.base) + (size_t)b * 32 + lane;
      const float4 w0 = __ldcs(wp);
      const float4 w1 = b + 1 < nb ? __ldcs(wp + 32) : make_float4(0.f, 0.f, 0.f, 0.f);
      v[0] = __fmul_rn(v[0], w0.x);
      v[1] = __fmul_rn(v[1], w0.y);
      v[2] = __fmul_rn(v[2], w0.z);
      v[3] = __fmul_rn(v[3], w0.w);
      v[4] = __fmul_rn(v[4], w1.x);
      v[5] = __fmul_rn(v[5], w1.y);
      v[6] = __fmul_rn(v[6], w1.z);
      v[7] = __fmul_rn(v[7], w1.w);
    }
    add8(s, c, v, b + 1 < nb ? 8 : 4);
    a0 = n0;
    a1 = n1;
  }
  return F2{s, -c};
}

// 32-bit ids, one per lane per block, at most 8 blocks: every id is loaded
// at once, then every share gathered.
template <bool kW, bool kLight>
__device__ __forceinline__ F2 sum_u32x1(const PrArgs& a, const PrSmem& sm, SliceView sv,
                                        const float* x, PrChunk ch, int lane) {
  const uint32_t* p = a.ids32 + ch.base + lane;
  const uint32_t nb = ch.nblk;
  uint32_t id[8];
#pragma unroll
  for (int k = 0; k < 8; k++) id[k] = (uint32_t)k < nb ? __ldcs(p + k * 32) : (uint32_t)a.n;
  float v[8];
#pragma unroll
  for (int k = 0; k < 8; k++) v[k] = (uint32_t)k < nb ? (kLight ? g_light(sm, sv, x, id[k]) : g_far(x, id[k])) : 0.f;
  if (kW) {
#pragma unroll
    for (int k = 0; k < 8; k++)
      if ((uint32_t)k < nb) v[k] = __fmul_rn(v[k], __ldcs(a.w32 + ch.base + (size_t)k * 32 + lane));
  }
  float s = 0.f, c = 0.f;
  add8(s, c, v, (int)nb);
  return F2{s, -c};
}

// A chunk's descriptor and this lane's slot (loaded one chunk ahead).
struct ChunkRef {
  PrChunk ch;
  uint32_t slot;
};
__device__ __forceinline__ ChunkRef chunk_ref(const PrArgs& a, uint32_t c, int lane) {
  return ChunkRef{a.chunks[c], __ldg(a.chunk_slot + (size_t)c * 32 + lane)};
}

template <bool kW>
__device__ __forceinline__ void run_chunk(const PrArgs& a, const PrSmem& sm, SliceView sv, ChunkRef cr,
                                          int cur, double base, Fx& f) {
  const int lane = threadIdx.x & 31;
  const PrChunk ch = cr.ch;
  const uint32_t slot = cr.slot;
  const float* x = a.x[cur];
  if (ch.kind == kLight4 || ch.kind == kLight1) {
    double old = 0.0, div = 0.0;
    if (slot != kNoRow) {  // the row was finished last iteration, maybe on another SM
      old = __ldcg(a.rank[cur] + slot);
      div = row_divisor(a, slot);
    }
    const F2 r = ch.kind == kLight4 ? sum_u32x4<kW, true>(a, sm, sv, x, ch, lane)
                                    : sum_u32x1<kW, true>(a, sm, sv, x, ch, lane);
    if (slot != kNoRow) finish_row(a, slot, f2_value(r), old, div, base, cur, f);
    return;
  }
  F2 r;
  switch (ch.kind) {
    case kSeg8: r = sum_seg8<kW>(a, sm, ch, lane); break;
    case kSeg2: r = sum_seg2<kW>(a, sm, ch, lane); break;
    case kFar4: r = sum_u32x4<kW, false>(a, sm, sv, x, ch, lane); break;
    default: r = sum_u32x1<kW, false>(a, sm, sv, x, ch, lane); break;
  }
  a.partial[slot] = r;
}

// Fixed-order reduction over the 32 lanes; valid in lane 0.
__device__ __forceinline__ F2 warp_sum_f2(F2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    F2 t{__shfl_down_sync(0xffffffffu, v.hi, o), __shfl_down_sync(0xffffffffu, v.lo, o)};
    v = f2_combine(v, t);
  }
  return v;
}

// Partial sums written by other blocks in this iteration: read through L2.
__device__ __forceinline__ F2 ldcg_f2(const F2* p) {
  const float2 v = __ldcg(reinterpret_cast<const float2*>(p));
  return F2{v.x, v.y};
}

// Block sum of the fixed-point accumulators; result valid in thread 0.
__device__ __forceinline__ Fx block_sum_fx(Fx v, FxPair* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.delta += shfl_down_u128(v.delta, o);
    v.dang += shfl_down_u128(v.dang, o);
  }
  __syncthreads();
  if (lane == 0) sh[w] = fx_pack(v.delta, v.dang);
  __syncthreads();
  Fx r{0, 0};
  if (threadIdx.x == 0)
    for (int i = 0; i < kPrWarps; i++) {
      r.delta += fx_delta(sh[i]);
      r.dang += fx_dang(sh[i]);
    }
  return r;
}

// Bounded grid barrier whose last-arriving block sums the fixed-point block
// partials of parity p (exact, so the result does not depend on which block
// arrives last), adds `extra` (the closed-form terms of the rows without
// in-edges) and publishes the totals; every block returns them.  A wait
// longer than kWaitLimitNs sets the error flag and returns.
__device__ __forceinline__ Fin barrier_totals(const PrArgs& a, int p, PrSmem& sm, Fin extra) {
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.gen = *(volatile unsigned*)a.bar_gen;
    __threadfence();
    sm.last = atomicAdd(a.bar_count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (sm.last) {
    __threadfence();
    Fx acc{0, 0};
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += kPrBlock) {
      const FxPair v = fx_ldcg(&a.block_part[p][i]);
      acc.delta += fx_delta(v);
      acc.dang += fx_dang(v);
    }
    const Fx r = block_sum_fx(acc, sm.red);
    if (threadIdx.x == 0) {
      a.totals[p] = make_double2(__dadd_rn(fx_value(r.delta), extra.delta),
                                 __dadd_rn(fx_value(r.dang), extra.dang));
      __threadfence();
      atomicExch(a.bar_count, 0u);
      __threadfence();
      atomicAdd(a.bar_gen, 1u);
    }
  } else if (threadIdx.x == 0) {
    const uint64_t t0 = global_ns();
    while (*(volatile unsigned*)a.bar_gen == sm.gen) {
      __nanosleep(32);
      if (global_ns() - t0 > kWaitLimitNs) {
        atomicExch(a.err, 1);
        break;
      }
      if (*(volatile int*)a.err) break;
    }
    __threadfence();
  }
  __syncthreads();
  const double2 t = __ldcg(&a.totals[p]);
  return Fin{t.x, t.y};
}

// Sources without in-edges (rows [zi_lo, iso_lo)): their rank is `rank`
// (closed form, not stored per iteration); only the share they pass on is
// written, and a dangling one (weighted, all out-weights 0) adds its rank to
// the dangling mass.  A coalesced pass over all threads of the grid, four
// rows per thread per step so their divisor loads are in flight together.
__device__ __forceinline__ void sources_without_in_edges(const PrArgs& a, double rank, int buf,
                                                         Fx& f) {
  const uint64_t stride = (uint64_t)gridDim.x * kPrBlock;
  for (uint64_t u0 = a.zi_lo + (uint64_t)blockIdx.x * kPrBlock + threadIdx.x; u0 < a.iso_lo;
       u0 += 4 * stride) {
    double div[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint64_t u = u0 + q * stride;
      div[q] = u < a.iso_lo ? row_divisor(a, u) : 1.0;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint64_t u = u0 + q * stride;
      if (u >= a.iso_lo) break;
      const bool dangling = !(div[q] > 0.0);
      a.x[buf][u] = dangling ? 0.f : (float)(rank / div[q]);
      if (dangling) f.dang += fx_of(rank);
    }
  }
}

// This block's contiguous range of the segment chunks (by the cost prefix),
// cut at group boundaries into sub-ranges, each with the slice it needs.
__device__ __forceinline__ void block_ranges(const PrArgs& a, PrSmem& sm) {
  if (threadIdx.x != 0) return;
  const uint32_t ns = a.n_seg_chunks;  // the statically split part
  const uint64_t total = ns ? a.cost_prefix[ns] : 0;
  auto first_of = [&](uint32_t blk) -> uint32_t {  // first chunk whose start maps to >= blk
    if (total == 0) return ns;
    uint32_t lo = 0, hi = ns;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if ((uint64_t)a.cost_prefix[mid] * gridDim.x / total < blk) lo = mid + 1; else hi = mid;
    }
    return lo;
  };
  const uint32_t lo = first_of(blockIdx.x), hi = first_of(blockIdx.x + 1);
  uint32_t k = 0;
  for (uint32_t g = 0; g < a.n_groups; g++) {
    const uint32_t b = max(lo, a.group_begin[g]), e = min(hi, a.group_begin[g + 1]);
    if (b < e) {
      sm.sub_begin[k] = b;
      sm.sub_end[k] = e;
      sm.sub_slice[k] = a.group_slice[g];
      k++;
    }
  }
  sm.n_sub = k;
}

template <bool kW>
__global__ void __launch_bounds__(kPrBlock, 1) pr_seg_k(PrArgs a) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  PrSmem& sm = *reinterpret_cast<PrSmem*>(smem_raw);
  const double nf = (double)a.n;
  const int lane = threadIdx.x & 31;
  const uint32_t gwarp = blockIdx.x * kPrWarps + (threadIdx.x >> 5);
  const uint32_t nwarps = gridDim.x * kPrWarps;
  const uint64_t gtid = (uint64_t)blockIdx.x * kPrBlock + threadIdx.x;
  const uint64_t nthr = (uint64_t)gridDim.x * kPrBlock;
  if (threadIdx.x < 4) sm.x[kSegW + threadIdx.x] = 0.f;
  if (threadIdx.x == 0)
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sm.mbar)), "r"(1)
                 : "memory");
  block_ranges(a, sm);
  if (threadIdx.x == 0) asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  uint32_t phase = 0;
  // ---- prologue: rank_0 = 1/n, shares, dangling mass of rank_0
  {
    Fx f{0, 0};
    const double r0 = 1.0 / nf;
    for (uint64_t u = gtid; u < a.zi_lo; u += nthr) init_row(a, u, r0, f);
    sources_without_in_edges(a, r0, 0, f);
    const Fx b = block_sum_fx(f, sm.red);
    if (threadIdx.x == 0) a.block_part[0][blockIdx.x] = fx_pack(0, b.dang);
  }
  // rows without in-edges: next = base + d * 0 = base on every iteration
  // (1/n before the first), so their ranks follow in closed form; isolated
  // rows (no out-edges either) are dangling and are never gathered
  const double n_zi = (double)(a.n - a.zi_lo);
  const double n_iso = (double)(a.n - a.iso_lo);
  const double r0 = 1.0 / nf;
  Fin tot = barrier_totals(a, 0, sm, Fin{0.0, n_iso * r0});
  double dm = tot.dang;
  double prev_iso = r0;
  int cur = 0;
  uint32_t iters = 0;
  double delta = 0.0;
  for (uint32_t it = 0; it < a.max_iter; it++) {
    if (*(volatile int*)a.err) break;
    const int parity = (int)((it + 1) & 1u);
    // base = (1-d)/n + d*dangling_mass/n   (pagerank.rs:79)
    const double base = __dadd_rn(__ddiv_rn(1.0 - a.damping, nf),
                                  __ddiv_rn(__dmul_rn(a.damping, dm), nf));
    // ---- phase A, static part: this block's share of the segment chunks
    if (threadIdx.x < kMaxGroups) sm.ctr[threadIdx.x] = 0;
    if (threadIdx.x == 0) sm.dctr = 0;
    __syncthreads();
    Fx f{0, 0};
    int loaded = -1;
    const uint32_t n_sub = sm.n_sub;
    for (uint32_t j = 0; j < n_sub; j++) {
      const int sl = sm.sub_slice[j];
      if (sl >= 0 && sl != loaded) {
        __syncthreads();  // every warp is done with the previous slice
        load_slice(a, sm, a.x[cur], sl, phase);
        loaded = sl;
      }
      const SliceView sv{(uint32_t)(loaded < 0 ? 0 : loaded) * kSegW, loaded >= 0};
      const uint32_t cb = sm.sub_begin[j], ce = sm.sub_end[j];
      // the next chunk's descriptor and slot load while this one is summed
      uint32_t k = 0;
      if (lane == 0) k = atomicAdd(&sm.ctr[j], 1u);
      k = __shfl_sync(0xffffffffu, k, 0) + cb;
      ChunkRef cr{};
      if (k < ce) cr = chunk_ref(a, k, lane);
      while (k < ce) {
        uint32_t kn = 0;
        if (lane == 0) kn = atomicAdd(&sm.ctr[j], 1u);
        kn = __shfl_sync(0xffffffffu, kn, 0) + cb;
        ChunkRef nx{};
        if (kn < ce) nx = chunk_ref(a, kn, lane);
        run_chunk<kW>(a, sm, sv, cr, cur, base, f);
        k = kn;
        cr = nx;
      }
    }
    // ---- phase A, second part: far pieces, then light rows; light gathers
    // use the segment-0 slice (the most-gathered shares) as a cache
    if (loaded != 0 && a.n_chunks > a.n_seg_chunks) {
      __syncthreads();  // every warp is done with the previous slice
      load_slice(a, sm, a.x[cur], 0, phase);
      loaded = 0;
    }
    {
      const SliceView sv{(uint32_t)(loaded < 0 ? 0 : loaded) * kSegW, loaded >= 0};
      // the far and light chunks (sorted largest first) are dealt round-robin
      // to the blocks, which balances them to one chunk, and the warps of a
      // block take the block's share from a shared-memory counter
      const uint32_t nd = a.n_chunks - a.n_seg_chunks, c0 = a.n_seg_chunks;
      const uint32_t mine = blockIdx.x < nd ? (nd - blockIdx.x + gridDim.x - 1) / gridDim.x : 0u;
      uint32_t j = 0;
      if (lane == 0) j = atomicAdd(&sm.dctr, 1u);
      j = __shfl_sync(0xffffffffu, j, 0);
      ChunkRef cr{};
      if (j < mine) cr = chunk_ref(a, c0 + blockIdx.x + j * gridDim.x, lane);
      while (j < mine) {
        uint32_t jn = 0;
        if (lane == 0) jn = atomicAdd(&sm.dctr, 1u);
        jn = __shfl_sync(0xffffffffu, jn, 0);
        ChunkRef nx{};
        if (jn < mine) nx = chunk_ref(a, c0 + blockIdx.x + jn * gridDim.x, lane);
        run_chunk<kW>(a, sm, sv, cr, cur, base, f);
        j = jn;
        cr = nx;
      }
    }
    // Work that does not need the partials runs before the barrier, where a
    // block that finished early would otherwise wait: the sources without
    // in-edges (they write next-iteration shares, which phase A never reads),
    // and the loads of this warp's first phase-B rows (slot ranges, old
    // ranks, divisors; none of them changes during phase A).
    sources_without_in_edges(a, base, cur ^ 1, f);
    const uint32_t wrank = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;  // warps, block-interleaved
    const uint32_t n_rb = (a.H + 31) / 32;
    uint32_t w_r = 0, w_s0 = 0, w_s1 = 0;
    double w_old = 0.0, w_div = 0.0;
    if (wrank < a.n_wide) {
      w_r = a.wide_rows[wrank];
      w_s0 = a.first_slot[w_r];
      w_s1 = a.first_slot[w_r + 1];
      w_old = __ldcg(a.rank[cur] + w_r);
      w_div = row_divisor(a, w_r);
    }
    uint32_t n_s0 = 0, n_s1 = 0;
    double n_old = 0.0, n_div = 0.0;
    {
      const uint32_t r = wrank * 32 + lane;
      if (wrank < n_rb && r < a.H) {
        n_s0 = a.first_slot[r];
        n_s1 = a.first_slot[r + 1];
        n_old = __ldcg(a.rank[cur] + r);
        n_div = row_divisor(a, r);
      }
    }
    grid_barrier(a.bar_count, a.bar_gen, gridDim.x, a.err, kWaitLimitNs);  // partials written
    // ---- phase B: heavy rows combine their slots (slot order) and finish.
    // Rows are sorted by in-degree, heaviest first; consecutive rows go to
    // consecutive blocks so the heavy ones spread over the GPU.
    {
      for (uint32_t i = wrank; i < a.n_wide; i += nwarps) {
        uint32_t r = w_r, s0 = w_s0, s1 = w_s1;
        double old = w_old, div = w_div;
        if (i != wrank) {  // beyond the first (prefetched) one
          r = a.wide_rows[i];
          s0 = a.first_slot[r];
          s1 = a.first_slot[r + 1];
          old = __ldcg(a.rank[cur] + r);
          div = row_divisor(a, r);
        }
        // four independent streams per lane (slots lane + 32 j, j mod 4),
        // combined in a fixed order
        F2 acc[4] = {f2_zero(), f2_zero(), f2_zero(), f2_zero()};
        uint32_t k = s0 + lane;
        for (; k + 96 < s1; k += 128) {
          const F2 p0 = ldcg_f2(a.partial + k), p1 = ldcg_f2(a.partial + k + 32);
          const F2 p2 = ldcg_f2(a.partial + k + 64), p3 = ldcg_f2(a.partial + k + 96);
          acc[0] = f2_combine(acc[0], p0);
          acc[1] = f2_combine(acc[1], p1);
          acc[2] = f2_combine(acc[2], p2);
          acc[3] = f2_combine(acc[3], p3);
        }
        for (int j = 0; k < s1; k += 32, j++) acc[j & 3] = f2_combine(acc[j & 3], ldcg_f2(a.partial + k));
        F2 t = warp_sum_f2(f2_combine(f2_combine(acc[0], acc[1]), f2_combine(acc[2], acc[3])));
        if (lane == 0) finish_row(a, r, f2_value(t), old, div, base, cur, f);
      }
      // the other heavy rows one per lane: a warp takes 32 consecutive rows
      // (adjacent slot ranges: coalesced loads), and consecutive 32-row
      // blocks go to consecutive blocks of the grid
      for (uint32_t rb = wrank; rb < n_rb; rb += nwarps) {
        const uint32_t r = rb * 32 + lane;
        if (r >= a.H) continue;
        uint32_t s0 = n_s0, s1 = n_s1;
        double old = n_old, div = n_div;
        if (rb != wrank) {
          s0 = a.first_slot[r];
          s1 = a.first_slot[r + 1];
          old = __ldcg(a.rank[cur] + r);
          div = row_divisor(a, r);
        }
        if (s1 - s0 > kWideSlots) continue;
        F2 acc = f2_zero();
        uint32_t k = s0;
        for (; k + 8 <= s1; k += 8) {
          F2 p[8];
#pragma unroll
          for (int q = 0; q < 8; q++) p[q] = ldcg_f2(a.partial + k + q);
#pragma unroll
          for (int q = 0; q < 8; q++) acc = f2_combine(acc, p[q]);
        }
        for (; k < s1; k++) acc = f2_combine(acc, ldcg_f2(a.partial + k));
        finish_row(a, r, f2_value(acc), old, div, base, cur, f);
      }
    }
    const Fx b = block_sum_fx(f, sm.red);
    if (threadIdx.x == 0) a.block_part[parity][blockIdx.x] = fx_pack(b.delta, b.dang);
    tot = barrier_totals(a, parity, sm, Fin{n_zi * fabs(base - prev_iso), n_iso * base});
    prev_iso = base;
    delta = tot.delta;
    dm = tot.dang;
    cur ^= 1;
    iters++;
    if (delta < a.tol) break;  // every block sees the same delta
  }
  // rows without in-edges: the last iteration's base (1/n if none ran)
  for (uint64_t u = a.zi_lo + gtid; u < a.n; u += nthr) a.rank[cur][u] = prev_iso;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *a.out_iters = iters;
    *a.out_delta = delta;
    *a.out_buf = (uint32_t)cur;
  }
}

// Weighted helpers: out-strength in out-CSR slot order (pagerank.rs:148-150,
// the same sequential order, so the f64 sums are bit-identical), relabelled,
// and the f32 weight of every execution slot (0 for padding).
__global__ void out_strength_new_k(const uint32_t* __restrict__ off,
                                   const uint32_t* __restrict__ eid, const double* __restrict__ w,
                                   const uint32_t* __restrict__ old_of_new, uint64_t n,
                                   double* __restrict__ out_str) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u = old_of_new[i];
    double s = 0.0;
    for (uint32_t k = off[u]; k < off[u + 1]; k++) s += w[eid[k]];
    out_str[i] = s;
  }
}

__global__ void permute_w_f32_k(const uint32_t* __restrict__ eid, const double* __restrict__ w,
                                uint64_t count, float* __restrict__ out) {
  for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count;
       k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e = eid[k];
    out[k] = e == kPadEid ? 0.f : (float)w[e];
  }
}

__global__ void unpermute_k(const double* __restrict__ rank_new,
                            const uint32_t* __restrict__ new_of_old, uint64_t n,
                            double* __restrict__ out) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x)
    out[u] = rank_new[new_of_old[u]];
}

size_t pr_smem_bytes() { return sizeof(PrSmem); }

template <class T>
T read1(const T* d, cudaStream_t s) {
  T h;
  UG_CUDA(cudaMemcpyAsync(&h, d, sizeof(T), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  return h;
}

}  // namespace

// with_eids: also the original edge id of every sliced-ELL entry (eid16 /
// eid32), which only the weighted variant reads (to lay out its weights).
static PrPlan* build_pr_plan(TopoImpl* t, cudaStream_t s, bool with_eids) {
  const uint64_t n = t->n, m = t->m;
  auto* plan = new PrPlan();
  plan->with_eids = with_eids;
  // ---- relabel by in-degree, highest first (stable: ties keep id order)
  {
    Scratch<uint32_t> key(n, s), key_sorted(n, s);
    exec_order_key_k<<<grid_for(n), kBlock, 0, s>>>(t->in.off.get(), t->out.off.get(), n, key.get());
    UG_LAUNCH_CHECK();
    plan->old_of_new.alloc(n, s);
    radix_sort_pairs(key.get(), nullptr, n, 32, key_sorted.get(), plan->old_of_new.get(), nullptr,
                     nullptr, s);
  }
  plan->new_of_old.alloc(n, s);
  plan->outdeg.alloc(n, s);
  Scratch<uint32_t> deg(n + 1, s), off(n + 1, s);
  relabel_maps_k<<<grid_for(n), kBlock, 0, s>>>(plan->old_of_new.get(), n, t->in.off.get(),
                                                 t->out.off.get(), plan->new_of_old.get(),
                                                 deg.get(), plan->outdeg.get());
  UG_LAUNCH_CHECK();
  UG_CUDA(cudaMemsetAsync(deg.get() + n, 0, sizeof(uint32_t), s));
  exclusive_scan_u32(deg.get(), off.get(), n + 1, nullptr, s);
  // ---- row classes
  uint32_t bnd[3];
  {
    Scratch<uint32_t> d(3, s);
    row_bounds_k<<<1, 1, 0, s>>>(deg.get(), plan->outdeg.get(), n, d.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemcpyAsync(bnd, d.get(), sizeof(bnd), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  }
  const uint32_t H = bnd[0];
  plan->H = H;
  plan->zi_lo = bnd[1];
  plan->iso_lo = bnd[2];
  UG_CHECK(H < (1u << 27), URSA_GPU_EINVAL, "pagerank: too many rows above the light-row degree");
  // ---- the in-CSR in the new labels; heavy rows' per-segment counts and the
  // number of 16-bit segments
  uint32_t S = 0;
  Scratch<uint32_t> cnt((uint64_t)(H ? H : 1) * kBins, s);
  // tiles: at most one per heavy row plus one per kTile edges
  const uint64_t max_tiles = (uint64_t)H + m / kTile + 1;
  Scratch<uint32_t> tile_first((uint64_t)H + 1, s);
  Scratch<uint32_t> tile_row(H ? max_tiles : 1, s), th(H ? max_tiles * kBins : 1, s);
  Scratch<uint32_t> src(m ? m : 1, s), eid;
  if (with_eids) eid.alloc(m ? m : 1, s);
  if (plan->zi_lo > H) {
    relabel_light_k<<<grid_for(plan->zi_lo - H), kBlock, 0, s>>>(
        off.get(), plan->old_of_new.get(), plan->new_of_old.get(), t->in.off.get(),
        t->in.tgt.get(), t->in.eid.get(), H, plan->zi_lo, src.get(),
        with_eids ? eid.get() : nullptr);
    UG_LAUNCH_CHECK();
  }
  if (H) {
    tile_count_k<<<grid_for(H), kBlock, 0, s>>>(off.get(), H, tile_first.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemsetAsync(tile_first.get() + H, 0, sizeof(uint32_t), s));
    exclusive_scan_u32(tile_first.get(), tile_first.get(), (uint64_t)H + 1, nullptr, s);
    tile_row_k<<<grid_for(H), kBlock, 0, s>>>(tile_first.get(), H, tile_row.get());
    UG_LAUNCH_CHECK();
    relabel_heavy_k<<<grid_for(max_tiles * 32), kBlock, 0, s>>>(
        off.get(), plan->old_of_new.get(), plan->new_of_old.get(), t->in.off.get(),
        t->in.tgt.get(), t->in.eid.get(), tile_first.get(), tile_row.get(), tile_first.get() + H,
        src.get(), with_eids ? eid.get() : nullptr, th.get());
    UG_LAUNCH_CHECK();
    Scratch<unsigned long long> tot(2 * kBins, s);
    UG_CUDA(cudaMemsetAsync(tot.get(), 0, 2 * kBins * sizeof(unsigned long long), s));
    row_scan_k<<<grid_for((uint64_t)H * 32), kBlock, 0, s>>>(tile_first.get(), H, th.get(),
                                                             cnt.get(), tot.get());
    UG_LAUNCH_CHECK();
    unsigned long long h[2 * kBins];
    UG_CUDA(cudaMemcpyAsync(h, tot.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
    // a segment pays for its partial sums when its pieces average >= 5 edges
    while (S < kSegMax && (uint64_t)S * kSegW < plan->iso_lo && h[kBins + S] > 0 &&
           h[S] >= 5ull * h[kBins + S])
      S++;
  }
  plan->S = S;
  const uint32_t nb = S + 1;  // merged bins: segments 0..S-1, far
  // ---- pieces and their slots (slot order: row, bin, piece)
  Scratch<uint32_t> slot_base((uint64_t)(H ? H : 1) * nb, s);
  uint32_t n_slots = 0;
  plan->first_slot.alloc((uint64_t)H + 1, s);
  if (H) {
    Scratch<uint32_t> total(1, s);
    piece_count_k<<<grid_for((uint64_t)H * nb), kBlock, 0, s>>>(cnt.get(), H, S, slot_base.get());
    UG_LAUNCH_CHECK();
    exclusive_scan_u32(slot_base.get(), slot_base.get(), (uint64_t)H * nb, total.get(), s);
    first_slot_k<<<grid_for((uint64_t)H + 1), kBlock, 0, s>>>(slot_base.get(), H, S, total.get(),
                                                              plan->first_slot.get());
    UG_LAUNCH_CHECK();
    n_slots = read1(total.get(), s);
  } else {
    UG_CUDA(cudaMemsetAsync(plan->first_slot.get(), 0, sizeof(uint32_t), s));
  }
  plan->n_slots = n_slots;
  // ---- heavy rows' edges grouped by bin; pieces sorted by (bin, length desc)
  const uint64_t m_heavy = H ? (uint64_t)read1(off.get() + H, s) : 0;
  Scratch<uint32_t> segpre((uint64_t)(H ? H : 1) * nb, s);
  Scratch<uint32_t> gsrc(m_heavy ? m_heavy : 1, s), geid;
  if (with_eids) geid.alloc(m_heavy ? m_heavy : 1, s);
  Scratch<uint32_t> skey(n_slots ? n_slots : 1, s), order(n_slots ? n_slots : 1, s);
  Scratch<uint32_t> prs(n_slots ? n_slots : 1, s);
  uint32_t bb[kSegMax + 2] = {0};
  if (H) {
    seg_prefix_k<<<grid_for(H), kBlock, 0, s>>>(off.get(), cnt.get(), H, S, segpre.get());
    UG_LAUNCH_CHECK();
    group_tiles_k<<<grid_for(max_tiles * 32), kBlock, 0, s>>>(
        off.get(), src.get(), eid.get(), tile_first.get(), tile_row.get(), tile_first.get() + H,
        th.get(), segpre.get(), S, gsrc.get(), geid.get());
    UG_LAUNCH_CHECK();
    Scratch<uint32_t> key(n_slots ? n_slots : 1, s);
    piece_keys_k<<<grid_for((uint64_t)H * nb), kBlock, 0, s>>>(cnt.get(), slot_base.get(), H, S,
                                                               key.get(), prs.get());
    UG_LAUNCH_CHECK();
    radix_sort_pairs(key.get(), nullptr, n_slots, bits_for(((uint64_t)S << 7) | 127u), skey.get(),
                     order.get(), nullptr, nullptr, s);
    Scratch<uint32_t> d(kSegMax + 2, s);
    bin_bounds_k<<<1, 32, 0, s>>>(skey.get(), n_slots, S, d.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemcpyAsync(bb, d.get(), (S + 2) * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  }
  // ---- chunk groups, in execution order: segments S-1..1, far, segment 0,
  // light rows (segment 0 and the light rows share the segment-0 slice)
  std::vector<GroupDesc> groups;
  uint32_t n_chunks = 0;
  auto add_group = [&](int type, uint32_t bin, uint32_t ib, uint32_t ie, int slice) {
    GroupDesc g{n_chunks, ib, ie, type, bin};
    plan->group_begin[groups.size()] = n_chunks;
    plan->group_slice[groups.size()] = slice;
    groups.push_back(g);
    n_chunks += (ie - ib + 31) / 32;
  };
  for (uint32_t b = S; b-- > 0;) add_group(0, b, bb[b], bb[b + 1], (int)b);
  plan->n_seg_chunks = n_chunks;  // the rest (far, then light) is taken dynamically
  if (H) add_group(1, S, bb[S], bb[S + 1], -1);
  add_group(2, 0, H, plan->zi_lo, -1);
  plan->n_groups = (uint32_t)groups.size();
  plan->group_begin[groups.size()] = n_chunks;
  plan->n_chunks = n_chunks;
  plan->chunks.alloc(n_chunks ? n_chunks : 1, s);
  plan->chunk_slot.alloc((uint64_t)(n_chunks ? n_chunks : 1) * 32, s);
  plan->cost_prefix.alloc((uint64_t)n_chunks + 1, s);
  if (n_chunks) {
    Scratch<GroupDesc> dg(groups.size(), s);
    UG_CUDA(cudaMemcpyAsync(dg.get(), groups.data(), groups.size() * sizeof(GroupDesc),
                            cudaMemcpyHostToDevice, s));
    Scratch<uint32_t> size16((uint64_t)n_chunks + 1, s), size32((uint64_t)n_chunks + 1, s);
    Scratch<uint32_t> tot16(1, s), tot32(1, s);
    UG_CUDA(cudaMemsetAsync(plan->cost_prefix.get() + n_chunks, 0, sizeof(uint32_t), s));
    chunk_shape_k<<<grid_for(n_chunks), kBlock, 0, s>>>(dg.get(), (int)groups.size(), n_chunks,
                                                        skey.get(), deg.get(), plan->chunks.get(),
                                                        size16.get(), size32.get(),
                                                        plan->cost_prefix.get());
    UG_LAUNCH_CHECK();
    exclusive_scan_u32(size16.get(), size16.get(), n_chunks, tot16.get(), s);
    exclusive_scan_u32(size32.get(), size32.get(), n_chunks, tot32.get(), s);
    exclusive_scan_u32(plan->cost_prefix.get(), plan->cost_prefix.get(), (uint64_t)n_chunks + 1,
                       nullptr, s);
    chunk_base_k<<<grid_for(n_chunks), kBlock, 0, s>>>(n_chunks, size16.get(), size32.get(),
                                                       plan->chunks.get());
    UG_LAUNCH_CHECK();
    const uint32_t n16 = read1(tot16.get(), s), n32 = read1(tot32.get(), s);
    plan->n16 = n16;
    plan->n32 = n32;
    plan->ids16.alloc(n16 ? n16 : 8, s);
    if (with_eids) plan->eid16.alloc(n16 ? n16 : 8, s);
    plan->ids32.alloc(n32 ? n32 : 4, s);
    if (with_eids) plan->eid32.alloc(n32 ? n32 : 4, s);
    chunk_fill_k<<<grid_for((uint64_t)n_chunks * 32), kBlock, 0, s>>>(
        dg.get(), (int)groups.size(), n_chunks, plan->chunks.get(), skey.get(), order.get(),
        prs.get(), slot_base.get(), segpre.get(), gsrc.get(), geid.get(), off.get(), src.get(),
        eid.get(), deg.get(), S, n, n_slots, plan->ids16.get(), plan->eid16.get(),
        plan->ids32.get(), plan->eid32.get(), plan->chunk_slot.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaStreamSynchronize(s));  // dg's host source must outlive the copy
  } else {
    UG_CUDA(cudaMemsetAsync(plan->cost_prefix.get(), 0, sizeof(uint32_t), s));
  }
  // ---- heavy rows combined by a warp in phase B
  plan->wide_rows.alloc(H ? H : 1, s);
  if (H) {
    Scratch<uint32_t> flag(H, s), pos(H, s), tot(1, s);
    wide_flag_k<<<grid_for(H), kBlock, 0, s>>>(plan->first_slot.get(), H, flag.get());
    UG_LAUNCH_CHECK();
    exclusive_scan_u32(flag.get(), pos.get(), H, tot.get(), s);
    wide_scatter_k<<<grid_for(H), kBlock, 0, s>>>(flag.get(), pos.get(), H, plan->wide_rows.get());
    UG_LAUNCH_CHECK();
    plan->n_wide = read1(tot.get(), s);
  }
  UG_CUDA(cudaStreamSynchronize(s));
  return plan;
}

// The plan is cached on the topology; a weighted call on a plan built
// without edge ids replaces it with one that has them (once).
static PrPlan* ensure_pr_plan(TopoImpl* t, cudaStream_t s, bool with_eids) {
  ensure_in(t, s);
  std::lock_guard<std::mutex> g(t->mu);
  if (t->pr_plan && with_eids && !t->pr_plan->with_eids) {
    t->pr_plan_retired = t->pr_plan;  // at most once: plans with ids stay
    t->pr_plan = nullptr;
  }
  if (!t->pr_plan) t->pr_plan = build_pr_plan(t, s, with_eids);
  return t->pr_plan;
}

template <bool kW>
static int pr_grid(int device) {
  static std::mutex mu;
  static int cached[64] = {0};
  std::lock_guard<std::mutex> g(mu);
  if (device < 0 || device >= 64) device = 0;
  if (!cached[device]) {
    const int smem = (int)pr_smem_bytes();
    UG_CUDA(cudaFuncSetAttribute(pr_seg_k<kW>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    int per_sm = 0;
    UG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_seg_k<kW>, kPrBlock, smem));
    UG_CHECK(per_sm > 0, URSA_GPU_ECUDA, "pagerank kernel cannot be resident");
    cached[device] = per_sm * sm_count(device);
  }
  return cached[device];
}

// Runs the iteration; the final ranks (caller's ids) are left in d_out
// (device).  d_weights (device, by edge row) selects the weighted variant.
void pagerank_run(TopoImpl* t, const ursa_gpu_pagerank_params& p, const double* d_weights,
                  double* d_out, cudaStream_t s, ursa_gpu_pagerank_stats* stats) {
  const uint64_t n = t->n;
  if (stats) *stats = ursa_gpu_pagerank_stats{0, 0.0, 0.0};
  if (n == 0) return;
  const bool weighted = d_weights != nullptr;
  PrPlan* plan = ensure_pr_plan(t, s, weighted);
  const int G = weighted ? pr_grid<true>(t->device) : pr_grid<false>(t->device);
  const size_t smem = pr_smem_bytes();

  Scratch<double> rank(2 * n, s);
  // share buffers: every slice [s*kSegW, +kSegW) a CTA may load, and the zero
  // share of padding id n; entries beyond n stay zero
  uint64_t cap = std::max<uint64_t>(n + 1, (uint64_t)std::max<uint32_t>(plan->S, 1u) * kSegW);
  cap = (cap + 3) & ~3ull;
  Scratch<float> x(2 * cap, s);
  Scratch<F2> partial((uint64_t)plan->n_slots + 1, s);
  Scratch<FxPair> block_part(2 * (size_t)G, s);
  Scratch<double2> totals(2, s);
  Scratch<unsigned> ctl(8, s);  // bar_count, bar_gen, err, iters, buf
  Scratch<double> ctl_d(1, s);
  UG_CUDA(cudaMemsetAsync(x.get(), 0, 2 * cap * sizeof(float), s));
  UG_CUDA(cudaMemsetAsync(ctl.get(), 0, 8 * sizeof(unsigned), s));

  Scratch<double> out_str;
  Scratch<float> w16, w32;
  if (weighted) {
    out_str.alloc(n, s);
    out_strength_new_k<<<grid_for(n), kBlock, 0, s>>>(t->out.off.get(), t->out.eid.get(),
                                                       d_weights, plan->old_of_new.get(), n,
                                                       out_str.get());
    UG_LAUNCH_CHECK();
    w16.alloc(plan->n16 ? plan->n16 : 8, s);
    w32.alloc(plan->n32 ? plan->n32 : 4, s);
    if (plan->n16) {
      permute_w_f32_k<<<grid_for(plan->n16), kBlock, 0, s>>>(plan->eid16.get(), d_weights,
                                                              plan->n16, w16.get());
      UG_LAUNCH_CHECK();
    }
    if (plan->n32) {
      permute_w_f32_k<<<grid_for(plan->n32), kBlock, 0, s>>>(plan->eid32.get(), d_weights,
                                                              plan->n32, w32.get());
      UG_LAUNCH_CHECK();
    }
  }

  PrArgs a;
  a.n = n;
  a.H = plan->H;
  a.zi_lo = plan->zi_lo;
  a.iso_lo = plan->iso_lo;
  a.n_chunks = plan->n_chunks;
  a.n_groups = plan->n_groups;
  a.n_seg_chunks = plan->n_seg_chunks;
  a.n_wide = plan->n_wide;
  for (int g = 0; g <= kMaxGroups; g++) a.group_begin[g] = plan->group_begin[g];
  for (int g = 0; g < kMaxGroups; g++) a.group_slice[g] = plan->group_slice[g];
  a.chunks = plan->chunks.get();
  a.chunk_slot = plan->chunk_slot.get();
  a.cost_prefix = plan->cost_prefix.get();
  a.ids16 = plan->ids16.get();
  a.ids32 = plan->ids32.get();
  a.w16 = weighted ? w16.get() : nullptr;
  a.w32 = weighted ? w32.get() : nullptr;
  a.first_slot = plan->first_slot.get();
  a.wide_rows = plan->wide_rows.get();
  a.partial = partial.get();
  a.outdeg = plan->outdeg.get();
  a.out_str = weighted ? out_str.get() : nullptr;
  a.rank[0] = rank.get();
  a.rank[1] = rank.get() + n;
  a.x[0] = x.get();
  a.x[1] = x.get() + cap;
  a.block_part[0] = block_part.get();
  a.block_part[1] = block_part.get() + G;
  a.totals = totals.get();
  a.bar_count = ctl.get() + 0;
  a.bar_gen = ctl.get() + 1;
  a.err = (int*)(ctl.get() + 2);
  a.out_iters = ctl.get() + 3;
  a.out_buf = ctl.get() + 4;
  a.out_delta = ctl_d.get();
  a.damping = p.damping;
  a.tol = p.tol;
  a.max_iter = p.max_iter;

  cudaEvent_t e0, e1;
  UG_CUDA(cudaEventCreate(&e0));
  UG_CUDA(cudaEventCreate(&e1));
  UG_CUDA(cudaEventRecord(e0, s));
  void* args[] = {&a};
  void* fn = weighted ? (void*)pr_seg_k<true> : (void*)pr_seg_k<false>;
  UG_CUDA(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(kPrBlock), args, smem, s));
  count_launch();
  UG_CUDA(cudaEventRecord(e1, s));
  unsigned h[8];
  double hd;
  UG_CUDA(cudaMemcpyAsync(h, ctl.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaMemcpyAsync(&hd, ctl_d.get(), sizeof(double), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  UG_CHECK(h[2] == 0, URSA_GPU_ETIMEOUT, "pagerank: a bounded wait in the kernel expired");
  const uint32_t buf = p.max_iter == 0 ? 0u : h[4];
  unpermute_k<<<grid_for(n), kBlock, 0, s>>>(rank.get() + (size_t)buf * n, plan->new_of_old.get(),
                                             n, d_out);
  UG_LAUNCH_CHECK();
  if (stats) {
    stats->iterations = h[3];
    stats->last_delta = hd;
    stats->device_ms = ms;
  }
}

}  // namespace ug

// primitives.cu -- reduce-then-scan prefix sums and a stable LSD radix sort.
//
// The radix sort is the core of the byte-exact CSR build: a stable sort of
// edge rows by their grouping endpoint reproduces ursa-core's counting sort
// exactly (rows keep their original order inside each node's segment,
// ursa-core/src/topology.rs:109-114).  Each 8-bit pass is
//   upsweep:   per-tile digit histograms, written digit-major,
//   scan:      one exclusive scan over the digit-major histogram,
//   downsweep: per-tile stable ranking (warp match_any + per-warp digit
//              counters, warps own contiguous sub-tiles) and scatter.
#include "primitives.cuh"

namespace ug {

namespace {

constexpr int kScanTile = 2048;  // 256 threads x 8 items
constexpr int kRadixItems = 16;  // per thread
constexpr int kRadixTile = kBlock * kRadixItems;  // 4096
constexpr int kWarps = kBlock / 32;

__device__ __forceinline__ int pad(int i) { return i + (i >> 5); }

template <class T>
__device__ T block_exclusive_scan(T v, T* block_total) {
  __shared__ T warp_tot[kWarps];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    T t = lane < kWarps ? warp_tot[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < kWarps) warp_tot[lane] = t;  // inclusive
  }
  __syncthreads();
  T warp_excl = w ? warp_tot[w - 1] : T(0);
  if (block_total) *block_total = warp_tot[kWarps - 1];
  __syncthreads();
  return warp_excl + x - v;
}

template <class T>
__global__ void scan_reduce_k(const T* __restrict__ in, uint64_t n, T* __restrict__ sums) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  T acc = 0;
  for (int i = threadIdx.x; i < kScanTile; i += kBlock) {
    uint64_t idx = base + i;
    if (idx < n) acc += in[idx];
  }
  T tot;
  block_exclusive_scan<T>(acc, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class T>
__global__ void scan_tile_k(const T* in, T* out, uint64_t n, const T* __restrict__ block_offsets,
                            T* total) {
  __shared__ T s[kScanTile + kScanTile / 32];
  uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  for (int i = threadIdx.x; i < kScanTile; i += kBlock) {
    uint64_t idx = base + i;
    s[pad(i)] = idx < n ? in[idx] : T(0);
  }
  __syncthreads();
  T v[8];
  T tsum = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) {
    v[j] = s[pad(threadIdx.x * 8 + j)];
    tsum += v[j];
  }
  T btot;
  T run = block_exclusive_scan<T>(tsum, &btot);
  if (block_offsets) run += block_offsets[blockIdx.x];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    s[pad(threadIdx.x * 8 + j)] = run;
    run += v[j];
  }
  if (total && threadIdx.x == 0) *total = (block_offsets ? block_offsets[blockIdx.x] : T(0)) + btot;
  __syncthreads();
  for (int i = threadIdx.x; i < kScanTile; i += kBlock) {
    uint64_t idx = base + i;
    if (idx < n) out[idx] = s[pad(i)];
  }
}

template <class T>
void scan_impl(const T* in, T* out, uint64_t n, T* total, cudaStream_t s) {
  if (n == 0) {
    if (total) UG_CUDA(cudaMemsetAsync(total, 0, sizeof(T), s));
    return;
  }
  uint64_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 1) {
    scan_tile_k<T><<<1, kBlock, 0, s>>>(in, out, n, nullptr, total);
    UG_LAUNCH_CHECK();
    return;
  }
  Scratch<T> sums(nb, s);
  scan_reduce_k<T><<<(unsigned)nb, kBlock, 0, s>>>(in, n, sums.get());
  UG_LAUNCH_CHECK();
  // The last block's total must include its own offset, so the recursive call
  // produces both the block offsets and the grand total.
  scan_impl<T>(sums.get(), sums.get(), nb, total, s);
  scan_tile_k<T><<<(unsigned)nb, kBlock, 0, s>>>(in, out, n, sums.get(), nullptr);
  UG_LAUNCH_CHECK();
}

// ---------------------------------------------------------------- radix sort
// bad != nullptr: every key >= limit sets *bad (the caller's range check,
// folded into the pass that reads the keys anyway).
__global__ void __launch_bounds__(kBlock) radix_upsweep_k(const uint32_t* __restrict__ keys,
                                                          uint64_t n, int shift, uint32_t mask,
                                                          uint32_t* __restrict__ hist,
                                                          uint32_t num_tiles,
                                                          unsigned* __restrict__ bad,
                                                          uint64_t limit) {
  __shared__ uint32_t cnt[kWarps][256];
  for (int i = threadIdx.x; i < kWarps * 256; i += kBlock) (&cnt[0][0])[i] = 0;
  __syncthreads();
  uint32_t tile = blockIdx.x;
  uint64_t base = (uint64_t)tile * kRadixTile;
  int w = threadIdx.x >> 5;
  uint32_t k[kRadixItems];
#pragma unroll
  for (int i = 0; i < kRadixItems; i++) {
    const uint64_t idx = base + (uint64_t)i * kBlock + threadIdx.x;
    k[i] = idx < n ? __ldg(&keys[idx]) : 0u;
  }
  bool out_of_range = false;
#pragma unroll
  for (int i = 0; i < kRadixItems; i++) {
    const uint64_t idx = base + (uint64_t)i * kBlock + threadIdx.x;
    if (idx < n) {
      atomicAdd(&cnt[w][(k[i] >> shift) & mask], 1u);
      out_of_range |= (uint64_t)k[i] >= limit;
    }
  }
  if (bad && __any_sync(0xffffffffu, out_of_range) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += kBlock) {
    uint32_t s = 0;
#pragma unroll
    for (int ww = 0; ww < kWarps; ww++) s += cnt[ww][d];
    hist[(uint64_t)d * num_tiles + tile] = s;
  }
}

__global__ void __launch_bounds__(kBlock) radix_downsweep_k(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint64_t n,
    int shift, uint32_t mask, const uint32_t* __restrict__ hist_scanned, uint32_t num_tiles,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
    const uint32_t* __restrict__ gather_src, uint32_t* __restrict__ gather_out) {
  __shared__ uint32_t wcnt[kWarps][256];
  __shared__ uint32_t gofs[256];
  uint32_t tile = blockIdx.x;
  for (int i = threadIdx.x; i < kWarps * 256; i += kBlock) (&wcnt[0][0])[i] = 0;
  for (int d = threadIdx.x; d < 256; d += kBlock) gofs[d] = hist_scanned[(uint64_t)d * num_tiles + tile];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  // Warp w owns the contiguous sub-tile [w*512, (w+1)*512); round i covers
  // items w*512 + i*32 + lane, so (round, lane) order is input order.
  const uint64_t wbase = (uint64_t)tile * kRadixTile + (uint64_t)w * (32 * kRadixItems);
  uint32_t k[kRadixItems], v[kRadixItems], dr[kRadixItems];
  // all of the warp's loads in flight before the first ranking step
#pragma unroll
  for (int i = 0; i < kRadixItems; i++) {
    const uint64_t idx = wbase + (uint64_t)i * 32 + lane;
    const bool valid = idx < n;
    k[i] = valid ? __ldg(&keys_in[idx]) : 0u;
    v[i] = valid ? (vals_in ? __ldg(&vals_in[idx]) : (uint32_t)idx) : 0u;
  }
#pragma unroll
  for (int i = 0; i < kRadixItems; i++) {
    uint64_t idx = wbase + (uint64_t)i * 32 + lane;
    bool valid = idx < n;
    uint32_t key = k[i];
    uint32_t d = valid ? ((key >> shift) & mask) : 256u;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t rank_in = __popc(peers & lt);
    uint32_t before = d < 256u ? wcnt[w][d] : 0u;
    __syncwarp();
    if (d < 256u && rank_in == 0) wcnt[w][d] = before + __popc(peers);
    __syncwarp();
    dr[i] = (d << 16) | (before + rank_in);
  }
  __syncthreads();
  // Per digit: each warp's exclusive start, and the tile's digit total.
  static_assert(kBlock == 256, "one thread per digit");
  uint32_t run = 0;
  {
    const int d = threadIdx.x;
#pragma unroll
    for (int ww = 0; ww < kWarps; ww++) {
      uint32_t x = wcnt[ww][d];
      wcnt[ww][d] = run;
      run += x;
    }
  }
  // Tile-local digit starts, so the tile can be ordered in shared memory and
  // written out in coalesced runs (one run per digit).
  __shared__ uint32_t toff[256];
  __shared__ uint32_t sk[kRadixTile];
  __shared__ uint32_t sv[kRadixTile];
  toff[threadIdx.x] = block_exclusive_scan<uint32_t>(run, nullptr);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kRadixItems; i++) {
    uint32_t d = dr[i] >> 16;
    if (d < 256u) {
      uint32_t p = toff[d] + wcnt[w][d] + (dr[i] & 0xffffu);
      sk[p] = k[i];
      sv[p] = v[i];
    }
  }
  __syncthreads();
  const uint64_t tile0 = (uint64_t)tile * kRadixTile;
  const uint32_t tile_n = (uint32_t)(n - tile0 < (uint64_t)kRadixTile ? n - tile0 : kRadixTile);
  for (uint32_t i = threadIdx.x; i < tile_n; i += kBlock) {
    const uint32_t key = sk[i], val = sv[i];
    const uint32_t d = (key >> shift) & mask;
    const uint32_t dest = gofs[d] + (i - toff[d]);
    keys_out[dest] = key;
    vals_out[dest] = val;
    if (gather_src) gather_out[dest] = gather_src[val];
  }
}

__global__ void offsets_k(const uint32_t* __restrict__ keys, uint64_t m, uint64_t n,
                          uint32_t* __restrict__ off) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u <= n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t lo = 0, hi = m;
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if ((uint64_t)keys[mid] < u)
        lo = mid + 1;
      else
        hi = mid;
    }
    off[u] = (uint32_t)lo;
  }
}

}  // namespace

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total,
                        cudaStream_t s) {
  scan_impl<uint32_t>(in, out, n, total, s);
}
void exclusive_scan_u64(const uint64_t* in, uint64_t* out, uint64_t n, uint64_t* total,
                        cudaStream_t s) {
  scan_impl<uint64_t>(in, out, n, total, s);
}

void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint64_t n, int key_bits,
                      uint32_t* keys_out, uint32_t* vals_out, const uint32_t* gather_src,
                      uint32_t* gather_out, cudaStream_t s, cudaEvent_t gather_ready,
                      unsigned* bad, uint64_t limit) {
  UG_CHECK(n < (1ull << 32), URSA_GPU_EINVAL, "radix sort: more than 2^32-1 items");
  if (n == 0) return;
  int passes = key_bits <= 8 ? 1 : (key_bits + 7) / 8;
  uint32_t num_tiles = (uint32_t)((n + kRadixTile - 1) / kRadixTile);
  Scratch<uint32_t> hist((size_t)256 * num_tiles, s);
  Scratch<uint32_t> kb[2], vb[2];
  if (passes > 1) {
    kb[0].alloc(n, s);
    vb[0].alloc(n, s);
    if (passes > 2) {
      kb[1].alloc(n, s);
      vb[1].alloc(n, s);
    }
  }
  const uint32_t* kin = keys_in;
  const uint32_t* vin = vals_in;
  for (int p = 0; p < passes; p++) {
    int shift = 8 * p;
    int bits = key_bits - shift;
    if (bits > 8) bits = 8;
    if (bits < 0) bits = 0;
    uint32_t mask = bits == 0 ? 0u : ((1u << bits) - 1u);
    bool last = p == passes - 1;
    uint32_t* kout = last ? keys_out : kb[p & 1].get();
    uint32_t* vout = last ? vals_out : vb[p & 1].get();
    radix_upsweep_k<<<num_tiles, kBlock, 0, s>>>(kin, n, shift, mask, hist.get(), num_tiles,
                                                 p == 0 ? bad : nullptr, limit);
    UG_LAUNCH_CHECK();
    exclusive_scan_u32(hist.get(), hist.get(), (uint64_t)256 * num_tiles, nullptr, s);
    if (last && gather_ready) UG_CUDA(cudaStreamWaitEvent(s, gather_ready, 0));
    radix_downsweep_k<<<num_tiles, kBlock, 0, s>>>(kin, vin, n, shift, mask, hist.get(), num_tiles,
                                                   kout, vout, last ? gather_src : nullptr,
                                                   gather_out);
    UG_LAUNCH_CHECK();
    kin = kout;
    vin = vout;
  }
}

void offsets_from_sorted(const uint32_t* sorted_keys, uint64_t m, uint64_t n, uint32_t* offsets,
                         cudaStream_t s) {
  offsets_k<<<grid_for(n + 1), kBlock, 0, s>>>(sorted_keys, m, n, offsets);
  UG_LAUNCH_CHECK();
}

namespace {
__global__ void any_negative_k(const double* __restrict__ w, uint64_t m, unsigned* __restrict__ bad) {
  bool neg = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    neg |= __ldg(&w[i]) < 0.0;
  if (__any_sync(0xffffffffu, neg) && (threadIdx.x & 31) == 0) *bad = 1u;
}
}  // namespace

void check_sssp_weights_device(const double* d_w, uint64_t m, cudaStream_t s) {
  if (m == 0) return;
  Scratch<unsigned> bad(1, s);
  UG_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
  any_negative_k<<<grid_for(m, kBlock, 148u * 16u), kBlock, 0, s>>>(d_w, m, bad.get());
  UG_LAUNCH_CHECK();
  unsigned h = 0;
  UG_CUDA(cudaMemcpyAsync(&h, bad.get(), 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(h == 0, URSA_GPU_EINVAL, "weights must be non-negative");
}

}  // namespace ug

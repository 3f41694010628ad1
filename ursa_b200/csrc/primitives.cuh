// primitives.cuh -- device-wide scan and stable LSD radix sort used by the CSR
// builds.  Hand-written for sm_100a; no library sort is used.
#pragma once

#include "common.cuh"

namespace ug {

// Exclusive prefix sum of n elements (out may alias in). If total is non-null
// the grand total is written to *total (device pointer).
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* total,
                        cudaStream_t s);
void exclusive_scan_u64(const uint64_t* in, uint64_t* out, uint64_t n, uint64_t* total,
                        cudaStream_t s);

// Stable sort of n (key, value) pairs by the low key_bits bits of the key
// (LSD, 8-bit digits).  vals_in == nullptr means value = input position.
// If gather_src is given, gather_out[p] = gather_src[vals_out[p]] is written
// in the last pass (used to place the CSR targets next to their edge ids).
// keys_out/vals_out must not alias the inputs.  n < 2^32.  gather_ready
// (optional): an event the last pass waits for before it reads gather_src,
// so gather_src may still be arriving while the earlier passes run.
void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint64_t n, int key_bits,
                      uint32_t* keys_out, uint32_t* vals_out, const uint32_t* gather_src,
                      uint32_t* gather_out, cudaStream_t s, cudaEvent_t gather_ready = nullptr);

// offsets[u] = lower_bound(sorted_keys[0..m), u) for u in [0, n].
void offsets_from_sorted(const uint32_t* sorted_keys, uint64_t m, uint64_t n, uint32_t* offsets,
                         cudaStream_t s);

// Largest u in [0, n) with off[u] <= k (the row owning CSR slot k).
__device__ __forceinline__ uint32_t owner_of(const uint32_t* __restrict__ off, uint64_t n,
                                             uint64_t k) {
  uint64_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    uint64_t mid = (lo + hi) >> 1;
    if ((uint64_t)off[mid] <= k)
      lo = mid;
    else
      hi = mid;
  }
  return (uint32_t)lo;
}

// Visits every CSR slot k < m with its owning row: the grid walks the slots
// in block-sized chunks, one thread finds the rows owning the chunk's first
// and last slot, and each thread searches only between them.  body(k, u) is
// called by the thread owning slot k.  Every thread of the block must call
// this (it synchronises the block).
template <class F>
__device__ __forceinline__ void for_each_slot_owner(const uint32_t* __restrict__ off, uint64_t n,
                                                    uint64_t m, F&& body) {
  __shared__ uint32_t s_range[2];
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < m; base += stride) {
    if (threadIdx.x == 0) {
      uint64_t last = base + blockDim.x - 1;
      if (last >= m) last = m - 1;
      s_range[0] = owner_of(off, n, base);
      s_range[1] = owner_of(off, n, last);
    }
    __syncthreads();
    const uint64_t k = base + threadIdx.x;
    if (k < m) {
      uint32_t lo = s_range[0], hi = s_range[1];  // answer in [lo, hi]
      while (lo < hi) {
        uint32_t mid = lo + ((hi - lo + 1) >> 1);
        if ((uint64_t)off[mid] <= k)
          lo = mid;
        else
          hi = mid - 1;
      }
      body(k, lo);
    }
    __syncthreads();
  }
}

inline int bits_for(uint64_t max_value) {
  int b = 0;
  while (b < 64 && (max_value >> b) != 0) b++;
  return b;
}

}  // namespace ug

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
// so gather_src may still be arriving while the earlier passes run.  bad
// (optional): set to nonzero if any key is >= limit (checked in the first
// pass; the sort itself masks every digit, so such keys are sorted by their
// low key_bits bits and the result is meant to be discarded).
void radix_sort_pairs(const uint32_t* keys_in, const uint32_t* vals_in, uint64_t n, int key_bits,
                      uint32_t* keys_out, uint32_t* vals_out, const uint32_t* gather_src,
                      uint32_t* gather_out, cudaStream_t s, cudaEvent_t gather_ready = nullptr,
                      unsigned* bad = nullptr, uint64_t limit = 0);

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

// Largest u in [lo, n) with off[u] <= k, given off[lo] <= k; called by a
// whole warp with the same arguments.  Two forward probes of 32 rows each
// (one 128-byte load apiece) settle the usual case, where the owner is a few
// short rows ahead of lo; a 32-ary search over [lo, n) settles the rest.
__device__ __forceinline__ uint32_t warp_owner_from(const uint32_t* __restrict__ off, uint64_t n,
                                                    uint64_t lo, uint64_t k) {
  const int lane = threadIdx.x & 31;
  for (int probe = 0; probe < 2; probe++) {
    const uint64_t u = lo + 1 + (uint64_t)lane;
    const bool ok = u < n && (uint64_t)off[u] <= k;
    const unsigned msk = __ballot_sync(0xffffffffu, ok);
    if (msk != 0xffffffffu) return (uint32_t)(lo + __popc(msk));  // ok is a prefix of the lanes
    lo += 32;
  }
  uint64_t hi = n;  // the answer is in [lo, hi)
  while (hi - lo > 1) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + (uint64_t)(lane + 1) * step;
    const bool ok = p < hi && (uint64_t)off[p] <= k;
    const uint64_t c = (uint64_t)__popc(__ballot_sync(0xffffffffu, ok));
    lo += c * step;
    hi = (lo + step < hi) ? lo + step : hi;
  }
  return (uint32_t)lo;
}

// Visits every CSR slot k < m with its owning row.  Each block walks one
// contiguous run of spans (kOwnerItems slots per thread); warp 0 finds the
// rows owning a span's first and last slot by searching forward from the
// previous span's owner, and each thread binary-searches only between them.
// body(k, u) is called by the thread owning slot k.  Every thread of the
// block must call this (it synchronises the block).
constexpr int kOwnerItems = 4;

template <class F>
__device__ __forceinline__ void for_each_slot_owner(const uint32_t* __restrict__ off, uint64_t n,
                                                    uint64_t m, F&& body) {
  __shared__ uint32_t s_range[2];
  const uint64_t span = (uint64_t)blockDim.x * kOwnerItems;
  const uint64_t spans = (m + span - 1) / span;
  const uint64_t per = (spans + gridDim.x - 1) / gridDim.x;
  const uint64_t beg = min(m, (uint64_t)blockIdx.x * per * span);
  const uint64_t end = min(m, beg + per * span);
  uint64_t prev = 0;  // warp 0: a row with off[prev] <= the next span's first slot
  for (uint64_t base = beg; base < end; base += span) {
    const uint64_t last = min(base + span, end) - 1;
    if (threadIdx.x < 32) {
      const uint32_t lo = warp_owner_from(off, n, prev, base);
      const uint32_t hi = warp_owner_from(off, n, lo, last);
      if (threadIdx.x == 0) {
        s_range[0] = lo;
        s_range[1] = hi;
      }
      prev = hi;
    }
    __syncthreads();
    const uint32_t r0 = s_range[0], r1 = s_range[1];
#pragma unroll
    for (int j = 0; j < kOwnerItems; j++) {
      const uint64_t k = base + (uint64_t)j * blockDim.x + threadIdx.x;
      if (k <= last) {
        uint32_t lo = r0, hi = r1;  // answer in [lo, hi]
        while (lo < hi) {
          const uint32_t mid = lo + ((hi - lo + 1) >> 1);
          if ((uint64_t)off[mid] <= k)
            lo = mid;
          else
            hi = mid - 1;
        }
        body(k, lo);
      }
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

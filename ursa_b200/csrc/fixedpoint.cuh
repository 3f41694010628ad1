// fixedpoint.cuh -- order-independent sums of non-negative f64 terms.
//
// Each term is truncated to a multiple of 2^-96 and added as a 128-bit
// integer.  Integer addition is exact and associative, so a sum does not
// depend on which thread, warp or block added which term: reductions over
// dynamically scheduled work stay bit-reproducible.  The truncation error is
// below 2^-96 per term; sums of PageRank residuals and dangling masses stay
// far below 2^31, inside the 128-bit range.
#pragma once

#include <stdint.h>

namespace ug {

typedef unsigned __int128 u128;

// v >= 0 finite -> floor(v * 2^96) (0 for subnormals), saturating.
__device__ __forceinline__ u128 fx_of(double v) {
  const uint64_t b = (uint64_t)__double_as_longlong(v);
  const int e = (int)((b >> 52) & 0x7ff);
  if (e == 0) return 0;
  const uint64_t mant = (b & 0xFFFFFFFFFFFFFull) | (1ull << 52);
  const int sh = e - 1075 + 96;  // v * 2^96 = mant * 2^sh
  if (sh >= 75) return ~(u128)0;
  if (sh >= 0) return (u128)mant << sh;
  if (sh <= -53) return 0;
  return (u128)(mant >> -sh);
}

__device__ __forceinline__ double fx_value(u128 x) {
  const double hi = __ull2double_rn((unsigned long long)(x >> 64));
  const double lo = __ull2double_rn((unsigned long long)x);
  return __dmul_rn(__dadd_rn(__dmul_rn(hi, 0x1p64), lo), 0x1p-96);
}

__device__ __forceinline__ u128 shfl_down_u128(u128 v, int o) {
  unsigned long long lo = (unsigned long long)v, hi = (unsigned long long)(v >> 64);
  lo = __shfl_down_sync(0xffffffffu, lo, o);
  hi = __shfl_down_sync(0xffffffffu, hi, o);
  return ((u128)hi << 64) | lo;
}

// A pair of fixed-point sums (residual, dangling mass) as stored in global
// memory: four 64-bit words.
struct __align__(16) FxPair {
  unsigned long long v[4];  // delta lo, delta hi, dangling lo, dangling hi
};

__device__ __forceinline__ FxPair fx_pack(u128 d, u128 g) {
  FxPair p;
  p.v[0] = (unsigned long long)d;
  p.v[1] = (unsigned long long)(d >> 64);
  p.v[2] = (unsigned long long)g;
  p.v[3] = (unsigned long long)(g >> 64);
  return p;
}
// L2 (cache-global) load of a pair written by another block.
__device__ __forceinline__ FxPair fx_ldcg(const FxPair* p) {
  const ulonglong2* q = reinterpret_cast<const ulonglong2*>(p);
  const ulonglong2 a = __ldcg(q), b = __ldcg(q + 1);
  FxPair r;
  r.v[0] = a.x;
  r.v[1] = a.y;
  r.v[2] = b.x;
  r.v[3] = b.y;
  return r;
}
__device__ __forceinline__ u128 fx_delta(const FxPair& p) { return ((u128)p.v[1] << 64) | p.v[0]; }
__device__ __forceinline__ u128 fx_dang(const FxPair& p) { return ((u128)p.v[3] << 64) | p.v[2]; }

}  // namespace ug

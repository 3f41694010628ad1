// common.cuh -- shared helpers for the ursa_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/ursa_gpu.h"

namespace ug {

// A failed CUDA call or a contract violation inside the library; caught at the
// C-ABI boundary and turned into a status code plus a thread-local message.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define UG_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      throw ::ug::Error(URSA_GPU_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_) + \
                                          " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
    }                                                                                  \
  } while (0)

#define UG_CHECK(cond, code, msg)                  \
  do {                                             \
    if (!(cond)) throw ::ug::Error((code), (msg)); \
  } while (0)

// Every kernel launch in the library is followed by UG_LAUNCH_CHECK(), which
// also counts it (ursa_gpu_launch_count), so a benchmark can report how many
// of this library's kernels ran in a timed region.
void count_launch();
#define UG_LAUNCH_CHECK()          \
  do {                             \
    ::ug::count_launch();          \
    UG_CUDA(cudaGetLastError());   \
  } while (0)

constexpr int kBlock = 256;

// Edge weights for the shortest-path family, once on the device (d_w: m
// f64): URSA_GPU_EINVAL if any is negative, as evaluate_weight requires
// before any weighted kernel runs (ursa-plan/src/weight.rs:88-93; NaN
// passes there too).  Negative weights would also let a frontier
// Bellman-Ford cycle forever, so this runs before one starts.
void check_sssp_weights_device(const double* d_w, uint64_t m, cudaStream_t s);

inline unsigned grid_for(uint64_t n, int block = kBlock, unsigned cap = 148u * 32u) {
  uint64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// Device blocks, stream-ordered.  Blocks of 4 MB and more are kept at their
// addresses once freed and handed out again to later requests that fit (the
// stream of the new owner waits on an event recorded where the block was
// freed); smaller ones come from the device's default pool, which keeps every
// freed block (its release threshold is raised to the maximum once per
// device).  block_free never throws.
void* block_alloc(size_t bytes, cudaStream_t s);
void block_free(void* p, cudaStream_t s) noexcept;
uint64_t block_cache_idle_bytes(int device);  // large blocks kept, none in use
void block_cache_flush(int device);           // hands them back to the pool

// Stream-ordered device scratch (block_alloc on the given stream, freed on it).
template <class T>
struct Scratch {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  Scratch() = default;
  Scratch(size_t count, cudaStream_t st) { alloc(count, st); }
  void alloc(size_t count, cudaStream_t st) {
    release();
    s = st;
    n = count;
    if (count) p = static_cast<T*>(block_alloc(count * sizeof(T), st));
  }
  void release() {
    if (p) block_free(p, s);
    p = nullptr;
    n = 0;
  }
  ~Scratch() { release(); }
  Scratch(const Scratch&) = delete;
  Scratch& operator=(const Scratch&) = delete;
  Scratch(Scratch&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; o.n = 0; }
  T* get() const { return p; }
  friend void swap(Scratch& a, Scratch& b) noexcept {
    std::swap(a.p, b.p);
    std::swap(a.n, b.n);
    std::swap(a.s, b.s);
  }
};

// Device allocation owned by a topology object, taken with block_alloc on the
// building call's stream.  Every call that uses a
// topology has finished before it returns, so the free is ordered on the
// per-thread default stream (always valid, whichever thread frees).
template <class T>
struct DevArray {
  T* p = nullptr;
  size_t n = 0;
  DevArray() = default;
  void alloc(size_t count, cudaStream_t s) {
    release();
    n = count;
    if (count) p = static_cast<T*>(block_alloc(count * sizeof(T), s));
  }
  void release() {
    if (p) block_free(p, cudaStreamPerThread);
    p = nullptr;
    n = 0;
  }
  ~DevArray() { release(); }
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  DevArray(DevArray&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevArray& operator=(DevArray&& o) noexcept {
    release();
    p = o.p;
    n = o.n;
    o.p = nullptr;
    o.n = 0;
    return *this;
  }
  T* get() const { return p; }
};

// Records the message returned by ursa_gpu_last_error() on this thread.
void set_last_error(const std::string& msg);

// Runs f() and maps exceptions to a C-ABI status code (URSA_GPU_*).
template <class F>
int guard(F&& f) {
  try {
    f();
    return URSA_GPU_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return URSA_GPU_ENOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return URSA_GPU_EINVAL;
  }
}

// One non-blocking stream per (host thread, device): calls from different
// host threads never serialise on a shared stream.
cudaStream_t thread_stream(int device);
void prepare_device(int device);
int sm_count(int device);
// Bytes the device's memory pool holds that no buffer uses (free for the
// library's next allocations, not for other allocators).
uint64_t pool_cached_bytes(int device);

// Device-side timeout for bounded waits (ns since an epoch).
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded grid barrier for cooperative launches. Every block calls it the same
// number of times. A wait longer than limit_ns sets *err and returns, so a
// broken invariant ends the kernel with an error status instead of a hang.
__device__ __forceinline__ void grid_barrier(unsigned* count, unsigned* gen, unsigned nblocks,
                                             int* err, uint64_t limit_ns) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = gen;
    unsigned g = *vgen;
    __threadfence();
    unsigned arrived = atomicAdd(count, 1u);
    if (arrived == nblocks - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      uint64_t t0 = global_ns();
      while (*vgen == g) {
        __nanosleep(64);
        if (global_ns() - t0 > limit_ns) {
          atomicExch(err, 1);
          break;
        }
        if (*(volatile int*)err) break;
      }
    }
    __threadfence();
  }
  __syncthreads();
}

// Compensated f32 accumulator: value = hi + lo (TwoSum / Kahan-Babuska-Neumaier).
struct F2 {
  float hi, lo;
};
__device__ __forceinline__ F2 f2_zero() { return F2{0.f, 0.f}; }
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
__device__ __forceinline__ F2 f2_add(F2 a, float x) {
  float s, e;
  two_sum(a.hi, x, s, e);
  return F2{s, __fadd_rn(a.lo, e)};
}
__device__ __forceinline__ F2 f2_combine(F2 a, F2 b) {
  float s, e;
  two_sum(a.hi, b.hi, s, e);
  return F2{s, __fadd_rn(__fadd_rn(a.lo, b.lo), e)};
}
__device__ __forceinline__ double f2_value(F2 a) { return (double)a.hi + (double)a.lo; }

}  // namespace ug

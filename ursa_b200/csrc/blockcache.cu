// blockcache.cu -- large device blocks kept at their addresses between calls.
//
// Every build and PageRank plan takes the same handful of 100-MB-class
// blocks on each call (sort buffers, grouped edge arrays, sliced-ELL ids).
// Taken from the device's default stream-ordered pool, a cudaMallocAsync of
// that size cost 0.6-13 ms of host time on B200 even with the memory already
// reserved by the pool, which made a third of an end-to-end R-MAT-22 step.
// So blocks of kCacheMin bytes and more are not returned to the pool when
// freed: they wait here, keyed by size, and the next request that fits takes
// one back at the same address.
//
// Stream order is kept the way the pool keeps it: a freed block carries an
// event recorded on the stream that freed it, and the stream of the next
// request waits on that event before any of its work can touch the block.
// A request the cache cannot satisfy goes to the pool; if the pool is out of
// memory the device's cached blocks are handed back to it and the request is
// retried once.
#include "common.cuh"

#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

namespace ug {

namespace {

constexpr size_t kCacheMin = 4ull << 20;  // smaller blocks go straight to the pool
constexpr size_t kGrain = 2ull << 20;     // cached sizes are multiples of this
constexpr int kMaxDevices = 64;

struct Block {
  void* p;
  size_t bytes;
  cudaEvent_t ready;  // recorded on the freeing stream
};

struct DeviceCache {
  std::multimap<size_t, Block> idle;  // by size
  std::vector<cudaEvent_t> spare_events;
  uint64_t idle_bytes = 0;
};

struct Live {
  int device;
  size_t bytes;
};

std::mutex g_mu;
DeviceCache g_cache[kMaxDevices];
std::unordered_map<void*, Live> g_live;  // cache-class blocks in use

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int d) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != d) cudaSetDevice(d);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Hands every idle block of `device` back to the pool, each freed behind its
// own event on the device's per-thread stream.  g_mu held.
void flush_locked(int device) {
  DeviceCache& c = g_cache[device];
  if (c.idle.empty()) return;
  DeviceGuard dg(device);
  for (auto& kv : c.idle) {
    cudaStreamWaitEvent(cudaStreamPerThread, kv.second.ready, 0);
    cudaFreeAsync(kv.second.p, cudaStreamPerThread);
    c.spare_events.push_back(kv.second.ready);
  }
  c.idle.clear();
  c.idle_bytes = 0;
}

}  // namespace

void* block_alloc(size_t bytes, cudaStream_t s) {
  void* p = nullptr;
  if (bytes < kCacheMin) {
    UG_CUDA(cudaMallocAsync(&p, bytes, s));
    return p;
  }
  const size_t need = (bytes + kGrain - 1) / kGrain * kGrain;
  int dev = 0;
  UG_CUDA(cudaStreamGetDevice(s, &dev));
  UG_CHECK(dev >= 0 && dev < kMaxDevices, URSA_GPU_EINVAL, "device index out of range");
  {
    std::lock_guard<std::mutex> g(g_mu);
    DeviceCache& c = g_cache[dev];
    // best fit, wasting at most an eighth of the request
    auto it = c.idle.lower_bound(need);
    if (it != c.idle.end() && it->first <= need + std::max(need / 8, kGrain)) {
      const Block b = it->second;
      c.idle.erase(it);
      c.idle_bytes -= b.bytes;
      c.spare_events.push_back(b.ready);
      g_live[b.p] = Live{dev, b.bytes};
      DeviceGuard dg(dev);
      UG_CUDA(cudaStreamWaitEvent(s, b.ready, 0));
      return b.p;
    }
  }
  cudaError_t e = cudaMallocAsync(&p, need, s);
  if (e == cudaErrorMemoryAllocation) {
    (void)cudaGetLastError();
    {
      std::lock_guard<std::mutex> g(g_mu);
      flush_locked(dev);
    }
    e = cudaMallocAsync(&p, need, s);
  }
  UG_CUDA(e);
  std::lock_guard<std::mutex> g(g_mu);
  g_live[p] = Live{dev, need};
  return p;
}

void block_free(void* p, cudaStream_t s) noexcept {
  if (!p) return;
  std::unique_lock<std::mutex> g(g_mu);
  auto it = g_live.find(p);
  if (it == g_live.end()) {
    g.unlock();
    cudaFreeAsync(p, s);
    return;
  }
  const Live lv = it->second;
  g_live.erase(it);
  DeviceCache& c = g_cache[lv.device];
  DeviceGuard dg(lv.device);
  cudaEvent_t ev = nullptr;
  if (!c.spare_events.empty()) {
    ev = c.spare_events.back();
    c.spare_events.pop_back();
  } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
    (void)cudaGetLastError();
    cudaFreeAsync(p, s);
    return;
  }
  if (cudaEventRecord(ev, s) != cudaSuccess) {
    (void)cudaGetLastError();
    c.spare_events.push_back(ev);
    cudaFreeAsync(p, s);
    return;
  }
  c.idle.emplace(lv.bytes, Block{p, lv.bytes, ev});
  c.idle_bytes += lv.bytes;
}

uint64_t block_cache_idle_bytes(int device) {
  if (device < 0 || device >= kMaxDevices) return 0;
  std::lock_guard<std::mutex> g(g_mu);
  return g_cache[device].idle_bytes;
}

void block_cache_flush(int device) {
  if (device < 0 || device >= kMaxDevices) return;
  std::lock_guard<std::mutex> g(g_mu);
  flush_locked(device);
}

}  // namespace ug

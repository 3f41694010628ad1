// cc_noalloc.cu -- connected_components_weak without any device allocation.
//
// Some callers cannot let a library allocate device memory during a query:
// a serving loop that has already handed all free HBM to resident graphs
// (admission is by free memory, so a surprise cudaMalloc can fail or evict),
// or a host runtime that owns every device byte through its own pool or
// arena and forbids allocations it does not make.  This entry point needs
// only memory that exists before the call: the topology (built earlier), the
// caller's output buffer, and one scratch array declared at file scope
// below.  The array is part of this file's device code: a GPU gets its copy
// when that code is loaded on it -- with CUDA's default lazy loading, at the
// first call of this entry point on that GPU -- and keeps it until the
// process exits.
#include <mutex>

#include "topo.cuh"

namespace ug {
void cc_weak_with_parent(TopoImpl* t, uint32_t* parent, uint32_t* d_out, cudaStream_t s);
}

namespace {

// Union-find parent array for graphs of up to kNoAllocMaxNodes nodes
// (4,194,304 nodes, 16 MiB per GPU).
constexpr uint64_t kNoAllocMaxNodes = 1ull << 22;
__device__ __align__(256) uint32_t g_cc_scratch[kNoAllocMaxNodes];

std::mutex g_scratch_mu;
uint32_t* g_scratch_addr[64] = {};

// The array's name is a host-side stand-in in host code; the device address
// is looked up once per device, with that device current.  The lookup leaves
// the calling thread's current device as it found it.
uint32_t* scratch_on(int device) {
  std::lock_guard<std::mutex> g(g_scratch_mu);
  if (!g_scratch_addr[device]) {
    int prev = 0;
    UG_CUDA(cudaGetDevice(&prev));
    UG_CUDA(cudaSetDevice(device));
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_cc_scratch);
    cudaSetDevice(prev);
    if (e != cudaSuccess || !p)
      throw ug::Error(URSA_GPU_ECUDA, std::string("cudaGetSymbolAddress(scratch) failed: ") +
                                          cudaGetErrorString(e));
    g_scratch_addr[device] = static_cast<uint32_t*>(p);
  }
  return g_scratch_addr[device];
}

}  // namespace

using namespace ug;

extern "C" int ursa_gpu_connected_components_weak_noalloc(ursa_gpu_topo* t, uint32_t* d_labels,
                                                         void* stream) {
  return guard([&] {
    UG_CHECK(t, URSA_GPU_EINVAL, "topology is NULL");
    TopoImpl* ti = &t->impl;
    UG_CHECK(ti->n <= kNoAllocMaxNodes, URSA_GPU_EINVAL,
             "connected_components_weak_noalloc: graph has " + std::to_string(ti->n) +
                 " nodes; the allocation-free variant supports at most " +
                 std::to_string(kNoAllocMaxNodes));
    if (ti->n == 0) return;
    UG_CHECK(d_labels, URSA_GPU_EINVAL, "d_labels is NULL");
    UG_CHECK(ti->device >= 0 && ti->device < 64, URSA_GPU_EINVAL, "device index out of range");
    uint32_t* parent = scratch_on(ti->device);
    // like every other entry point: the topology's device becomes current on
    // this thread, so the launches below go to that device even when the
    // caller's stream is given and another device was current
    cudaStream_t s = thread_stream(ti->device);
    if (stream) s = (cudaStream_t)stream;
    // every entry of the shared array that the kernels read is rewritten first
    cc_weak_with_parent(ti, parent, d_labels, s);
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

// api.cu -- the extern "C" boundary (include/ursa_gpu.h): status codes, a
// thread-local error message, per-thread streams, topology lifecycle and the
// host-mirror downloads, plus degree and PageRank.
#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "primitives.cuh"
#include "topo.cuh"

namespace ug {

namespace {
thread_local std::string g_last_error;
thread_local int g_device = 0;

struct StreamSlot {
  cudaStream_t s[64] = {};
  ~StreamSlot() {
    for (auto& x : s)
      if (x) cudaStreamDestroy(x);
  }
};
thread_local StreamSlot g_streams;
thread_local StreamSlot g_aux_streams;  // a second stream per thread: copies that overlap work
std::mutex g_dev_mu;
int g_sm_count[64] = {0};
bool g_prepared[64] = {false};

__global__ void widen_k(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

__global__ void degree_dir_k(const uint32_t* __restrict__ a, const uint32_t* __restrict__ b,
                             uint64_t n, uint32_t* __restrict__ out) {
  for (uint64_t u = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t d = a[u + 1] - a[u];
    if (b) d += b[u + 1] - b[u];
    out[u] = d;
  }
}

}  // namespace

// degree.rs:12-30: out-, in- or total degree per node.
void degree_run(TopoImpl* t, int dir, uint32_t* d_out, cudaStream_t s) {
  if (t->n == 0) return;
  if (dir != 0) ensure_in(t, s);
  const uint32_t* a = dir == 1 ? t->in.off.get() : t->out.off.get();
  const uint32_t* b = dir == 2 ? t->in.off.get() : nullptr;
  degree_dir_k<<<grid_for(t->n), kBlock, 0, s>>>(a, b, t->n, d_out);
  UG_LAUNCH_CHECK();
}

static std::atomic<uint64_t> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void prepare_device(int device) {
  std::lock_guard<std::mutex> g(g_dev_mu);
  if (device < 0 || device >= 64) throw Error(URSA_GPU_EINVAL, "device index out of range");
  if (g_prepared[device]) return;
  int cnt = 0;
  UG_CUDA(cudaGetDeviceCount(&cnt));
  UG_CHECK(device < cnt, URSA_GPU_ENODEV, "no such CUDA device");
  UG_CUDA(cudaSetDevice(device));
  UG_CUDA(cudaDeviceGetAttribute(&g_sm_count[device], cudaDevAttrMultiProcessorCount, device));
  // Keep every freed stream-ordered block in the pool instead of returning it
  // to the driver at the next synchronisation: a build whose transient
  // scratch exceeded a finite threshold otherwise unmapped and re-mapped
  // gigabytes on each call.  ursa_gpu_pool_release gives the cache back.
  cudaMemPool_t pool;
  UG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t threshold = UINT64_MAX;
  UG_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  g_prepared[device] = true;
}

uint64_t pool_cached_bytes(int device) {
  prepare_device(device);
  cudaMemPool_t pool;
  UG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t reserved = 0, used = 0;  // the attributes are 64-bit
  UG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
  UG_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
  return (reserved > used ? (uint64_t)(reserved - used) : 0) + block_cache_idle_bytes(device);
}

int sm_count(int device) {
  prepare_device(device);
  return g_sm_count[device];
}

cudaStream_t thread_stream(int device) {
  prepare_device(device);
  UG_CUDA(cudaSetDevice(device));
  cudaStream_t& s = g_streams.s[device];
  if (!s) UG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

// The thread's second stream on `device` (overlapping host-to-device copies).
static cudaStream_t thread_aux_stream(int device) {
  thread_stream(device);
  cudaStream_t& s = g_aux_streams.s[device];
  if (!s) UG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  return s;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

static cudaStream_t call_stream(TopoImpl* t, void* stream) {
  cudaStream_t s = thread_stream(t->device);
  return stream ? (cudaStream_t)stream : s;
}

static void require(const void* p, const char* what) {
  if (!p) throw Error(URSA_GPU_EINVAL, std::string(what) + " is NULL");
}

TopoImpl* topo_from_device(uint64_t n, const uint32_t* d_src, const uint32_t* d_dst, uint64_t m,
                           cudaStream_t s, int device, ursa_gpu_topo** holder, cudaEvent_t dst_ready) {
  UG_CHECK(m <= 0xFFFFFFFFull, URSA_GPU_EINVAL,
           "more than u32::MAX (~4.29B) edges is beyond the edge-id cap");
  UG_CHECK(n <= 0xFFFFFFFFull, URSA_GPU_EINVAL, "more than u32::MAX nodes");
  auto* h = new ursa_gpu_topo();
  *holder = h;
  TopoImpl* t = &h->impl;
  t->device = device;
  t->n = n;
  t->m = m;
  // The endpoint range check is done by the first radix pass of each sort
  // (which reads every key) and read once at the end: the sort masks every
  // digit and its gathers index row positions, so out-of-range ids cannot
  // make it touch memory out of bounds -- the result is only discarded.
  Scratch<unsigned> bad(1, s);
  UG_CUDA(cudaMemsetAsync(bad.get(), 0, sizeof(unsigned), s));
  // Out-CSR: rows by source; the destinations are only gathered in the last
  // radix pass, so they may still be arriving (dst_ready) until then.
  build_csr(n, d_src, d_dst, m, t->out, s, dst_ready, bad.get());
  // The endpoint columns are on the device in row order right now, so the
  // transpose is a second stable sort by destination -- the same in-CSR the
  // lazy reconstruction would produce (topology.rs:343-348), without
  // un-permuting the out-CSR later.
  build_csr(n, d_dst, d_src, m, t->in, s, nullptr, bad.get());
  t->has_in = true;
  unsigned hb = 0;
  UG_CUDA(cudaMemcpyAsync(&hb, bad.get(), sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(hb == 0, URSA_GPU_EINVAL, "dense endpoint id out of range (>= n_nodes)");
  return t;
}

}  // namespace ug

using namespace ug;

extern "C" {

const char* ursa_gpu_last_error(void) { return g_last_error.c_str(); }

int ursa_gpu_version(void) { return 100; }

uint64_t ursa_gpu_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int ursa_gpu_set_device(int device) {
  return guard([&] {
    prepare_device(device);
    g_device = device;
  });
}

int ursa_gpu_pool_cached_bytes(int device, uint64_t* cached) {
  return guard([&] {
    require(cached, "cached");
    *cached = pool_cached_bytes(device);
  });
}

int ursa_gpu_pool_release(int device) {
  return guard([&] {
    prepare_device(device);
    cudaMemPool_t pool;
    UG_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    UG_CUDA(cudaSetDevice(device));
    block_cache_flush(device);
    UG_CUDA(cudaDeviceSynchronize());  // frees still ordered on streams land in the pool first
    UG_CUDA(cudaMemPoolTrimTo(pool, 0));
  });
}

int ursa_gpu_thread_stream(int device, void** stream) {
  return guard([&] {
    require(stream, "stream");
    *stream = (void*)thread_stream(device);
  });
}

int ursa_gpu_topo_build(uint64_t n_nodes, const uint32_t* src, const uint32_t* dst,
                        uint64_t n_edges, ursa_gpu_topo** out) {
  return guard([&] {
    require(out, "out");
    *out = nullptr;
    if (n_edges) {
      require(src, "src");
      require(dst, "dst");
    }
    UG_CHECK(n_edges <= 0xFFFFFFFFull, URSA_GPU_EINVAL,
             "more than u32::MAX (~4.29B) edges is beyond the edge-id cap");
    int dev = g_device;
    cudaStream_t s = thread_stream(dev);
    cudaStream_t s2 = thread_aux_stream(dev);
    Scratch<uint32_t> d_src(n_edges, s), d_dst(n_edges, s);
    // src first on this stream; dst on the second stream right behind it, so
    // the out-CSR's radix passes over src run while dst crosses the link
    cudaEvent_t src_in = nullptr, dst_in = nullptr;
    UG_CUDA(cudaEventCreateWithFlags(&src_in, cudaEventDisableTiming));
    UG_CUDA(cudaEventCreateWithFlags(&dst_in, cudaEventDisableTiming));
    ursa_gpu_topo* h = nullptr;
    try {
      if (n_edges) UG_CUDA(cudaMemcpyAsync(d_src.get(), src, n_edges * 4, cudaMemcpyHostToDevice, s));
      UG_CUDA(cudaEventRecord(src_in, s));
      UG_CUDA(cudaStreamWaitEvent(s2, src_in, 0));
      if (n_edges) UG_CUDA(cudaMemcpyAsync(d_dst.get(), dst, n_edges * 4, cudaMemcpyHostToDevice, s2));
      UG_CUDA(cudaEventRecord(dst_in, s2));
      topo_from_device(n_nodes, d_src.get(), d_dst.get(), n_edges, s, dev, &h, dst_in);
    } catch (...) {
      UG_CUDA(cudaStreamWaitEvent(s, dst_in, 0));  // d_dst is freed on s
      delete h;
      cudaEventDestroy(src_in);
      cudaEventDestroy(dst_in);
      throw;
    }
    cudaEventDestroy(src_in);
    cudaEventDestroy(dst_in);
    *out = h;
  });
}

int ursa_gpu_topo_build_device(uint64_t n_nodes, const uint32_t* d_src, const uint32_t* d_dst,
                               uint64_t n_edges, void* stream, ursa_gpu_topo** out) {
  return guard([&] {
    require(out, "out");
    *out = nullptr;
    int dev = g_device;
    cudaStream_t s = stream ? (cudaStream_t)stream : thread_stream(dev);
    prepare_device(dev);
    ursa_gpu_topo* h = nullptr;
    try {
      topo_from_device(n_nodes, d_src, d_dst, n_edges, s, dev, &h);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

void ursa_gpu_topo_free(ursa_gpu_topo* t) {
  if (!t) return;
  cudaSetDevice(t->impl.device);
  delete t;
}

uint64_t ursa_gpu_topo_n_nodes(const ursa_gpu_topo* t) { return t ? t->impl.n : 0; }
uint64_t ursa_gpu_topo_n_edges(const ursa_gpu_topo* t) { return t ? t->impl.m : 0; }

uint64_t ursa_gpu_topo_device_bytes(const ursa_gpu_topo* t) {
  if (!t) return 0;
  const TopoImpl& i = t->impl;
  uint64_t b = 0;
  for (const DevCsr* c : {&i.out, &i.in}) b += (c->off.n + c->tgt.n + c->eid.n) * 4ull;
  b += (i.und_off.n + i.und_tgt.n + i.outdeg.n) * 4ull;
  b += pr_plan_bytes(i.pr_plan) + pr_plan_bytes(i.pr_plan_retired);
  return b;
}

int ursa_gpu_topo_prepare(ursa_gpu_topo* t, int what) {
  return guard([&] {
    require(t, "topology");
    cudaStream_t s = call_stream(&t->impl, nullptr);
    if (what & 1) ensure_in(&t->impl, s);
    if (what & 2) ensure_undirected(&t->impl, s);
  });
}

int ursa_gpu_topo_adjacency(ursa_gpu_topo* t, int dir, uint64_t* offsets, uint32_t* targets,
                            uint32_t* edge_ids) {
  return guard([&] {
    require(t, "topology");
    UG_CHECK(dir == 0 || dir == 1, URSA_GPU_EINVAL, "adjacency direction must be 0 (out) or 1 (in)");
    TopoImpl* ti = &t->impl;
    cudaStream_t s = call_stream(ti, nullptr);
    if (dir == 1) ensure_in(ti, s);
    const DevCsr& c = dir == 0 ? ti->out : ti->in;
    if (offsets) {
      Scratch<uint64_t> wide(ti->n + 1, s);
      widen_k<<<grid_for(ti->n + 1), kBlock, 0, s>>>(c.off.get(), ti->n + 1, wide.get());
      UG_LAUNCH_CHECK();
      UG_CUDA(cudaMemcpyAsync(offsets, wide.get(), (ti->n + 1) * 8, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
    }
    if (targets && ti->m)
      UG_CUDA(cudaMemcpyAsync(targets, c.tgt.get(), ti->m * 4, cudaMemcpyDeviceToHost, s));
    if (edge_ids && ti->m)
      UG_CUDA(cudaMemcpyAsync(edge_ids, c.eid.get(), ti->m * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_topo_undirected_len(ursa_gpu_topo* t, uint64_t* len) {
  return guard([&] {
    require(t, "topology");
    require(len, "len");
    cudaStream_t s = call_stream(&t->impl, nullptr);
    ensure_undirected(&t->impl, s);
    *len = t->impl.m_und;
  });
}

int ursa_gpu_topo_undirected(ursa_gpu_topo* t, uint64_t* offsets, uint32_t* targets) {
  return guard([&] {
    require(t, "topology");
    TopoImpl* ti = &t->impl;
    cudaStream_t s = call_stream(ti, nullptr);
    ensure_undirected(ti, s);
    if (offsets) {
      Scratch<uint64_t> wide(ti->n + 1, s);
      widen_k<<<grid_for(ti->n + 1), kBlock, 0, s>>>(ti->und_off.get(), ti->n + 1, wide.get());
      UG_LAUNCH_CHECK();
      UG_CUDA(cudaMemcpyAsync(offsets, wide.get(), (ti->n + 1) * 8, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
    }
    if (targets && ti->m_und)
      UG_CUDA(cudaMemcpyAsync(targets, ti->und_tgt.get(), ti->m_und * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_degree(ursa_gpu_topo* t, int dir, uint32_t* out) {
  return guard([&] {
    require(t, "topology");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    TopoImpl* ti = &t->impl;
    if (ti->n == 0) return;
    require(out, "out");
    cudaStream_t s = call_stream(ti, nullptr);
    Scratch<uint32_t> d(ti->n, s);
    degree_run(ti, dir, d.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d.get(), ti->n * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

static void check_params(const ursa_gpu_pagerank_params* p) {
  require(p, "params");
  UG_CHECK(p->damping == p->damping && p->tol == p->tol, URSA_GPU_EINVAL,
           "pagerank parameters must not be NaN");
}

int ursa_gpu_pagerank(ursa_gpu_topo* t, const ursa_gpu_pagerank_params* params, double* out,
                      ursa_gpu_pagerank_stats* stats) {
  return guard([&] {
    require(t, "topology");
    check_params(params);
    TopoImpl* ti = &t->impl;
    if (stats) *stats = ursa_gpu_pagerank_stats{0, 0.0, 0.0};
    if (ti->n == 0) return;  // pagerank.rs:100-102
    require(out, "out");
    cudaStream_t s = call_stream(ti, nullptr);
    Scratch<double> d_out(ti->n, s);
    pagerank_run(ti, *params, nullptr, d_out.get(), s, stats);
    UG_CUDA(cudaMemcpyAsync(out, d_out.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_pagerank_device(ursa_gpu_topo* t, const ursa_gpu_pagerank_params* params,
                             double* d_out, void* stream, ursa_gpu_pagerank_stats* stats) {
  return guard([&] {
    require(t, "topology");
    check_params(params);
    TopoImpl* ti = &t->impl;
    if (stats) *stats = ursa_gpu_pagerank_stats{0, 0.0, 0.0};
    if (ti->n == 0) return;
    require(d_out, "d_out");
    cudaStream_t s = call_stream(ti, stream);
    pagerank_run(ti, *params, nullptr, d_out, s, stats);
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_pagerank_weighted(ursa_gpu_topo* t, const double* weights, uint64_t n_weights,
                               const ursa_gpu_pagerank_params* params, double* out,
                               ursa_gpu_pagerank_stats* stats) {
  return guard([&] {
    require(t, "topology");
    check_params(params);
    TopoImpl* ti = &t->impl;
    if (stats) *stats = ursa_gpu_pagerank_stats{0, 0.0, 0.0};
    if (ti->n == 0) return;  // pagerank.rs:137-139
    UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
    require(out, "out");
    if (ti->m) require(weights, "weights");
    cudaStream_t s = call_stream(ti, nullptr);
    Scratch<double> d_w(ti->m ? ti->m : 1, s), d_out(ti->n, s);
    if (ti->m)
      UG_CUDA(cudaMemcpyAsync(d_w.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
    pagerank_run(ti, *params, d_w.get(), d_out.get(), s, stats);
    UG_CUDA(cudaMemcpyAsync(out, d_out.get(), ti->n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"

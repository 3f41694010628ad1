// result.cu -- Arrow results (ursa-plan/src/result.rs:144-261): query_batch,
// hop_batch and path_batch as Arrow C Data Interface record batches.
//
// Every column of a result is computed on the device into one staging block
// laid out exactly as the Arrow value buffers (64-byte aligned, back to
// back); ids are translated dense -> user on the device (IdMap::gather_user,
// id_map.rs:381-396, and the user-id column, id_map.rs:359-376); one
// device-to-host copy moves the block into pinned host memory, and the
// exported arrays point into that block.  Pinned blocks come from a small
// pool because page-locking a large block costs more than the copy into it.
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "topo.cuh"

namespace ug {

// One column of a result: Arrow format ("l" Int64, "I" UInt32, "g" Float64),
// value width and offset of its buffer in the block.
struct ResultCol {
  std::string name;
  const char* format;
  size_t width;
  size_t offset;
};

namespace {

constexpr size_t kAlign = 64;             // Arrow's buffer alignment
constexpr size_t kPoolKeep = 1ull << 30;  // pinned bytes kept for reuse

struct PinnedPool {
  std::mutex mu;
  std::multimap<size_t, void*> blocks;
  size_t kept = 0;

  void* take(size_t bytes, size_t* got) {
    {
      std::lock_guard<std::mutex> g(mu);
      auto it = blocks.lower_bound(bytes);
      if (it != blocks.end() && it->first <= 2 * bytes + (1u << 20)) {
        void* p = it->second;
        *got = it->first;
        kept -= it->first;
        blocks.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    UG_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocPortable));
    *got = bytes;
    return p;
  }
  void give(void* p, size_t bytes) {
    std::lock_guard<std::mutex> g(mu);
    if (kept + bytes <= kPoolKeep) {
      blocks.emplace(bytes, p);
      kept += bytes;
    } else {
      cudaFreeHost(p);
    }
  }
};

// Process-lifetime pool (blocks still kept at exit go with the process).
PinnedPool& pinned_pool() {
  static PinnedPool* p = new PinnedPool();
  return *p;
}

__global__ void iota_u32_k(uint32_t* out, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)i;
}

}  // namespace
}  // namespace ug

using namespace ug;

struct ursa_gpu_result {
  std::atomic<int> refs{1};
  void* host = nullptr;  // pinned block
  size_t cap = 0;
  uint64_t rows = 0;
  std::vector<ResultCol> cols;

  // Appends a column of `rows` values; returns its offset in the block.
  size_t add(const char* name, const char* format, size_t width) {
    size_t off = 0;
    if (!cols.empty()) {
      const ResultCol& b = cols.back();
      off = (b.offset + b.width * rows + kAlign - 1) / kAlign * kAlign;
    }
    cols.push_back(ResultCol{name, format, width, off});
    return off;
  }
  size_t bytes() const {
    if (cols.empty()) return kAlign;
    const ResultCol& b = cols.back();
    const size_t end = b.offset + b.width * rows;
    return end < kAlign ? kAlign : (end + kAlign - 1) / kAlign * kAlign;
  }
  void alloc_host() { host = pinned_pool().take(bytes(), &cap); }
  uint8_t* at(size_t off) { return (uint8_t*)host + off; }
  ~ursa_gpu_result() {
    if (host) pinned_pool().give(host, cap);
  }
};

namespace {

void result_unref(ursa_gpu_result* r) {
  if (r->refs.fetch_sub(1, std::memory_order_acq_rel) == 1) delete r;
}

// ---- Arrow C Data Interface export.  Each child holds its own reference on
// the result, so a consumer may move a child out and release the parent.
struct ChildSchemaPriv {
  std::string name;
};
void release_child_schema(ArrowSchema* s) {
  delete (ChildSchemaPriv*)s->private_data;
  s->release = nullptr;
}
struct SchemaPriv {
  std::vector<ArrowSchema> kids;
  std::vector<ArrowSchema*> kid_ptrs;
};
void release_schema(ArrowSchema* s) {
  auto* p = (SchemaPriv*)s->private_data;
  for (ArrowSchema& k : p->kids)
    if (k.release) k.release(&k);
  delete p;
  s->release = nullptr;
}

struct ChildArrayPriv {
  const void* bufs[2];
  ursa_gpu_result* r;
};
void release_child_array(ArrowArray* a) {
  auto* p = (ChildArrayPriv*)a->private_data;
  result_unref(p->r);
  delete p;
  a->release = nullptr;
}
struct ArrayPriv {
  const void* bufs[1] = {nullptr};
  std::vector<ArrowArray> kids;
  std::vector<ArrowArray*> kid_ptrs;
  ursa_gpu_result* r = nullptr;
};
void release_array(ArrowArray* a) {
  auto* p = (ArrayPriv*)a->private_data;
  for (ArrowArray& k : p->kids)
    if (k.release) k.release(&k);
  result_unref(p->r);
  delete p;
  a->release = nullptr;
}

// Validates an output column; returns its Arrow format and value width
// (result.rs:52-63: Float64 for pagerank, clustering, closeness, betweenness).
const char* column_format(const ursa_gpu_output_column& c, uint64_t m, size_t* width) {
  UG_CHECK(c.name, URSA_GPU_EINVAL, "output column name is NULL");
  const bool weighted = c.weights != nullptr;
  switch (c.algo) {
    case URSA_GPU_ALGO_PAGERANK:
      UG_CHECK(c.damping == c.damping && c.tol == c.tol, URSA_GPU_EINVAL,
               "pagerank parameters must not be NaN");
      UG_CHECK(!weighted || c.n_weights == m, URSA_GPU_EINVAL,
               "weights length must equal the edge count");
      *width = 8;
      return "g";
    case URSA_GPU_ALGO_CONNECTED_COMPONENTS:
      UG_CHECK(!c.strong, URSA_GPU_EINVAL,
               "strong components run on the host (not on the device path)");
      *width = 4;
      return "I";
    case URSA_GPU_ALGO_DEGREE:
      UG_CHECK(c.direction >= 0 && c.direction <= 2, URSA_GPU_EINVAL,
               "direction must be 0, 1 or 2");
      *width = 4;
      return "I";
    case URSA_GPU_ALGO_TRIANGLE_COUNT:
      *width = 4;
      return "I";
    case URSA_GPU_ALGO_CLUSTERING_COEFFICIENT:
      *width = 8;
      return "g";
    case URSA_GPU_ALGO_BETWEENNESS:
    case URSA_GPU_ALGO_CLOSENESS:
      UG_CHECK(!weighted || c.n_weights == m, URSA_GPU_EINVAL,
               "weights length must equal the edge count");
      *width = 8;
      return "g";
    case URSA_GPU_ALGO_LABEL_PROPAGATION:
    case URSA_GPU_ALGO_LOUVAIN:
      throw Error(URSA_GPU_EINVAL, "label propagation and louvain run on the host (not on the device path)");
    default:
      throw Error(URSA_GPU_EINVAL, "unknown output column algorithm");
  }
}

// algo_array (result.rs:82-140) into the device column at d_dst.
void compute_column(TopoImpl* t, const ursa_gpu_output_column& c, uint8_t* d_dst, cudaStream_t s) {
  Scratch<double> dw;
  if (c.weights && t->m) {
    dw.alloc(t->m, s);
    UG_CUDA(cudaMemcpyAsync(dw.get(), c.weights, t->m * 8, cudaMemcpyHostToDevice, s));
    if (c.algo == URSA_GPU_ALGO_BETWEENNESS || c.algo == URSA_GPU_ALGO_CLOSENESS)
      check_sssp_weights_device(dw.get(), t->m, s);
  }
  const double* w = c.weights ? (t->m ? dw.get() : nullptr) : nullptr;
  const bool weighted = c.weights != nullptr;
  switch (c.algo) {
    case URSA_GPU_ALGO_PAGERANK: {
      ursa_gpu_pagerank_params p{c.damping, c.max_iter, c.tol};
      Scratch<double> none;
      if (weighted && !w) none.alloc(1, s);  // zero edges: any non-null weight array
      pagerank_run(t, p, weighted ? (w ? w : none.get()) : nullptr, (double*)d_dst, s, nullptr);
      break;
    }
    case URSA_GPU_ALGO_CONNECTED_COMPONENTS:
      cc_weak_run(t, (uint32_t*)d_dst, s);
      break;
    case URSA_GPU_ALGO_DEGREE:
      degree_run(t, c.direction, (uint32_t*)d_dst, s);
      break;
    case URSA_GPU_ALGO_TRIANGLE_COUNT:
      triangle_count_run(t, (uint32_t*)d_dst, s);
      break;
    case URSA_GPU_ALGO_CLUSTERING_COEFFICIENT:
      clustering_run(t, (double*)d_dst, s);
      break;
    case URSA_GPU_ALGO_BETWEENNESS: {
      Scratch<double> none;
      if (weighted && !w) none.alloc(1, s);
      betweenness_run(t, weighted ? (w ? w : none.get()) : nullptr, c.has_sample != 0, c.sample,
                      c.has_seed != 0, c.seed, (double*)d_dst, s);
      break;
    }
    case URSA_GPU_ALGO_CLOSENESS:
      if (weighted) {
        Scratch<double> none;
        if (!w) none.alloc(1, s);
        closeness_weighted_device(t, w ? w : none.get(), (double*)d_dst, s);
      } else {
        closeness_device(t, (double*)d_dst, s, nullptr);
      }
      break;
  }
}

// The IdMap for a result over topology t: same device, one user id per node.
void check_ids(TopoImpl* t, ursa_gpu_idmap* ids) {
  if (!ids) return;
  uint64_t n_ids = 0;
  int dev = 0;
  idmap_users(ids, &n_ids, &dev);
  UG_CHECK(n_ids == t->n, URSA_GPU_EINVAL, "idmap and topology disagree on the node count");
  UG_CHECK(dev == t->device, URSA_GPU_EINVAL, "idmap and topology live on different devices");
}

// Writes rows dense node ids as the result's id-typed column at block offset
// off: user ids gathered on the device, or the dense ids themselves.
void write_ids(ursa_gpu_result* r, ursa_gpu_idmap* ids, const uint32_t* host_dense, uint64_t rows,
               size_t off, cudaStream_t s) {
  if (rows == 0) return;
  if (!ids) {
    std::memcpy(r->at(off), host_dense, rows * 4);
    return;
  }
  Scratch<uint32_t> d_dense(rows, s);
  Scratch<int64_t> d_user(rows, s);
  UG_CUDA(cudaMemcpyAsync(d_dense.get(), host_dense, rows * 4, cudaMemcpyHostToDevice, s));
  idmap_gather_device(ids, d_dense.get(), rows, d_user.get(), s);
  UG_CUDA(cudaMemcpyAsync(r->at(off), d_user.get(), rows * 8, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

extern "C" {

int ursa_gpu_query_batch(ursa_gpu_topo* t, ursa_gpu_idmap* ids, const ursa_gpu_output_column* cols,
                         uint64_t n_cols, ursa_gpu_result** out) {
  return guard([&] {
    UG_CHECK(t && out, URSA_GPU_EINVAL, "topology or out is NULL");
    UG_CHECK(n_cols == 0 || cols, URSA_GPU_EINVAL, "columns is NULL");
    *out = nullptr;
    TopoImpl* ti = &t->impl;
    check_ids(ti, ids);
    const uint64_t n = ti->n;
    auto* r = new ursa_gpu_result();
    try {
      r->rows = n;
      r->add("id", ids ? "l" : "I", ids ? 8 : 4);
      for (uint64_t i = 0; i < n_cols; i++) {
        size_t width = 0;
        const char* fmt = column_format(cols[i], ti->m, &width);
        r->add(cols[i].name, fmt, width);
      }
      r->alloc_host();
      cudaStream_t s = thread_stream(ti->device);
      if (n > 0) {
        const size_t bytes = r->bytes();
        Scratch<uint8_t> dev(bytes, s);
        if (ids) {
          uint64_t n_ids = 0;
          int d = 0;
          const int64_t* users = idmap_users(ids, &n_ids, &d);
          UG_CUDA(cudaMemcpyAsync(dev.get() + r->cols[0].offset, users, n * 8, cudaMemcpyDeviceToDevice, s));
        } else {
          iota_u32_k<<<grid_for(n), kBlock, 0, s>>>((uint32_t*)(dev.get() + r->cols[0].offset), n);
          UG_LAUNCH_CHECK();
        }
        for (uint64_t i = 0; i < n_cols; i++) compute_column(ti, cols[i], dev.get() + r->cols[i + 1].offset, s);
        UG_CUDA(cudaMemcpyAsync(r->host, dev.get(), bytes, cudaMemcpyDeviceToHost, s));
        UG_CUDA(cudaStreamSynchronize(s));
      }
    } catch (...) {
      result_unref(r);
      throw;
    }
    *out = r;
  });
}

int ursa_gpu_hop_batch(ursa_gpu_topo* t, ursa_gpu_idmap* ids, const uint32_t* seeds, uint64_t n_seeds,
                       uint32_t k, int dir, ursa_gpu_result** out) {
  return guard([&] {
    UG_CHECK(t && out, URSA_GPU_EINVAL, "topology or out is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    UG_CHECK(n_seeds == 0 || seeds, URSA_GPU_EINVAL, "seeds is NULL");
    *out = nullptr;
    TopoImpl* ti = &t->impl;
    check_ids(ti, ids);
    cudaStream_t s = thread_stream(ti->device);
    PairsHost ph;
    k_hop_run(ti, seeds, n_seeds, k, dir, ph, s);
    auto* r = new ursa_gpu_result();
    try {
      r->rows = ph.reached.size();
      const size_t o_src = r->add("src", ids ? "l" : "I", ids ? 8 : 4);
      const size_t o_dst = r->add("dst", ids ? "l" : "I", ids ? 8 : 4);
      r->alloc_host();
      write_ids(r, ids, ph.seeds.data(), r->rows, o_src, s);
      write_ids(r, ids, ph.reached.data(), r->rows, o_dst, s);
    } catch (...) {
      result_unref(r);
      throw;
    }
    *out = r;
  });
}

int ursa_gpu_path_batch(ursa_gpu_topo* t, ursa_gpu_idmap* ids, uint32_t source, uint32_t target,
                        int dir, const double* weights, uint64_t n_weights, ursa_gpu_result** out) {
  return guard([&] {
    UG_CHECK(t && out, URSA_GPU_EINVAL, "topology or out is NULL");
    UG_CHECK(dir >= 0 && dir <= 2, URSA_GPU_EINVAL, "direction must be 0, 1 or 2");
    *out = nullptr;
    TopoImpl* ti = &t->impl;
    check_ids(ti, ids);
    if (weights) {
      UG_CHECK(n_weights == ti->m, URSA_GPU_EINVAL, "weights length must equal the edge count");
      UG_CHECK(ti->m == 0 || weights, URSA_GPU_EINVAL, "weights is NULL");
    }
    const uint64_t n = ti->n;
    cudaStream_t s = thread_stream(ti->device);
    std::vector<uint32_t> path(n ? n : 1);
    std::vector<double> costs(weights ? (n ? n : 1) : 0);
    int64_t len;
    if (weights) {
      Scratch<double> dw(ti->m ? ti->m : 1, s);
      if (ti->m) UG_CUDA(cudaMemcpyAsync(dw.get(), weights, ti->m * 8, cudaMemcpyHostToDevice, s));
      check_sssp_weights_device(dw.get(), ti->m, s);
      len = weighted_path_run(ti, dw.get(), source, target, dir, path.data(), costs.data(), path.size(), s);
    } else {
      len = shortest_path_run(ti, source, target, dir, path.data(), path.size(), s);
    }
    UG_CHECK(len >= -1, URSA_GPU_ECUDA, "path longer than the node count");
    // result.rs:237-251: one row per consecutive pair of the route
    const uint64_t rows = len > 1 ? (uint64_t)len - 1 : 0;
    std::vector<uint32_t> a(rows), b(rows);
    for (uint64_t i = 0; i < rows; i++) {
      a[i] = path[i];
      b[i] = path[i + 1];
    }
    auto* r = new ursa_gpu_result();
    try {
      r->rows = rows;
      const size_t o_src = r->add("src", ids ? "l" : "I", ids ? 8 : 4);
      const size_t o_dst = r->add("dst", ids ? "l" : "I", ids ? 8 : 4);
      const size_t o_hop = r->add("hop", "l", 8);
      const size_t o_cost = r->add("cost", "g", 8);
      r->alloc_host();
      write_ids(r, ids, a.data(), rows, o_src, s);
      write_ids(r, ids, b.data(), rows, o_dst, s);
      auto* hop = (int64_t*)r->at(o_hop);
      auto* cost = (double*)r->at(o_cost);
      for (uint64_t i = 0; i < rows; i++) {
        hop[i] = (int64_t)i;
        cost[i] = weights ? costs[i + 1] : (double)(i + 1);
      }
    } catch (...) {
      result_unref(r);
      throw;
    }
    *out = r;
  });
}

uint64_t ursa_gpu_result_num_rows(const ursa_gpu_result* r) { return r ? r->rows : 0; }

uint64_t ursa_gpu_result_num_columns(const ursa_gpu_result* r) { return r ? r->cols.size() : 0; }

int ursa_gpu_result_export(ursa_gpu_result* r, ArrowSchema* schema, ArrowArray* array) {
  return guard([&] {
    UG_CHECK(r && schema && array, URSA_GPU_EINVAL, "result, schema or array is NULL");
    const size_t k = r->cols.size();
    auto* sp = new SchemaPriv();
    sp->kids.resize(k);
    sp->kid_ptrs.resize(k);
    for (size_t i = 0; i < k; i++) {
      auto* cp = new ChildSchemaPriv{r->cols[i].name};
      ArrowSchema& c = sp->kids[i];
      c.format = r->cols[i].format;
      c.name = cp->name.c_str();
      c.metadata = nullptr;
      c.flags = 0;  // result.rs:144-153: no algorithm or id column is nullable
      c.n_children = 0;
      c.children = nullptr;
      c.dictionary = nullptr;
      c.release = release_child_schema;
      c.private_data = cp;
      sp->kid_ptrs[i] = &c;
    }
    schema->format = "+s";
    schema->name = "";
    schema->metadata = nullptr;
    schema->flags = 0;
    schema->n_children = (int64_t)k;
    schema->children = sp->kid_ptrs.data();
    schema->dictionary = nullptr;
    schema->release = release_schema;
    schema->private_data = sp;

    auto* ap = new ArrayPriv();
    ap->kids.resize(k);
    ap->kid_ptrs.resize(k);
    for (size_t i = 0; i < k; i++) {
      r->refs.fetch_add(1, std::memory_order_relaxed);
      auto* cp = new ChildArrayPriv{{nullptr, r->at(r->cols[i].offset)}, r};
      ArrowArray& c = ap->kids[i];
      c.length = (int64_t)r->rows;
      c.null_count = 0;
      c.offset = 0;
      c.n_buffers = 2;  // validity (absent), values
      c.n_children = 0;
      c.buffers = cp->bufs;
      c.children = nullptr;
      c.dictionary = nullptr;
      c.release = release_child_array;
      c.private_data = cp;
      ap->kid_ptrs[i] = &c;
    }
    r->refs.fetch_add(1, std::memory_order_relaxed);
    ap->r = r;
    array->length = (int64_t)r->rows;
    array->null_count = 0;
    array->offset = 0;
    array->n_buffers = 1;  // a struct array has only its (absent) validity buffer
    array->n_children = (int64_t)k;
    array->buffers = ap->bufs;
    array->children = ap->kid_ptrs.data();
    array->dictionary = nullptr;
    array->release = release_array;
    array->private_data = ap;
  });
}

void ursa_gpu_result_free(ursa_gpu_result* r) {
  if (r) result_unref(r);
}

}  // extern "C"

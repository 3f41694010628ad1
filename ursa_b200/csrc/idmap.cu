// idmap.cu -- IdMap interning of Int64 node ids on the device
// (ursa-core/src/id_map.rs:197-320 from_edge_arrays / from_edge_batches /
// intern_i64, :381-440 gather_user / dense_from_array), feeding
// Topology::build directly from the id columns (ursa-plan/src/topology.rs:39-45).
//
// The reference walks the edges in chunk order and interns src before dst,
// so an id's dense index is the number of distinct ids whose first
// occurrence in the stream src[0], dst[0], src[1], dst[1], ... comes before
// its own.  Here:
//  1. every occurrence p (2i for src[i], 2i + 1 for dst[i]) is inserted into
//     an open-addressing table (2^k slots, load <= 1/2, linear probing, a
//     compare-and-swap claims an empty slot) that keeps the smallest p per id
//     (atomicMin), and the slot of every occurrence is recorded;
//  2. the occupied slots are compacted and stably radix-sorted by that first
//     position: the rank is the dense id, exactly the reference's order;
//  3. each occurrence's dense id is a gather through its recorded slot.
// The id equal to the table's empty marker (0xFFFF_FFFF_FFFF_FFFF, i.e. -1)
// is kept in a separate cell.  The table takes 20 bytes per slot and 4 slots
// per edge, so one map takes at most 2^29 edges (43 GB of table at that
// size); dense ids are u32 as in the reference.
#include <memory>
#include <vector>

#include "frontier.cuh"
#include "primitives.cuh"

namespace ug {

namespace {

constexpr unsigned long long kEmpty = 0xFFFFFFFFFFFFFFFFull;

// MurmurHash3's 64-bit finalizer (a published bit mixer).
__device__ __forceinline__ uint64_t id_mix(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

__global__ void id_insert_k(const int64_t* __restrict__ src, const int64_t* __restrict__ dst,
                            uint64_t n_occ, uint64_t mask, unsigned long long* __restrict__ keys,
                            uint32_t* __restrict__ first, uint32_t* __restrict__ slot_of,
                            uint32_t* __restrict__ special_first, unsigned* __restrict__ overflow) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_occ;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long key = (unsigned long long)((p & 1) ? dst[p >> 1] : src[p >> 1]);
    if (key == kEmpty) {
      atomicMin(special_first, (uint32_t)p);
      slot_of[p] = (uint32_t)(mask + 1);  // the separate cell
      continue;
    }
    uint64_t h = id_mix(key) & mask;
    // the table is at most half full, so a free or matching slot is found
    // within mask + 1 probes
    uint64_t probes = 0;
    while (true) {
      unsigned long long k = keys[h];
      if (k == kEmpty) k = atomicCAS(&keys[h], kEmpty, key);
      if (k == kEmpty || k == key) {
        atomicMin(&first[h], (uint32_t)p);
        slot_of[p] = (uint32_t)h;
        break;
      }
      h = (h + 1) & mask;
      if (++probes > mask) {
        atomicOr(overflow, 1u);
        break;
      }
    }
  }
}

// Occupied slot flags (the separate cell is slot mask + 1).
__global__ void id_flags_k(const unsigned long long* __restrict__ keys, uint64_t cap,
                           const uint32_t* __restrict__ special_first,
                           uint32_t* __restrict__ flag) {
  for (uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; h <= cap;
       h += (uint64_t)gridDim.x * blockDim.x)
    flag[h] = h < cap ? (keys[h] != kEmpty ? 1u : 0u) : (*special_first != 0xFFFFFFFFu ? 1u : 0u);
}

__global__ void id_compact_k(const uint32_t* __restrict__ pos, uint64_t cap,
                             const uint32_t* __restrict__ first,
                             const uint32_t* __restrict__ special_first,
                             uint32_t* __restrict__ c_first, uint32_t* __restrict__ c_slot) {
  for (uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; h <= cap;
       h += (uint64_t)gridDim.x * blockDim.x) {
    if (pos[h + 1] == pos[h]) continue;
    c_first[pos[h]] = h < cap ? first[h] : *special_first;
    c_slot[pos[h]] = (uint32_t)h;
  }
}

// dense[slot] = rank; to_user[rank] = the slot's id.
__global__ void id_rank_k(const uint32_t* __restrict__ sorted_idx, const uint32_t* __restrict__ c_slot,
                          uint64_t n, uint64_t cap, const unsigned long long* __restrict__ keys,
                          uint32_t* __restrict__ dense_of_slot, int64_t* __restrict__ to_user) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t slot = c_slot[sorted_idx[r]];
    dense_of_slot[slot] = (uint32_t)r;
    to_user[r] = slot < cap ? (int64_t)keys[slot] : (int64_t)kEmpty;
  }
}

__global__ void id_gather_k(const uint32_t* __restrict__ slot_of, uint64_t n_occ,
                            const uint32_t* __restrict__ dense_of_slot, uint32_t* __restrict__ ds,
                            uint32_t* __restrict__ dd) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_occ;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = dense_of_slot[slot_of[p]];
    if (p & 1)
      dd[p >> 1] = d;
    else
      ds[p >> 1] = d;
  }
}

__global__ void id_lookup_k(const int64_t* __restrict__ ids, uint64_t n, uint64_t mask,
                            const unsigned long long* __restrict__ keys,
                            const uint32_t* __restrict__ dense_of_slot, uint32_t special_dense,
                            uint32_t* __restrict__ out, uint8_t* __restrict__ found) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long key = (unsigned long long)ids[i];
    uint32_t d = 0xFFFFFFFFu;
    if (key == kEmpty) {
      d = special_dense;
    } else {
      uint64_t h = id_mix(key) & mask;
      for (uint64_t probes = 0; probes <= mask; probes++) {
        const unsigned long long k = keys[h];
        if (k == key) {
          d = dense_of_slot[h];
          break;
        }
        if (k == kEmpty) break;
        h = (h + 1) & mask;
      }
    }
    out[i] = d == 0xFFFFFFFFu ? 0u : d;
    found[i] = d == 0xFFFFFFFFu ? 0 : 1;
  }
}

}  // namespace

}  // namespace ug

using namespace ug;

struct ursa_gpu_idmap {
  int device = 0;
  uint64_t n_edges = 0, n_ids = 0, cap = 0;
  DevArray<unsigned long long> keys;
  DevArray<uint32_t> dense_of_slot;  // cap + 1 (the last is the separate cell)
  DevArray<uint32_t> src, dst;       // dense edge columns
  DevArray<int64_t> to_user;
  uint32_t special_dense = 0xFFFFFFFFu;
};

namespace ug {

namespace {

// IdMap::gather_user (id_map.rs:381-396): out[i] = to_user[dense[i]]; an
// index past the map (the reference's slice index would panic) sets *bad.
__global__ void gather_user_k(const int64_t* __restrict__ to_user, uint64_t n_ids,
                              const uint32_t* __restrict__ dense, uint64_t n, int64_t* __restrict__ out,
                              unsigned* __restrict__ bad) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t d = dense[i];
    if (d < n_ids) {
      out[i] = to_user[d];
    } else {
      out[i] = 0;
      *bad = 1u;
    }
  }
}

}  // namespace

const int64_t* idmap_users(ursa_gpu_idmap* m, uint64_t* n_ids, int* device) {
  *n_ids = m->n_ids;
  *device = m->device;
  return m->to_user.get();
}

void idmap_gather_device(ursa_gpu_idmap* m, const uint32_t* d_dense, uint64_t n, int64_t* d_out,
                         cudaStream_t s) {
  if (n == 0) return;
  Scratch<unsigned> bad(1, s);
  UG_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
  gather_user_k<<<grid_for(n), kBlock, 0, s>>>(m->to_user.get(), m->n_ids, d_dense, n, d_out, bad.get());
  UG_LAUNCH_CHECK();
  unsigned h = 0;
  UG_CUDA(cudaMemcpyAsync(&h, bad.get(), 4, cudaMemcpyDeviceToHost, s));
  UG_CUDA(cudaStreamSynchronize(s));
  UG_CHECK(h == 0, URSA_GPU_EINVAL, "gather_user: dense index out of range");
}

}  // namespace ug

extern "C" {

int ursa_gpu_idmap_build(uint64_t n_chunks, const int64_t* const* src_chunks,
                         const int64_t* const* dst_chunks, const uint64_t* chunk_lens,
                         ursa_gpu_idmap** out) {
  return guard([&] {
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    *out = nullptr;
    UG_CHECK(n_chunks == 0 || (src_chunks && dst_chunks && chunk_lens), URSA_GPU_EINVAL,
             "chunk arrays are NULL");
    uint64_t m = 0;
    for (uint64_t c = 0; c < n_chunks; c++) {
      UG_CHECK(chunk_lens[c] == 0 || (src_chunks[c] && dst_chunks[c]), URSA_GPU_EINVAL,
               "a chunk's src / dst column is NULL");
      m += chunk_lens[c];
    }
    UG_CHECK(m <= (1ull << 29), URSA_GPU_EINVAL,
             "idmap: at most 2^29 edges per map (the table takes 20 bytes per slot, 4 slots per edge)");
    int dev = 0;
    UG_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = thread_stream(dev);
    std::unique_ptr<ursa_gpu_idmap> M(new ursa_gpu_idmap());
    M->device = dev;
    M->n_edges = m;
    uint64_t cap = 1024;
    while (cap < 4 * m) cap <<= 1;  // at most 2m distinct ids: load <= 1/2
    M->cap = cap;
    M->src.alloc(m ? m : 1, s);
    M->dst.alloc(m ? m : 1, s);
    M->keys.alloc(cap, s);
    M->dense_of_slot.alloc(cap + 1, s);
    if (m == 0) {
      M->to_user.alloc(1, s);
      UG_CUDA(cudaStreamSynchronize(s));
      *out = M.release();
      return;
    }
    const uint64_t n_occ = 2 * m;
    {
      Scratch<int64_t> d_src(m, s), d_dst(m, s);
      uint64_t at = 0;
      for (uint64_t c = 0; c < n_chunks; c++) {
        if (!chunk_lens[c]) continue;
        UG_CUDA(cudaMemcpyAsync(d_src.get() + at, src_chunks[c], chunk_lens[c] * 8,
                                cudaMemcpyHostToDevice, s));
        UG_CUDA(cudaMemcpyAsync(d_dst.get() + at, dst_chunks[c], chunk_lens[c] * 8,
                                cudaMemcpyHostToDevice, s));
        at += chunk_lens[c];
      }
      Scratch<uint32_t> first(cap, s), slot_of(n_occ, s), ctl(2, s);  // special first, overflow
      UG_CUDA(cudaMemsetAsync(M->keys.get(), 0xFF, cap * 8, s));
      UG_CUDA(cudaMemsetAsync(first.get(), 0xFF, cap * 4, s));
      UG_CUDA(cudaMemsetAsync(ctl.get(), 0xFF, 4, s));
      UG_CUDA(cudaMemsetAsync(ctl.get() + 1, 0, 4, s));
      id_insert_k<<<grid_for(n_occ), kBlock, 0, s>>>(d_src.get(), d_dst.get(), n_occ, cap - 1,
                                                     M->keys.get(), first.get(), slot_of.get(),
                                                     ctl.get(), ctl.get() + 1);
      UG_LAUNCH_CHECK();
      // compact occupied slots, sort them by first occurrence
      Scratch<uint32_t> pos(cap + 2, s), total(1, s);
      UG_CUDA(cudaMemsetAsync(pos.get(), 0, (cap + 2) * 4, s));
      id_flags_k<<<grid_for(cap + 1), kBlock, 0, s>>>(M->keys.get(), cap, ctl.get(), pos.get());
      UG_LAUNCH_CHECK();
      exclusive_scan_u32(pos.get(), pos.get(), cap + 2, total.get(), s);
      uint32_t h[2] = {0, 0};
      UG_CUDA(cudaMemcpyAsync(&h[0], total.get(), 4, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaMemcpyAsync(&h[1], ctl.get() + 1, 4, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
      UG_CHECK(h[1] == 0, URSA_GPU_ECUDA, "idmap: hash table overflow");
      const uint64_t n = h[0];
      M->n_ids = n;
      Scratch<uint32_t> c_first(n, s), c_slot(n, s), k_sorted(n, s), idx_sorted(n, s);
      id_compact_k<<<grid_for(cap + 1), kBlock, 0, s>>>(pos.get(), cap, first.get(), ctl.get(),
                                                        c_first.get(), c_slot.get());
      UG_LAUNCH_CHECK();
      radix_sort_pairs(c_first.get(), nullptr, n, 32, k_sorted.get(), idx_sorted.get(), nullptr,
                       nullptr, s);
      M->to_user.alloc(n, s);
      id_rank_k<<<grid_for(n), kBlock, 0, s>>>(idx_sorted.get(), c_slot.get(), n, cap,
                                               M->keys.get(), M->dense_of_slot.get(),
                                               M->to_user.get());
      UG_LAUNCH_CHECK();
      id_gather_k<<<grid_for(n_occ), kBlock, 0, s>>>(slot_of.get(), n_occ, M->dense_of_slot.get(),
                                                      M->src.get(), M->dst.get());
      UG_LAUNCH_CHECK();
      // dense id of the separate cell, if the id -1 occurs
      UG_CUDA(cudaMemcpyAsync(&M->special_dense, M->dense_of_slot.get() + cap, 4,
                              cudaMemcpyDeviceToHost, s));
      uint32_t sf = 0;
      UG_CUDA(cudaMemcpyAsync(&sf, ctl.get(), 4, cudaMemcpyDeviceToHost, s));
      UG_CUDA(cudaStreamSynchronize(s));
      if (sf == 0xFFFFFFFFu) M->special_dense = 0xFFFFFFFFu;
    }
    *out = M.release();
  });
}

void ursa_gpu_idmap_free(ursa_gpu_idmap* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  delete m;
}

uint64_t ursa_gpu_idmap_len(const ursa_gpu_idmap* m) { return m ? m->n_ids : 0; }
uint64_t ursa_gpu_idmap_n_edges(const ursa_gpu_idmap* m) { return m ? m->n_edges : 0; }

int ursa_gpu_idmap_user_ids(ursa_gpu_idmap* m, int64_t* out) {
  return guard([&] {
    UG_CHECK(m, URSA_GPU_EINVAL, "idmap is NULL");
    if (!m->n_ids) return;
    UG_CHECK(out, URSA_GPU_EINVAL, "out is NULL");
    cudaStream_t s = thread_stream(m->device);
    UG_CUDA(cudaMemcpyAsync(out, m->to_user.get(), m->n_ids * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_idmap_dense_edges(ursa_gpu_idmap* m, uint32_t* src_out, uint32_t* dst_out) {
  return guard([&] {
    UG_CHECK(m, URSA_GPU_EINVAL, "idmap is NULL");
    if (!m->n_edges) return;
    cudaStream_t s = thread_stream(m->device);
    if (src_out)
      UG_CUDA(cudaMemcpyAsync(src_out, m->src.get(), m->n_edges * 4, cudaMemcpyDeviceToHost, s));
    if (dst_out)
      UG_CUDA(cudaMemcpyAsync(dst_out, m->dst.get(), m->n_edges * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_idmap_topology(ursa_gpu_idmap* m, ursa_gpu_topo** out) {
  return guard([&] {
    UG_CHECK(m && out, URSA_GPU_EINVAL, "idmap / out is NULL");
    *out = nullptr;
    int st = ursa_gpu_topo_build_device(m->n_ids, m->src.get(), m->dst.get(), m->n_edges, nullptr, out);
    if (st != URSA_GPU_OK) throw Error(st, ursa_gpu_last_error());
  });
}

int ursa_gpu_idmap_gather_user(ursa_gpu_idmap* m, const uint32_t* dense, uint64_t n, int64_t* out) {
  return guard([&] {
    UG_CHECK(m, URSA_GPU_EINVAL, "idmap is NULL");
    if (!n) return;
    UG_CHECK(dense && out, URSA_GPU_EINVAL, "dense / out is NULL");
    cudaStream_t s = thread_stream(m->device);
    Scratch<uint32_t> d_dense(n, s);
    Scratch<int64_t> d_out(n, s);
    UG_CUDA(cudaMemcpyAsync(d_dense.get(), dense, n * 4, cudaMemcpyHostToDevice, s));
    idmap_gather_device(m, d_dense.get(), n, d_out.get(), s);
    UG_CUDA(cudaMemcpyAsync(out, d_out.get(), n * 8, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

int ursa_gpu_idmap_lookup(ursa_gpu_idmap* m, const int64_t* ids, uint64_t n, uint32_t* dense_out,
                          uint8_t* found) {
  return guard([&] {
    UG_CHECK(m, URSA_GPU_EINVAL, "idmap is NULL");
    if (!n) return;
    UG_CHECK(ids && dense_out && found, URSA_GPU_EINVAL, "ids / dense_out / found is NULL");
    cudaStream_t s = thread_stream(m->device);
    Scratch<int64_t> d_ids(n, s);
    Scratch<uint32_t> d_out(n, s);
    Scratch<uint8_t> d_found(n, s);
    UG_CUDA(cudaMemcpyAsync(d_ids.get(), ids, n * 8, cudaMemcpyHostToDevice, s));
    id_lookup_k<<<grid_for(n), kBlock, 0, s>>>(d_ids.get(), n, m->cap - 1, m->keys.get(),
                                                m->dense_of_slot.get(), m->special_dense,
                                                d_out.get(), d_found.get());
    UG_LAUNCH_CHECK();
    UG_CUDA(cudaMemcpyAsync(dense_out, d_out.get(), n * 4, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaMemcpyAsync(found, d_found.get(), n, cudaMemcpyDeviceToHost, s));
    UG_CUDA(cudaStreamSynchronize(s));
  });
}

}  // extern "C"

// batch.cuh -- the per-graph descriptor and launch arguments of the batched
// kernels (batch.cu), shared with the serving loop (serve.cu), which runs
// pagerank queries on uploaded graphs through the same bucket kernel.
#pragma once

#include "topo.cuh"

struct ursa_gpu_batch;

namespace ug {

constexpr uint32_t kBkWhatPr = 1, kBkWhatCc = 2, kBkWhatTc = 4;

// One graph of a batch.  Row pointers are offset to the graph's first row;
// ids stored in in_src / o_tgt are `id_base` + local id.
struct __align__(16) GraphDesc {
  const uint32_t* in_off;   // n + 1 (values index in_src)
  const uint32_t* in_src;
  const uint32_t* out_off;  // n + 1 (out-degree only)
  const uint32_t* o_off;    // n + 1 (values index o_tgt)
  const uint32_t* o_tgt;    // oriented undirected lists, ascending ids
  const uint32_t* rows;     // local rows grouped by degree class
  double* rank;             // n (pagerank result, updated in place)
  float* x0;                // n (global share row: staging or shares)
  float* x1;                // n
  uint32_t* cc;             // n
  uint32_t* tri;            // n
  uint32_t cls[8];          // class c rows: rows[cls[c] .. cls[c+1]), cls[6] = n
  uint32_t n;
  uint32_t id_base;
  uint32_t pad[2];
};

struct BucketArgs {
  const GraphDesc* desc;
  const uint32_t* work;  // descriptor indices, largest graph first
  uint32_t n_work;
  uint32_t* next;        // work counter (zeroed before the launch)
  uint32_t cap;          // nodes whose state fits in the CTA's shared memory
  uint32_t what;
  uint32_t max_iter;
  double damping, tol;
  uint32_t* iters;       // per descriptor
  double* delta;         // per descriptor
};

// The bucket kernel for a CTA size (128, 256, 512 or 1024), its resident
// CTAs for a dynamic shared-memory size (sets the size attribute), and the
// host copy of a batch graph's descriptor.
void* batch_kernel_for(uint32_t threads);
int batch_kernel_resident(uint32_t threads, size_t smem, int device);
const GraphDesc* batch_host_desc(const ursa_gpu_batch* b, uint64_t g);

}  // namespace ug

// pending.cu -- entry points whose device kernels are not in this build yet.
// Each returns URSA_GPU_EINVAL with a clear message (never a CPU fallback).
#include "common.cuh"

extern "C" {

static int pending(const char* what) {
  ug::set_last_error(std::string(what) + ": not available in this build");
  return URSA_GPU_EINVAL;
}

int ursa_gpu_betweenness(ursa_gpu_topo*, int, double, int, uint64_t, double*) {
  return pending("betweenness");
}
int ursa_gpu_betweenness_weighted(ursa_gpu_topo*, const double*, uint64_t, int, double, int,
                                  uint64_t, double*) {
  return pending("betweenness_weighted");
}
}

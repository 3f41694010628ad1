// unionfind.cuh -- lock-free union-find over a parent array (global or
// shared memory through a generic pointer), used by weak connected components
// (ursa-core/src/algo/components.rs:14-68).
//
// A union always hooks the larger root under the smaller one with a
// compare-and-swap (a failed CAS means the root moved; the walk continues from
// the new parent), and finds compress paths by pointer jumping.  Parents only
// ever decrease, so each tree's root is the minimum id of its component.
#pragma once

#include <stdint.h>

namespace ug {

__device__ __forceinline__ uint32_t uf_parent(const uint32_t* p, uint32_t x) {
  return *(const volatile uint32_t*)&p[x];
}

// Root of x with intermediate pointer jumping (parent[x] < x off the root).
__device__ __forceinline__ uint32_t uf_find(uint32_t* p, uint32_t x) {
  uint32_t par = uf_parent(p, x);
  if (par != x) {
    uint32_t prev = x, next;
    while (par > (next = uf_parent(p, par))) {
      p[prev] = next;
      prev = par;
      par = next;
    }
  }
  return par;
}

__device__ __forceinline__ void uf_unite(uint32_t* p, uint32_t a, uint32_t b) {
  uint32_t ra = uf_find(p, a), rb = uf_find(p, b);
  // bounded by the depth of the forest; each failed CAS moves one link up
  while (ra != rb) {
    if (ra < rb) {
      uint32_t old = atomicCAS(&p[rb], rb, ra);
      if (old == rb) return;
      rb = old;
    } else {
      uint32_t old = atomicCAS(&p[ra], ra, rb);
      if (old == ra) return;
      ra = old;
    }
  }
}

// Final root of x without writes (valid once every union has finished).
__device__ __forceinline__ uint32_t uf_root(const uint32_t* p, uint32_t x) {
  uint32_t par = uf_parent(p, x);
  while (par != x) {
    x = par;
    par = uf_parent(p, x);
  }
  return par;
}

}  // namespace ug

// Grid-wide barrier for cooperative (co-resident) launches, with a bounded wait.
//
// Arrival counter whose top bit flips once every CTA of the grid has arrived:
// CTA 0 adds 0x80000000 - (nblocks - 1), every other CTA adds 1, so the sum of one
// barrier's arrivals is exactly 0x80000000 and the counter needs no reset. A CTA
// waits for the flip with __nanosleep back-off; after `limit` polls it records
// an error and returns false instead of spinning forever.
#pragma once
#include <cuda_runtime.h>

namespace sp {

struct GridBar {
  unsigned int arrived;
  int error;  // nonzero once any CTA gave up waiting
};

// The same barrier over a group of nb co-resident CTAs that share gb; `first` marks
// exactly one CTA of the group.
__device__ __forceinline__ bool group_barrier(GridBar* gb, unsigned int nb, bool first,
                                              unsigned long long limit = (1ull << 24)) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int inc = first ? (0x80000000u - (nb - 1u)) : 1u;
    __threadfence();
    const unsigned int old = atomicAdd(&gb->arrived, inc);
    volatile unsigned int* ap = &gb->arrived;
    volatile int* ep = &gb->error;
    unsigned long long polls = 0;
    int ok = 1;
    while (((old ^ *ap) & 0x80000000u) == 0u) {
      if (*ep || ++polls > limit) {
        atomicExch(&gb->error, 1);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ bool grid_barrier(GridBar* gb, unsigned long long limit = (1ull << 24)) {
  return group_barrier(gb, gridDim.x * gridDim.y * gridDim.z, (blockIdx.x | blockIdx.y | blockIdx.z) == 0, limit);
}

}  // namespace sp

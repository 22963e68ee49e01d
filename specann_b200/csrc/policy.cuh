// Execution policies shared by the persistent kernels: which threads work on one problem and how
// its phases are separated.
#pragma once
#include "common.cuh"

namespace sa {

// GridPolicy: one problem on the whole cooperative grid; phases are separated by grid_barrier on
// the control block's GridSync (epilogue by the last CTA to arrive).
struct GridPolicy {
  __device__ __forceinline__ long long tid() const { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ __forceinline__ long long nthr() const { return (long long)gridDim.x * blockDim.x; }
  __device__ __forceinline__ int block() const { return blockIdx.x; }
  __device__ __forceinline__ int nblocks() const { return gridDim.x; }
  template <class E>
  __device__ __forceinline__ bool sync(GridSync* gs, E&& e) const { return grid_barrier(gs, e); }
  __device__ __forceinline__ bool sync(GridSync* gs) const { return grid_barrier(gs); }
};

// TeamPolicy: one problem on the CTAs [b0, b0 + nb) of a cooperative grid (batched solves: every
// team works through its own list of problems). Phases are separated by a barrier of the nb CTAs
// on the team's own GridSync (the control block's is not used); a team of one CTA uses
// __syncthreads, with the epilogue run by the whole CTA.
struct TeamPolicy {
  int b0, nb;
  GridSync* gs;
  __device__ __forceinline__ long long tid() const { return (long long)(blockIdx.x - b0) * blockDim.x + threadIdx.x; }
  __device__ __forceinline__ long long nthr() const { return (long long)nb * blockDim.x; }
  __device__ __forceinline__ int block() const { return (int)blockIdx.x - b0; }
  __device__ __forceinline__ int nblocks() const { return nb; }
  template <class E>
  __device__ __forceinline__ bool sync(GridSync*, E&& e) const {
    if (nb == 1) {
      __syncthreads();
      e();
      __syncthreads();
      return true;
    }
    return grid_barrier_n(gs, (unsigned int)nb, e);
  }
  __device__ __forceinline__ bool sync(GridSync* g) const { return sync(g, [] {}); }
};

}  // namespace sa

// Execution policies shared by the persistent kernels.
#pragma once
#include "common.cuh"

namespace sa {

// GridPolicy: one problem on a cooperative grid, phases
// separated by grid_barrier (epilogue by the last CTA). CtaPolicy: one problem per CTA (batched
// solves), phases separated by __syncthreads (epilogue by the whole CTA).
struct GridPolicy {
  __device__ __forceinline__ long long tid() const { return (long long)blockIdx.x * blockDim.x + threadIdx.x; }
  __device__ __forceinline__ long long nthr() const { return (long long)gridDim.x * blockDim.x; }
  __device__ __forceinline__ int block() const { return blockIdx.x; }
  __device__ __forceinline__ int nblocks() const { return gridDim.x; }
  template <class E>
  __device__ __forceinline__ bool sync(GridSync* gs, E&& e) const { return grid_barrier(gs, e); }
  __device__ __forceinline__ bool sync(GridSync* gs) const { return grid_barrier(gs); }
};

struct CtaPolicy {
  __device__ __forceinline__ long long tid() const { return threadIdx.x; }
  __device__ __forceinline__ long long nthr() const { return blockDim.x; }
  __device__ __forceinline__ int block() const { return 0; }
  __device__ __forceinline__ int nblocks() const { return 1; }
  template <class E>
  __device__ __forceinline__ bool sync(GridSync*, E&& e) const {
    __syncthreads();
    e();
    __syncthreads();
    return true;
  }
  __device__ __forceinline__ bool sync(GridSync*) const {
    __syncthreads();
    return true;
  }
};

}  // namespace sa

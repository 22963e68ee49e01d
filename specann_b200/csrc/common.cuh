// Shared device helpers for the SpecAnn kernels (sm_100a).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/specann_b200.h"

namespace sa {

constexpr int kThreads = 512;             // threads per CTA of the persistent kernels
constexpr int kWarps = kThreads / 32;
constexpr int kShortMax = 64;             // rows with at most this many entries are "short"
constexpr int kChunk = 256;               // entries per chunk of a long row
constexpr int kSegMax = 256;              // entries per short segment at most (= one warp tile)
constexpr int kSegRows = 64;              // rows per short segment at most
constexpr int kTileIt = kSegMax / 32;     // entries per lane of a tile
constexpr int kNcvMax = 64;               // largest Lanczos basis
constexpr int kDotBatch = 8;              // basis vectors per register batch in the dot phase
constexpr unsigned long long kSpinLimit = 1ull << 25;   // ~2 s of 64 ns sleeps
constexpr int kMaxSplits = 8;             // column splits of an operator larger than L2 (split.cu)

// One tile of the SpMV work list: at most kSegMax stored entries starting at e0.
//   row >= 0: a short segment of rows [row, row + nrows);
//   row < 0:  a chunk of the long row -(row + 1).
//   meta bits 0-8: entries in the tile; segment: bits 9-15 nrows; chunk: bits 9-31 hold
//   (multi-chunk row id + 1), 0 when the row fits in one chunk.
struct WorkItem {
  long long e0;
  int row;
  int meta;
};
__host__ __device__ __forceinline__ int item_len(int meta) { return meta & 511; }
__host__ __device__ __forceinline__ int item_nrows(int meta) { return (meta >> 9) & 127; }
__host__ __device__ __forceinline__ int item_mc(int meta) { return (int)((unsigned)meta >> 9) - 1; }

// Device-resident synchronisation block of a persistent kernel (zeroed before launch).
struct GridSync {
  unsigned int count;
  unsigned int gen;
  int error;
  int pad;
};

__device__ __forceinline__ unsigned int ld_volatile_u32(const unsigned int* p) {
  return *((volatile const unsigned int*)p);
}
__device__ __forceinline__ int ld_volatile_i32(const int* p) {
  return *((volatile const int*)p);
}

// Barrier of `expected` co-resident CTAs (a cooperative grid, or a team of CTAs inside one),
// with an epilogue run by the last CTA to arrive (the whole CTA runs it, after every other CTA's
// writes are visible) before the others are released. Waits are bounded: after spin_limit sleeps
// the barrier records SA_ERR_BARRIER_TIMEOUT in gs->error and returns false, and a waiting CTA
// also stops as soon as another CTA has recorded an error; the caller must then return. The
// decision is taken by thread 0 and shared through shared memory, so the whole CTA returns the
// same value.
template <class Epilogue>
__device__ __forceinline__ bool grid_barrier_n(GridSync* gs, unsigned int expected, Epilogue&& epi,
                                               unsigned long long spin_limit = kSpinLimit) {
  __shared__ unsigned int s_last, s_gen;
  __shared__ int s_err;
  __syncthreads();
  if (threadIdx.x == 0) {
    s_gen = ld_volatile_u32(&gs->gen);
    __threadfence();
    unsigned int arrived = atomicAdd(&gs->count, 1u);
    s_last = (arrived == expected - 1) ? 1u : 0u;
    s_err = 0;
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    epi();
    __syncthreads();
    if (threadIdx.x == 0) {
      gs->count = 0;
      __threadfence();
      atomicAdd(&gs->gen, 1u);
      if (ld_volatile_i32(&gs->error)) s_err = 1;
    }
  } else if (threadIdx.x == 0) {
    unsigned long long spins = 0;
    while (ld_volatile_u32(&gs->gen) == s_gen) {
      __nanosleep(64);
      if (ld_volatile_i32(&gs->error)) break;
      if (++spins > spin_limit) {
        atomicExch(&gs->error, SA_ERR_BARRIER_TIMEOUT);
        break;
      }
    }
    __threadfence();
    if (ld_volatile_i32(&gs->error)) s_err = 1;
  }
  __syncthreads();
  return s_err == 0;
}

template <class Epilogue>
__device__ __forceinline__ bool grid_barrier(GridSync* gs, Epilogue&& epi) {
  return grid_barrier_n(gs, gridDim.x, epi);
}

__device__ __forceinline__ bool grid_barrier(GridSync* gs) {
  return grid_barrier_n(gs, gridDim.x, [] {});
}

// Device clock in ns (phase timers of the persistent kernels).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// ---------------------------------------------------------------------------------------------
// Counter-based random streams (identical to oracle/selection.py and the host code).
// ---------------------------------------------------------------------------------------------
constexpr unsigned long long kSelSalt = 0x5E1EC7ED5EED0001ull;
constexpr long long kFinalStreamBase = 1ll << 20;

__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  unsigned long long z = x;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct SelKeys {
  unsigned long long k[4];
  unsigned long long mask;
  unsigned int shift;
};

__host__ __device__ inline int domain_bits(long long n) {
  int b = 0;
  unsigned long long v = (unsigned long long)(n - 1);
  while (v) { ++b; v >>= 1; }
  return b < 1 ? 1 : b;
}

__host__ __device__ inline SelKeys make_sel_keys(unsigned long long seed, long long stream, long long n) {
  SelKeys s;
  unsigned long long base = splitmix64(seed ^ kSelSalt);
  for (int r = 0; r < 4; ++r) s.k[r] = splitmix64(base + 4ull * (unsigned long long)stream + (unsigned long long)r);
  int b = domain_bits(n);
  s.mask = (b >= 64) ? ~0ull : ((1ull << b) - 1ull);
  s.shift = (unsigned int)((b + 1) / 2);
  return s;
}

__host__ __device__ __forceinline__ unsigned long long sel_perm(unsigned long long x, const SelKeys& s) {
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const unsigned long long add = s.k[r] & s.mask;
    const unsigned long long mul = ((s.k[r] >> 32) | 1ull) & 0xFFFFFFFFull;
    x = (x + add) & s.mask;
    x = (x * mul) & s.mask;
    x = x ^ (x >> s.shift);
  }
  return x;
}

// rank(i): a bijection of [0, n) (cycle walking; terminates because i's cycle contains i < n).
__host__ __device__ __forceinline__ long long sel_rank(long long i, const SelKeys& s, long long n) {
  unsigned long long y = sel_perm((unsigned long long)i, s);
  while (y >= (unsigned long long)n) y = sel_perm(y, s);
  return (long long)y;
}

// Standard normal from a counter (Box-Muller on two 53-bit uniforms in (0, 1]).
__device__ __forceinline__ double normal_from_counter(unsigned long long key, long long i) {
  const unsigned long long h1 = splitmix64(key ^ (2ull * (unsigned long long)i));
  const unsigned long long h2 = splitmix64(key ^ (2ull * (unsigned long long)i + 1ull));
  const double u1 = ((double)(h1 >> 11) + 1.0) * (1.0 / 9007199254740992.0);
  const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// ---------------------------------------------------------------------------------------------
// Reductions (fixed order: results do not depend on timing).
// ---------------------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum of one double (all threads get the result). Uses a kWarps scratch array.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = (lane < (int)(blockDim.x >> 5)) ? scratch[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) scratch[0] = t;
  }
  __syncthreads();
  t = scratch[0];
  __syncthreads();
  return t;
}

__device__ __forceinline__ long long rp_load(const int* rp, long long i) { return (long long)__ldg(rp + i); }
__device__ __forceinline__ long long rp_load(const long long* rp, long long i) { return __ldg(rp + i); }

}  // namespace sa

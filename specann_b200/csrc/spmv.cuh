// Fused CSR SpMV work-list processor shared by the standalone operator, the Lanczos kernel and
// the residual check.
//
// The rows are cut once per matrix (sa_set_matrix) into a work list in row order whose items are
// warp tiles of at most kSegMax = 256 entries:
//   * short segments: runs of consecutive rows with at most kShortMax entries each (at most
//     kSegRows rows, at most kSegMax entries);
//   * long-row chunks: rows with more than kShortMax entries cut into chunks of kChunk entries.
// A warp streams its tile's columns and values with kTileIt fully coalesced, independent loads per
// lane (lane l takes entries l, l + 32, ...), issues the kTileIt gathers of u, and multiplies. For
// a segment the products go to a per-warp shared buffer and one lane per row adds its contiguous
// range in order; for a chunk the lanes' partial sums are combined by a fixed xor-shuffle tree.
// A row of one chunk is finished by its warp. For a row of several chunks every warp stores its
// partial sum and the warp that finishes last (an atomic ticket per row) adds the partials in chunk
// order and finishes the row. No spin-waits, and no summation order depends on timing.
//
// Warps take items round robin (item t -> warp t mod warps), so concurrent warps stream
// neighbouring parts of col/val. col, val, rowptr and the work list are read through the
// read-only path. The gathered vector u is read through the read-only path too when it is
// immutable for the whole kernel (kReadOnlyU, the standalone operator); the persistent kernels
// rewrite u between phases, so there it is read with ordinary L1-allocating loads, which see the
// writes of other CTAs because every phase boundary is a grid barrier (gpu-scope fence by the
// waiting thread, then bar.sync).
#pragma once
#include "common.cuh"

namespace sa {

template <typename T, typename RP>
struct SpmvArgs {
  const RP* rowptr;
  const int* col;
  const T* val;
  const WorkItem* items;
  long long n_items;
  const long long* mc_base;
  int* mc_count;
  T* long_part;
};

// Per-warp shared staging of a tile: kSegMax products and kSegRows + 1 row offsets.
template <typename T>
struct SpmvSmem {
  T prod[kWarps][kSegMax];
  int rp[kWarps][kSegRows + 1];
};

// fin(row, sum) is called exactly once per row with sum = sum_j val_ij * u_j (T arithmetic).
template <bool kReadOnlyU, typename T>
__device__ __forceinline__ T gather(const T* u, int j) {
  if (kReadOnlyU) return __ldg(u + j);
  return u[j];
}

template <typename T, typename RP, bool kReadOnlyU = false, class Fin>
__device__ __forceinline__ void spmv_items(const SpmvArgs<T, RP>& S, const T* u, long long gwarp,
                                           long long nwarps, SpmvSmem<T>& sm, Fin&& fin) {
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  T* prod = sm.prod[wid];
  int* srp = sm.rp[wid];
  for (long long it = gwarp; it < S.n_items; it += nwarps) {
    const long long ix = __ldg(&S.items[it].x);
    const int iy = __ldg(&S.items[it].y);
    long long e0, e1, row = 0;
    int z = -1;
    if (ix >= 0) {
      e0 = rp_load(S.rowptr, ix);
      e1 = rp_load(S.rowptr, iy);
    } else {
      row = -(ix + 1);
      z = __ldg(&S.items[it].z);
      const long long rs = rp_load(S.rowptr, row), re = rp_load(S.rowptr, row + 1);
      e0 = rs + (long long)iy * kChunk;
      e1 = (e0 + kChunk < re) ? e0 + kChunk : re;
    }
    const int len = (int)(e1 - e0);
    int ci[kTileIt];
    T v[kTileIt];
#pragma unroll
    for (int q = 0; q < kTileIt; ++q) {
      const int k = lane + 32 * q;
      ci[q] = 0;
      v[q] = T(0);
      if (k < len) {
        ci[q] = __ldg(S.col + e0 + k);
        v[q] = __ldg(S.val + e0 + k);
      }
    }
#pragma unroll
    for (int q = 0; q < kTileIt; ++q) {
      const int k = lane + 32 * q;
      if (k < len) v[q] *= gather<kReadOnlyU>(u, ci[q]);
    }
    if (ix >= 0) {
      const int nr = iy - (int)ix;
      for (int k = lane; k <= nr; k += 32) srp[k] = (int)(rp_load(S.rowptr, ix + k) - e0);
#pragma unroll
      for (int q = 0; q < kTileIt; ++q) {
        const int k = lane + 32 * q;
        if (k < len) prod[k] = v[q];
      }
      __syncwarp();
      for (int r = lane; r < nr; r += 32) {
        const int b = srp[r], e = srp[r + 1];
        T acc = T(0);
        for (int q = b; q < e; ++q) acc += prod[q];
        fin(ix + r, acc);
      }
      __syncwarp();
    } else {
      T acc = T(0);
#pragma unroll
      for (int q = 0; q < kTileIt; ++q) acc += v[q];
      acc = warp_sum(acc);
      if (lane == 0) {
        if (z < 0) {
          fin(row, acc);
        } else {
          const long long rs = rp_load(S.rowptr, row), re = rp_load(S.rowptr, row + 1);
          const long long base = __ldg(S.mc_base + z);
          const int nch = (int)((re - rs + kChunk - 1) / kChunk);
          S.long_part[base + iy] = acc;
          __threadfence();
          const int ticket = atomicAdd(S.mc_count + z, 1);
          if (ticket == nch - 1) {
            __threadfence();
            T tot = T(0);
            for (int c = 0; c < nch; ++c) tot += *((volatile T*)(S.long_part + base + c));
            S.mc_count[z] = 0;
            fin(row, tot);
          }
        }
      }
    }
  }
}

}  // namespace sa

// Fused CSR SpMV work-list processor shared by the standalone operator, the Lanczos kernel and
// the residual check.
//
// The rows are cut once per matrix (sa_set_matrix) into a work list in row order:
//   * short segments: runs of consecutive rows with at most kShortMax entries each, closed after
//     kSegRows rows or more than kSegElems entries. A warp processes a segment with G lanes per
//     row (G = 4, 8, 16 or 32 from the mean short-row degree); each group reduces with a fixed
//     xor-shuffle tree.
//   * long-row chunks: rows with more than kShortMax entries, cut into chunks of kChunk entries, one
//     warp per chunk. A row of one chunk is finished by its warp. For a row of several chunks
//     every warp stores its partial sum and the warp that finishes last (an atomic ticket per row)
//     adds the partials in chunk order and finishes the row. No spin-waits, and the summation
//     order never depends on timing.
// Warps take work items round robin (item t -> warp t mod warps), so concurrent warps stream
// neighbouring parts of col/val. col, val, rowptr and the work list are read through the
// read-only path; the gathered vector u is written by the same kernel in other phases, so it is
// read with plain loads.
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

// fin(row, sum) is called exactly once per row with sum = sum_j val_ij * u_j (T arithmetic).
template <typename T, typename RP, int G, class Fin>
__device__ __forceinline__ void spmv_items(const SpmvArgs<T, RP>& S, const T* u, long long gwarp,
                                           long long nwarps, Fin&& fin) {
  const int lane = threadIdx.x & 31;
  constexpr int NG = 32 / G;
  const int g = lane / G, gl = lane % G;
  for (long long it = gwarp; it < S.n_items; it += nwarps) {
    const long long ix = __ldg(&S.items[it].x);
    const int iy = __ldg(&S.items[it].y);
    if (ix >= 0) {
      for (long long base = ix; base < iy; base += NG) {
        const long long r = base + g;
        T acc = T(0);
        if (r < iy) {
          const long long rs = rp_load(S.rowptr, r), re = rp_load(S.rowptr, r + 1);
#pragma unroll 4
          for (long long p = rs + gl; p < re; p += G) {
            acc += __ldg(S.val + p) * u[__ldg(S.col + p)];
          }
        }
        acc = group_sum<G>(acc);
        if (r < iy && gl == 0) fin(r, acc);
      }
    } else {
      const long long row = -(ix + 1);
      const int chunk = iy;
      const int z = __ldg(&S.items[it].z);
      const long long rs = rp_load(S.rowptr, row), re = rp_load(S.rowptr, row + 1);
      const long long cb = rs + (long long)chunk * kChunk;
      const long long ce = (cb + kChunk < re) ? cb + kChunk : re;
      T acc = T(0);
#pragma unroll 4
      for (long long p = cb + lane; p < ce; p += 32) acc += __ldg(S.val + p) * u[__ldg(S.col + p)];
      acc = warp_sum(acc);
      if (lane == 0) {
        if (z < 0) {
          fin(row, acc);
        } else {
          const long long base = __ldg(S.mc_base + z);
          const int nch = (int)((re - rs + kChunk - 1) / kChunk);
          S.long_part[base + chunk] = acc;
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

// Dispatch on the short-row group width chosen for the matrix.
template <typename T, typename RP, class Fin>
__device__ __forceinline__ void spmv_dispatch(int group, const SpmvArgs<T, RP>& S, const T* u,
                                              long long gwarp, long long nwarps, Fin&& fin) {
  switch (group) {
    case 4: spmv_items<T, RP, 4>(S, u, gwarp, nwarps, fin); break;
    case 8: spmv_items<T, RP, 8>(S, u, gwarp, nwarps, fin); break;
    case 16: spmv_items<T, RP, 16>(S, u, gwarp, nwarps, fin); break;
    default: spmv_items<T, RP, 32>(S, u, gwarp, nwarps, fin); break;
  }
}

}  // namespace sa

// Fused CSR SpMV work-list processor shared by the standalone operator, the Lanczos kernel and
// the residual check.
//
// The rows are cut once per matrix (sa_set_matrix) into a work list in row order whose items are
// warp tiles of at most kSegMax = 256 stored entries (start offset and length stored in the item):
//   * short segments: runs of consecutive rows with at most kShortMax entries each (at most
//     kSegRows rows);
//   * long-row chunks: rows with more than kShortMax entries cut into chunks of kChunk entries.
// A warp streams a tile's columns and values with kTileIt fully coalesced, independent loads per
// lane (lane l takes entries l, l + 32, ...), gathers u and multiplies. For a segment the products
// go to a per-warp shared buffer and one lane per row adds its contiguous range in order; for a
// chunk the lanes' partial sums are combined by a fixed xor-shuffle tree. A row of one chunk is
// finished by its warp. For a row of several chunks every warp stores its partial sum and the warp
// that finishes last (an atomic ticket per row) adds the partials in chunk order and finishes the
// row. No spin-waits, and no summation order depends on timing.
//
// Warps take items round robin (item t -> warp t mod warps), so concurrent warps stream
// neighbouring parts of col/val. Each warp runs a three-stage software pipeline: the descriptor of
// the tile after next and the columns/values of the next tile are in flight while the current
// tile's gathers and row sums run, so the HBM stream overlaps the gather latency.
// col, val, rowptr and the work list are read through the read-only path. The gathered vector u
// is read through the read-only path too when it is immutable for the whole kernel (kReadOnlyU,
// the standalone operator); the persistent kernels rewrite u between phases, so there it is read
// with ordinary L1-allocating loads, which see the writes of other CTAs because every phase
// boundary is a grid barrier (gpu-scope fence by the waiting thread, then bar.sync).
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
  // Couplings of one magnitude (every |val| == wmag): scol[k] = col[k] with the sign of val[k] in
  // bit 31, streamed instead of col and val (4 bytes per entry instead of 4 + sizeof(T)); null
  // when the magnitudes differ. The products are the same: val[k] is exactly +-wmag.
  const int* scol;
  T wmag;
  // (No default member initialisers: the batch kernel keeps these arguments in shared memory;
  // brace-initialised copies zero the trailing fields.)
};

// Per-warp shared staging of a tile: kSegMax products and kSegRows + 1 row offsets, for CTAs of
// at most NW warps.
template <typename T, int NW = kWarps>
struct SpmvSmem {
  T prod[NW][kSegMax];
  int rp[NW][kSegRows + 1];
};

// L2 cache policies (createpolicy): the streams read once per SpMV (columns, values, descriptors)
// are first in line for eviction and skip L1, so L1 and L2 keep the gathered vector (its hub rows
// are hit again and again; at large n it is about the size of L2), whose gathers are marked
// evict_last.
__device__ __forceinline__ unsigned long long l2_policy_evict_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_policy_evict_last() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ int ld_stream(const int* p, unsigned long long pol) {
  int v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ long long ld_stream(const long long* p, unsigned long long pol) {
  long long v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.s64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p, unsigned long long pol) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p, unsigned long long pol) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

// Gathers of the SpMV's input vector (read-only path when it is immutable for the kernel).
__device__ __forceinline__ float ld_gather(const float* p, unsigned long long pol, bool nc) {
  float v;
  if (nc) asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  else asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_gather(const double* p, unsigned long long pol, bool nc) {
  double v;
  if (nc) asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  else asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

template <bool kReadOnlyU, typename T>
__device__ __forceinline__ T gather(const T* u, int j, unsigned long long pol) {
  return ld_gather(u + j, pol, kReadOnlyU);
}

struct TileDesc {
  long long e0;
  int row;
  int meta;
};

__device__ __forceinline__ TileDesc load_desc(const WorkItem* items, long long t, long long n_items,
                                              unsigned long long pol) {
  TileDesc d{0, 0, 0};
  if (t < n_items) {
    d.e0 = ld_stream(&items[t].e0, pol);
    d.row = ld_stream(&items[t].row, pol);
    d.meta = ld_stream(&items[t].meta, pol);
  }
  return d;
}

template <typename T, typename RP>
__device__ __forceinline__ void load_tile(const SpmvArgs<T, RP>& S, const TileDesc& d, int lane,
                                          int (&ci)[kTileIt], T (&v)[kTileIt], unsigned long long pol) {
  const int len = item_len(d.meta);
  if (S.scol) {
#pragma unroll
    for (int q = 0; q < kTileIt; ++q) {
      const int k = lane + 32 * q;
      ci[q] = 0;
      if (k < len) ci[q] = ld_stream(S.scol + d.e0 + k, pol);
    }
#pragma unroll
    for (int q = 0; q < kTileIt; ++q) {
      v[q] = (ci[q] < 0) ? -S.wmag : S.wmag;
      ci[q] &= 0x7fffffff;
      if (lane + 32 * q >= len) v[q] = T(0);
    }
    return;
  }
#pragma unroll
  for (int q = 0; q < kTileIt; ++q) {
    const int k = lane + 32 * q;
    ci[q] = 0;
    v[q] = T(0);
    if (k < len) {
      ci[q] = ld_stream(S.col + d.e0 + k, pol);
      v[q] = ld_stream(S.val + d.e0 + k, pol);
    }
  }
}

// fin(row, sum) is called exactly once per row with sum = sum_j val_ij * u_j (T arithmetic).
template <typename T, typename RP, bool kReadOnlyU = false, int NW = kWarps, class Fin>
__device__ __forceinline__ void spmv_items(const SpmvArgs<T, RP>& S, const T* u, long long gwarp,
                                           long long nwarps, SpmvSmem<T, NW>& sm, Fin&& fin) {
  const int lane = threadIdx.x & 31;
  const int wid = threadIdx.x >> 5;
  T* prod = sm.prod[wid];
  int* srp = sm.rp[wid];
  const unsigned long long pol_stream = l2_policy_evict_first();
  const unsigned long long pol_gather = l2_policy_evict_last();
  long long it = gwarp;
  TileDesc cur = load_desc(S.items, it, S.n_items, pol_stream);
  int ci[kTileIt];
  T v[kTileIt];
  load_tile(S, cur, lane, ci, v, pol_stream);
  TileDesc nxt = load_desc(S.items, it + nwarps, S.n_items, pol_stream);
  while (it < S.n_items) {
    // stage 1: next tile's entries and the descriptor after it are put in flight
    int cn[kTileIt];
    T vn[kTileIt];
    load_tile(S, nxt, lane, cn, vn, pol_stream);
    const TileDesc nn = load_desc(S.items, it + 2 * nwarps, S.n_items, pol_stream);
    // stage 2: the current tile
    const int len = item_len(cur.meta);
#pragma unroll
    for (int q = 0; q < kTileIt; ++q) {
      const int k = lane + 32 * q;
      if (k < len) v[q] *= gather<kReadOnlyU>(u, ci[q], pol_gather);
    }
    if (cur.row >= 0) {
      const int nr = item_nrows(cur.meta);
      for (int k = lane; k <= nr; k += 32) srp[k] = (int)(rp_load(S.rowptr, cur.row + k) - cur.e0);
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
        fin((long long)cur.row + r, acc);
      }
      __syncwarp();
    } else {
      const long long row = -((long long)cur.row + 1);
      const int z = item_mc(cur.meta);
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
          const int chunk = (int)((cur.e0 - rs) / kChunk);
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
    // rotate the pipeline
    cur = nxt;
    nxt = nn;
#pragma unroll
    for (int q = 0; q < kTileIt; ++q) {
      ci[q] = cn[q];
      v[q] = vn[q];
    }
    it += nwarps;
  }
}

}  // namespace sa

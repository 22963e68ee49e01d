// Instance matrix built on the device from an edge list: the COO -> CSR step of the reference's loader
// (utils/data_loader.py:112-204: both triangles appended edge by edge, coo_matrix(...).tocsr() summing
// duplicates, then _remove_isolated_nodes) for edge lists parsed on the host (loader.cpp's text rules).
//
// Steps (all on the caller's stream, scratch in a caller-owned workspace):
//   1. expand: entry 2e = (i_e, j_e, w_e), entry 2e + 1 = (j_e, i_e, w_e), key = row * nv + col;
//   2. a stable LSD radix sort of (key, entry index), 8 bits per pass over the key bits in use: per
//      tile a histogram, a digit-major scan over the tiles, and a scatter in which each warp walks
//      its part of the tile in order (peers of a digit from __match_any_sync), so equal keys keep
//      their entry order;
//   3. duplicates summed in entry (= file) order, one thread per run of equal keys, in FP64;
//   4. rows whose entries are all zero are removed (when any entry exists), the kept rows renumbered,
//      entries to removed columns dropped; row pointers from the kept entries.
// The result equals the host loader's CSR bit for bit (same summation order).
#include <cstdint>
#include <cstring>
#include <vector>

#include "handle.cuh"

namespace sa {
void count_launches(int k);
}

namespace {

constexpr int kTile = 4096;          // entries per tile of the radix passes
constexpr int kSortThreads = 256;    // 8 warps, 512 entries each
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kPerWarp = kTile / kSortWarps;

#define CO_CUDA(call)                          \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return SA_ERR_CUDA; \
  } while (0)

__global__ void co_expand(const int64_t* ei, const int64_t* ej, long long ne, long long nv, unsigned long long* key,
                          long long* idx) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < ne; e += (long long)gridDim.x * blockDim.x) {
    const long long i = ei[e], j = ej[e];
    key[2 * e] = (unsigned long long)i * (unsigned long long)nv + (unsigned long long)j;
    key[2 * e + 1] = (unsigned long long)j * (unsigned long long)nv + (unsigned long long)i;
    idx[2 * e] = 2 * e;
    idx[2 * e + 1] = 2 * e + 1;
  }
}

// per tile: counts of each digit, stored digit-major (hist[d * ntiles + t])
__global__ void co_hist(const unsigned long long* key, long long E, int shift, long long ntiles, unsigned* hist) {
  __shared__ unsigned cnt[256];
  for (int d = threadIdx.x; d < 256; d += blockDim.x) cnt[d] = 0;
  __syncthreads();
  const long long t = blockIdx.x;
  const long long b = t * kTile, e = min(b + kTile, E);
  for (long long q = b + threadIdx.x; q < e; q += blockDim.x) atomicAdd(&cnt[(key[q] >> shift) & 255u], 1u);
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(long long)d * ntiles + t] = cnt[d];
}

// exclusive scan of hist in digit-major order (one CTA; each thread a contiguous range, then a
// block scan of the range totals)
__global__ void co_scan(const unsigned* hist, long long len, long long* off) {
  __shared__ long long part[1024];
  const long long per = (len + blockDim.x - 1) / blockDim.x;
  const long long b = threadIdx.x * per, e = min(b + per, len);
  long long s = 0;
  for (long long q = b; q < e; ++q) s += hist[q];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int w = 0; w < (int)blockDim.x; ++w) {
      const long long x = part[w];
      part[w] = run;
      run += x;
    }
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (long long q = b; q < e; ++q) {
    off[q] = run;
    run += hist[q];
  }
}

// stable scatter of one tile: warp w walks entries [b + w kPerWarp, ...) in order, 32 at a time
__global__ void __launch_bounds__(kSortThreads) co_scatter(const unsigned long long* key, const long long* idx, long long E,
                                                           int shift, long long ntiles, const long long* off,
                                                           unsigned long long* key_out, long long* idx_out) {
  __shared__ unsigned wcnt[kSortWarps][256];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int d = lane; d < 256; d += 32) wcnt[wid][d] = 0;
  __syncwarp();
  const long long t = blockIdx.x;
  const long long wb = t * kTile + (long long)wid * kPerWarp;
  const long long we = min(wb + kPerWarp, min(t * kTile + kTile, E));
  // pass 1: each warp's digit counts
  for (long long q0 = wb; q0 < we; q0 += 32) {
    const long long q = q0 + lane;
    const bool ok = q < we;
    const unsigned d = ok ? (unsigned)((key[q] >> shift) & 255u) : 256u + lane;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (ok && lane == __ffs(peers) - 1) wcnt[wid][d] += __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // exclusive prefix over the warps, per digit
  for (int d = threadIdx.x; d < 256; d += blockDim.x) {
    unsigned run = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const unsigned x = wcnt[w][d];
      wcnt[w][d] = run;
      run += x;
    }
  }
  __syncthreads();
  // pass 2: positions in entry order
  for (long long q0 = wb; q0 < we; q0 += 32) {
    const long long q = q0 + lane;
    const bool ok = q < we;
    const unsigned long long k = ok ? key[q] : 0ull;
    const unsigned d = ok ? (unsigned)((k >> shift) & 255u) : 256u + lane;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const unsigned rank = __popc(peers & ((1u << lane) - 1u));
    if (ok) {
      const long long dst = off[(long long)d * ntiles + t] + wcnt[wid][d] + rank;
      key_out[dst] = k;
      idx_out[dst] = idx[q];
    }
    __syncwarp();
    if (ok && lane == __ffs(peers) - 1) wcnt[wid][d] += __popc(peers);
    __syncwarp();
  }
}

// heads of runs of equal keys
__global__ void co_heads(const unsigned long long* key, long long E, int* head) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < E; q += (long long)gridDim.x * blockDim.x)
    head[q] = (q == 0 || key[q] != key[q - 1]) ? 1 : 0;
}

// inclusive block-level scan helpers for int counts (one CTA over a whole array)
__global__ void co_scan_int(const int* in, long long len, long long* out_excl, long long* total) {
  __shared__ long long part[1024];
  const long long per = (len + blockDim.x - 1) / blockDim.x;
  const long long b = threadIdx.x * per, e = min(b + per, len);
  long long s = 0;
  for (long long q = b; q < e; ++q) s += in[q];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int w = 0; w < (int)blockDim.x; ++w) {
      const long long x = part[w];
      part[w] = run;
      run += x;
    }
    *total = run;
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (long long q = b; q < e; ++q) {
    out_excl[q] = run;
    run += in[q];
  }
}

// one thread per run: the run's FP64 sum in entry order, its row and column, |sum| into the row's flag
__global__ void co_reduce(const unsigned long long* key, const long long* idx, const double* ew, long long E, long long nv,
                          const int* head, const long long* run_of, long long* urow, int* ucol, double* uval, int* nonzero) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < E; q += (long long)gridDim.x * blockDim.x) {
    if (!head[q]) continue;
    const unsigned long long k = key[q];
    double s = ew[idx[q] >> 1];
    for (long long p = q + 1; p < E && key[p] == k; ++p) s += ew[idx[p] >> 1];
    const long long u = run_of[q];
    const long long r = (long long)(k / (unsigned long long)nv);
    urow[u] = r;
    ucol[u] = (int)(k % (unsigned long long)nv);
    uval[u] = s;
    if (s != 0.0) nonzero[r] = 1;
  }
}

__global__ void co_keep_all(int* keep, long long nv) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nv; q += (long long)gridDim.x * blockDim.x)
    keep[q] = 1;
}

// kept unique entries: flag, then compaction into the CSR arrays
__global__ void co_entry_flags(const long long* urow, const int* ucol, long long U, const int* keep, int* flag) {
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x)
    flag[u] = (keep[urow[u]] && keep[ucol[u]]) ? 1 : 0;
}

__global__ void co_emit(const long long* urow, const int* ucol, const double* uval, long long U, const int* flag,
                        const long long* pos, const long long* newid, int* col, double* val, long long* rowcnt) {
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x) {
    if (!flag[u]) continue;
    const long long p = pos[u];
    col[p] = (int)newid[ucol[u]];
    val[p] = uval[u];
    atomicAdd((unsigned long long*)&rowcnt[newid[urow[u]] + 1], 1ull);
  }
}

__global__ void co_node_ids(const int* keep, const long long* newid, long long nv, long long* node_ids) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < nv; q += (long long)gridDim.x * blockDim.x)
    if (keep[q]) node_ids[newid[q]] = q;
}

// in-place inclusive prefix sum of a[0 .. len) (one CTA: contiguous ranges per thread, then a scan of
// the range totals)
__global__ void co_inclusive(long long* a, long long len) {
  __shared__ long long part[1024];
  const long long per = (len + blockDim.x - 1) / blockDim.x;
  const long long b = threadIdx.x * per, e = min(b + per, len);
  long long s = 0;
  for (long long q = b; q < e; ++q) s += a[q];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long run = 0;
    for (int w = 0; w < (int)blockDim.x; ++w) {
      const long long x = part[w];
      part[w] = run;
      run += x;
    }
  }
  __syncthreads();
  long long run = part[threadIdx.x];
  for (long long q = b; q < e; ++q) {
    run += a[q];
    a[q] = run;
  }
}

struct CooPlan {
  long long E, ntiles, U_cap;
  size_t off_key[2], off_idx[2], off_hist, off_off, off_head, off_run, off_urow, off_ucol, off_uval, off_nz, off_keep,
      off_newid, off_flag, off_pos, off_tot, total;
};

CooPlan coo_plan(long long ne, long long nv) {
  CooPlan P;
  P.E = 2 * ne;
  P.ntiles = (P.E + kTile - 1) / kTile;
  P.U_cap = P.E;
  sa::Layout L;
  const size_t E = (size_t)std::max(1ll, P.E);
  P.off_key[0] = L.off(8 * E);
  P.off_key[1] = L.off(8 * E);
  P.off_idx[0] = L.off(8 * E);
  P.off_idx[1] = L.off(8 * E);
  P.off_hist = L.off(4 * 256 * (size_t)std::max(1ll, P.ntiles));
  P.off_off = L.off(8 * 256 * (size_t)std::max(1ll, P.ntiles));
  P.off_head = L.off(4 * E);
  P.off_run = L.off(8 * E);
  P.off_urow = L.off(8 * E);
  P.off_ucol = L.off(4 * E);
  P.off_uval = L.off(8 * E);
  P.off_nz = L.off(4 * (size_t)std::max(1ll, nv));
  P.off_keep = L.off(4 * (size_t)std::max(1ll, nv));
  P.off_newid = L.off(8 * (size_t)std::max(1ll, nv));
  P.off_flag = L.off(4 * E);
  P.off_pos = L.off(8 * E);
  P.off_tot = L.off(8 * 4);
  P.total = L.total;
  return P;
}

}  // namespace

extern "C" {

int sa_coo_workspace_size(int64_t num_edges, int64_t num_vertices, size_t* bytes) {
  if (!bytes || num_edges < 0 || num_vertices < 1 || num_vertices > (int64_t)INT32_MAX) return SA_ERR_INVALID_ARG;
  *bytes = coo_plan(num_edges, num_vertices).total;
  return SA_OK;
}

int sa_coo_to_csr(int64_t num_edges, int64_t num_vertices, const int64_t* ei, const int64_t* ej, const double* ew,
                  void* workspace, size_t bytes, int64_t* rowptr, int32_t* col, double* val, int64_t* node_ids,
                  int64_t* n_out, int64_t* nnz_out, void* stream) {
  const long long ne = num_edges, nv = num_vertices;
  if (ne < 0 || nv < 1 || nv > (long long)INT32_MAX || !workspace || ((uintptr_t)workspace & 255) || !rowptr ||
      !node_ids || !n_out || !nnz_out || (ne > 0 && (!ei || !ej || !ew || !col || !val)))
    return SA_ERR_INVALID_ARG;
  const CooPlan P = coo_plan(ne, nv);
  if (bytes < P.total) return SA_ERR_OOM;
  cudaStream_t s = (cudaStream_t)stream;
  char* w = (char*)workspace;
  int dev = 0, sms = 0;
  CO_CUDA(cudaGetDevice(&dev));
  CO_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const long long E = P.E;
  auto grid = [&](long long work) { return (int)std::max(1ll, std::min((work + 255) / 256, (long long)sms * 8)); };
  unsigned long long* key[2] = {(unsigned long long*)(w + P.off_key[0]), (unsigned long long*)(w + P.off_key[1])};
  long long* idx[2] = {(long long*)(w + P.off_idx[0]), (long long*)(w + P.off_idx[1])};
  int* keep = (int*)(w + P.off_keep);
  long long* newid = (long long*)(w + P.off_newid);
  long long* tot = (long long*)(w + P.off_tot);
  int cur = 0;
  long long U = 0;
  CO_CUDA(cudaMemsetAsync(w + P.off_nz, 0, 4 * (size_t)nv, s));
  if (E > 0) {
    co_expand<<<grid(ne), 256, 0, s>>>((const int64_t*)ei, (const int64_t*)ej, ne, nv, key[0], idx[0]);
    sa::count_launches(1);
    // key bits in use: keys < nv^2
    const unsigned long long kmax = (unsigned long long)nv * (unsigned long long)nv;
    int bits = 0;
    while (bits < 64 && (kmax - 1) >> bits) ++bits;
    for (int shift = 0; shift < bits; shift += 8) {
      co_hist<<<(unsigned)P.ntiles, 256, 0, s>>>(key[cur], E, shift, P.ntiles, (unsigned*)(w + P.off_hist));
      co_scan<<<1, 1024, 0, s>>>((const unsigned*)(w + P.off_hist), 256 * P.ntiles, (long long*)(w + P.off_off));
      co_scatter<<<(unsigned)P.ntiles, kSortThreads, 0, s>>>(key[cur], idx[cur], E, shift, P.ntiles,
                                                              (const long long*)(w + P.off_off), key[cur ^ 1],
                                                              idx[cur ^ 1]);
      sa::count_launches(3);
      cur ^= 1;
    }
    int* head = (int*)(w + P.off_head);
    long long* run = (long long*)(w + P.off_run);
    co_heads<<<grid(E), 256, 0, s>>>(key[cur], E, head);
    co_scan_int<<<1, 1024, 0, s>>>(head, E, run, tot);
    co_reduce<<<grid(E), 256, 0, s>>>(key[cur], idx[cur], ew, E, nv, head, run, (long long*)(w + P.off_urow),
                                      (int*)(w + P.off_ucol), (double*)(w + P.off_uval), (int*)(w + P.off_nz));
    sa::count_launches(3);
    CO_CUDA(cudaMemcpyAsync(&U, tot, 8, cudaMemcpyDeviceToHost, s));
    CO_CUDA(cudaStreamSynchronize(s));
  }
  // isolated rows: removed only when the matrix has entries (as the reference)
  long long nk = nv;
  if (U > 0) {
    CO_CUDA(cudaMemcpyAsync(keep, w + P.off_nz, 4 * (size_t)nv, cudaMemcpyDeviceToDevice, s));
  } else {
    co_keep_all<<<grid(nv), 256, 0, s>>>(keep, nv);
    sa::count_launches(1);
  }
  co_scan_int<<<1, 1024, 0, s>>>(keep, nv, newid, tot + 1);
  sa::count_launches(1);
  CO_CUDA(cudaMemcpyAsync(&nk, tot + 1, 8, cudaMemcpyDeviceToHost, s));
  CO_CUDA(cudaStreamSynchronize(s));
  if (nk > (long long)INT32_MAX) return SA_ERR_INVALID_ARG;
  CO_CUDA(cudaMemsetAsync(rowptr, 0, 8 * (size_t)(nk + 1), s));
  long long nnz = 0;
  if (U > 0) {
    int* flag = (int*)(w + P.off_flag);
    long long* pos = (long long*)(w + P.off_pos);
    co_entry_flags<<<grid(U), 256, 0, s>>>((const long long*)(w + P.off_urow), (const int*)(w + P.off_ucol), U, keep, flag);
    co_scan_int<<<1, 1024, 0, s>>>(flag, U, pos, tot + 2);
    co_emit<<<grid(U), 256, 0, s>>>((const long long*)(w + P.off_urow), (const int*)(w + P.off_ucol),
                                    (const double*)(w + P.off_uval), U, flag, pos, newid, col, val, (long long*)rowptr);
    co_inclusive<<<1, 1024, 0, s>>>((long long*)rowptr + 1, nk);
    sa::count_launches(4);
    CO_CUDA(cudaMemcpyAsync(&nnz, tot + 2, 8, cudaMemcpyDeviceToHost, s));
  }
  co_node_ids<<<grid(nv), 256, 0, s>>>(keep, newid, nv, (long long*)node_ids);
  sa::count_launches(1);
  CO_CUDA(cudaGetLastError());
  CO_CUDA(cudaStreamSynchronize(s));
  *n_out = nk;
  *nnz_out = nnz;
  return SA_OK;
}

}  // extern "C"

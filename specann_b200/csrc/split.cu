// L2 column splits of the operator, for gathered vectors larger than L2.
//
// When u = sigma * x no longer fits in L2 (n = 2^25 in FP32: 134 MB against 126 MB of L2), most random
// gathers of the work-list SpMV go to DRAM. Cutting the columns into S ranges whose slice of u fits in
// L2 (at most 48 MB each) and applying the operator as S work-list passes, one per range, keeps the
// gathers of every pass in L2. Each pass adds its row sums to a partial vector; the last pass hands
// the total to the caller's epilogue (in the persistent kernels a grid barrier separates the passes;
// the standalone operator runs them as successive launches). The summation order is fixed (pass
// after pass, each pass as the work list).
//
// Layout (sa_split_build, on the device): per split s a CSR of the entries with a column in range s
// (row pointers of the handle's type, the entries of every row in CSR order, packed signed columns when
// every coupling has one magnitude, else columns and values), and its work list (built on the host
// from the split's row pointers, as for the whole matrix).
#include <algorithm>
#include <cmath>
#include <vector>

#include "handle.cuh"
#include "spmv.cuh"

namespace sa {
void count_launches(int k);
}

using namespace sa;

namespace {

#define SP_CUDA(call)                          \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return SA_ERR_CUDA; \
  } while (0)

constexpr double kSplitBytes = 48.0 * 1024 * 1024;   // slice of u per split
constexpr int kScanBlock = 1024;                    // rows per block of the row-pointer scan

struct SplitPlan {
  int S = 0;
  long long width = 0;   // columns per split (the last may be shorter)
  size_t off_cnt = 0, off_rp = 0, off_col = 0, off_val = 0, off_items = 0, off_mcb = 0, off_mcc = 0,
         off_lp = 0, off_part = 0, off_tot = 0, total = 0;
  long long cap_items = 0, cap_mc = 0, cap_lp = 0;
};

int auto_splits(const sa_handle* h) {
  const double bytes = (double)h->n * (h->prec == 32 ? 4.0 : 8.0);
  return (int)std::min<double>(kMaxSplits, std::max(1.0, std::ceil(bytes / kSplitBytes)));
}

int plan_splits(const sa_handle* h, int S, SplitPlan* pl) {
  if (S < 2 || S > kMaxSplits) return SA_ERR_INVALID_ARG;
  const size_t T = h->prec == 32 ? 4 : 8, RP = h->rp64 ? 8 : 4;
  const bool uniform = h->wmag > 0.0;
  const long long n = h->n, nnz = std::max(1ll, h->nnz);
  pl->S = S;
  pl->width = (n + S - 1) / S;
  // work-list bounds summed over the splits (each split has n rows and nnz_s entries)
  pl->cap_items = (long long)S * (n / kSegRows + 8) + max_items(0, nnz);
  pl->cap_mc = max_multichunk_rows(nnz) + S;
  pl->cap_lp = max_long_partials(nnz) + 2 * S;
  Layout L;
  pl->off_cnt = L.off(4 * (size_t)S * (size_t)(n + 1));
  pl->off_rp = L.off(RP * (size_t)S * (size_t)(n + 1));
  pl->off_col = L.off(4 * (size_t)nnz);
  pl->off_val = uniform ? 0 : L.off(T * (size_t)nnz);
  pl->off_items = L.off(sizeof(WorkItem) * (size_t)pl->cap_items);
  pl->off_mcb = L.off(8 * (size_t)pl->cap_mc);
  pl->off_mcc = L.off(4 * (size_t)pl->cap_mc);
  pl->off_lp = L.off(T * (size_t)pl->cap_lp);
  pl->off_part = L.off(T * (size_t)n);
  pl->off_tot = L.off(8 * (size_t)(n / kScanBlock + 2) * S);
  pl->total = L.total;
  return SA_OK;
}

// entries of every row in each split: a warp per row
template <typename RP>
__global__ void sp_count(const RP* rp, const int* col, long long n, int S, long long width, int* cnt) {
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    int c[kMaxSplits];
#pragma unroll
    for (int q = 0; q < kMaxSplits; ++q) c[q] = 0;
    for (long long k = rp_load(rp, r) + lane; k < rp_load(rp, r + 1); k += 32) {
      const int s = (int)(__ldg(col + k) / width);
#pragma unroll
      for (int q = 0; q < kMaxSplits; ++q) c[q] += (q == s) ? 1 : 0;
    }
#pragma unroll
    for (int q = 0; q < kMaxSplits; ++q) {
      const int v = warp_sum(c[q]);
      if (lane == 0 && q < S) cnt[(long long)q * (n + 1) + r] = v;
    }
  }
}

// row pointers of every split from its counts (exclusive scan of n + 1 values with cnt[n] = 0):
// block sums, a scan of the block sums (one CTA per split), the block scans with their offsets
__global__ void sp_scan_blocks(const int* cnt, long long n1, long long nblk, long long* tot) {
  __shared__ long long sm[kScanBlock / 32];
  const int s = blockIdx.y;
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  long long v = (i < n1) ? cnt[(long long)s * n1 + i] : 0;
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long t = 0;
    for (int q = 0; q < kScanBlock / 32; ++q) t += sm[q];
    tot[(long long)s * nblk + blockIdx.x] = t;
  }
}

__global__ void sp_scan_totals(long long* tot, long long nblk) {
  const int s = blockIdx.x;
  if (threadIdx.x == 0) {
    long long run = 0;
    for (long long b = 0; b < nblk; ++b) {
      const long long v = tot[(long long)s * nblk + b];
      tot[(long long)s * nblk + b] = run;
      run += v;
    }
  }
}

template <typename RP>
__global__ void sp_scan_rows(const int* cnt, long long n1, long long nblk, const long long* tot, RP* rp_out) {
  __shared__ long long sm[kScanBlock];
  const int s = blockIdx.y;
  const long long i = (long long)blockIdx.x * kScanBlock + threadIdx.x;
  sm[threadIdx.x] = (i < n1) ? cnt[(long long)s * n1 + i] : 0;
  __syncthreads();
  // inclusive Hillis-Steele scan of the block
  for (int d = 1; d < kScanBlock; d <<= 1) {
    const long long t = (threadIdx.x >= (unsigned)d) ? sm[threadIdx.x - d] : 0;
    __syncthreads();
    sm[threadIdx.x] += t;
    __syncthreads();
  }
  // exclusive value at i = inclusive at i - the count at i
  if (i < n1) {
    const long long excl = sm[threadIdx.x] - (long long)cnt[(long long)s * n1 + i];
    rp_out[(long long)s * n1 + i] = (RP)(tot[(long long)s * nblk + blockIdx.x] + excl);
  }
}

// entries to their split, in CSR order within every row: a warp per row
template <typename T, typename RP>
__global__ void sp_scatter(const RP* rp, const int* col, const T* val, long long n, int S, long long width,
                           const RP* rps, long long n1, const long long* base, int uniform, int* cols, T* vals) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    long long pos[kMaxSplits];
#pragma unroll
    for (int q = 0; q < kMaxSplits; ++q) pos[q] = (q < S) ? base[q] + (long long)rps[(long long)q * n1 + r] : 0;
    const long long b = rp_load(rp, r), e = rp_load(rp, r + 1);
    for (long long k0 = b; k0 < e; k0 += 32) {
      const long long k = k0 + lane;
      const bool ok = k < e;
      const int c = ok ? __ldg(col + k) : 0;
      const int s = ok ? (int)(c / width) : -1;
      long long dst = -1;
#pragma unroll
      for (int q = 0; q < kMaxSplits; ++q) {
        const unsigned m = __ballot_sync(0xffffffffu, s == q);
        if (s == q) dst = pos[q] + __popc(m & lt);
        pos[q] += __popc(m);
      }
      if (ok) {
        const T v = __ldg(val + k);
        if (uniform) {
          cols[dst] = c | ((v < T(0)) ? (int)0x80000000u : 0);
        } else {
          cols[dst] = c;
          vals[dst] = v;
        }
      }
    }
  }
}

// one pass of the standalone operator: mode 0 writes the partial sums, 1 adds to them, 2 finishes
// y = rho x - sigma (partial + this pass)
template <typename T, typename RP>
__global__ void __launch_bounds__(kThreads, 2) split_spmv_kernel(SpmvArgs<T, RP> S, int mode, const T* u, const T* x,
                                                               const T* sigma, T rho, T* part, T* y) {
  __shared__ SpmvSmem<T> ssp;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  spmv_items<T, RP, true>(S, u, gtid >> 5, nthreads >> 5, ssp, [&](long long r, T acc) {
    if (mode == 0) part[r] = acc;
    else if (mode == 1) part[r] = part[r] + acc;
    else y[r] = rho * x[r] - sigma[r] * (part[r] + acc);
  });
}

template <typename T, typename RP>
int build_splits(sa_handle* h, const SplitPlan& pl, char* base) {
  const int S = pl.S;
  const long long n = h->n, n1 = n + 1, nblk = (n1 + kScanBlock - 1) / kScanBlock;
  const bool uniform = h->wmag > 0.0;
  int* cnt = (int*)(base + pl.off_cnt);
  RP* rps = (RP*)(base + pl.off_rp);
  long long* tot = (long long*)(base + pl.off_tot);
  const RP* rp = (const RP*)h->rowptr;
  const int g = h->sm_count * 8;
  SP_CUDA(cudaMemsetAsync(cnt, 0, 4 * (size_t)S * (size_t)n1, h->stream));
  sp_count<RP><<<g, 256, 0, h->stream>>>(rp, h->col, n, S, pl.width, cnt);
  sp_scan_blocks<<<dim3((unsigned)nblk, S), kScanBlock, 0, h->stream>>>(cnt, n1, nblk, tot);
  sp_scan_totals<<<S, 32, 0, h->stream>>>(tot, nblk);
  sp_scan_rows<RP><<<dim3((unsigned)nblk, S), kScanBlock, 0, h->stream>>>(cnt, n1, nblk, tot, rps);
  count_launches(4);
  SP_CUDA(cudaGetLastError());
  // host: every split's row pointers (work lists) and entry counts (offsets of the column arrays)
  std::vector<std::vector<long long>> hrp(S, std::vector<long long>((size_t)n1));
  std::vector<RP> tmp((size_t)n1);
  std::vector<long long> off(S + 1, 0);
  for (int s = 0; s < S; ++s) {
    SP_CUDA(cudaMemcpyAsync(tmp.data(), rps + (size_t)s * n1, sizeof(RP) * (size_t)n1, cudaMemcpyDeviceToHost, h->stream));
    SP_CUDA(cudaStreamSynchronize(h->stream));
    for (long long i = 0; i < n1; ++i) hrp[s][(size_t)i] = (long long)tmp[(size_t)i];
    off[s + 1] = off[s] + hrp[s][(size_t)n];
  }
  if (off[S] != h->nnz) return SA_ERR_INVALID_ARG;
  long long* d_off = tot;   // the scan totals are no longer needed
  SP_CUDA(cudaMemcpyAsync(d_off, off.data(), 8 * (size_t)S, cudaMemcpyHostToDevice, h->stream));
  int* cols = (int*)(base + pl.off_col);
  T* vals = uniform ? nullptr : (T*)(base + pl.off_val);
  sp_scatter<T, RP><<<g, 256, 0, h->stream>>>(rp, h->col, (const T*)h->val, n, S, pl.width, rps, n1, d_off,
                                               uniform ? 1 : 0, cols, vals);
  count_launches(1);
  SP_CUDA(cudaGetLastError());
  // work lists
  WorkItem* items = (WorkItem*)(base + pl.off_items);
  long long* mcb = (long long*)(base + pl.off_mcb);
  int* mcc = (int*)(base + pl.off_mcc);
  T* lp = (T*)(base + pl.off_lp);
  long long used_items = 0, used_mc = 0, used_lp = 0;
  double bytes = 0.0;
  for (int s = 0; s < S; ++s) {
    std::vector<WorkItem> it;
    std::vector<long long> mc;
    long long npart = 0;
    double mean_short = 0.0;
    build_items(hrp[s], n, it, mc, &npart, &mean_short);
    if (used_items + (long long)it.size() > pl.cap_items || used_mc + (long long)mc.size() > pl.cap_mc ||
        used_lp + npart > pl.cap_lp)
      return SA_ERR_OOM;
    // the work items address the split's own arrays: entry offsets are relative to the split
    if (!it.empty())
      SP_CUDA(cudaMemcpyAsync(items + used_items, it.data(), sizeof(WorkItem) * it.size(), cudaMemcpyHostToDevice, h->stream));
    if (!mc.empty()) {
      SP_CUDA(cudaMemcpyAsync(mcb + used_mc, mc.data(), 8 * mc.size(), cudaMemcpyHostToDevice, h->stream));
      SP_CUDA(cudaMemsetAsync(mcc + used_mc, 0, 4 * mc.size(), h->stream));
    }
    auto& d = h->split[s];
    d.rowptr = rps + (size_t)s * n1;
    d.col = cols + off[s];
    d.val = uniform ? nullptr : (const void*)(vals + off[s]);
    d.items = items + used_items;
    d.n_items = (long long)it.size();
    d.nnz = off[s + 1] - off[s];
    d.mc_base = mcb + used_mc;
    d.mc_count = mcc + used_mc;
    d.long_part = lp + used_lp;
    used_items += (long long)it.size();
    used_mc += (long long)mc.size();
    used_lp += npart;
    bytes += (double)d.nnz * (uniform ? 4.0 : 4.0 + sizeof(T)) + (double)n1 * sizeof(RP) +
             (double)d.n_items * sizeof(WorkItem);
  }
  SP_CUDA(cudaStreamSynchronize(h->stream));
  h->split_part = base + pl.off_part;
  h->split_bytes = bytes + 2.0 * (double)(S - 1) * (double)n * sizeof(T);
  h->n_splits = S;
  return SA_OK;
}

template <typename T, typename RP>
SpmvArgs<T, RP> split_args_t(const sa_handle* h, int s) {
  const auto& d = h->split[s];
  SpmvArgs<T, RP> A{};
  A.rowptr = (const RP*)d.rowptr;
  A.col = d.val ? d.col : nullptr;
  A.val = (const T*)d.val;
  A.items = d.items;
  A.n_items = d.n_items;
  A.mc_base = d.mc_base;
  A.mc_count = d.mc_count;
  A.long_part = (T*)d.long_part;
  A.scol = d.val ? nullptr : d.col;
  A.wmag = (T)h->wmag;
  return A;
}

template <typename T, typename RP>
int launch_split_spmv(sa_handle* h, const T* u, const T* x, const T* sigma, double rho, T* y) {
  const int gs = h->sm_count * 2;
  for (int s = 0; s < h->n_splits; ++s) {
    const int mode = (s == 0) ? 0 : (s + 1 < h->n_splits ? 1 : 2);
    split_spmv_kernel<T, RP><<<gs, kThreads, 0, h->stream>>>(split_args_t<T, RP>(h, s), mode, u, x, sigma, (T)rho,
                                                              (T*)h->split_part, y);
  }
  count_launches(h->n_splits);
  SP_CUDA(cudaGetLastError());
  return SA_OK;
}

}  // namespace

namespace sa {

// Per-split operator arguments for the persistent kernels.
template <typename T, typename RP>
SpmvArgs<T, RP> split_args(const sa_handle* h, int s) {
  return split_args_t<T, RP>(h, s);
}
template SpmvArgs<float, int> split_args<float, int>(const sa_handle*, int);
template SpmvArgs<float, long long> split_args<float, long long>(const sa_handle*, int);
template SpmvArgs<double, int> split_args<double, int>(const sa_handle*, int);
template SpmvArgs<double, long long> split_args<double, long long>(const sa_handle*, int);

// The standalone operator through the column splits (sa_spmv_scaled when they are on).
int split_spmv_launch(sa_handle* h, const void* u, const void* x, const void* sigma, double rho, void* y) {
  if (h->prec == 32)
    return h->rp64 ? launch_split_spmv<float, long long>(h, (const float*)u, (const float*)x, (const float*)sigma, rho, (float*)y)
                   : launch_split_spmv<float, int>(h, (const float*)u, (const float*)x, (const float*)sigma, rho, (float*)y);
  return h->rp64 ? launch_split_spmv<double, long long>(h, (const double*)u, (const double*)x, (const double*)sigma, rho, (double*)y)
                 : launch_split_spmv<double, int>(h, (const double*)u, (const double*)x, (const double*)sigma, rho, (double*)y);
}

}  // namespace sa

extern "C" {

int sa_split_workspace_size(sa_handle* h, int32_t splits, size_t* bytes, int32_t* splits_used) {
  if (!h || !h->bound || !bytes || splits < 0 || splits > kMaxSplits) return SA_ERR_INVALID_ARG;
  const int S = splits ? splits : std::max(2, auto_splits(h));
  SplitPlan pl;
  const int st = plan_splits(h, S, &pl);
  if (st != SA_OK) return st;
  *bytes = pl.total;
  if (splits_used) *splits_used = S;
  return SA_OK;
}

int sa_split_build(sa_handle* h, int32_t splits, void* workspace, size_t bytes) {
  if (!h || !h->bound || !workspace || ((uintptr_t)workspace & 255) || splits < 0 || splits > kMaxSplits)
    return SA_ERR_INVALID_ARG;
  const int S = splits ? splits : std::max(2, auto_splits(h));
  SplitPlan pl;
  int st = plan_splits(h, S, &pl);
  if (st != SA_OK) return st;
  if (bytes < pl.total) return SA_ERR_OOM;
  h->split_ready = h->split_on = 0;
  if (h->prec == 32) st = h->rp64 ? build_splits<float, long long>(h, pl, (char*)workspace) : build_splits<float, int>(h, pl, (char*)workspace);
  else st = h->rp64 ? build_splits<double, long long>(h, pl, (char*)workspace) : build_splits<double, int>(h, pl, (char*)workspace);
  if (st != SA_OK) return st;
  h->split_ready = 1;
  h->split_on = 1;
  h->panel_on = 0;
  return SA_OK;
}

int sa_split_enable(sa_handle* h, int32_t on) {
  if (!h || (on && !h->split_ready)) return SA_ERR_INVALID_ARG;
  h->split_on = on ? 1 : 0;
  if (on) h->panel_on = 0;
  return SA_OK;
}

int sa_split_count(sa_handle* h, int32_t* splits, double* matrix_bytes) {
  if (!h || !splits) return SA_ERR_INVALID_ARG;
  *splits = h->split_on ? h->n_splits : 0;
  if (matrix_bytes) *matrix_bytes = h->split_on ? h->split_bytes : 0.0;
  return SA_OK;
}

}  // extern "C"

// C-ABI entry points of libspecann_b200.so: handle and workspace, matrix set-up (prelude of the
// reference solve), the standalone fused SpMV, rounding, and the candidate store.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "handle.cuh"
#include "spmv.cuh"

#include <atomic>

namespace sa {
static std::atomic<unsigned long long> g_launches{0};
void count_launches(int k) { g_launches.fetch_add((unsigned long long)k, std::memory_order_relaxed); }
int alpha_solve_impl(sa_handle* h, const sa_alpha_params* p);
const void* alpha_kernel_for(int prec, int rp64);
const void* ls_kernel_for(int prec, int rp64, int integer);
size_t ls_workspace_bytes(long long n, long long nnz, int k, int integer);
int ls_run_impl(sa_handle* h, const sa_ls_params* p, void* ws, size_t bytes, double* eb, double* ea,
                sa_ls_result* res);
}  // namespace sa

using namespace sa;

#define SA_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return SA_ERR_CUDA;          \
  } while (0)

namespace sa {
int panel_spmv_launch(sa_handle* h, const void* u, const void* x, const void* sigma, double rho, void* y);
int split_spmv_launch(sa_handle* h, const void* u, const void* x, const void* sigma, double rho, void* y);
}

namespace {

struct Carve {
  size_t sigma, ld, deg, V, w, u, y0, y1, y2, items, mc_base, mc_count, long_part, blk_part, actrl, red,
      cand, refined, scratch, dense, scol, total;
};

constexpr int kMaxBlocks = 1024;
constexpr int kPartWidth = 2 * kNcvMax + kDotBatch + 8;

Carve carve(long long n, long long nnz, int prec, int ncv_max, int max_cand) {
  const size_t T = prec == 32 ? 4 : 8;
  const long long ldv = (n + 63) & ~63ll;
  const long long W = (n + 31) / 32;
  Layout L;
  Carve c;
  c.sigma = L.off(T * n);
  c.ld = L.off(8 * n);
  c.deg = L.off(8 * n);
  c.V = L.off(T * (size_t)ldv * ncv_max);
  c.w = L.off(T * n);
  c.u = L.off(T * n);
  c.y0 = L.off(T * n);
  c.y1 = L.off(T * n);
  c.y2 = L.off(T * n);
  c.items = L.off(sizeof(WorkItem) * (size_t)max_items(n, nnz));
  c.mc_base = L.off(8 * (size_t)max_multichunk_rows(nnz));
  c.mc_count = L.off(4 * (size_t)max_multichunk_rows(nnz));
  c.long_part = L.off(T * (size_t)max_long_partials(nnz));
  c.blk_part = L.off(8 * (size_t)kMaxBlocks * kPartWidth);
  c.actrl = L.off(sizeof(AlphaCtrl));
  c.red = L.off(8 * 64);
  c.cand = L.off(4 * (size_t)W * max_cand);
  c.refined = L.off(4 * (size_t)W * max_cand);
  c.scratch = L.off(4 * (size_t)W);
  c.dense = L.off(8 * 2 * (size_t)kNcvMax * kNcvMax);
  c.scol = L.off(4 * (size_t)std::max(1ll, nnz));
  c.total = L.total;
  return c;
}

// ---- set-up kernels ---------------------------------------------------------------------------

struct DegRed {
  unsigned long long dmax_bits, dmin_bits;
  int nonint;
  int badcol;   // a column index outside [0, n)
};

template <typename T, typename RP>
__global__ void degree_kernel(const RP* rp, const int* col, const T* val, long long n, double* deg, DegRed* red) {
  __shared__ unsigned long long s_max, s_min;
  __shared__ int s_nonint;
  if (threadIdx.x == 0) { s_max = 0ull; s_min = ~0ull; s_nonint = 0; }
  __syncthreads();
  unsigned long long lmax = 0ull, lmin = ~0ull;
  int nonint = 0, badcol = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long b = rp_load(rp, i), e = rp_load(rp, i + 1);
    double s = 0.0;
    for (long long p = b; p < e; ++p) {
      const int cidx = __ldg(col + p);
      if (cidx < 0 || (long long)cidx >= n) badcol = 1;
      const double v = (double)__ldg(val + p);
      s += fabs(v);
      if (!(v == rint(v)) || fabs(v) > 16777216.0) nonint = 1;
    }
    deg[i] = s;
    const unsigned long long bits = __double_as_longlong(s);
    lmax = bits > lmax ? bits : lmax;
    lmin = bits < lmin ? bits : lmin;
  }
  atomicMax(&s_max, lmax);
  atomicMin(&s_min, lmin);
  if (nonint) s_nonint = 1;
  if (badcol) atomicOr(&red->badcol, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicMax(&red->dmax_bits, s_max);
    atomicMin(&red->dmin_bits, s_min);
    if (s_nonint) atomicOr(&red->nonint, 1);
  }
}

// Packed signed columns for couplings of one magnitude w: scol[k] = col[k] | sign(val[k]) << 31;
// *mixed is set when some |val[k]| differs from w (then scol is not used).
template <typename T>
__global__ void pack_kernel(const int* col, const T* val, long long nnz, T w, int* scol, int* mixed) {
  int bad = 0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += (long long)gridDim.x * blockDim.x) {
    const T v = __ldg(val + k);
    if (!(fabs(v) == w)) bad = 1;
    scol[k] = __ldg(col + k) | ((v < T(0)) ? (int)0x80000000u : 0);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(mixed, 1);
}

__global__ void logdeg_kernel(const double* deg, long long n, double c, double* ld) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double d = deg[i] / c;
    ld[i] = d > 0.0 ? log2(d) : -INFINITY;
  }
}

// sigma = D^{-1/2} / sqrt(c) for this alpha and u = sigma * x.
template <typename T>
__global__ void scale_kernel(const double* ld, long long n, double alpha, double half_log2_c, const T* x,
                             T* sigma, T* u) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double logD = (alpha == 0.0) ? 0.0 : alpha * (double)ld[i];
    const double logDc = fmax(logD, -39.86313713864835);
    const T s = (T)exp2(-0.5 * logDc - half_log2_c);
    sigma[i] = s;
    u[i] = s * x[i];
  }
}

template <typename T, typename RP>
__global__ void __launch_bounds__(kThreads, 2) spmv_kernel(SpmvArgs<T, RP> S, int group, const T* u, const T* x,
                                                         const T* sigma, T rho, T* y) {
  __shared__ SpmvSmem<T> ssp;
  const long long gtid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nthreads = (long long)gridDim.x * blockDim.x;
  spmv_items<T, RP, true>(S, u, gtid >> 5, nthreads >> 5, ssp, [&](long long r, T acc) {
    y[r] = rho * x[r] - sigma[r] * acc;
  });
}

// Norm and alignment dot of a vector (for sa_round_vector).
template <typename T>
__global__ void norm_dot_kernel(const T* y, const T* yl, long long n, int use_last, double* out) {
  __shared__ double sm[kWarps];
  double a = 0.0, b = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)y[i];
    a += v * v;
    if (use_last) b += v * (double)yl[i];
  }
  a = block_sum(a, sm);
  b = block_sum(b, sm);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = a;
    out[2 * blockIdx.x + 1] = b;
  }
}

__device__ __forceinline__ unsigned long long word_mix_host(long long widx, unsigned int word) {
  return splitmix64(((unsigned long long)widx << 32) ^ (unsigned long long)word ^ 0xA5A5000000000000ull);
}

template <typename T>
__global__ void round_kernel(const T* y, long long n, double alpha, double half_log2_c, double sqrt_c,
                             const double* ld, T scale, T* yout, uint32_t* bits, unsigned long long* sig) {
  const long long nr = (n + 31) & ~31ll;
  unsigned long long hs = 0ull;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nr; i += (long long)gridDim.x * blockDim.x) {
    bool bit = false;
    if (i < n) {
      const double logD = (alpha == 0.0) ? 0.0 : alpha * (double)ld[i];
      const double logDc = fmax(logD, -39.86313713864835);
      const T sg = (T)exp2(-0.5 * logDc - half_log2_c);
      const T yv = (T)(y[i] * scale);
      yout[i] = yv;
      const T x = yv * (T)((double)sg * sqrt_c);
      bit = x >= T(0);
    }
    const unsigned int word = __ballot_sync(0xffffffffu, bit);
    if ((threadIdx.x & 31) == 0) {
      bits[i >> 5] = word;
      hs += word_mix_host(i >> 5, word);
    }
  }
  if ((threadIdx.x & 31) == 0 && hs) atomicAdd(sig, hs);
}

__global__ void compare_kernel(const uint32_t* a, const uint32_t* b, long long W, int* differ) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < W; i += (long long)gridDim.x * blockDim.x)
    if (a[i] != b[i]) *differ = 1;
}

__global__ void unpack_kernel(const uint32_t* bits, long long n, int8_t* out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = ((bits[i >> 5] >> (i & 31)) & 1u) ? (int8_t)1 : (int8_t)-1;
}

// One bounded grid barrier of `expected` arrivals (sa_barrier_selftest): bit 0 of out[block] is the
// barrier's result in that CTA, bit 1 is set in the CTA that ran the epilogue.
__global__ void barrier_selftest_kernel(GridSync* gs, unsigned expected, unsigned long long spin_limit, int* out) {
  __shared__ int s_epi;
  if (threadIdx.x == 0) s_epi = 0;
  const bool ok = grid_barrier_n(gs, expected, [&] { if (threadIdx.x == 0) s_epi = 1; }, spin_limit);
  if (threadIdx.x == 0) out[blockIdx.x] = (ok ? 1 : 0) | (s_epi ? 2 : 0);
}

int grid_for(long long work, int threads, int sm_count) {
  long long b = (work + threads - 1) / threads;
  const long long cap = (long long)sm_count * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

// Work list (host): short segments and long-row chunks in row order.
}  // namespace

namespace sa {

// SpMV work list of a CSR (host row pointers): see max_items for the bound.
void build_items(const std::vector<long long>& rp, long long n, std::vector<WorkItem>& items,
                 std::vector<long long>& mc_base, long long* n_long_part, double* mean_short) {
  items.clear();
  mc_base.clear();
  long long part = 0, seg_begin = -1, seg_rows = 0, seg_elems = 0;
  long long short_rows = 0, short_elems = 0;
  auto flush = [&](long long end) {
    if (seg_begin >= 0)
      items.push_back(WorkItem{rp[seg_begin], (int)seg_begin, (int)((rp[end] - rp[seg_begin]) | ((end - seg_begin) << 9))});
    seg_begin = -1;
    seg_rows = 0;
    seg_elems = 0;
  };
  for (long long r = 0; r < n; ++r) {
    const long long d = rp[r + 1] - rp[r];
    if (d > kShortMax) {
      flush(r);
      const long long nch = (d + kChunk - 1) / kChunk;
      int zcode = 0;
      if (nch > 1) {
        zcode = (int)mc_base.size() + 1;
        mc_base.push_back(part);
        part += nch;
      }
      for (long long c = 0; c < nch; ++c) {
        const long long len = std::min<long long>(kChunk, d - c * kChunk);
        items.push_back(WorkItem{rp[r] + c * kChunk, (int)(-(r + 1)), (int)(len | ((long long)zcode << 9))});
      }
    } else {
      if (seg_begin >= 0 && seg_elems + d > kSegMax) flush(r);
      if (seg_begin < 0) seg_begin = r;
      ++seg_rows;
      seg_elems += d;
      ++short_rows;
      short_elems += d;
      if (seg_rows >= kSegRows) flush(r + 1);
    }
  }
  flush(n);
  *n_long_part = part;
  *mean_short = short_rows ? (double)short_elems / (double)short_rows : 0.0;
}

}  // namespace sa

template <typename T, typename RP>
static void set_policy(SpmvArgs<T, RP>& S, const sa_handle* h) {
  S.scol = h->packed ? h->scol : nullptr;
  S.wmag = (T)h->wmag;
}

extern "C" {

const char* sa_version(void) { return "specann_b200 0.1 (sm_100a)"; }

uint64_t sa_kernel_launches(void) { return (uint64_t)g_launches.load(std::memory_order_relaxed); }

int sa_workspace_size(int64_t n, int64_t nnz, int32_t rowptr64, int32_t precision, int32_t ncv_max,
                      int32_t max_candidates, size_t* bytes) {
  (void)rowptr64;
  if (!bytes || n < 1 || nnz < 0 || (precision != 32 && precision != 64) || ncv_max < 2 ||
      ncv_max > kNcvMax || max_candidates < 1 || max_candidates > 128 || n > INT32_MAX)
    return SA_ERR_INVALID_ARG;
  *bytes = carve(n, nnz, precision, ncv_max, max_candidates).total;
  return SA_OK;
}

int sa_create(sa_handle** out, int64_t n, int64_t nnz, int32_t rowptr64, int32_t precision, int32_t ncv_max,
              int32_t max_candidates, void* workspace, size_t workspace_bytes, void* stream) {
  if (!out) return SA_ERR_INVALID_ARG;
  *out = nullptr;
  size_t need = 0;
  int st = sa_workspace_size(n, nnz, rowptr64, precision, ncv_max, max_candidates, &need);
  if (st != SA_OK) return st;
  if (!rowptr64 && nnz > INT32_MAX) return SA_ERR_INVALID_ARG;
  if (!workspace || workspace_bytes < need) return SA_ERR_OOM;
  if (((uintptr_t)workspace) & 255) return SA_ERR_INVALID_ARG;
  sa_handle* h = new sa_handle();
  h->n = n;
  h->nnz = nnz;
  h->rp64 = rowptr64 ? 1 : 0;
  h->prec = precision;
  h->ncv_max = ncv_max;
  h->max_cand = max_candidates;
  h->stream = (cudaStream_t)stream;
  h->ws = (char*)workspace;
  h->ws_bytes = workspace_bytes;
  const Carve c = carve(n, nnz, precision, ncv_max, max_candidates);
  h->ldv = (n + 63) & ~63ll;
  h->W = (n + 31) / 32;
  h->sigma = h->ws + c.sigma;
  h->ld = (double*)(h->ws + c.ld);
  h->deg = (double*)(h->ws + c.deg);
  h->V = h->ws + c.V;
  h->w = h->ws + c.w;
  h->u = h->ws + c.u;
  h->yv[0] = h->ws + c.y0;
  h->yv[1] = h->ws + c.y1;
  h->yv[2] = h->ws + c.y2;
  h->items = (WorkItem*)(h->ws + c.items);
  h->cap_items = max_items(n, nnz);
  h->mc_base = (long long*)(h->ws + c.mc_base);
  h->mc_count = (int*)(h->ws + c.mc_count);
  h->cap_mc = max_multichunk_rows(nnz);
  h->long_part = h->ws + c.long_part;
  h->cap_long_part = max_long_partials(nnz);
  h->blk_part = (double*)(h->ws + c.blk_part);
  h->blk_part_width = kPartWidth;
  h->actrl = (AlphaCtrl*)(h->ws + c.actrl);
  h->red = (double*)(h->ws + c.red);
  h->cand = (uint32_t*)(h->ws + c.cand);
  h->refined = (uint32_t*)(h->ws + c.refined);
  h->scratch = (uint32_t*)(h->ws + c.scratch);
  h->dense = (double*)(h->ws + c.dense);
  h->scol = (int32_t*)(h->ws + c.scol);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) { delete h; return SA_ERR_CUDA; }
  if (cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) { delete h; return SA_ERR_CUDA; }
  int occ_a = 0, occ_l = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a, alpha_kernel_for(precision, h->rp64), kThreads, 0) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_l, ls_kernel_for(precision, h->rp64, 1), kThreads, 0) != cudaSuccess) {
    delete h;
    return SA_ERR_CUDA;
  }
  int occ_l2 = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_l2, ls_kernel_for(precision, h->rp64, 0), kThreads, 0) != cudaSuccess) {
    delete h;
    return SA_ERR_CUDA;
  }
  int occ = std::min(std::min(occ_a, occ_l), occ_l2);
  occ = std::min(occ, 2);
  if (occ < 1) { delete h; return SA_ERR_CUDA; }
  h->max_blocks = std::min(h->sm_count * occ, kMaxBlocks);
  h->blocks = h->max_blocks;
  if (cudaMemsetAsync(h->red, 0, 8 * 64, h->stream) != cudaSuccess) { delete h; return SA_ERR_CUDA; }
  *out = h;
  return SA_OK;
}

int sa_destroy(sa_handle* h) {
  delete h;
  return SA_OK;
}

int sa_operator_status(sa_handle* h, int32_t* status) {
  if (!h || !status) return SA_ERR_INVALID_ARG;
  int* word = operator_status_word(h);
  int v = 0;
  SA_CUDA(cudaMemcpyAsync(&v, word, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  SA_CUDA(cudaMemsetAsync(word, 0, sizeof(int), h->stream));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  *status = v;
  return SA_OK;
}

int sa_barrier_selftest(int32_t blocks, int32_t expected, uint64_t spin_limit, void* scratch, size_t scratch_bytes,
                        int32_t* status, int32_t* passed_blocks, int32_t* epilogues, void* stream) {
  int dev = 0, sms = 0;
  SA_CUDA(cudaGetDevice(&dev));
  SA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (blocks < 1 || blocks > sms || expected < 1 || spin_limit < 1 || spin_limit > kSpinLimit || !scratch ||
      ((uintptr_t)scratch & 15) || scratch_bytes < sizeof(GridSync) + 4 * (size_t)blocks || !status ||
      !passed_blocks || !epilogues)
    return SA_ERR_INVALID_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  GridSync* gs = (GridSync*)scratch;
  int* out = (int*)((char*)scratch + sizeof(GridSync));
  SA_CUDA(cudaMemsetAsync(scratch, 0, sizeof(GridSync) + 4 * (size_t)blocks, st));
  barrier_selftest_kernel<<<blocks, 128, 0, st>>>(gs, (unsigned)expected, (unsigned long long)spin_limit, out);
  count_launches(1);
  SA_CUDA(cudaGetLastError());
  GridSync g;
  std::vector<int> flags(blocks);
  SA_CUDA(cudaMemcpyAsync(&g, gs, sizeof(GridSync), cudaMemcpyDeviceToHost, st));
  SA_CUDA(cudaMemcpyAsync(flags.data(), out, 4 * (size_t)blocks, cudaMemcpyDeviceToHost, st));
  SA_CUDA(cudaStreamSynchronize(st));
  int passed = 0, epi = 0;
  for (int b = 0; b < blocks; ++b) {
    passed += flags[b] & 1;
    epi += (flags[b] >> 1) & 1;
  }
  *status = g.error;
  *passed_blocks = passed;
  *epilogues = epi;
  return SA_OK;
}

int sa_set_matrix(sa_handle* h, const void* rowptr, const int32_t* col, const void* val, double* norm_c,
                  double* d_min, double* d_max, int32_t* integer_couplings) {
  if (!h || !rowptr || (!col && h->nnz > 0) || (!val && h->nnz > 0)) return SA_ERR_INVALID_ARG;
  h->rowptr = rowptr;
  h->col = col;
  h->val = val;
  // row pointers to the host first: validated before any kernel reads through them
  std::vector<long long> rp(h->n + 1);
  if (h->rp64) {
    SA_CUDA(cudaMemcpyAsync(rp.data(), rowptr, sizeof(long long) * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
    SA_CUDA(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<int> rp32(h->n + 1);
    SA_CUDA(cudaMemcpyAsync(rp32.data(), rowptr, sizeof(int) * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
    SA_CUDA(cudaStreamSynchronize(h->stream));
    for (long long i = 0; i <= h->n; ++i) rp[i] = rp32[i];
  }
  if (rp[0] != 0 || rp[h->n] != h->nnz) return SA_ERR_INVALID_ARG;
  for (long long i = 0; i < h->n; ++i)
    if (rp[i + 1] < rp[i]) return SA_ERR_INVALID_ARG;
  DegRed init{0ull, ~0ull, 0, 0};
  DegRed* dred = (DegRed*)h->red;
  SA_CUDA(cudaMemcpyAsync(dred, &init, sizeof(DegRed), cudaMemcpyHostToDevice, h->stream));
  const int g = grid_for(h->n, 256, h->sm_count);
  if (h->prec == 32) {
    if (h->rp64) degree_kernel<float, long long><<<g, 256, 0, h->stream>>>((const long long*)rowptr, col, (const float*)val, h->n, h->deg, dred);
    else degree_kernel<float, int><<<g, 256, 0, h->stream>>>((const int*)rowptr, col, (const float*)val, h->n, h->deg, dred);
    count_launches(1);
  } else {
    if (h->rp64) degree_kernel<double, long long><<<g, 256, 0, h->stream>>>((const long long*)rowptr, col, (const double*)val, h->n, h->deg, dred);
    else degree_kernel<double, int><<<g, 256, 0, h->stream>>>((const int*)rowptr, col, (const double*)val, h->n, h->deg, dred);
    count_launches(1);
  }
  SA_CUDA(cudaGetLastError());
  DegRed r;
  SA_CUDA(cudaMemcpyAsync(&r, dred, sizeof(DegRed), cudaMemcpyDeviceToHost, h->stream));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  if (r.badcol) return SA_ERR_INVALID_ARG;
  double dmax, dmin;
  memcpy(&dmax, &r.dmax_bits, 8);
  memcpy(&dmin, &r.dmin_bits, 8);
  h->c = dmax;
  h->dmax = dmax > 0 ? 1.0 : 0.0;
  h->dmin = dmax > 0 ? dmin / dmax : 0.0;
  h->integer_J = (r.nonint == 0 && dmax < 1073741824.0) ? 1 : 0;
  if (!(dmax > 0.0) || !std::isfinite(dmax)) return SA_ERR_INVALID_ARG;
  logdeg_kernel<<<g, 256, 0, h->stream>>>(h->deg, h->n, h->c, h->ld);
  count_launches(1);
  SA_CUDA(cudaGetLastError());
  // one coupling magnitude: the SpMV streams packed signed columns instead of col and val
  h->wmag = 0.0;
  h->packed = 0;
  if (h->nnz > 0) {
    int* mixed = (int*)(h->red + 16);
    double w0 = 0.0;
    SA_CUDA(cudaMemsetAsync(mixed, 0, sizeof(int), h->stream));
    const int gp = grid_for(h->nnz, 256, h->sm_count);
    if (h->prec == 32) {
      float f0 = 0.0f;
      SA_CUDA(cudaMemcpyAsync(&f0, val, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
      SA_CUDA(cudaStreamSynchronize(h->stream));
      w0 = std::fabs((double)f0);
      pack_kernel<float><<<gp, 256, 0, h->stream>>>(col, (const float*)val, h->nnz, (float)w0, h->scol, mixed);
    } else {
      SA_CUDA(cudaMemcpyAsync(&w0, val, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
      SA_CUDA(cudaStreamSynchronize(h->stream));
      w0 = std::fabs(w0);
      pack_kernel<double><<<gp, 256, 0, h->stream>>>(col, (const double*)val, h->nnz, w0, h->scol, mixed);
    }
    count_launches(1);
    SA_CUDA(cudaGetLastError());
    int mx = 1;
    SA_CUDA(cudaMemcpyAsync(&mx, mixed, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    SA_CUDA(cudaStreamSynchronize(h->stream));
    if (!mx && w0 > 0.0 && std::isfinite(w0)) h->wmag = w0;
    h->packed = (h->wmag > 0.0 && h->packed_allowed) ? 1 : 0;
  }
  std::vector<WorkItem> items;
  std::vector<long long> mc_base;
  long long n_part = 0;
  double mean_short = 0.0;
  build_items(rp, h->n, items, mc_base, &n_part, &mean_short);
  if ((long long)items.size() > h->cap_items || (long long)mc_base.size() > h->cap_mc || n_part > h->cap_long_part)
    return SA_ERR_OOM;
  h->n_items = (long long)items.size();
  h->n_mc = (long long)mc_base.size();
  h->n_long_part = n_part;
  if (!items.empty())
    SA_CUDA(cudaMemcpyAsync(h->items, items.data(), sizeof(WorkItem) * items.size(), cudaMemcpyHostToDevice, h->stream));
  if (!mc_base.empty()) {
    SA_CUDA(cudaMemcpyAsync(h->mc_base, mc_base.data(), 8 * mc_base.size(), cudaMemcpyHostToDevice, h->stream));
    SA_CUDA(cudaMemsetAsync(h->mc_count, 0, 4 * mc_base.size(), h->stream));
  }
  const double target = mean_short / 3.0;
  h->group = target <= 4.0 ? 4 : (target <= 8.0 ? 8 : (target <= 16.0 ? 16 : 32));
  const long long want = std::max((h->n_items + 7) / 8, (h->n + 2047) / 2048);
  h->blocks = (int)std::max(1ll, std::min((long long)h->max_blocks, want));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  h->bound = true;
  h->panel_ready = h->panel_on = 0;
  h->split_ready = h->split_on = 0;
  h->has_last = h->has_prev = false;
  if (norm_c) *norm_c = h->c;
  if (d_min) *d_min = h->dmin;
  if (d_max) *d_max = h->dmax;
  if (integer_couplings) *integer_couplings = h->integer_J;
  return SA_OK;
}

int sa_set_spmv_policy(sa_handle* h, int32_t packed_columns) {
  if (!h || (packed_columns != 0 && packed_columns != 1)) return SA_ERR_INVALID_ARG;
  h->packed_allowed = packed_columns;
  h->packed = (h->bound && h->wmag > 0.0 && packed_columns) ? 1 : 0;
  return SA_OK;
}

int sa_get_spmv_policy(sa_handle* h, int32_t* packed_columns, double* magnitude) {
  if (!h) return SA_ERR_INVALID_ARG;
  if (packed_columns) *packed_columns = h->packed;
  if (magnitude) *magnitude = h->wmag;
  return SA_OK;
}

int sa_spmv_scaled(sa_handle* h, double alpha, double rho, const void* x, void* y) {
  if (!h || !h->bound || !x || !y) return SA_ERR_INVALID_ARG;
  const int g = grid_for(h->n, 256, h->sm_count);
  const double hl = 0.5 * std::log2(h->c);
  const int gs = h->sm_count * 2;
  if (h->panel_on || h->split_on) {
    if (h->prec == 32)
      scale_kernel<float><<<g, 256, 0, h->stream>>>(h->ld, h->n, alpha, hl, (const float*)x, (float*)h->sigma, (float*)h->u);
    else
      scale_kernel<double><<<g, 256, 0, h->stream>>>(h->ld, h->n, alpha, hl, (const double*)x, (double*)h->sigma, (double*)h->u);
    count_launches(1);
    SA_CUDA(cudaGetLastError());
    return h->panel_on ? panel_spmv_launch(h, h->u, x, h->sigma, rho, y) : split_spmv_launch(h, h->u, x, h->sigma, rho, y);
  }
  if (h->n_mc) SA_CUDA(cudaMemsetAsync(h->mc_count, 0, 4 * h->n_mc, h->stream));
  if (h->prec == 32) {
    scale_kernel<float><<<g, 256, 0, h->stream>>>(h->ld, h->n, alpha, hl, (const float*)x, (float*)h->sigma, (float*)h->u);
    count_launches(1);
    SpmvArgs<float, int> S32;
    SpmvArgs<float, long long> S64;
    if (h->rp64) {
      S64 = SpmvArgs<float, long long>{(const long long*)h->rowptr, h->col, (const float*)h->val, h->items, h->n_items, h->mc_base, h->mc_count, (float*)h->long_part};
      set_policy(S64, h);
      spmv_kernel<float, long long><<<gs, kThreads, 0, h->stream>>>(S64, h->group, (const float*)h->u, (const float*)x, (const float*)h->sigma, (float)rho, (float*)y);
      count_launches(1);
    } else {
      S32 = SpmvArgs<float, int>{(const int*)h->rowptr, h->col, (const float*)h->val, h->items, h->n_items, h->mc_base, h->mc_count, (float*)h->long_part};
      set_policy(S32, h);
      spmv_kernel<float, int><<<gs, kThreads, 0, h->stream>>>(S32, h->group, (const float*)h->u, (const float*)x, (const float*)h->sigma, (float)rho, (float*)y);
      count_launches(1);
    }
  } else {
    scale_kernel<double><<<g, 256, 0, h->stream>>>(h->ld, h->n, alpha, hl, (const double*)x, (double*)h->sigma, (double*)h->u);
    count_launches(1);
    if (h->rp64) {
      SpmvArgs<double, long long> S{(const long long*)h->rowptr, h->col, (const double*)h->val, h->items, h->n_items, h->mc_base, h->mc_count, (double*)h->long_part};
      set_policy(S, h);
      spmv_kernel<double, long long><<<gs, kThreads, 0, h->stream>>>(S, h->group, (const double*)h->u, (const double*)x, (const double*)h->sigma, rho, (double*)y);
      count_launches(1);
    } else {
      SpmvArgs<double, int> S{(const int*)h->rowptr, h->col, (const double*)h->val, h->items, h->n_items, h->mc_base, h->mc_count, (double*)h->long_part};
      set_policy(S, h);
      spmv_kernel<double, int><<<gs, kThreads, 0, h->stream>>>(S, h->group, (const double*)h->u, (const double*)x, (const double*)h->sigma, rho, (double*)y);
      count_launches(1);
    }
  }
  SA_CUDA(cudaGetLastError());
  return SA_OK;
}

int sa_alpha_solve(sa_handle* h, const sa_alpha_params* p, sa_alpha_record* rec) {
  if (!h || !h->bound || !p || !rec) return SA_ERR_INVALID_ARG;
  if (p->ncv < 2 || p->ncv > h->ncv_max || p->ncv > std::max<long long>(2, h->n) || p->maxiter < 1)
    return SA_ERR_INVALID_ARG;
  const int m = p->start_mode;
  if (m < SA_START_RANDOM || m > SA_START_TANGENT) return SA_ERR_INVALID_ARG;
  if ((m == SA_START_PREV || m == SA_START_DIAGONAL || m == SA_START_SECANT || m == SA_START_TANGENT) && !h->has_last)
    return SA_ERR_INVALID_ARG;
  if ((m == SA_START_GIVEN || m == SA_START_TANGENT) && !p->v0) return SA_ERR_INVALID_ARG;
  SA_CUDA(cudaMemsetAsync(h->actrl, 0, sizeof(GridSync), h->stream));
  if (h->n_mc) SA_CUDA(cudaMemsetAsync(h->mc_count, 0, 4 * h->n_mc, h->stream));
  int st = alpha_solve_impl(h, p);
  if (st != SA_OK) return st;
  AlphaCtrl ctl;
  SA_CUDA(cudaMemcpyAsync(&ctl, h->actrl, sizeof(AlphaCtrl), cudaMemcpyDeviceToHost, h->stream));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  memset(rec, 0, sizeof(*rec));
  rec->status = ctl.gs.error ? ctl.gs.error : ctl.status;
  if (ctl.nonfinite && rec->status == SA_OK) rec->status = SA_ERR_NONFINITE;
  rec->iterations = ctl.iters;
  rec->restarts = ctl.restarts;
  rec->pred_accepted = ctl.pred_accepted;
  rec->pred_residual = ctl.pred_residual;
  rec->mu = ctl.theta;
  rec->lambda1 = p->rho - ctl.theta;
  rec->residual = p->residual_check ? (ctl.nrm_y > 0 ? std::sqrt(ctl.rr) / ctl.nrm_y : NAN) : NAN;
  rec->res_estimate = ctl.res_est;
  rec->degree_scale = ctl.degree_scale;
  rec->align_dot = ctl.align_dot;
  rec->signature = ctl.sig;
  rec->nonfinite = ctl.nonfinite;
  rec->basis_used = ctl.j + 1;
  rec->spmv_count = ctl.spmvs;
  rec->alg_bytes = ctl.bytes;
  for (int q = 0; q < 6; ++q) rec->phase_ms[q] = (double)ctl.tph[q] * 1e-6;
  if (rec->status != SA_OK && std::getenv("SPECANN_DEBUG")) {
    std::fprintf(stderr, "[specann] alpha_solve status %d: j=%d iters=%d restarts=%d action=%d theta=%.17g ww=%.6g inv_b=%.6g\n",
                 rec->status, ctl.j, ctl.iters, ctl.restarts, ctl.action, ctl.theta, ctl.ww, ctl.inv_b);
    for (int i = 0; i <= ctl.j && i < kNcvMax; ++i)
      std::fprintf(stderr, "  a[%d]=%.17g b[%d]=%.17g h[%d]=%.17g\n", i, ctl.a[i], i, ctl.b[i], i, ctl.h[i]);
  }
  return SA_OK;
}

int sa_result_vector(sa_handle* h, const void** y) {
  if (!h || !y) return SA_ERR_INVALID_ARG;
  *y = h->yv[h->iy_out];
  return SA_OK;
}

int sa_commit_alpha(sa_handle* h) {
  if (!h) return SA_ERR_INVALID_ARG;
  const int old_prev = h->iy_prev;
  h->iy_prev = h->iy_last;
  h->iy_last = h->iy_out;
  h->iy_out = old_prev;
  h->has_prev = h->has_last;
  h->has_last = true;
  return SA_OK;
}

int sa_set_last_vector(sa_handle* h, const void* y) {
  if (!h || !y) return SA_ERR_INVALID_ARG;
  const size_t T = h->prec == 32 ? 4 : 8;
  SA_CUDA(cudaMemcpyAsync(h->yv[h->iy_last], y, T * h->n, cudaMemcpyDeviceToDevice, h->stream));
  h->has_last = true;
  h->has_prev = false;
  return SA_OK;
}

int sa_round_vector(sa_handle* h, double alpha, const void* y, int32_t align, uint64_t* signature) {
  if (!h || !h->bound || !y) return SA_ERR_INVALID_ARG;
  const int g = std::min(grid_for(h->n, 256, h->sm_count), 512);
  double* part = h->blk_part;
  const int use_last = (align && h->has_last) ? 1 : 0;
  if (h->prec == 32) norm_dot_kernel<float><<<g, 256, 0, h->stream>>>((const float*)y, (const float*)h->yv[h->iy_last], h->n, use_last, part);
  else norm_dot_kernel<double><<<g, 256, 0, h->stream>>>((const double*)y, (const double*)h->yv[h->iy_last], h->n, use_last, part);
  count_launches(1);
  SA_CUDA(cudaGetLastError());
  std::vector<double> hp(2 * g);
  SA_CUDA(cudaMemcpyAsync(hp.data(), part, sizeof(double) * 2 * g, cudaMemcpyDeviceToHost, h->stream));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  double a = 0, b = 0;
  for (int i = 0; i < g; ++i) { a += hp[2 * i]; b += hp[2 * i + 1]; }
  const double nrm = std::sqrt(a);
  const double sg = (use_last && b < 0.0) ? -1.0 : 1.0;
  const double scale = nrm > 0 ? sg / nrm : sg;
  unsigned long long* sig = (unsigned long long*)h->red;
  SA_CUDA(cudaMemsetAsync(sig, 0, 8, h->stream));
  const double hl = 0.5 * std::log2(h->c), sc = std::sqrt(h->c);
  if (h->prec == 32) round_kernel<float><<<g, 256, 0, h->stream>>>((const float*)y, h->n, alpha, hl, sc, h->ld, (float)scale, (float*)h->yv[h->iy_out], h->scratch, sig);
  else round_kernel<double><<<g, 256, 0, h->stream>>>((const double*)y, h->n, alpha, hl, sc, h->ld, scale, (double*)h->yv[h->iy_out], h->scratch, sig);
  count_launches(1);
  SA_CUDA(cudaGetLastError());
  unsigned long long s = 0;
  SA_CUDA(cudaMemcpyAsync(&s, sig, 8, cudaMemcpyDeviceToHost, h->stream));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  if (signature) *signature = s;
  return SA_OK;
}

int sa_candidate_keep(sa_handle* h, int32_t slot) {
  if (!h || slot < 0 || slot >= h->max_cand) return SA_ERR_INVALID_ARG;
  SA_CUDA(cudaMemcpyAsync(h->cand + (size_t)slot * h->W, h->scratch, 4 * h->W, cudaMemcpyDeviceToDevice, h->stream));
  return SA_OK;
}

int sa_candidate_equal(sa_handle* h, int32_t slot, int32_t* equal) {
  if (!h || !equal || slot < 0 || slot >= h->max_cand) return SA_ERR_INVALID_ARG;
  int* flag = (int*)h->red;
  SA_CUDA(cudaMemsetAsync(flag, 0, 4, h->stream));
  compare_kernel<<<grid_for(h->W, 256, h->sm_count), 256, 0, h->stream>>>(h->cand + (size_t)slot * h->W, h->scratch, h->W, flag);
  count_launches(1);
  SA_CUDA(cudaGetLastError());
  int d = 0;
  SA_CUDA(cudaMemcpyAsync(&d, flag, 4, cudaMemcpyDeviceToHost, h->stream));
  SA_CUDA(cudaStreamSynchronize(h->stream));
  *equal = d ? 0 : 1;
  return SA_OK;
}

int sa_candidate_set(sa_handle* h, int32_t slot, const uint32_t* packed_device) {
  if (!h || !packed_device || slot < 0 || slot >= h->max_cand) return SA_ERR_INVALID_ARG;
  SA_CUDA(cudaMemcpyAsync(h->cand + (size_t)slot * h->W, packed_device, 4 * h->W, cudaMemcpyDeviceToDevice, h->stream));
  return SA_OK;
}

int sa_candidate_get(sa_handle* h, int32_t slot, int32_t refined, uint32_t* packed_device) {
  if (!h || !packed_device || slot < -1 || slot >= h->max_cand) return SA_ERR_INVALID_ARG;
  const uint32_t* src = slot < 0 ? h->scratch : (refined ? h->refined : h->cand) + (size_t)slot * h->W;
  SA_CUDA(cudaMemcpyAsync(packed_device, src, 4 * h->W, cudaMemcpyDeviceToDevice, h->stream));
  return SA_OK;
}

int sa_candidate_unpack(sa_handle* h, int32_t slot, int32_t refined, int8_t* spins_device) {
  if (!h || !spins_device || slot < -1 || slot >= h->max_cand) return SA_ERR_INVALID_ARG;
  const uint32_t* src = slot < 0 ? h->scratch : (refined ? h->refined : h->cand) + (size_t)slot * h->W;
  unpack_kernel<<<grid_for(h->n, 256, h->sm_count), 256, 0, h->stream>>>(src, h->n, spins_device);
  count_launches(1);
  SA_CUDA(cudaGetLastError());
  return SA_OK;
}

int sa_ls_workspace_size(sa_handle* h, int32_t k, size_t* bytes) {
  if (!h || !bytes || k < 1 || k > 128) return SA_ERR_INVALID_ARG;
  *bytes = ls_workspace_bytes(h->n, h->nnz, k, h->integer_J);
  return SA_OK;
}

int sa_local_search(sa_handle* h, const sa_ls_params* p, void* ls_workspace, size_t ls_bytes,
                    double* energies_before, double* energies_after, sa_ls_result* result) {
  if (!h || !h->bound || !p || !ls_workspace || p->k < 1 || p->first_slot < 0 ||
      p->first_slot + p->k > h->max_cand || p->max_iterations < 0 || p->semantics < 0 || p->semantics > 1 ||
      p->num_rounds < 0 || p->final_sweep_iters < 0)
    return SA_ERR_INVALID_ARG;
  if (((uintptr_t)ls_workspace) & 255) return SA_ERR_INVALID_ARG;
  return ls_run_impl(h, p, ls_workspace, ls_bytes, energies_before, energies_after, result);
}

int sa_energies(sa_handle* h, int32_t k, void* ls_workspace, size_t ls_bytes, double* energies) {
  sa_ls_params p;
  memset(&p, 0, sizeof(p));
  p.k = k;
  p.max_iterations = 0;
  p.subset_fraction = 1.0;
  p.final_sweep_fraction = 1.0;
  p.final_sweep_iters = 0;
  p.num_rounds = 0;
  p.seed = 0;
  return sa_local_search(h, &p, ls_workspace, ls_bytes, energies, nullptr, nullptr);
}

}  // extern "C"

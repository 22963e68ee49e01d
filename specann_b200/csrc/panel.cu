// Column-panel SpMV: the layout builder (on the device) and the standalone panel operator kernel.
//
// sa_panel_workspace_size / sa_panel_build lay the bound matrix out as panel segments (see
// panel.cuh) in a caller-owned workspace; sa_panel_enable switches the handle's operator kernels to
// the panel SpMV. The row blocks are cut on the host from the row pointers (a binary search per
// block); everything per entry runs on the device in five launches:
//   1. pl_words: each entry's 32-bit word (row in block, sign, column in panel), in CSR order;
//   2. pl_sort: per block, a stable counting sort of the words by panel (one CTA per block, 512
//      entries per round in CSR order; ranks from warp match-any and per-warp panel counts);
//   3. pl_pieces (twice: count, then write): every segment, in row order, packed into pieces of
//      at most kPanelBatchEntries entries: rows are added whole while they fit, a row longer than
//      a piece fills whole pieces; every piece is padded to kPanelBatchEntries slots, so a warp
//      processes exactly one piece per batch. The segment's pieces are cut into kWarps contiguous
//      runs, one per warp (a cut never separates the pieces of one row);
//   4. pl_scan: the pieces' offsets (one CTA);
//   5. pl_copy: the pieces copied to their slots, padding words appended.
// The layout is a deterministic function of the CSR (stable sort, fixed cut rule).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "handle.cuh"
#include "panel.cuh"

namespace sa {
void count_launches(int k);
}

using namespace sa;

namespace {

#define PN_CUDA(call)                          \
  do {                                         \
    cudaError_t e_ = (call);                   \
    if (e_ != cudaSuccess) return SA_ERR_CUDA; \
  } while (0)

constexpr int kPlMaxPanels = 256;   // panels the device builder supports (smem of pl_sort)

struct PanelPlan {
  std::vector<int> row0;   // block first rows (n_blocks + 1)
  int n_panels = 0, width = 0;
  long long chunks = 0;    // n_blocks * n_panels * kWarps
  long long max_pieces = 0;
  size_t cap = 0;          // entry slots, padding included (upper bound)
  // final layout
  size_t off_ent = 0, off_val = 0, off_chunk = 0, off_row0 = 0;
  // build scratch
  size_t off_w = 0, off_ws = 0, off_vs = 0, off_seg = 0, off_npc = 0, off_pbase = 0, off_pstart = 0, off_plen = 0;
  size_t total = 0;
};

// Row blocks of about nnz / SMs entries and at most max_rows rows (block b ends at the first row
// whose entry offset reaches (b + 1) nnz / SMs, or after max_rows rows); panels of `width` columns.
int plan_panels(const sa_handle* h, const std::vector<long long>& rp, PanelPlan* pl) {
  const size_t T = h->prec == 32 ? 4 : 8;
  const long long max_rows = std::min<long long>(kPanelRowBytes / (long long)T, 65535);
  pl->width = (int)(panel_buf_bytes((int)T) / T);
  pl->n_panels = (int)((h->n + pl->width - 1) / pl->width);
  if (pl->n_panels > kPlMaxPanels) return SA_ERR_INVALID_ARG;
  const double target = (double)h->nnz / (double)std::max(1, h->sm_count);
  pl->row0.assign(1, 0);
  long long start = 0;
  int b = 0;
  while (start < h->n) {
    const double goal = target * (double)(b + 1);
    // first row index in [start + 1, n) whose offset reaches the goal, else n
    const long long idx =
        std::lower_bound(rp.begin() + start + 1, rp.begin() + h->n, goal,
                         [](long long v, double g) { return (double)v < g; }) - rp.begin();
    const long long end = std::min(std::min(idx, start + max_rows), h->n);
    pl->row0.push_back((int)end);
    start = end;
    ++b;
  }
  const long long nb = (long long)pl->row0.size() - 1;
  pl->chunks = nb * pl->n_panels * kWarps;
  // a piece that is closed before it is full is longer than kPanelBatchEntries together with the
  // row that follows it, so a segment of L entries has at most 2 L / kPanelBatchEntries + 1 pieces
  const long long nseg = nb * pl->n_panels;
  pl->max_pieces = 2 * (std::max(1ll, h->nnz) / kPanelBatchEntries) + nseg + 1;
  pl->cap = (size_t)pl->max_pieces * kPanelBatchEntries;
  const bool uniform = h->wmag > 0.0;
  const size_t nz = (size_t)std::max(1ll, h->nnz);
  Layout L;
  pl->off_ent = L.off(4 * pl->cap);
  pl->off_val = uniform ? 0 : L.off(T * pl->cap);
  pl->off_chunk = L.off(8 * ((size_t)pl->chunks + 1));
  pl->off_row0 = L.off(4 * (size_t)(nb + 1));
  pl->off_w = L.off(4 * nz);
  pl->off_ws = L.off(4 * nz);
  pl->off_vs = uniform ? 0 : L.off(T * nz);
  pl->off_seg = L.off(4 * (size_t)nseg);
  pl->off_npc = L.off(4 * (size_t)nseg);
  pl->off_pbase = L.off(8 * ((size_t)nseg + 1));
  pl->off_pstart = L.off(8 * (size_t)pl->max_pieces);
  pl->off_plen = L.off(4 * (size_t)pl->max_pieces);
  pl->total = L.total;
  return SA_OK;
}

int host_rowptr(const sa_handle* h, std::vector<long long>& rp) {
  rp.resize(h->n + 1);
  if (h->rp64) {
    PN_CUDA(cudaMemcpyAsync(rp.data(), h->rowptr, 8 * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
    PN_CUDA(cudaStreamSynchronize(h->stream));
  } else {
    std::vector<int> r32(h->n + 1);
    PN_CUDA(cudaMemcpyAsync(r32.data(), h->rowptr, 4 * (h->n + 1), cudaMemcpyDeviceToHost, h->stream));
    PN_CUDA(cudaStreamSynchronize(h->stream));
    for (long long i = 0; i <= h->n; ++i) rp[i] = r32[i];
  }
  return SA_OK;
}

// ---- device builder ------------------------------------------------------------------------

// 1. words in CSR order; a warp per row
template <typename T, typename RP>
__global__ void pl_words(const RP* rp, const int* col, const T* val, long long n, const int* row0, int nb, int width,
                         unsigned* W) {
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long r = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < n; r += nw) {
    int lo = 0, hi = nb;   // row0[lo] <= r < row0[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (__ldg(row0 + mid) <= r) lo = mid;
      else hi = mid;
    }
    const unsigned rl = (unsigned)(r - __ldg(row0 + lo)) << 16;
    const long long b = rp_load(rp, r), e = rp_load(rp, r + 1);
    for (long long k = b + lane; k < e; k += 32) {
      const int c = __ldg(col + k);
      W[k] = rl | ((__ldg(val + k) < T(0)) ? 0x8000u : 0u) | (unsigned)(c % width);
    }
  }
}

// 2. stable counting sort of one block's words by panel (CTA b = block b, kThreads threads)
template <typename T, typename RP>
__global__ void __launch_bounds__(kThreads) pl_sort(const RP* rp, const int* col, const T* val, const unsigned* W,
                                                    const int* row0, int np, int width, int with_val, unsigned* Ws,
                                                    T* Vs, int* seg_len) {
  __shared__ int run[kPlMaxPanels];
  __shared__ int wcnt[kWarps][kPlMaxPanels];
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const long long e0 = rp_load(rp, __ldg(row0 + b)), e1 = rp_load(rp, __ldg(row0 + b + 1));
  for (int p = tid; p < np; p += blockDim.x) run[p] = 0;
  __syncthreads();
  for (long long k = e0 + tid; k < e1; k += blockDim.x) atomicAdd(&run[__ldg(col + k) / width], 1);
  __syncthreads();
  if (tid == 0) {
    int s = 0;
    for (int p = 0; p < np; ++p) {
      const int c = run[p];
      seg_len[(long long)b * np + p] = c;
      run[p] = s;
      s += c;
    }
  }
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (long long base = e0; base < e1; base += blockDim.x) {
    const long long k = base + tid;
    const bool ok = k < e1;
    const int p = ok ? __ldg(col + k) / width : np;
    const unsigned m = __match_any_sync(0xffffffffu, p);
    const int rank = __popc(m & lt);
    for (int q = lane; q < np; q += 32) wcnt[wid][q] = 0;
    __syncwarp();
    if (ok && rank == 0) wcnt[wid][p] = __popc(m);
    __syncthreads();
    int off = 0;
    if (ok) {
      for (int w = 0; w < wid; ++w) off += wcnt[w][p];
      off += run[p] + rank;
    }
    __syncthreads();
    for (int q = tid; q < np; q += blockDim.x) {
      int s = 0;
      for (int w = 0; w < kWarps; ++w) s += wcnt[w][q];
      run[q] += s;
    }
    if (ok) {
      Ws[e0 + off] = W[k];
      if (with_val) Vs[e0 + off] = __ldg(val + k);
    }
    __syncthreads();
  }
}

// offset of segment (b, p) inside block b's range, from the segment lengths
__device__ __forceinline__ long long seg_offset(const int* seg_len, int b, int p, int np) {
  long long s = 0;
  for (int q = 0; q < p; ++q) s += seg_len[(long long)b * np + q];
  return s;
}

// 3. pieces of every segment; a thread per segment walks its rows. WRITE = false: count them into
// npc; WRITE = true: record each piece (start in the sorted words, length), starting at the
// segment's piece offset pbase, and the chunk table (warp w's first slot).
template <bool WRITE, typename RP>
__global__ void pl_pieces(const RP* rp, const int* row0, int nb, int np, const int* seg_len, const unsigned* Ws,
                          int* npc, const long long* pbase, long long* pstart, int* plen, long long* chunk) {
  const long long nseg = (long long)nb * np;
  for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < nseg; g += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(g / np), p = (int)(g % np);
    const long long s = rp_load(rp, __ldg(row0 + b)) + seg_offset(seg_len, b, p, np);
    const long long e = s + seg_len[g];
    const long long base = WRITE ? pbase[g] : 0;
    long long cnt = 0, open = -1;   // pieces so far; start of the open piece
    int fill = 0;
    for (long long k = s; k < e;) {
      const unsigned row = Ws[k] >> 16;
      long long k2 = k + 1;
      while (k2 < e && (Ws[k2] >> 16) == row) ++k2;
      long long left = k2 - k;
      if (fill > 0 && fill + left > kPanelBatchEntries) {   // the row does not fit: close the piece
        if (WRITE) { pstart[base + cnt] = open; plen[base + cnt] = fill; }
        ++cnt;
        fill = 0;
      }
      while (left > 0) {
        if (fill == 0) open = k;
        const long long take = min(left, (long long)(kPanelBatchEntries - fill));
        fill += (int)take;
        k += take;
        left -= take;
        if (fill == kPanelBatchEntries) {
          if (WRITE) { pstart[base + cnt] = open; plen[base + cnt] = fill; }
          ++cnt;
          fill = 0;
        }
      }
    }
    if (fill > 0) {
      if (WRITE) { pstart[base + cnt] = open; plen[base + cnt] = fill; }
      ++cnt;
    }
    if (!WRITE) {
      npc[g] = (int)cnt;
    } else {
      // warp w starts at piece w cnt / kWarps, moved forward past pieces that continue a row
      for (int w = 0; w < kWarps; ++w) {
        long long t = cnt * w / kWarps;
        while (t > 0 && t < cnt && pstart[base + t] > s &&
               (Ws[pstart[base + t]] >> 16) == (Ws[pstart[base + t] - 1] >> 16))
          ++t;
        chunk[g * kWarps + w] = (base + t) * kPanelBatchEntries;
      }
    }
  }
}

// 4. exclusive scan of the pieces per segment (one CTA of kThreads); out[m] = total
__global__ void __launch_bounds__(kThreads) pl_scan(const int* cnt, long long m, long long* out) {
  __shared__ long long part[kThreads];
  const int t = threadIdx.x;
  const long long per = (m + blockDim.x - 1) / blockDim.x;
  const long long a = min(m, (long long)t * per), z = min(m, a + per);
  long long s = 0;
  for (long long i = a; i < z; ++i) s += cnt[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    long long run = 0;
    for (int q = 0; q < (int)blockDim.x; ++q) {
      const long long v = part[q];
      part[q] = run;
      run += v;
    }
    out[m] = run;
  }
  __syncthreads();
  long long run = part[t];
  for (long long i = a; i < z; ++i) {
    out[i] = run;
    run += cnt[i];
  }
}

// 5. pieces to their slots (kPanelBatchEntries each); a warp per piece
template <typename T>
__global__ void pl_copy(const long long* pstart, const int* plen, long long pieces, const unsigned* Ws, const T* Vs,
                        int with_val, unsigned* ent, T* pval) {
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < pieces; c += nw) {
    const long long src = pstart[c], dst = c * kPanelBatchEntries;
    const int len = plen[c];
    for (int j = lane; j < kPanelBatchEntries; j += 32) {
      ent[dst + j] = (j < len) ? Ws[src + j] : kPanelPad;
      if (with_val) pval[dst + j] = (j < len) ? Vs[src + j] : T(0);
    }
  }
}

template <typename T, typename RP>
int build_on_device(sa_handle* h, const PanelPlan& pl, char* base) {
  const int nb = (int)pl.row0.size() - 1, np = pl.n_panels;
  const bool uniform = h->wmag > 0.0;
  const int* row0 = (const int*)(base + pl.off_row0);
  unsigned* W = (unsigned*)(base + pl.off_w);
  unsigned* Ws = (unsigned*)(base + pl.off_ws);
  T* Vs = uniform ? nullptr : (T*)(base + pl.off_vs);
  int* seg = (int*)(base + pl.off_seg);
  int* npc = (int*)(base + pl.off_npc);
  long long* pbase = (long long*)(base + pl.off_pbase);
  long long* pstart = (long long*)(base + pl.off_pstart);
  int* plen = (int*)(base + pl.off_plen);
  long long* chunk = (long long*)(base + pl.off_chunk);
  unsigned* ent = (unsigned*)(base + pl.off_ent);
  T* pval = uniform ? nullptr : (T*)(base + pl.off_val);
  const RP* rp = (const RP*)h->rowptr;
  const T* val = (const T*)h->val;
  const int g = h->sm_count * 4;
  const long long nseg = (long long)nb * np;
  pl_words<T, RP><<<g, 256, 0, h->stream>>>(rp, h->col, val, h->n, row0, nb, pl.width, W);
  pl_sort<T, RP><<<nb, kThreads, 0, h->stream>>>(rp, h->col, val, W, row0, np, pl.width, uniform ? 0 : 1, Ws, Vs, seg);
  const int gs = (int)std::max(1ll, std::min<long long>((nseg + 127) / 128, g));
  pl_pieces<false, RP><<<gs, 128, 0, h->stream>>>(rp, row0, nb, np, seg, Ws, npc, nullptr, nullptr, nullptr, nullptr);
  pl_scan<<<1, kThreads, 0, h->stream>>>(npc, nseg, pbase);
  pl_pieces<true, RP><<<gs, 128, 0, h->stream>>>(rp, row0, nb, np, seg, Ws, nullptr, pbase, pstart, plen, chunk);
  long long pieces = 0;
  PN_CUDA(cudaMemcpyAsync(&pieces, pbase + nseg, 8, cudaMemcpyDeviceToHost, h->stream));
  PN_CUDA(cudaStreamSynchronize(h->stream));
  if (pieces < 0 || pieces > pl.max_pieces) return SA_ERR_OOM;
  const long long total = pieces * kPanelBatchEntries;
  PN_CUDA(cudaMemcpyAsync(chunk + pl.chunks, &total, 8, cudaMemcpyHostToDevice, h->stream));
  if (pieces > 0) pl_copy<T><<<g, 256, 0, h->stream>>>(pstart, plen, pieces, Ws, Vs, uniform ? 0 : 1, ent, pval);
  count_launches(pieces > 0 ? 6 : 5);
  PN_CUDA(cudaGetLastError());
  return SA_OK;
}

template <typename T, typename RP>
__global__ void __launch_bounds__(kThreads, 1) panel_spmv_kernel(PanelArgs P, const T* u, const T* x, const T* sigma,
                                                               T rho, T* y, int* err) {
  extern __shared__ __align__(128) char psm[];
  __shared__ unsigned long long bars[kPanelBufs];
  panel_init(bars);
  unsigned par = 0;
  panel_spmv<T>(P, u, blockIdx.x, gridDim.x, psm, bars, par, err,
                [&](long long r, T acc) { y[r] = rho * x[r] - sigma[r] * acc; });
}

}  // namespace

namespace sa {

PanelArgs panel_args(const sa_handle* h) {
  PanelArgs P;
  P.ent = h->panel_ent;
  P.val = h->panel_val;
  P.chunk = h->panel_chunk;
  P.row0 = h->panel_row0;
  P.n_blocks = h->panel_blocks;
  P.n_panels = h->panel_count;
  P.width = h->panel_width;
  P.pad = 0;
  P.n = h->n;
  P.wmag = h->panel_val ? 0.0 : h->wmag;
  return P;
}

// Algorithmic bytes of one panel SpMV read from DRAM: the entry stream (padding included), the
// values when they differ in magnitude, the chunk bounds and the block rows. The staged input is
// read from L2 by every CTA and counted once with the vectors by the caller.
double panel_alg_bytes(const sa_handle* h) {
  const double T = h->prec == 32 ? 4.0 : 8.0;
  double b = 4.0 * (double)h->panel_slots + 16.0 * (double)h->panel_blocks * h->panel_count * kWarps +
             4.0 * (double)(h->panel_blocks + 1);
  if (h->panel_val) b += T * (double)h->panel_slots;
  return b;
}

// The standalone operator through the panel layout (sa_spmv_scaled when the panel SpMV is on). The
// dynamic shared-memory attribute is set on every launch: it belongs to the current device.
int panel_spmv_launch(sa_handle* h, const void* u, const void* x, const void* sigma, double rho, void* y) {
  int* err = operator_status_word(h);   // sticky until sa_operator_status reads it
  const PanelArgs P = panel_args(h);
  const int grid = std::min(h->panel_blocks, h->sm_count);
  if (h->prec == 32) {
    auto k = panel_spmv_kernel<float, int>;
    PN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_smem_bytes(4)));
    k<<<grid, kThreads, panel_smem_bytes(4), h->stream>>>(P, (const float*)u, (const float*)x, (const float*)sigma,
                                                          (float)rho, (float*)y, err);
  } else {
    auto k = panel_spmv_kernel<double, int>;
    PN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_smem_bytes(8)));
    k<<<grid, kThreads, panel_smem_bytes(8), h->stream>>>(P, (const double*)u, (const double*)x, (const double*)sigma,
                                                          rho, (double*)y, err);
  }
  count_launches(1);
  PN_CUDA(cudaGetLastError());
  return SA_OK;
}

}  // namespace sa

extern "C" {

int sa_panel_workspace_size(sa_handle* h, size_t* bytes, int32_t* row_blocks) {
  if (!h || !h->bound || !bytes) return SA_ERR_INVALID_ARG;
  std::vector<long long> rp;
  int st = host_rowptr(h, rp);
  if (st != SA_OK) return st;
  PanelPlan pl;
  st = plan_panels(h, rp, &pl);
  if (st != SA_OK) return st;
  *bytes = pl.total;
  if (row_blocks) *row_blocks = (int32_t)(pl.row0.size() - 1);
  return SA_OK;
}

int sa_panel_build(sa_handle* h, void* workspace, size_t bytes) {
  if (!h || !h->bound || !workspace || ((uintptr_t)workspace & 255)) return SA_ERR_INVALID_ARG;
  std::vector<long long> rp;
  int st = host_rowptr(h, rp);
  if (st != SA_OK) return st;
  PanelPlan pl;
  st = plan_panels(h, rp, &pl);
  if (st != SA_OK) return st;
  if (bytes < pl.total) return SA_ERR_OOM;
  char* base = (char*)workspace;
  h->panel_ready = h->panel_on = 0;
  PN_CUDA(cudaMemcpyAsync(base + pl.off_row0, pl.row0.data(), 4 * pl.row0.size(), cudaMemcpyHostToDevice, h->stream));
  if (h->prec == 32) st = h->rp64 ? build_on_device<float, long long>(h, pl, base) : build_on_device<float, int>(h, pl, base);
  else st = h->rp64 ? build_on_device<double, long long>(h, pl, base) : build_on_device<double, int>(h, pl, base);
  if (st != SA_OK) return st;
  long long slots = 0;
  PN_CUDA(cudaMemcpyAsync(&slots, base + pl.off_chunk + 8 * (size_t)pl.chunks, 8, cudaMemcpyDeviceToHost, h->stream));
  PN_CUDA(cudaStreamSynchronize(h->stream));
  if (slots < 0 || (size_t)slots > pl.cap) return SA_ERR_OOM;
  const bool uniform = h->wmag > 0.0;
  h->panel_ent = (const unsigned int*)(base + pl.off_ent);
  h->panel_val = uniform ? nullptr : (const void*)(base + pl.off_val);
  h->panel_chunk = (const long long*)(base + pl.off_chunk);
  h->panel_row0 = (const int*)(base + pl.off_row0);
  h->panel_blocks = (int)pl.row0.size() - 1;
  h->panel_slots = slots;
  h->panel_count = pl.n_panels;
  h->panel_width = pl.width;
  h->panel_ready = 1;
  h->panel_on = 1;
  h->split_on = 0;
  return SA_OK;
}

int sa_panel_info(sa_handle* h, int64_t* slots, int32_t* row_blocks, int32_t* panels, int32_t* width,
                  double* alg_bytes) {
  if (!h || !h->panel_ready) return SA_ERR_INVALID_ARG;
  if (slots) *slots = h->panel_slots;
  if (row_blocks) *row_blocks = h->panel_blocks;
  if (panels) *panels = h->panel_count;
  if (width) *width = h->panel_width;
  if (alg_bytes) *alg_bytes = panel_alg_bytes(h);
  return SA_OK;
}

int sa_panel_tables(sa_handle* h, const void** entries, const void** chunk_starts, const void** block_rows) {
  if (!h || !h->panel_ready) return SA_ERR_INVALID_ARG;
  if (entries) *entries = h->panel_ent;
  if (chunk_starts) *chunk_starts = h->panel_chunk;
  if (block_rows) *block_rows = h->panel_row0;
  return SA_OK;
}

int sa_panel_enable(sa_handle* h, int32_t on) {
  if (!h || (on && !h->panel_ready)) return SA_ERR_INVALID_ARG;
  h->panel_on = on ? 1 : 0;
  if (on) h->split_on = 0;
  return SA_OK;
}

}  // extern "C"

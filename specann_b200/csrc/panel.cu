// Column-panel SpMV layout builder (host) and the standalone panel operator kernel.
//
// sa_panel_workspace_size / sa_panel_build lay the bound matrix out as panel segments (see
// panel.cuh) in a caller-owned workspace; sa_panel_enable switches the handle's operator kernels to
// the panel SpMV. The builder reads the CSR back to the host once and sorts it by (block, panel)
// with a counting sort (O(nnz)).
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

struct PanelPlan {
  std::vector<int> row0;   // block first rows (n_blocks + 1)
  int n_panels = 0, width = 0;
  size_t cap = 0;   // entry slots, padding included
  size_t off_ent = 0, off_val = 0, off_chunk = 0, off_row0 = 0, total = 0;
};

// Row blocks of about nnz / blocks entries and at most max_rows rows; column panels of `width`.
int plan_panels(const sa_handle* h, const std::vector<long long>& rp, PanelPlan* pl) {
  const size_t T = h->prec == 32 ? 4 : 8;
  const long long max_rows = std::min<long long>(kPanelRowBytes / (long long)T, 65535);
  pl->width = (int)(panel_buf_bytes((int)T) / T);
  pl->n_panels = (int)((h->n + pl->width - 1) / pl->width);
  const long long want = std::max(1, h->sm_count);
  const double target = (double)h->nnz / (double)want;
  pl->row0.clear();
  pl->row0.push_back(0);
  long long start = 0;
  int b = 0;
  while (start < h->n) {
    // close the block when it reaches its share of the entries or max_rows rows
    const double goal = target * (double)(b + 1);
    long long end = start + 1;
    while (end < h->n && end - start < max_rows && (double)rp[end] < goal) ++end;
    pl->row0.push_back((int)end);
    start = end;
    ++b;
  }
  const long long nb = (long long)pl->row0.size() - 1;
  Layout L;
  // every chunk is padded to a multiple of kPanelLane entries
  pl->cap = (size_t)std::max(1ll, h->nnz) + (size_t)(kPanelLane - 1) * (size_t)nb * pl->n_panels * kWarps;
  pl->off_ent = L.off(4 * pl->cap);
  pl->off_val = (h->wmag > 0.0) ? 0 : L.off(T * pl->cap);
  pl->off_chunk = L.off(8 * ((size_t)nb * pl->n_panels * kWarps + 1));
  pl->off_row0 = L.off(4 * (size_t)(nb + 1));
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

// The standalone operator through the panel layout (sa_spmv_scaled when the panel SpMV is on).
int panel_spmv_launch(sa_handle* h, const void* u, const void* x, const void* sigma, double rho, void* y) {
  static bool attr_set[2] = {false, false};
  int* err = (int*)(h->red + 20);
  PN_CUDA(cudaMemsetAsync(err, 0, sizeof(int), h->stream));
  const PanelArgs P = panel_args(h);
  const int grid = std::min(h->panel_blocks, h->sm_count);
  if (h->prec == 32) {
    auto k = panel_spmv_kernel<float, int>;
    if (!attr_set[0]) {
      PN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_smem_bytes(4)));
      attr_set[0] = true;
    }
    k<<<grid, kThreads, panel_smem_bytes(4), h->stream>>>(P, (const float*)u, (const float*)x, (const float*)sigma, (float)rho,
                                                 (float*)y, err);
  } else {
    auto k = panel_spmv_kernel<double, int>;
    if (!attr_set[1]) {
      PN_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, panel_smem_bytes(8)));
      attr_set[1] = true;
    }
    k<<<grid, kThreads, panel_smem_bytes(8), h->stream>>>(P, (const double*)u, (const double*)x, (const double*)sigma, rho,
                                                 (double*)y, err);
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
  const long long nnz = h->nnz;
  const size_t T = h->prec == 32 ? 4 : 8;
  const bool uniform = h->wmag > 0.0;
  std::vector<int> col(std::max(1ll, nnz));
  std::vector<char> val((size_t)std::max(1ll, nnz) * T);
  if (nnz > 0) {
    PN_CUDA(cudaMemcpyAsync(col.data(), h->col, 4 * (size_t)nnz, cudaMemcpyDeviceToHost, h->stream));
    PN_CUDA(cudaMemcpyAsync(val.data(), h->val, T * (size_t)nnz, cudaMemcpyDeviceToHost, h->stream));
    PN_CUDA(cudaStreamSynchronize(h->stream));
  }
  auto negative = [&](long long k) {
    if (T == 4) { float v; memcpy(&v, &val[(size_t)k * 4], 4); return v < 0.0f; }
    double v; memcpy(&v, &val[(size_t)k * 8], 8); return v < 0.0;
  };
  const int nb = (int)pl.row0.size() - 1, np = pl.n_panels, width = pl.width;
  std::vector<unsigned int> ent(pl.cap, kPanelPad);
  std::vector<char> pv(uniform ? 0 : pl.cap * T, 0);
  std::vector<long long> chunk((size_t)nb * np * kWarps + 1);
  std::vector<long long> cnt(np + 1), pos(np);
  std::vector<unsigned> seg;   // the current block's entries in segment order (unpadded)
  std::vector<long long> src;  // their CSR positions
  long long out = 0;           // next padded slot
  for (int b = 0; b < nb; ++b) {
    const long long r0 = pl.row0[b], r1 = pl.row0[b + 1];
    const long long e0 = rp[r0], e1 = rp[r1];
    std::fill(cnt.begin(), cnt.end(), 0);
    for (long long k = e0; k < e1; ++k) cnt[col[k] / width + 1] += 1;
    for (int p = 0; p < np; ++p) cnt[p + 1] += cnt[p];
    for (int p = 0; p < np; ++p) pos[p] = cnt[p];
    seg.assign((size_t)(e1 - e0), 0u);
    src.assign((size_t)(e1 - e0), 0);
    for (long long r = r0; r < r1; ++r) {
      for (long long k = rp[r]; k < rp[r + 1]; ++k) {
        const int c = col[k];
        const int p = c / width;
        const long long d = pos[p]++;
        seg[(size_t)d] = ((unsigned)(r - r0) << 16) | (negative(k) ? 0x8000u : 0u) | (unsigned)(c - p * width);
        src[(size_t)d] = k;
      }
    }
    // each segment cut at row boundaries into kWarps chunks of about equal length; every chunk is
    // written at a multiple of kPanelLane slots and padded to one
    for (int p = 0; p < np; ++p) {
      const long long s0 = cnt[p], s1 = cnt[p + 1];
      long long cut[kWarps + 1];
      cut[0] = s0;
      cut[kWarps] = s1;
      for (int w = 1; w < kWarps; ++w) {
        long long t = s0 + (s1 - s0) * w / kWarps;
        if (t < cut[w - 1]) t = cut[w - 1];
        while (t > s0 && t < s1 && (seg[(size_t)t] >> 16) == (seg[(size_t)t - 1] >> 16)) ++t;
        cut[w] = t;
      }
      for (int w = 0; w < kWarps; ++w) {
        chunk[((size_t)b * np + p) * kWarps + w] = out;
        for (long long q = cut[w]; q < cut[w + 1]; ++q, ++out) {
          ent[(size_t)out] = seg[(size_t)q];
          if (!uniform) memcpy(&pv[(size_t)out * T], &val[(size_t)src[(size_t)q] * T], T);
        }
        out = (out + kPanelLane - 1) / kPanelLane * kPanelLane;
      }
    }
  }
  chunk[(size_t)nb * np * kWarps] = out;
  if ((size_t)out > pl.cap) return SA_ERR_OOM;
  char* base = (char*)workspace;
  if (out > 0) PN_CUDA(cudaMemcpyAsync(base + pl.off_ent, ent.data(), 4 * (size_t)out, cudaMemcpyHostToDevice, h->stream));
  if (!uniform && out > 0)
    PN_CUDA(cudaMemcpyAsync(base + pl.off_val, pv.data(), T * (size_t)out, cudaMemcpyHostToDevice, h->stream));
  PN_CUDA(cudaMemcpyAsync(base + pl.off_chunk, chunk.data(), 8 * chunk.size(), cudaMemcpyHostToDevice, h->stream));
  PN_CUDA(cudaMemcpyAsync(base + pl.off_row0, pl.row0.data(), 4 * pl.row0.size(), cudaMemcpyHostToDevice, h->stream));
  PN_CUDA(cudaStreamSynchronize(h->stream));
  h->panel_ent = (const unsigned int*)(base + pl.off_ent);
  h->panel_val = uniform ? nullptr : (const void*)(base + pl.off_val);
  h->panel_chunk = (const long long*)(base + pl.off_chunk);
  h->panel_row0 = (const int*)(base + pl.off_row0);
  h->panel_blocks = nb;
  h->panel_slots = out;
  h->panel_count = np;
  h->panel_width = width;
  h->panel_ready = 1;
  h->panel_on = 1;
  return SA_OK;
}

int sa_panel_enable(sa_handle* h, int32_t on) {
  if (!h || (on && !h->panel_ready)) return SA_ERR_INVALID_ARG;
  h->panel_on = on ? 1 : 0;
  return SA_OK;
}

}  // extern "C"

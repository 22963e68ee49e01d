// Host launch of the single-problem alpha solve (cooperative grid; device code in alpha_body.cuh).
#include "alpha_body.cuh"

namespace sa {

PanelArgs panel_args(const sa_handle* h);
double panel_alg_bytes(const sa_handle* h);
template <typename T, typename RP>
SpmvArgs<T, RP> split_args(const sa_handle* h, int s);

template <typename T, typename RP>
__global__ void __launch_bounds__(kThreads, 1) alpha_kernel(AlphaArgs<T, RP> A) {
  alpha_body<T, RP>(A, GridPolicy{});
}

// ---- host side ------------------------------------------------------------------------------

template <typename T, typename RP>
static int launch_alpha(sa_handle* h, const sa_alpha_params* p) {
  AlphaArgs<T, RP> A;
  A.S.rowptr = (const RP*)h->rowptr;
  A.S.col = h->col;
  A.S.val = (const T*)h->val;
  A.S.items = h->items;
  A.S.n_items = h->n_items;
  A.S.mc_base = h->mc_base;
  A.S.mc_count = h->mc_count;
  A.S.long_part = (T*)h->long_part;
  A.S.scol = h->packed ? h->scol : nullptr;
  A.S.wmag = (T)h->wmag;
  A.n = h->n;
  A.ldv = h->ldv;
  A.sigma = (T*)h->sigma;
  A.ld = h->ld;
  A.aoff = h->aoff;
  A.V = (T*)h->V;
  A.w = (T*)h->w;
  A.u = (T*)h->u;
  A.ylast = (const T*)h->yv[h->iy_last];
  A.yprev = (const T*)h->yv[h->iy_prev];
  A.yout = (T*)h->yv[h->iy_out];
  A.v0 = (const T*)p->v0;
  A.part = h->blk_part;
  A.pw = h->blk_part_width;
  A.ctrl = h->actrl;
  A.bits = h->scratch;
  A.W = h->W;
  A.p = *p;
  A.has_last = h->has_last ? 1 : 0;
  A.has_prev = h->has_prev ? 1 : 0;
  A.half_log2_c = 0.5 * std::log2(h->c);
  A.sqrt_c = std::sqrt(h->c);
  A.group = h->group;
  A.dense = h->dense;
  // Algorithmic bytes of one operator application, whatever the layout: the CSR (column + value per
  // entry, row pointers) and the vectors x, sigma, y. The panel and split layouts stream their own
  // (smaller or larger) encodings; the roofline is stated against this figure.
  A.spmv_bytes = (double)h->nnz * (4.0 + sizeof(T)) + (double)(h->n + 1) * sizeof(RP) + 3.0 * (double)h->n * sizeof(T);
  A.use_panel = h->panel_on ? 1 : 0;
  int dyn = 0;
  if (A.use_panel) {
    A.panel = panel_args(h);
    dyn = panel_smem_bytes((int)sizeof(T));
    // set on every launch: the attribute belongs to the current device
    if (cudaFuncSetAttribute((const void*)alpha_kernel<T, RP>, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn) !=
        cudaSuccess)
      return SA_ERR_CUDA;
  } else {
    A.panel = PanelArgs{};
  }
  A.n_splits = 0;
  A.split_part = nullptr;
  if (!A.use_panel && h->split_on) {
    A.n_splits = h->n_splits;
    for (int q = 0; q < h->n_splits; ++q) A.split[q] = split_args<T, RP>(h, q);
    A.split_part = (T*)h->split_part;
  }
  void* args[] = {&A};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)alpha_kernel<T, RP>, dim3(h->blocks),
                                              dim3(kThreads), args, (size_t)dyn, h->stream);
  count_launches(1);
  return e == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}

int alpha_solve_impl(sa_handle* h, const sa_alpha_params* p) {
  if (h->prec == 32) {
    return h->rp64 ? launch_alpha<float, long long>(h, p) : launch_alpha<float, int>(h, p);
  }
  return h->rp64 ? launch_alpha<double, long long>(h, p) : launch_alpha<double, int>(h, p);
}

template <typename T, typename RP>
static const void* alpha_kernel_ptr() { return (const void*)alpha_kernel<T, RP>; }

const void* alpha_kernel_for(int prec, int rp64) {
  if (prec == 32) return rp64 ? alpha_kernel_ptr<float, long long>() : alpha_kernel_ptr<float, int>();
  return rp64 ? alpha_kernel_ptr<double, long long>() : alpha_kernel_ptr<double, int>();
}

}  // namespace sa

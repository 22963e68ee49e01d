// Host launch of the batched local search (cooperative grid; device code in ls_body.cuh).
#include "ls_body.cuh"

namespace sa {

template <typename VT, typename RP, typename GT>
__global__ void __launch_bounds__(kThreads) ls_kernel(LsArgs<VT, RP, GT> A) {
  ls_body<VT, RP, GT>(A, GridPolicy{});
}

template <typename VT, typename RP, typename GT>
static int launch_ls(sa_handle* h, const sa_ls_params* p, char* ws, int kp, int kw, int cp,
                     long long wl_cap) {
  LsArgs<VT, RP, GT> A;
  A.rowptr = (const RP*)h->rowptr;
  A.col = h->col;
  A.val = (const VT*)h->val;
  A.items = h->items;
  A.n_items = h->n_items;
  A.n = h->n;
  A.k = p->k;
  A.kp = kp;
  A.kw = kw;
  A.cp = cp;
  Layout L;
  const size_t o_ctrl = L.off(sizeof(LsCtrl));
  const size_t o_eb = L.off(sizeof(double) * 128);
  const size_t o_ea = L.off(sizeof(double) * 128);
  const size_t o_sb = L.off(sizeof(uint32_t) * (size_t)h->n * kw);
  const size_t o_fm = L.off(sizeof(uint32_t) * (size_t)h->n * kw);
  const size_t o_h = L.off(sizeof(GT) * (size_t)h->n * kp);
  const size_t o_wl = L.off(sizeof(long long) * (size_t)wl_cap);
  const size_t o_wm = L.off(sizeof(uint32_t) * (size_t)h->n * kw);
  const size_t o_pr = L.off(sizeof(int) * (size_t)h->n);
  const size_t o_wq = L.off(sizeof(int) * (size_t)h->n);
  A.wm = (uint32_t*)(ws + o_wm);
  A.prio = (int*)(ws + o_pr);
  A.wq = (int*)(ws + o_wq);
  A.priority = p->semantics == 0 ? 1 : 0;
  A.ctrl = (LsCtrl*)(ws + o_ctrl);
  A.ebefore = (typename LsArgs<VT, RP, GT>::EAccPtr)(ws + o_eb);
  A.eafter = (typename LsArgs<VT, RP, GT>::EAccPtr)(ws + o_ea);
  A.sb = (uint32_t*)(ws + o_sb);
  A.flipm = (uint32_t*)(ws + o_fm);
  A.h = (GT*)(ws + o_h);
  A.wl = (long long*)(ws + o_wl);
  A.wl_cap = wl_cap;
  A.cand = h->cand + (size_t)p->first_slot * h->W;
  A.refined = h->refined + (size_t)p->first_slot * h->W;
  A.W = h->W;
  A.p = *p;
  A.m_main = (long long)(p->subset_fraction * (double)h->n);
  if (A.m_main < 1) A.m_main = 1;
  A.m_final = (long long)(p->final_sweep_fraction * (double)h->n);
  if (A.m_final < 1) A.m_final = 1;
  if (cudaMemsetAsync(A.ctrl, 0, sizeof(GridSync), h->stream) != cudaSuccess) return SA_ERR_CUDA;
  void* args[] = {&A};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)ls_kernel<VT, RP, GT>, dim3(h->blocks),
                                              dim3(kThreads), args, 0, h->stream);
  count_launches(1);
  return e == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}

void ls_geometry(int k, int* kp, int* kw, int* cp) {
  int p = k <= 8 ? 8 : (k <= 16 ? 16 : 32 * ((k + 31) / 32));
  *kp = p;
  *kw = p >= 32 ? p / 32 : 1;
  *cp = p >= 32 ? 32 : p;
}

size_t ls_workspace_bytes(long long n, long long nnz, int k, int integer) {
  int kp, kw, cp;
  ls_geometry(k, &kp, &kw, &cp);
  const long long wl_cap = n + nnz / kChunk + 2;
  Layout L;
  L.off(sizeof(LsCtrl));
  L.off(sizeof(double) * 128);
  L.off(sizeof(double) * 128);
  L.off(sizeof(uint32_t) * (size_t)n * kw);
  L.off(sizeof(uint32_t) * (size_t)n * kw);
  L.off((integer ? sizeof(int) : sizeof(double)) * (size_t)n * kp);
  L.off(sizeof(long long) * (size_t)wl_cap);
  L.off(sizeof(uint32_t) * (size_t)n * kw);
  L.off(sizeof(int) * (size_t)n);
  L.off(sizeof(int) * (size_t)n);
  return L.total;
}

int ls_run_impl(sa_handle* h, const sa_ls_params* p, void* ws, size_t bytes, double* eb, double* ea,
                sa_ls_result* res) {
  int kp, kw, cp;
  ls_geometry(p->k, &kp, &kw, &cp);
  const long long wl_cap = h->n + h->nnz / kChunk + 2;
  if (bytes < ls_workspace_bytes(h->n, h->nnz, p->k, h->integer_J)) return SA_ERR_OOM;
  char* w = (char*)ws;
  int st;
  const bool integer = h->integer_J != 0;
  if (h->prec == 32) {
    if (h->rp64) st = integer ? launch_ls<float, long long, int>(h, p, w, kp, kw, cp, wl_cap)
                              : launch_ls<float, long long, double>(h, p, w, kp, kw, cp, wl_cap);
    else st = integer ? launch_ls<float, int, int>(h, p, w, kp, kw, cp, wl_cap)
                      : launch_ls<float, int, double>(h, p, w, kp, kw, cp, wl_cap);
  } else {
    if (h->rp64) st = integer ? launch_ls<double, long long, int>(h, p, w, kp, kw, cp, wl_cap)
                              : launch_ls<double, long long, double>(h, p, w, kp, kw, cp, wl_cap);
    else st = integer ? launch_ls<double, int, int>(h, p, w, kp, kw, cp, wl_cap)
                      : launch_ls<double, int, double>(h, p, w, kp, kw, cp, wl_cap);
  }
  if (st != SA_OK) return st;
  // read back the control block and the energy sums
  LsCtrl ctl;
  Layout L;
  const size_t o_ctrl = L.off(sizeof(LsCtrl));
  const size_t o_eb = L.off(sizeof(double) * 128);
  const size_t o_ea = L.off(sizeof(double) * 128);
  long long sb_raw[128], sa_raw[128];
  if (cudaMemcpyAsync(&ctl, w + o_ctrl, sizeof(LsCtrl), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaMemcpyAsync(sb_raw, w + o_eb, sizeof(long long) * 128, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaMemcpyAsync(sa_raw, w + o_ea, sizeof(long long) * 128, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (ctl.gs.error) return ctl.gs.error;
  for (int q = 0; q < p->k; ++q) {
    if (integer) {
      if (eb) eb[q] = -0.5 * (double)sb_raw[q];
      if (ea) ea[q] = -0.5 * (double)sa_raw[q];
    } else {
      double x, y;
      memcpy(&x, &sb_raw[q], 8);
      memcpy(&y, &sa_raw[q], 8);
      if (eb) eb[q] = -0.5 * x;
      if (ea) ea[q] = -0.5 * y;
    }
  }
  if (res) {
    res->status = SA_OK;
    res->iterations = ctl.it;
    res->final_passes = ctl.final_passes;
    res->integer_gains = integer ? 1 : 0;
    res->total_flips = ctl.total_flips;
    for (int q = 0; q < 4; ++q) res->phase_ms[q] = (double)ctl.tph[q] * 1e-6;
  }
  return SA_OK;
}

const void* ls_kernel_for(int prec, int rp64, int integer) {
  if (prec == 32) {
    if (rp64) return integer ? (const void*)ls_kernel<float, long long, int> : (const void*)ls_kernel<float, long long, double>;
    return integer ? (const void*)ls_kernel<float, int, int> : (const void*)ls_kernel<float, int, double>;
  }
  if (rp64) return integer ? (const void*)ls_kernel<double, long long, int> : (const void*)ls_kernel<double, long long, double>;
  return integer ? (const void*)ls_kernel<double, int, int> : (const void*)ls_kernel<double, int, double>;
}

}  // namespace sa

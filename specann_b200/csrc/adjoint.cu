// Differentiation form: the adjoint of the leading eigenvector of N_a = D_a^{-1/2} (J/c) D_a^{-1/2}
// with per-vertex exponents a (D_a = max(d^a, 1e-12) per vertex; a_i = alpha + offset_i).
// No counterpart in the reference (it has no gradients); derived from first-order perturbation
// theory of a simple eigenpair:
//   (lambda, y) leading pair, |y| = 1; x = D^{-1/2} y (the rounding vector); t = tanh(beta x);
//   L = -1/2 t^T J t;  g_x = dL/dx = -beta (1 - t^2) o (J t);  g_y = D^{-1/2} g_x.
//   dy = -(M - lambda)^+ (I - y y^T) dM y, so dL = w^T dM y with w the solution of
//   (lambda I - M) w = (I - y y^T) g_y, w orthogonal to y (MINRES on the projected operator);
//   dM/da_k = l_k (e_k e_k^T M + M e_k e_k^T), l_k = -1/2 ln d_k (0 where the clamp is active), so
//   dL/da_k = l_k [y_k (M w)_k + w_k (M y)_k] + l_k g_x,k x_k   (the last term: x's own D^{-1/2}).
// The tangent dy/dalpha solves (lambda I - M) t = (I - y y^T) (dM/dalpha) y with
// (dM/dalpha) y = l o (M y) + M (l o y); it is the third eigenvector predictor (SA_START_TANGENT).
//
// One persistent cooperative kernel per call: set-up and right-hand side, MINRES (Paige-Saunders
// recurrences in FP64 scalars, vectors in the working precision, every inner product in FP64),
// the projection of the solution, and for the gradient the two SpMVs M w and M y and the assembly.
// The operator is the fused scaled SpMV of the alpha solve with rho = lambda, which applies
// lambda I - M exactly as the Lanczos kernel applies S_rho.
#include "alpha_body.cuh"

namespace sa {

constexpr int kAdjWindow = 50;          // MINRES iterations between stagnation checks
constexpr double kAdjStallOk = 1e-3;    // a stalled solve counts as converged below this residual

struct AdjCtrl {
  GridSync gs;
  double beta1, beta, oldb, alfa, dbar, epsln, oldeps, phibar, phi, cs, sn, delta, gamma, denom;
  double loss, rhs_dot, xproj, dalpha;
  double chk_phibar;        // residual estimate at the last stagnation checkpoint
  int itn, done, status, spmvs;
  int iy, ir1, ir2, iw, iw1, iw2;
};

template <typename T, typename RP>
struct AdjArgs {
  SpmvArgs<T, RP> S;
  long long n;
  const double* ld;
  const double* aoff;
  double alpha, lambda, beta_s, sqrt_c, half_log2_c, tol;
  int maxiter, mode;
  const T* yhat;
  const T* b;
  T* sigma;
  T* u;
  T* V;
  T* R[3];
  T* Wb[3];
  T* X;
  T* Z;
  T* G;
  double* grad;
  T* out;
  double* part;
  int pw;
  AdjCtrl* ctrl;
  PanelArgs panel;   // column-panel layout of the operator (use_panel = 1, with
  int use_panel;     // panel_smem_bytes(sizeof(T)) of dynamic shared memory), else the work list
};

// l_i = -1/2 ln d_i where d_i^{a_i} is above the clamp (else 0: D_i does not depend on a_i there)
template <typename T, typename RP>
__device__ __forceinline__ double dlog_of(const AdjArgs<T, RP>& A, long long i) {
  const double ldi = A.ld[i];
  const double ai = A.aoff ? A.alpha + A.aoff[i] : A.alpha;
  if (!isfinite(ldi)) return 0.0;
  const double logD = (ai == 0.0) ? 0.0 : ai * ldi;
  return logD > kLog2Clamp ? -0.5 * 0.69314718055994530942 * ldi : 0.0;
}

template <typename T, typename RP>
__global__ void __launch_bounds__(kThreads, 1) adjoint_kernel(AdjArgs<T, RP> A) {
  __shared__ double sm[kWarps * 4];
  __shared__ double sh[8];
  __shared__ SpmvSmem<T> ssp;
  __shared__ unsigned long long pbars[kPanelBufs];
  extern __shared__ __align__(128) char panel_smem[];
  const GridPolicy pol;
  AdjCtrl* C = A.ctrl;
  const long long n = A.n;
  const long long gtid = pol.tid(), nthreads = pol.nthr();
  const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
  unsigned ppar = 0;
  if (A.use_panel) panel_init(pbars);
  // one operator application: fin(row, sum_j val_ij u_j) once per row; false on a timed-out wait
  auto apply = [&](auto&& fin) -> bool {
    if (A.use_panel)
      return panel_spmv<T>(A.panel, A.u, pol.block(), pol.nblocks(), panel_smem, pbars, ppar, &C->gs.error, fin);
    spmv_items<T, RP>(A.S, A.u, gwarp, nwarps, ssp, fin);
    return true;
  };
  const T tlam = (T)A.lambda;

  // ---- P0: scaling for the exponents, zero the recurrences' vectors, mode set-up ------------
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    C->status = SA_OK;
    C->spmvs = 0;
    C->itn = 0;
    C->done = 0;
    C->loss = 0.0;
    C->dalpha = 0.0;
  }
  for (long long i = gtid; i < n; i += nthreads) {
    const double ldi = A.ld[i];
    const double ai = A.aoff ? A.alpha + A.aoff[i] : A.alpha;
    const double logD = (ai == 0.0) ? 0.0 : ai * ldi;
    const T sg = (T)exp2(-0.5 * fmax(logD, kLog2Clamp) - A.half_log2_c);
    A.sigma[i] = sg;
    A.Wb[0][i] = T(0);
    A.Wb[1][i] = T(0);
    A.Wb[2][i] = T(0);
    A.X[i] = T(0);
    const T yh = __ldg(A.yhat + i);
    if (A.mode == 0) {
      const double x = A.sqrt_c * (double)sg * (double)yh;
      A.u[i] = (T)tanh(A.beta_s * x);
    } else if (A.mode == 1) {
      A.u[i] = sg * yh;
    }
  }
  if (!grid_barrier(&C->gs)) return;

  // ---- P1: right-hand side G (and the loss) ---------------------------------------------------
  if (A.mode == 0) {
    double v[2] = {0.0, 0.0};
    if (!apply([&](long long r, T acc) {
      const double t = (double)__ldcg(A.u + r);
      const double jt = (double)acc;
      const double gx = -A.beta_s * (1.0 - t * t) * jt;
      const T gy = (T)(A.sqrt_c * (double)__ldcg(A.sigma + r) * gx);
      A.G[r] = gy;
      v[0] += t * jt;
      v[1] += (double)__ldg(A.yhat + r) * (double)gy;
    })) return;
    block_store_partials<2>(v, A.part, A.pw, 0, sm, blockIdx.x);
    if (!grid_barrier(&C->gs, [&] {
          reduce_partials(A.part, A.pw, gridDim.x, 2, sh);
          if (threadIdx.x == 0) {
            C->loss = -0.5 * sh[0];
            C->rhs_dot = sh[1];
            C->spmvs += 1;
          }
        })) return;
  } else if (A.mode == 1) {
    if (!apply([&](long long r, T acc) {
      A.Z[r] = __ldcg(A.sigma + r) * acc;                     // (M y)_r
    })) return;
    if (!grid_barrier(&C->gs)) return;
    for (long long i = gtid; i < n; i += nthreads)
      A.u[i] = (T)((double)__ldcg(A.sigma + i) * dlog_of(A, i) * (double)__ldg(A.yhat + i));
    if (!grid_barrier(&C->gs)) return;
    double v[1] = {0.0};
    if (!apply([&](long long r, T acc) {
      const T g = (T)(dlog_of(A, r) * (double)__ldcg(A.Z + r) + (double)__ldcg(A.sigma + r) * (double)acc);
      A.G[r] = g;
      v[0] += (double)__ldg(A.yhat + r) * (double)g;
    })) return;
    block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
    if (!grid_barrier(&C->gs, [&] {
          reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
          if (threadIdx.x == 0) { C->rhs_dot = sh[0]; C->spmvs += 2; }
        })) return;
  } else {
    double v[1] = {0.0};
    for (long long i = gtid; i < n; i += nthreads) {
      const T g = __ldg(A.b + i);
      A.G[i] = g;
      v[0] += (double)__ldg(A.yhat + i) * (double)g;
    }
    block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
    if (!grid_barrier(&C->gs, [&] {
          reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
          if (threadIdx.x == 0) C->rhs_dot = sh[0];
        })) return;
  }

  // ---- P2: b = (I - y y^T) G; r1 = r2 = b; explicit gradient term ----------------------------
  {
    const double rd = vload(&C->rhs_dot);
    double v[1] = {0.0};
    for (long long i = gtid; i < n; i += nthreads) {
      const double g = (double)__ldcg(A.G + i);
      const double yh = (double)__ldg(A.yhat + i);
      const T bi = (T)(g - rd * yh);
      A.R[0][i] = bi;
      A.R[1][i] = bi;
      v[0] += (double)bi * (double)bi;
      if (A.mode == 0) A.grad[i] = dlog_of(A, i) * g * yh;   // g_x,i x_i l_i with g_y = D^{-1/2} g_x
    }
    block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
    if (!grid_barrier(&C->gs, [&] {
          reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
          if (threadIdx.x == 0) {
            const double b1 = sqrt(sh[0]);
            C->beta1 = b1;
            C->beta = b1;
            C->oldb = 0.0;
            C->dbar = 0.0;
            C->epsln = 0.0;
            C->phibar = b1;
            C->cs = -1.0;
            C->sn = 0.0;
            C->chk_phibar = b1;
            C->ir1 = 0; C->ir2 = 1; C->iy = 2;
            C->iw = 0; C->iw1 = 1; C->iw2 = 2;
            C->done = (b1 > 0.0 && isfinite(b1)) ? 0 : 1;
            if (!isfinite(b1)) C->status = SA_ERR_NONFINITE;
          }
        })) return;
  }
  // first Lanczos vector v = r2 / beta and its scaled copy for the SpMV gather
  if (!vload(&C->done)) {
    const double ib = 1.0 / vload(&C->beta);
    for (long long i = gtid; i < n; i += nthreads) {
      const T vi = (T)((double)__ldcg(A.R[1] + i) * ib);
      A.V[i] = vi;
      A.u[i] = __ldcg(A.sigma + i) * vi;
    }
  }
  if (!grid_barrier(&C->gs)) return;

  // ---- MINRES on (lambda I - M) restricted to y's complement ----------------------------------
  while (!vload(&C->done)) {
    const int ir1 = vload(&C->ir1), ir2 = vload(&C->ir2), iy = vload(&C->iy);
    const double beta = vload(&C->beta), oldb = vload(&C->oldb);
    const int itn = vload(&C->itn);
    // PS: y = (lambda I - M) v - (beta / oldb) r1; alfa = v.y. The Krylov vectors are not
    // re-projected: applying (I - y y^T) after the operator alone would make it unsymmetric and
    // break the short recurrence; the right-hand side is orthogonal to y and the operator maps y's
    // complement into itself up to the eigenpair's error, and the solution is projected at the end.
    {
      double v[1] = {0.0};
      const double fr1 = itn >= 1 ? beta / oldb : 0.0;
      const T* r1 = A.R[ir1];
      T* yv = A.R[iy];
      if (!apply([&](long long r, T acc) {
        const T vr = __ldcg(A.V + r);
        double y = (double)(tlam * vr - __ldcg(A.sigma + r) * acc);
        if (itn >= 1) y -= fr1 * (double)__ldcg(r1 + r);
        const T yt = (T)y;
        yv[r] = yt;
        v[0] += (double)vr * (double)yt;
      })) return;
      block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
      if (!grid_barrier(&C->gs, [&] {
            reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
            if (threadIdx.x == 0) {
              C->alfa = sh[0];
              C->itn = itn + 1;
              C->spmvs += 1;
            }
          })) return;
    }
    // PU: y <- y - (alfa / beta) r2 ; |y|^2
    {
      const double fa = vload(&C->alfa) / beta;
      const T* r2 = A.R[ir2];
      T* yv = A.R[iy];
      double v[1] = {0.0};
      for (long long i = gtid; i < n; i += nthreads) {
        const double y = (double)__ldcg(yv + i) - fa * (double)__ldcg(r2 + i);
        const T yt = (T)y;
        yv[i] = yt;
        v[0] += (double)yt * (double)yt;
      }
      block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
      if (!grid_barrier(&C->gs, [&] {
            reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
            if (threadIdx.x == 0) {
              // r1 <- r2, r2 <- y (index rotation); Givens update of the QR factor of T_k
              C->ir1 = ir2;
              C->ir2 = iy;
              C->iy = ir1;
              C->oldb = beta;
              const double nb = sqrt(sh[0]);
              C->beta = nb;
              const double alfa = C->alfa;
              C->oldeps = C->epsln;
              C->delta = C->cs * C->dbar + C->sn * alfa;
              const double gbar = C->sn * C->dbar - C->cs * alfa;
              C->epsln = C->sn * nb;
              C->dbar = -C->cs * nb;
              const double gamma = fmax(hypot(gbar, nb), 1e-300);
              C->cs = gbar / gamma;
              C->sn = nb / gamma;
              C->phi = C->cs * C->phibar;
              C->phibar = C->sn * C->phibar;
              C->denom = 1.0 / gamma;
              const bool conv = C->phibar <= A.tol * C->beta1 || !(nb > 0.0);
              // stagnation: the right-hand side keeps a component along the true eigenvector as
              // large as the eigenpair's error, which the projected operator cannot resolve; the
              // residual estimate then stops decreasing and further iterations change nothing
              bool stalled = false;
              if (C->itn % kAdjWindow == 0) {
                stalled = C->phibar > 0.99 * C->chk_phibar;
                C->chk_phibar = C->phibar;
              }
              if (!isfinite(nb) || !isfinite(alfa)) {
                C->status = SA_ERR_NONFINITE;
                C->done = 1;
              } else if (conv || stalled || C->itn >= A.maxiter) {
                C->status = (conv || (stalled && C->phibar <= kAdjStallOk * C->beta1)) ? SA_OK : SA_ERR_NOT_CONVERGED;
                C->done = 1;
              }
            }
          })) return;
    }
    // PW: w = (v - oldeps w1 - delta w2) / gamma into the oldest buffer; x += phi w; next v
    {
      const int iw = vload(&C->iw), iw1 = vload(&C->iw1), iw2 = vload(&C->iw2);
      const double oldeps = vload(&C->oldeps), delta = vload(&C->delta), denom = vload(&C->denom);
      const double phi = vload(&C->phi);
      const int done = vload(&C->done);
      const double nb = vload(&C->beta);
      const double ib = done ? 0.0 : 1.0 / nb;
      const int nr2 = vload(&C->ir2);
      for (long long i = gtid; i < n; i += nthreads) {
        const double vi = (double)__ldcg(A.V + i);
        const double w = (vi - oldeps * (double)__ldcg(A.Wb[iw2] + i) - delta * (double)__ldcg(A.Wb[iw] + i)) * denom;
        A.Wb[iw1][i] = (T)w;
        A.X[i] = (T)((double)__ldcg(A.X + i) + phi * w);
        if (!done) {
          const T vn = (T)((double)__ldcg(A.R[nr2] + i) * ib);
          A.V[i] = vn;
          A.u[i] = __ldcg(A.sigma + i) * vn;
        }
      }
      if (!grid_barrier(&C->gs, [&] {
            if (threadIdx.x == 0) {
              C->iw = iw1;
              C->iw1 = iw2;
              C->iw2 = iw;
            }
          })) return;
    }
  }

  // ---- the solution, kept orthogonal to y -----------------------------------------------------
  {
    double v[1] = {0.0};
    for (long long i = gtid; i < n; i += nthreads) v[0] += (double)__ldg(A.yhat + i) * (double)__ldcg(A.X + i);
    block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
    if (!grid_barrier(&C->gs, [&] {
          reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
          if (threadIdx.x == 0) C->xproj = sh[0];
        })) return;
  }
  {
    const double xp = vload(&C->xproj);
    for (long long i = gtid; i < n; i += nthreads) {
      const T xi = (T)((double)__ldcg(A.X + i) - xp * (double)__ldg(A.yhat + i));
      A.X[i] = xi;
      if (A.mode == 0) A.u[i] = __ldcg(A.sigma + i) * xi;
      else A.out[i] = xi;
    }
  }
  if (A.mode != 0) return;
  if (!grid_barrier(&C->gs)) return;

  // ---- gradient: M w, then M y and the assembly --------------------------------------------------
  if (!apply([&](long long r, T acc) {
    A.Z[r] = __ldcg(A.sigma + r) * acc;
  })) return;
  if (!grid_barrier(&C->gs)) return;
  for (long long i = gtid; i < n; i += nthreads) A.u[i] = __ldcg(A.sigma + i) * __ldg(A.yhat + i);
  if (!grid_barrier(&C->gs)) return;
  {
    double v[1] = {0.0};
    if (!apply([&](long long r, T acc) {
      const double my = (double)__ldcg(A.sigma + r) * (double)acc;
      const double g = A.grad[r] + dlog_of(A, r) * ((double)__ldg(A.yhat + r) * (double)__ldcg(A.Z + r) +
                                                    (double)__ldcg(A.X + r) * my);
      A.grad[r] = g;
      v[0] += g;
    })) return;
    block_store_partials<1>(v, A.part, A.pw, 0, sm, blockIdx.x);
    grid_barrier(&C->gs, [&] {
      reduce_partials(A.part, A.pw, gridDim.x, 1, sh);
      if (threadIdx.x == 0) { C->dalpha = sh[0]; C->spmvs += 2; }
    });
  }
}

// ---- host side ------------------------------------------------------------------------------

constexpr int kAdjPartWidth = 8;

struct AdjCarve {
  size_t sigma, u, V, R[3], W[3], X, Z, G, part, ctrl, total;
};

static AdjCarve adj_carve(long long n, int prec, int blocks) {
  const size_t T = prec == 32 ? 4 : 8;
  Layout L;
  AdjCarve c;
  c.sigma = L.off(T * n);
  c.u = L.off(T * n);
  c.V = L.off(T * n);
  for (int q = 0; q < 3; ++q) c.R[q] = L.off(T * n);
  for (int q = 0; q < 3; ++q) c.W[q] = L.off(T * n);
  c.X = L.off(T * n);
  c.Z = L.off(T * n);
  c.G = L.off(T * n);
  c.part = L.off(8 * (size_t)blocks * kAdjPartWidth);
  c.ctrl = L.off(sizeof(AdjCtrl));
  c.total = L.total;
  return c;
}

PanelArgs panel_args(const sa_handle* h);

template <typename T, typename RP>
static int launch_adjoint(sa_handle* h, const sa_adjoint_params* p, char* ws, int blocks) {
  const AdjCarve c = adj_carve(h->n, h->prec, blocks);
  AdjArgs<T, RP> A;
  A.S = SpmvArgs<T, RP>{(const RP*)h->rowptr, h->col, (const T*)h->val, h->items, h->n_items, h->mc_base,
                         h->mc_count, (T*)h->long_part};
  A.S.scol = h->packed ? h->scol : nullptr;
  A.S.wmag = (T)h->wmag;
  A.n = h->n;
  A.ld = h->ld;
  A.aoff = h->aoff;
  A.alpha = p->alpha;
  A.lambda = p->lambda1;
  A.beta_s = p->beta;
  A.sqrt_c = std::sqrt(h->c);
  A.half_log2_c = 0.5 * std::log2(h->c);
  A.tol = p->tol;
  A.maxiter = p->maxiter;
  A.mode = p->mode;
  A.yhat = (const T*)p->y;
  A.b = (const T*)p->rhs;
  A.sigma = (T*)(ws + c.sigma);
  A.u = (T*)(ws + c.u);
  A.V = (T*)(ws + c.V);
  for (int q = 0; q < 3; ++q) { A.R[q] = (T*)(ws + c.R[q]); A.Wb[q] = (T*)(ws + c.W[q]); }
  A.X = (T*)(ws + c.X);
  A.Z = (T*)(ws + c.Z);
  A.G = (T*)(ws + c.G);
  A.grad = p->grad;
  A.out = (T*)p->out;
  A.part = (double*)(ws + c.part);
  A.pw = kAdjPartWidth;
  A.ctrl = (AdjCtrl*)(ws + c.ctrl);
  if (cudaMemsetAsync(A.ctrl, 0, sizeof(GridSync), h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (h->n_mc && cudaMemsetAsync(h->mc_count, 0, 4 * h->n_mc, h->stream) != cudaSuccess) return SA_ERR_CUDA;
  A.use_panel = h->panel_on ? 1 : 0;
  A.panel = A.use_panel ? panel_args(h) : PanelArgs{};
  size_t dyn = 0;
  if (A.use_panel) {
    dyn = (size_t)panel_smem_bytes((int)sizeof(T));
    // set on every launch: the attribute belongs to the current device
    if (cudaFuncSetAttribute((const void*)adjoint_kernel<T, RP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dyn) != cudaSuccess)
      return SA_ERR_CUDA;
  }
  void* args[] = {&A};
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)adjoint_kernel<T, RP>, dim3(blocks), dim3(kThreads),
                                                    args, dyn, h->stream);
  count_launches(1);
  return e == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}

// the handle's grid, clamped to what the adjoint kernel keeps resident at once (cooperative launch)
static int adj_blocks(sa_handle* h) {
  int occ = 0;
  const void* fn = h->prec == 32 ? (h->rp64 ? (const void*)adjoint_kernel<float, long long> : (const void*)adjoint_kernel<float, int>)
                                 : (h->rp64 ? (const void*)adjoint_kernel<double, long long> : (const void*)adjoint_kernel<double, int>);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kThreads, 0) != cudaSuccess || occ < 1) occ = 1;
  return std::max(1, std::min(h->blocks, h->sm_count * occ));
}

}  // namespace sa

using namespace sa;

extern "C" {

int sa_set_exponent_offsets(sa_handle* h, const double* offsets_device) {
  if (!h) return SA_ERR_INVALID_ARG;
  h->aoff = offsets_device;
  return SA_OK;
}

int sa_adjoint_workspace_size(sa_handle* h, size_t* bytes) {
  if (!h || !bytes) return SA_ERR_INVALID_ARG;
  *bytes = adj_carve(h->n, h->prec, adj_blocks(h)).total;
  return SA_OK;
}

int sa_adjoint(sa_handle* h, const sa_adjoint_params* p, void* work, size_t bytes, sa_adjoint_result* res) {
  if (!h || !h->bound || !p || !res || !p->y || p->maxiter < 1 || !(p->tol > 0.0)) return SA_ERR_INVALID_ARG;
  if (p->mode < SA_ADJ_GRADIENT || p->mode > SA_ADJ_SOLVE) return SA_ERR_INVALID_ARG;
  if (p->mode == SA_ADJ_GRADIENT && !p->grad) return SA_ERR_INVALID_ARG;
  if (p->mode != SA_ADJ_GRADIENT && !p->out) return SA_ERR_INVALID_ARG;
  if (p->mode == SA_ADJ_SOLVE && !p->rhs) return SA_ERR_INVALID_ARG;
  const int blocks = adj_blocks(h);
  const AdjCarve c = adj_carve(h->n, h->prec, blocks);
  if (!work || bytes < c.total) return SA_ERR_OOM;
  if (((uintptr_t)work) & 255) return SA_ERR_INVALID_ARG;
  char* ws = (char*)work;
  int st;
  if (h->prec == 32) st = h->rp64 ? launch_adjoint<float, long long>(h, p, ws, blocks) : launch_adjoint<float, int>(h, p, ws, blocks);
  else st = h->rp64 ? launch_adjoint<double, long long>(h, p, ws, blocks) : launch_adjoint<double, int>(h, p, ws, blocks);
  if (st != SA_OK) return st;
  AdjCtrl ctl;
  if (cudaMemcpyAsync(&ctl, ws + c.ctrl, sizeof(AdjCtrl), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) return SA_ERR_CUDA;
  memset(res, 0, sizeof(*res));
  res->status = ctl.gs.error ? ctl.gs.error : ctl.status;
  res->iterations = ctl.itn;
  res->spmv_count = ctl.spmvs;
  res->residual = ctl.beta1 > 0.0 ? ctl.phibar / ctl.beta1 : 0.0;
  res->loss = ctl.loss;
  res->dloss_dalpha = ctl.dalpha;
  return SA_OK;
}

}  // extern "C"

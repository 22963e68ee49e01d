// One alpha of the SpecAnn sweep as one persistent cooperative kernel: start vector / predictor,
// warm-started thick-restart Lanczos for the smallest eigenpair of S_rho = rho I - N_alpha with
// FP64 inner products and an FP64 tridiagonal Ritz solve, the Ritz-matrix guard, sign alignment,
// the true residual, and rounding to packed spins with an order-independent signature.
//
// CTAs rewrite V, w, u and y between phases and the per-SM L1 is not coherent with writes from
// other SMs, so every read of those arrays inside this kernel uses ld.global.cg (L2).
//
// Vectors (basis V, w, u, y) are in T (float or double); every inner product and norm is
// accumulated in double; the projected tridiagonal T_j lives in double in the control block.
// Between phases the CTAs meet at grid_barrier, whose epilogue (run by the last CTA to arrive)
// reduces the per-CTA partial sums in CTA order and takes the Lanczos decisions, so every CTA
// follows the same control path and results do not depend on timing.
#pragma once
#include <cmath>
#include <cstdio>

#include "common.cuh"
#include "handle.cuh"
#include "spmv.cuh"
#include "panel.cuh"
#include "policy.cuh"

namespace sa {

void count_launches(int k);

enum Action : int { ACT_NEXT = 0, ACT_REPASS = 1, ACT_RESTART = 2, ACT_REJECT = 3, ACT_DONE = 4, ACT_ERROR = 5,
                    ACT_P0_AGAIN = 6 };

constexpr double kLog2Clamp = -39.86313713864835;   // log2(1e-12)
constexpr int kRestartDefault = 8;   // Ritz vectors kept by an implicit restart (at most ncv / 2)
constexpr int kRestartMax = 16;
constexpr double kTinyNorm = 1e-12;

template <typename T, typename RP>
struct AlphaArgs {
  SpmvArgs<T, RP> S;
  long long n, ldv;
  T* sigma;
  const double* ld;
  const double* aoff;    // per-vertex exponent offsets (a_i = alpha + aoff[i]) or null
  T* V;
  T* w;
  T* u;
  const T* ylast;
  const T* yprev;
  T* yout;
  const T* v0;
  double* part;          // per-CTA partial sums, blocks x pw
  int pw;
  AlphaCtrl* ctrl;
  uint32_t* bits;        // scratch candidate (W words)
  long long W;
  sa_alpha_params p;
  int has_last, has_prev;
  double half_log2_c;
  double sqrt_c;
  int group;
  double spmv_bytes;     // algorithmic bytes of one fused SpMV
  double* dense;         // implicit-restart scratch (dense T, then dense Q)
  PanelArgs panel;       // column-panel layout of the operator (use_panel = 1; needs
  int use_panel;         // panel_smem_bytes(sizeof(T)) of dynamic shared memory), else the work list
  SpmvArgs<T, RP> split[kMaxSplits];   // L2 column splits of the operator (n_splits > 0): one
  int n_splits;                        // work-list pass per split, partial row sums in split_part
  T* split_part;
};

// ---- small dense helpers for the projected tridiagonal (double, one CTA) --------------------

// Biased exponent of a double (integer pipe: the recurrences below test signs and magnitudes on
// the bit pattern, keeping double compares off their dependency chains).
__device__ __forceinline__ int dexp_bits(double v) { return (int)((__double_as_longlong(v) >> 52) & 0x7FF); }

// Number of eigenvalues of the tridiagonal (a, b; size m) below x: sign changes of the leading
// principal minors det(T_k - x I), computed with the three-term recurrence. The pair (p_k, p_k-1) is
// rescaled by exact powers of two every 4 steps when its exponent leaves [2^-500, 2^500] (four steps
// of entries bounded by the Gershgorin radius cannot leave the double range from there).
__device__ inline int sturm_count(const double* a, const double* b, int m, double x) {
  double pp = 1.0, pc = a[0] - x;
  bool neg = pc < 0.0;
  int cnt = neg ? 1 : 0;
  for (int i = 1; i < m; ++i) {
    const double pn = (a[i] - x) * pc - b[i - 1] * b[i - 1] * pp;
    pp = pc;
    pc = pn;
    const long long bits = __double_as_longlong(pc);
    const bool nneg = ((bits << 1) != 0) ? (bits < 0) : !neg;   // a zero minor takes the opposite sign
    cnt += (nneg != neg);
    neg = nneg;
    if ((i & 3) == 0) {
      const int e = max(dexp_bits(pc), dexp_bits(pp));
      if (e > 1023 + 500) { pc *= 0x1p-500; pp *= 0x1p-500; }
      else if (e < 1023 - 500) { pc *= 0x1p500; pp *= 0x1p500; }
    }
  }
  return cnt;
}

// s_last^2 of the unit eigenvector for eigenvalue x: -det(T_{m-1} - x) / det'(T_m - x) (the same
// rescaling as sturm_count).
__device__ inline double last_component_sq(const double* a, const double* b, int m, double x) {
  double pp = 1.0, pc = a[0] - x, dp = 0.0, dc = -1.0;
  for (int i = 1; i < m; ++i) {
    const double bb = b[i - 1] * b[i - 1];
    const double pn = (a[i] - x) * pc - bb * pp;
    const double dn = -pc + (a[i] - x) * dc - bb * dp;
    pp = pc; pc = pn; dp = dc; dc = dn;
    if ((i & 3) == 0) {
      const int e = max(max(dexp_bits(pc), dexp_bits(dc)), max(dexp_bits(pp), dexp_bits(dp)));
      if (e > 1023 + 500) { pc *= 0x1p-500; pp *= 0x1p-500; dc *= 0x1p-500; dp *= 0x1p-500; }
      else if (e < 1023 - 500 && e > 0) { pc *= 0x1p500; pp *= 0x1p500; dc *= 0x1p500; dp *= 0x1p500; }
    }
  }
  // pp = det(T_{m-1} - x) (1 for m = 1), dc = det'(T_m - x)
  if (dc == 0.0) return 1.0;
  double s2 = -pp / dc;
  if (!(s2 >= 0.0)) s2 = 0.0;
  if (s2 > 1.0) s2 = 1.0;
  return s2;
}

// Smallest eigenvalue by multisection over the whole CTA (blockDim.x points per round), and the
// squared last component of its unit eigenvector in *s2 (every thread gets both). The tridiagonal
// is first copied from the control block to shared memory: every Sturm count walks it
// sequentially, so its loads must be short.
// hint_lo < hint_hi: a bracket to try first (from the previous step: by interlacing the smallest
// eigenvalue of T_m is at most the previous smallest Ritz value, and the previous residual bounds how
// far below it can be unless a new, lower eigenvalue appears); it is used only if the Sturm counts
// confirm no eigenvalue below hint_lo and at least one below hint_hi, else the Gershgorin interval.
__device__ inline double smallest_eig_block(const double* ag, const double* bg, int m, double* s2,
                                            double hint_lo = 0.0, double hint_hi = -1.0) {
  __shared__ double s_lo, s_hi, s_s2;
  __shared__ int s_first, s_cnt_lo, s_cnt_hi;
  __shared__ double a[kNcvMax], b[kNcvMax];
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    a[i] = ag[i];
    b[i] = (i + 1 < m) ? bg[i] : 0.0;
  }
  __syncthreads();
  const bool hint = hint_lo < hint_hi;
  if (hint && threadIdx.x == 1) s_cnt_lo = sturm_count(a, b, m, hint_lo);
  if (hint && threadIdx.x == 2) s_cnt_hi = sturm_count(a, b, m, hint_hi);
  if (threadIdx.x == 0) {
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < m; ++i) {
      const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < m ? fabs(b[i]) : 0.0);
      lo = fmin(lo, a[i] - r);
      hi = fmax(hi, a[i] + r);
    }
    const double pad = 1e-12 * fmax(1.0, fmax(fabs(lo), fabs(hi)));
    s_lo = lo - pad;
    s_hi = hi + pad;
  }
  __syncthreads();
  if (threadIdx.x == 0 && hint && s_cnt_lo == 0 && s_cnt_hi >= 1 && hint_lo > s_lo && hint_hi < s_hi) {
    s_lo = hint_lo;
    s_hi = hint_hi;
  }
  __syncthreads();
  const int P = blockDim.x;
  for (int round = 0; round < 7; ++round) {
    const double lo = s_lo, hi = s_hi;
    if (threadIdx.x == 0) s_first = P;
    __syncthreads();
    const double x = lo + (hi - lo) * (double)(threadIdx.x + 1) / (double)(P + 1);
    if (sturm_count(a, b, m, x) >= 1) atomicMin(&s_first, (int)threadIdx.x);
    __syncthreads();
    if (threadIdx.x == 0) {
      const int f = s_first;
      const double nlo = (f == 0) ? lo : lo + (hi - lo) * (double)f / (double)(P + 1);
      const double nhi = (f >= P) ? hi : lo + (hi - lo) * (double)(f + 1) / (double)(P + 1);
      s_lo = nlo;
      s_hi = nhi;
    }
    __syncthreads();
    if (s_hi - s_lo <= 1e-15 * fmax(1.0, fabs(s_hi))) break;
  }
  const double r = 0.5 * (s_lo + s_hi);
  if (threadIdx.x == 0) s_s2 = last_component_sq(a, b, m, r);
  __syncthreads();
  *s2 = s_s2;
  __syncthreads();
  return r;
}

// Unit eigenvector of the tridiagonal for eigenvalue theta by inverse iteration (one thread):
// LU with partial pivoting of (T - theta I), two solves from a constant start.
__device__ inline void tridiag_eigvec(const double* a, const double* b, int m, double theta, double* s) {
  if (m == 1) { s[0] = 1.0; return; }
  double dl[kNcvMax], d[kNcvMax], du[kNcvMax], du2[kNcvMax];
  int ipiv[kNcvMax];
  double anorm = 0.0;
  for (int i = 0; i < m; ++i) {
    d[i] = a[i] - theta;
    if (i + 1 < m) { dl[i] = b[i]; du[i] = b[i]; }
    anorm = fmax(anorm, fabs(a[i]) + (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < m ? fabs(b[i]) : 0.0));
  }
  const double tiny = fmax(anorm, 1e-300) * 1e-15;
  for (int i = 0; i < m; ++i) du2[i] = 0.0;
  for (int i = 0; i < m - 1; ++i) {
    if (fabs(d[i]) >= fabs(dl[i])) {
      ipiv[i] = i;
      if (d[i] == 0.0) d[i] = tiny;
      const double f = dl[i] / d[i];
      dl[i] = f;
      d[i + 1] -= f * du[i];
    } else {
      ipiv[i] = i + 1;
      const double f = d[i] / dl[i];
      d[i] = dl[i];
      dl[i] = f;
      const double t = du[i];
      du[i] = d[i + 1];
      d[i + 1] = t - f * d[i + 1];
      if (i < m - 2) {
        du2[i] = du[i + 1];
        du[i + 1] = -f * du[i + 1];
      }
    }
  }
  ipiv[m - 1] = m - 1;
  if (d[m - 1] == 0.0) d[m - 1] = tiny;
  for (int i = 0; i < m; ++i) s[i] = 1.0;
  for (int iter = 0; iter < 3; ++iter) {
    // forward: L
    for (int i = 0; i < m - 1; ++i) {
      if (ipiv[i] == i) {
        s[i + 1] -= dl[i] * s[i];
      } else {
        const double t = s[i];
        s[i] = s[i + 1];
        s[i + 1] = t - dl[i] * s[i];
      }
    }
    // backward: U
    s[m - 1] /= d[m - 1];
    if (m > 1) s[m - 2] = (s[m - 2] - du[m - 2] * s[m - 1]) / d[m - 2];
    for (int i = m - 3; i >= 0; --i) s[i] = (s[i] - du[i] * s[i + 1] - du2[i] * s[i + 2]) / d[i];
    double nrm = 0.0;
    for (int i = 0; i < m; ++i) nrm += s[i] * s[i];
    nrm = sqrt(nrm);
    if (!(nrm > 0.0) || !isfinite(nrm)) { for (int i = 0; i < m; ++i) s[i] = (i == 0) ? 1.0 : 0.0; return; }
    for (int i = 0; i < m; ++i) s[i] /= nrm;
  }
}

// The (q+1)-th smallest eigenvalue of the tridiagonal by bisection on the Sturm count.
__device__ inline double kth_eig(const double* a, const double* b, int m, int q) {
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? fabs(b[i - 1]) : 0.0) + (i + 1 < m ? fabs(b[i]) : 0.0);
    lo = fmin(lo, a[i] - r);
    hi = fmax(hi, a[i] + r);
  }
  lo -= 1e-12 * fmax(1.0, fabs(lo));
  hi += 1e-12 * fmax(1.0, fabs(hi));
  for (int it = 0; it < 80 && hi - lo > 1e-15 * fmax(1.0, fabs(hi)); ++it) {
    const double mid = 0.5 * (lo + hi);
    if (sturm_count(a, b, m, mid) >= q + 1) hi = mid;
    else lo = mid;
  }
  return 0.5 * (lo + hi);
}

// Implicit restart with exact shifts (the CTA): the m - kk largest Ritz values of the tridiagonal
// (a, b; size m) are the shifts of implicit QR steps. Each step is a bulge chase on the tridiagonal
// itself (diagonal d, off-diagonal e and the one bulge entry, O(m) work by one thread: rotation r
// acts on rows and columns r, r + 1 as T <- G T G^T with G = [[c, s], [-s, c]]); its m - 1 rotations
// are then applied to the rows of Q (Qd, m x m row-major, Q <- Q G^T) by all threads, one row each,
// with the row's moving entry kept in a register. Afterwards Q^T T Q has a leading kk x kk
// tridiagonal, written back to a and b, and the residual of the kept basis is
// V Q[:, kk] T+[kk][kk-1] + w Q[m-1][kk-1] (w: the pending unnormalised Lanczos vector).
// scratch: 5 kNcvMax doubles of shared memory.
__device__ inline void implicit_restart(AlphaCtrl* C, double* Qd, int m, int kk, double* scratch) {
  double* d = scratch;
  double* e = scratch + kNcvMax;
  double* ritz = scratch + 2 * kNcvMax;
  double* rc = scratch + 3 * kNcvMax;
  double* rs = scratch + 4 * kNcvMax;
  const int t = threadIdx.x;
  for (int i = t; i < m; i += blockDim.x) {
    d[i] = C->a[i];
    e[i] = (i + 1 < m) ? C->b[i] : 0.0;
  }
  __syncthreads();
  if (t < m) ritz[t] = kth_eig(d, e, m, t);
  for (int idx = t; idx < m * m; idx += blockDim.x) Qd[idx] = (idx / m == idx % m) ? 1.0 : 0.0;
  __syncthreads();
  for (int sft = m - 1; sft >= kk; --sft) {
    if (t == 0) {
      const double mu = ritz[sft];
      double g = 0.0;                          // bulge T[r+1][r-1]
      for (int r = 0; r < m - 1; ++r) {
        const double x = (r == 0) ? d[0] - mu : e[r - 1];
        const double z = (r == 0) ? e[0] : g;
        const double rr = hypot(x, z);
        const double c = (rr == 0.0) ? 1.0 : x / rr;
        const double sn = (rr == 0.0) ? 0.0 : z / rr;
        if (r > 0) e[r - 1] = rr;
        const double dr = d[r], dn = d[r + 1], er = e[r];
        d[r] = c * c * dr + 2.0 * c * sn * er + sn * sn * dn;
        d[r + 1] = sn * sn * dr - 2.0 * c * sn * er + c * c * dn;
        e[r] = c * sn * (dn - dr) + (c * c - sn * sn) * er;
        if (r + 2 < m) {
          g = sn * e[r + 1];
          e[r + 1] = c * e[r + 1];
        }
        rc[r] = c;
        rs[r] = sn;
      }
    }
    __syncthreads();
    for (int q = t; q < m; q += blockDim.x) {
      double* row = Qd + (long long)q * m;
      double pv = row[0];
      for (int r = 0; r < m - 1; ++r) {
        const double qv = row[r + 1];
        const double c = rc[r], sn = rs[r];
        row[r] = c * pv + sn * qv;
        pv = -sn * pv + c * qv;
      }
      row[m - 1] = pv;
    }
    __syncthreads();
  }
  if (t < kk) {
    C->a[t] = d[t];
    if (t + 1 < kk) C->b[t] = e[t];
  }
  if (t == 0) {
    C->irl_beta = e[kk - 1];
    C->irl_sigma = Qd[(m - 1) * m + (kk - 1)];
    C->irl_k = kk;
  }
  __syncthreads();
}

// sum_{k <= jmax} coef[k] V[k][i] in double, with the basis loads issued 8 at a time (independent
// loads keep the memory pipeline full; a plain loop over k would wait for each load in turn).
template <typename T>
__device__ __forceinline__ double basis_combine(const T* V, long long ldv, long long i, int jmax, const double* coef) {
  double acc = 0.0;
  for (int kb = 0; kb <= jmax; kb += 8) {
    T vv[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) vv[q] = (kb + q <= jmax) ? __ldcg(V + (long long)(kb + q) * ldv + i) : T(0);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      if (kb + q <= jmax) acc += coef[kb + q] * (double)vv[q];
  }
  return acc;
}

// 16-byte vector access to VW = 16 / sizeof(T) consecutive rows (rows of V, w, u, sigma are
// 256-byte aligned). Vector phases handle VW rows per thread per iteration, so every load
// instruction moves 16 bytes and a thread keeps several of them in flight.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };

template <typename T>
__device__ __forceinline__ void ld16(const T* p, T* out) {
  const typename Vec16<T>::type v = __ldcg(reinterpret_cast<const typename Vec16<T>::type*>(p));
  const T* c = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int r = 0; r < (int)(16 / sizeof(T)); ++r) out[r] = c[r];
}

template <typename T>
__device__ __forceinline__ void st16(T* p, const T* in) {
  typename Vec16<T>::type v;
  T* c = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int r = 0; r < (int)(16 / sizeof(T)); ++r) c[r] = in[r];
  *reinterpret_cast<typename Vec16<T>::type*>(p) = v;
}

// ---- reductions of per-CTA partials --------------------------------------------------------

// Sum part[blk * pw + col] over blocks for cols [0, ncols) into out[col] (fixed order).
__device__ inline void reduce_partials(const double* part, int pw, int nblocks, int ncols, double* out) {
  // a warp takes kCols adjacent columns and puts all their loads in flight at once (one L2 round trip
  // per 256 blocks instead of one per column); each column is summed in the same order as alone
  constexpr int kCols = 3;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c0 = wid * kCols; c0 < ncols; c0 += nw * kCols) {
    double acc[kCols];
#pragma unroll
    for (int cc = 0; cc < kCols; ++cc) acc[cc] = 0.0;
    for (int b0 = 0; b0 < nblocks; b0 += 32 * 8) {
      double pv[kCols][8];
#pragma unroll
      for (int cc = 0; cc < kCols; ++cc) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int bk = b0 + lane + 32 * q;
          pv[cc][q] = (bk < nblocks && c0 + cc < ncols) ? __ldcg(part + (long long)bk * pw + c0 + cc) : 0.0;
        }
      }
#pragma unroll
      for (int cc = 0; cc < kCols; ++cc) {
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[cc] += pv[cc][q];
      }
    }
#pragma unroll
    for (int cc = 0; cc < kCols; ++cc) {
      const double v = warp_sum(acc[cc]);
      if (lane == 0 && c0 + cc < ncols) out[c0 + cc] = v;
    }
  }
  __syncthreads();
}

// Block-reduce NV per-thread values and store them as this CTA's partials [col0, col0 + NV).
template <int NV>
__device__ void block_store_partials(const double (&v)[NV], double* part, int pw, int col0, double* sm, int blk) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double r[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) r[q] = warp_sum(v[q]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) sm[wid * NV + q] = r[q];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double acc = 0.0;
    for (int wv = 0; wv < nw; ++wv) acc += sm[wv * NV + threadIdx.x];
    part[(long long)blk * pw + col0 + threadIdx.x] = acc;
  }
  __syncthreads();
}

template <typename T>
__device__ __forceinline__ T vload(const T* p) { return *((volatile const T*)p); }

__device__ __forceinline__ unsigned long long word_mix(long long widx, unsigned int word) {
  return splitmix64(((unsigned long long)widx << 32) ^ (unsigned long long)word ^ 0xA5A5000000000000ull);
}

// ---- the alpha-solve kernel ----------------------------------------------------------------

// Shared scratch of the reductions: per-warp partials of block_store_partials (NW x 9) and the
// reduced columns of the dot phase (up to 2 kNcvMax + kDotBatch + 8 partial columns).
constexpr int kRedCols = 2 * kNcvMax + kDotBatch + 8;

// NW: warps per CTA at most (sizes the shared staging). kLayouts: the operator may use the column-panel
// layout or the L2 column splits (the single-problem kernel); without it only the work list is compiled
// (the batch kernel, whose register budget the other paths would spill).
template <typename T, typename RP, class Pol, int NW = kWarps, bool kLayouts = true>
__device__ __forceinline__ void alpha_body(const AlphaArgs<T, RP>& A, const Pol& pol) {
  static_assert(NW * (kDotBatch + 1) <= kRedCols, "reduction scratch too small");
  __shared__ double sm[kRedCols];
  __shared__ double sh[kNcvMax];
  __shared__ double s_theta, s_s2;
  __shared__ SpmvSmem<T, NW> ssp;
  __shared__ double sq[kNcvMax * (kRestartMax + 1)];
  __shared__ unsigned long long pbars[kPanelBufs];
  extern __shared__ __align__(128) char panel_smem[];
  AlphaCtrl* C = A.ctrl;
  const long long n = A.n;
  const long long gtid = pol.tid();
  const long long nthreads = pol.nthr();
  const sa_alpha_params& P = A.p;
  const double rho = P.rho;
  const double bound = 10.0 * (P.rho + P.gershgorin);
  const int ncv = P.ncv;
  unsigned ppar = 0;   // phase bits of the panel barriers
  if (kLayouts && A.use_panel) panel_init(pbars);
  // one operator application: fin(row, sum_j val_ij u_j) once per row; false on a timed-out wait
  auto apply = [&](auto&& fin) -> bool {
    if constexpr (kLayouts) {
      if (A.use_panel)
        return panel_spmv<T>(A.panel, A.u, pol.block(), pol.nblocks(), panel_smem, pbars, ppar, &C->gs.error, fin);
    }
    if constexpr (kLayouts) {
      if (A.n_splits > 0) {
        // pass s adds the row sums of split s; a barrier makes them visible to the next pass
        for (int q = 0; q < A.n_splits; ++q) {
          const bool first = q == 0, last = q + 1 == A.n_splits;
          spmv_items<T, RP>(A.split[q], A.u, gtid >> 5, nthreads >> 5, ssp, [&](long long r, T acc) {
            const T sum = first ? acc : __ldcg(A.split_part + r) + acc;
            if (last) fin(r, sum);
            else __stcg(A.split_part + r, sum);
          });
          if (!last && !pol.sync(&C->gs)) return false;
        }
        return true;
      }
    }
    spmv_items<T, RP>(A.S, A.u, gtid >> 5, nthreads >> 5, ssp, fin);
    return true;
  };

  // phase timer: CTA 0 thread 0 charges the time since the previous barrier exit to a phase
  unsigned long long t_mark = (pol.block() == 0 && threadIdx.x == 0) ? global_ns() : 0ull;
  auto mark = [&](int ph) {
    if (pol.block() == 0 && threadIdx.x == 0) {
      const unsigned long long t = global_ns();
      C->tph[ph] += t - t_mark;
      t_mark = t;
    }
  };

  // ---------------- P0: sigma, degree scale, start vector --------------------------------------
  int mode = P.start_mode;
  if (pol.block() == 0 && threadIdx.x == 0) {
    C->mode = mode;
    C->test_pred = (mode == SA_START_DIAGONAL || mode == SA_START_SECANT || mode == SA_START_TANGENT) ? 1 : 0;
    C->pred_accepted = -1;
    C->pred_residual = nan("");
    C->iters = 0;
    C->restarts = 0;
    C->status = SA_OK;
    C->nonfinite = 0;
    C->sig = 0ull;
    C->secant_sign = 1;
    C->bytes = 0.0;
    C->spmvs = 0;
    for (int q = 0; q < 6; ++q) C->tph[q] = 0ull;
  }
  {
    double ds = 0.0;
    for (long long i = gtid; i < n; i += nthreads) {
      const double ldi = (double)A.ld[i];
      const double ai = A.aoff ? P.alpha + A.aoff[i] : P.alpha;
      const double logD = (ai == 0.0) ? 0.0 : ai * ldi;
      const double logDc = fmax(logD, kLog2Clamp);
      A.sigma[i] = (T)exp2(-0.5 * logDc - A.half_log2_c);
      ds += exp2(logD);
    }
    double v[1] = {ds};
    block_store_partials<1>(v, A.part, A.pw, 0, sm, pol.block());
  }
  if (!pol.sync(&C->gs, [&] {
        reduce_partials(A.part, A.pw, pol.nblocks(), 1, sh);
        if (threadIdx.x == 0) {
          C->degree_scale = sh[0];
          C->bytes += (double)n * (8.0 + sizeof(T));
        }
      })) return;
  mark(0);

  if (mode == SA_START_SECANT && A.has_prev) {
    double v[1] = {0.0};
    for (long long i = gtid; i < n; i += nthreads) v[0] += (double)A.ylast[i] * (double)A.yprev[i];
    block_store_partials<1>(v, A.part, A.pw, 0, sm, pol.block());
    if (!pol.sync(&C->gs, [&] {
          reduce_partials(A.part, A.pw, pol.nblocks(), 1, sh);
          if (threadIdx.x == 0) {
            C->secant_sign = (sh[0] < 0.0) ? -1 : 1;
            C->bytes += 2.0 * (double)n * sizeof(T);
          }
        })) return;
    mark(0);
  }

  while (true) {   // P0 loop (repeats for a predictor fallback or rejection)
    mode = vload(&C->mode);
    const int sgn = vload(&C->secant_sign);
    const unsigned long long key = splitmix64(P.seed ^ 0x57A27000ull) ^ splitmix64((unsigned long long)P.stream_id + 0x1234567ull);
    double v[3] = {0.0, 0.0, 0.0};   // ||v0||^2, ||s||^2 (secant), ||y||^2 (secant)
    for (long long i = gtid; i < n; i += nthreads) {
      double x;
      if (mode == SA_START_RANDOM) {
        x = (double)(T)normal_from_counter(key, i);
      } else if (mode == SA_START_PREV) {
        x = (double)A.ylast[i];
      } else if (mode == SA_START_GIVEN) {
        x = (double)A.v0[i];
      } else if (mode == SA_START_TANGENT) {
        // first-order step along the eigenvector tangent dy/dalpha at alpha_prev (given in v0)
        x = (double)(T)(A.ylast[i] + (T)(P.alpha - P.alpha_prev) * A.v0[i]);
      } else if (mode == SA_START_DIAGONAL) {
        const double ldi = fmax((double)A.ld[i], kLog2Clamp);
        const T wgt = (T)exp2(0.5 * (P.alpha - P.alpha_prev) * ldi);
        x = (double)(T)(wgt * A.ylast[i]);
      } else {   // SECANT
        const T yl = A.ylast[i];
        const T yp = A.has_prev ? (T)(sgn * A.yprev[i]) : yl;
        const T sdiff = (T)(yl - yp);
        x = (double)(T)(yl + (T)P.secant_gamma * sdiff);
        v[1] += (double)sdiff * (double)sdiff;
      }
      const T xt = (T)x;
      A.w[i] = xt;
      A.u[i] = A.sigma[i] * xt;
      v[0] += (double)xt * (double)xt;
    }
    v[2] = v[0];
    block_store_partials<3>(v, A.part, A.pw, 0, sm, pol.block());
    if (!pol.sync(&C->gs, [&] {
          reduce_partials(A.part, A.pw, pol.nblocks(), 3, sh);
          if (threadIdx.x == 0) {
            const int md = C->mode;
            const double nrm = sqrt(sh[0]);
            const double nin = (md == SA_START_RANDOM) ? 0.0 : ((md == SA_START_SECANT || md == SA_START_TANGENT) ? 2.0 : 1.0);
            C->bytes += (double)n * sizeof(T) * (2.0 + nin) + (md == SA_START_DIAGONAL ? 8.0 * n : 0.0);
            C->action = ACT_NEXT;
            if (md == SA_START_DIAGONAL && nrm < kTinyNorm) {
              C->mode = SA_START_RANDOM;           // utils/predictors.py:22-25
              C->action = ACT_P0_AGAIN;
            } else if (md == SA_START_SECANT &&
                       (!A.has_prev || sqrt(sh[1]) < kTinyNorm || nrm < kTinyNorm)) {
              C->mode = SA_START_PREV;             // utils/predictors.py:44-55
              C->action = ACT_P0_AGAIN;
            } else if (md == SA_START_TANGENT && (!A.has_last || !(nrm >= kTinyNorm) || !isfinite(nrm))) {
              C->mode = SA_START_PREV;             // as the secant fallback
              C->action = ACT_P0_AGAIN;
            } else if (!(nrm > 0.0) || !isfinite(nrm)) {
              C->status = SA_ERR_NONFINITE;
              C->action = ACT_ERROR;
            } else {
              C->inv_b = 1.0 / nrm;
              C->j = 0;
              C->pass2 = 0;
            }
          }
        })) return;
    mark(0);
    const int act = vload(&C->action);
    if (act == ACT_P0_AGAIN) continue;
    if (act == ACT_ERROR) return;

    // ---------------- Lanczos steps ----------------------------------------------------------
    bool restart_p0 = false;
    if (pol.block() == 0 && threadIdx.x == 0) C->ritz_ok = 0;
    while (true) {
      const int j = vload(&C->j);
      const int pass2 = vload(&C->pass2);
      if (!pass2) {
        // P1: V[j] = w * inv_b; w <- S V[j]; partial sums of a_j = V[j] . w
        const T inv_b = (T)vload(&C->inv_b);
        T* Vj = A.V + (long long)j * A.ldv;
        const T trho = (T)rho;
        double pa[1] = {0.0};
        if (!apply([&](long long r, T acc) {
              const T wr = __ldcg(A.w + r);
              const T vr = wr * inv_b;
              const T wn = (trho * wr - __ldcg(A.sigma + r) * acc) * inv_b;
              Vj[r] = vr;
              A.w[r] = wn;
              pa[0] += (double)vr * (double)wn;
            })) return;
        block_store_partials<1>(pa, A.part, A.pw, 0, sm, pol.block());
        if (!pol.sync(&C->gs, [&] {
              reduce_partials(A.part, A.pw, pol.nblocks(), 1, sm);
              if (threadIdx.x == 0) {
                C->a[j] = sm[0];
                C->bytes += A.spmv_bytes + (double)n * sizeof(T);
                C->spmvs += 1;
              }
            })) return;
        mark(1);
      }
      // P2: three-term step w -= a_j V[j] + b_{j-1} V[j-1] (first pass only), then the
      // reorthogonalisation coefficients h_k = V_k . w (k <= j) and ww = w . w. Removing the
      // dominant components explicitly first keeps the single Gram-Schmidt pass stable.
      {
        const double a3 = pass2 ? 0.0 : vload(&C->a[j]);
        const double b3 = (pass2 || j == 0) ? 0.0 : vload(&C->b[j - 1]);
        const T* Vj = A.V + (long long)j * A.ldv;
        const T* Vm = A.V + (long long)(j > 0 ? j - 1 : 0) * A.ldv;
        constexpr int VW = 16 / sizeof(T);
        const long long nvec = n / VW;
        for (int kb = 0; kb <= j; kb += kDotBatch) {
          double acc[kDotBatch + 1];
#pragma unroll
          for (int q = 0; q <= kDotBatch; ++q) acc[q] = 0.0;
          const int nk = (j + 1 - kb < kDotBatch) ? (j + 1 - kb) : kDotBatch;
          for (long long iv = gtid; iv < nvec; iv += nthreads) {
            const long long i0 = iv * VW;
            T wv[VW];
            ld16(A.w + i0, wv);
            double wd[VW];
            if (kb == 0 && !pass2) {
              T vj[VW], vm[VW];
              ld16(Vj + i0, vj);
              ld16(Vm + i0, vm);
#pragma unroll
              for (int r = 0; r < VW; ++r) {
                double x = (double)wv[r] - a3 * (double)vj[r];
                if (j > 0) x -= b3 * (double)vm[r];
                wv[r] = (T)x;
              }
              st16(A.w + i0, wv);
            }
#pragma unroll
            for (int r = 0; r < VW; ++r) wd[r] = (double)wv[r];
#pragma unroll
            for (int q = 0; q < kDotBatch; ++q) {
              if (q < nk) {
                T vk[VW];
                ld16(A.V + (long long)(kb + q) * A.ldv + i0, vk);
#pragma unroll
                for (int r = 0; r < VW; ++r) acc[q] += (double)vk[r] * wd[r];
              }
            }
            if (kb == 0) {
#pragma unroll
              for (int r = 0; r < VW; ++r) acc[kDotBatch] += wd[r] * wd[r];
            }
          }
          for (long long i = nvec * VW + gtid; i < n; i += nthreads) {
            double wi = (double)__ldcg(A.w + i);
            if (kb == 0 && !pass2) {
              wi -= a3 * (double)__ldcg(Vj + i);
              if (j > 0) wi -= b3 * (double)__ldcg(Vm + i);
              const T wt = (T)wi;
              A.w[i] = wt;
              wi = (double)wt;
            }
#pragma unroll
            for (int q = 0; q < kDotBatch; ++q)
              if (q < nk) acc[q] += (double)__ldcg(A.V + (long long)(kb + q) * A.ldv + i) * wi;
            if (kb == 0) acc[kDotBatch] += wi * wi;
          }
          block_store_partials<kDotBatch + 1>(acc, A.part, A.pw, kb * 2, sm, pol.block());
        }
        if (!pol.sync(&C->gs, [&] {
              // batch kb stored its 8 dots at cols [2kb, 2kb + 8) and ww (kb = 0) at col 8
              const int nb = (j + kDotBatch) / kDotBatch;
              reduce_partials(A.part, A.pw, pol.nblocks(), 2 * kDotBatch * (nb - 1) + kDotBatch + 1, sm);
              if (threadIdx.x <= j) {
                const int kb = (threadIdx.x / kDotBatch) * kDotBatch;
                C->h[threadIdx.x] = sm[2 * kb + (threadIdx.x - kb)];
              }
              if (threadIdx.x == 0) {
                C->ww = sm[kDotBatch];
                C->a[j] += sm[2 * ((j / kDotBatch) * kDotBatch) + (j % kDotBatch)];
                C->bytes += (double)n * sizeof(T) * (double)(j + 2 + (C->pass2 ? 0 : 3));
              }
            })) return;
        mark(2);
      }
      // P3: w -= sum_k h_k V_k ; u = sigma w ; ww2
      {
        if (threadIdx.x <= j) sh[threadIdx.x] = vload(&C->h[threadIdx.x]);
        __syncthreads();
        double v[1] = {0.0};
        constexpr int VW = 16 / sizeof(T);
        const long long nvec = n / VW;
        // U positions per thread and iteration (iv, iv + nthreads), whose loads are in flight
        // together, and KB3 basis vectors per batch (the same registers as one position and
        // kDotBatch vectors); the batch kernel keeps one position within its register budget
        constexpr int U = kLayouts ? 2 : 1;
        constexpr int KB3 = kDotBatch / U;
        for (long long iv = gtid; iv < nvec; iv += U * nthreads) {
          const bool two = U == 2 && iv + nthreads < nvec;
          const long long i0[2] = {iv * VW, (two ? iv + nthreads : iv) * VW};
          // w and sigma are put in flight first; the basis is read kDotBatch vectors at a time
          T wv[2][VW], sg[2][VW];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            ld16(A.w + i0[u], wv[u]);
            ld16(A.sigma + i0[u], sg[u]);
          }
          double corr[2][VW];
#pragma unroll
          for (int u = 0; u < U; ++u)
#pragma unroll
            for (int r = 0; r < VW; ++r) corr[u][r] = 0.0;
          for (int kb = 0; kb <= j; kb += KB3) {
            T vk[KB3][2][VW];
#pragma unroll
            for (int q = 0; q < KB3; ++q) {
              if (kb + q <= j) {
#pragma unroll
                for (int u = 0; u < U; ++u) ld16(A.V + (long long)(kb + q) * A.ldv + i0[u], vk[q][u]);
              }
            }
#pragma unroll
            for (int q = 0; q < KB3; ++q) {
              if (kb + q <= j) {
#pragma unroll
                for (int u = 0; u < U; ++u)
#pragma unroll
                  for (int r = 0; r < VW; ++r) corr[u][r] += sh[kb + q] * (double)vk[q][u][r];
              }
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
            T uv[VW];
#pragma unroll
            for (int r = 0; r < VW; ++r) {
              wv[u][r] = (T)((double)wv[u][r] - corr[u][r]);
              uv[r] = sg[u][r] * wv[u][r];
              if (u == 0 || two) v[0] += (double)wv[u][r] * (double)wv[u][r];
            }
            if (u == 0 || two) {
              st16(A.w + i0[u], wv[u]);
              st16(A.u + i0[u], uv);
            }
          }
        }
        for (long long i = nvec * VW + gtid; i < n; i += nthreads) {
          const double corr = basis_combine(A.V, A.ldv, i, j, sh);
          const T wi = (T)((double)__ldcg(A.w + i) - corr);
          A.w[i] = wi;
          A.u[i] = A.sigma[i] * wi;
          v[0] += (double)wi * (double)wi;
        }
        block_store_partials<1>(v, A.part, A.pw, 0, sm, pol.block());
      }
      if (!pol.sync(&C->gs, [&] {
            reduce_partials(A.part, A.pw, pol.nblocks(), 1, sm);
            const double ww2 = sm[0];
            const double bj = sqrt(ww2);
            const double aj = C->a[j];
            if (threadIdx.x == 0) {
              C->action = ACT_NEXT;
              C->bytes += (double)n * sizeof(T) * (double)(j + 5);
              if (!C->pass2) C->iters += 1;
              if (!isfinite(aj) || !isfinite(bj) || fabs(aj) > bound || bj > bound) {
                C->status = SA_ERR_BREAKDOWN;   // models/spectral_annealing.py:85-120
                C->action = ACT_ERROR;
              } else if (C->test_pred && j == 0) {
                C->test_pred = 0;
                C->pred_residual = bj;
                C->pred_accepted = (bj > P.pred_tol) ? 0 : 1;
                if (bj > P.pred_tol) {           // models/spectral_annealing.py:610-612
                  C->mode = SA_START_PREV;
                  C->iters = 0;
                  C->action = ACT_REJECT;
                }
              }
              if (C->action == ACT_NEXT && !C->pass2 && ww2 < 1e-4 * C->ww && bj > 1e-14 * bound) {
                C->pass2 = 1;                    // second Gram-Schmidt pass
                C->action = ACT_REPASS;
              }
              C->pass2 = (C->action == ACT_REPASS) ? 1 : 0;
            }
            __syncthreads();
            const int act0 = C->action;
            if (act0 == ACT_NEXT) {
              const int m = j + 1;
              double s2;
              // previous step's Ritz value and residual estimate as the bracket to try first
              double hlo = 0.0, hhi = -1.0;
              if (m >= 2 && C->ritz_ok) {
                const double th0 = C->theta, r0 = C->res_est;
                const double pad = 1e-12 * fmax(1.0, fabs(th0));
                hlo = th0 - 2.0 * r0 - pad;
                hhi = th0 + pad;
              }
              const double th = smallest_eig_block(C->a, C->b, m, &s2, hlo, hhi);
              if (threadIdx.x == 0) {
                s_theta = th;
                s_s2 = s2;
              }
              __syncthreads();
              if (threadIdx.x == 0) {
                const double res = bj * sqrt(s_s2);
                const bool invariant = bj <= 1e-14 * bound;
                C->theta = s_theta;
                C->res_est = invariant ? 0.0 : res;
                C->ritz_ok = 1;
                const bool conv = invariant || res <= P.tol;
                if (conv || C->iters >= P.maxiter) {
                  tridiag_eigvec(C->a, C->b, m, s_theta, C->s);
                  C->status = conv ? SA_OK : SA_ERR_NOT_CONVERGED;
                  C->b[j] = bj;
                  C->action = ACT_DONE;
                } else if (m >= ncv) {
                  C->restarts += 1;
                  C->action = ACT_RESTART;
                } else {
                  C->b[j] = bj;
                  C->inv_b = 1.0 / bj;
                  C->j = j + 1;
                }
              }
              __syncthreads();
              if (C->action == ACT_RESTART) {
                const int keep = P.restart_keep > 0 ? P.restart_keep : kRestartDefault;
                const int kk = max(1, min(min(keep, kRestartMax), ncv / 2));
                implicit_restart(C, A.dense + kNcvMax * kNcvMax, m, kk, sq);
              }
            }
          })) return;
      mark(3);
      const int act = vload(&C->action);
      if (act == ACT_NEXT) continue;
      if (act == ACT_REPASS) continue;
      if (act == ACT_ERROR) return;
      if (act == ACT_REJECT) { restart_p0 = true; break; }
      if (act == ACT_RESTART) {
        // kept basis V[0..kk) <- V Q[:, 0..kk) and the new residual
        // f = V Q[:, kk] T+[kk][kk-1] + w Q[m-1][kk-1], row by row in place (all m inputs of a row
        // are read before its kk outputs are written)
        const int m = j + 1;
        const int kk = vload(&C->irl_k);
        const double beta_hat = vload(&C->irl_beta), sig_q = vload(&C->irl_sigma);
        const double* Qd = A.dense + kNcvMax * kNcvMax;
        for (int idx = threadIdx.x; idx < m * (kk + 1); idx += blockDim.x) {
          const int r = idx / (kk + 1), c = idx % (kk + 1);
          sq[idx] = vload(Qd + r * m + c);
        }
        __syncthreads();
        double v[1] = {0.0};
        for (long long i = gtid; i < n; i += nthreads) {
          double y[kRestartMax + 1];
#pragma unroll
          for (int c = 0; c <= kRestartMax; ++c) y[c] = 0.0;
#pragma unroll 2
          for (int r = 0; r < m; ++r) {
            const double vr = (double)A.V[(long long)r * A.ldv + i];
#pragma unroll
            for (int c = 0; c <= kRestartMax; ++c)
              if (c <= kk) y[c] += vr * sq[r * (kk + 1) + c];
          }
#pragma unroll
          for (int c = 0; c < kRestartMax; ++c)
            if (c < kk) A.V[(long long)c * A.ldv + i] = (T)y[c];
          double yk = 0.0;
#pragma unroll
          for (int c = 0; c <= kRestartMax; ++c)
            if (c == kk) yk = y[c];
          const T f = (T)(yk * beta_hat + (double)A.w[i] * sig_q);
          A.w[i] = f;
          A.u[i] = A.sigma[i] * f;
          v[0] += (double)f * (double)f;
        }
        block_store_partials<1>(v, A.part, A.pw, 0, sm, pol.block());
        if (!pol.sync(&C->gs, [&] {
              reduce_partials(A.part, A.pw, pol.nblocks(), 1, sm);
              if (threadIdx.x == 0) {
                const double nf = sqrt(sm[0]);
                C->pass2 = 0;
                C->bytes += (double)n * sizeof(T) * (double)(m + kk + 3);
                if (!(nf > 1e-14 * bound) || !isfinite(nf)) {
                  // the kept basis spans an invariant subspace: finish with its Ritz vector
                  const double th = kth_eig(C->a, C->b, kk, 0);
                  C->theta = th;
                  tridiag_eigvec(C->a, C->b, kk, th, C->s);
                  C->j = kk - 1;
                  C->res_est = 0.0;
                  C->status = SA_OK;
                  C->action = ACT_DONE;
                } else {
                  C->b[kk - 1] = nf;
                  C->inv_b = 1.0 / nf;
                  C->j = kk;
                  C->action = ACT_NEXT;
                }
              }
            })) return;
        mark(4);
        if (vload(&C->action) == ACT_DONE) break;
        continue;
      }
      break;   // ACT_DONE
    }
    if (restart_p0) continue;
    break;
  }

  // ---------------- F1: Ritz vector y = V s, norm, alignment dot ------------------------------
  const int jf = vload(&C->j);
  if (threadIdx.x <= jf) sh[threadIdx.x] = vload(&C->s[threadIdx.x]);
  __syncthreads();
  {
    double v[2] = {0.0, 0.0};
    int bad = 0;
    const bool align = P.align && A.has_last;
    for (long long i = gtid; i < n; i += nthreads) {
      const double y = basis_combine(A.V, A.ldv, i, jf, sh);
      const T yt = (T)y;
      if (!isfinite((double)yt)) bad = 1;
      A.yout[i] = yt;
      A.u[i] = A.sigma[i] * yt;
      v[0] += (double)yt * (double)yt;
      if (align) v[1] += (double)yt * (double)A.ylast[i];
    }
    if (bad) atomicOr(&C->nonfinite, 1);
    block_store_partials<2>(v, A.part, A.pw, 0, sm, pol.block());
  }
  if (!pol.sync(&C->gs, [&] {
        reduce_partials(A.part, A.pw, pol.nblocks(), 2, sh);
        if (threadIdx.x == 0) {
          const double nrm = sqrt(sh[0]);
          const bool align = P.align && A.has_last;
          C->nrm_y = nrm;
          C->align_dot = align ? sh[1] : 0.0;
          C->bytes += (double)n * sizeof(T) * (double)(jf + 3 + (align ? 1 : 0));
          const double sg = (align && sh[1] < 0.0) ? -1.0 : 1.0;
          C->scale = (nrm > 0.0) ? sg / nrm : sg;
        }
      })) return;
  mark(5);

  // ---------------- F2: true residual (one SpMV) and rounding -----------------------------------
  const double theta = vload(&C->theta);
  const double scale = vload(&C->scale);
  {
    double v[1] = {0.0};
    if (P.residual_check) {
      const T trho = (T)rho;
      if (!apply([&](long long r, T acc) {
            const T yt = __ldcg(A.yout + r);
            const double yr = (double)yt;
            const double sy = (double)(trho * yt - __ldcg(A.sigma + r) * acc);
            const double rr = sy - theta * yr;
            v[0] += rr * rr;
          })) return;
    }
    if (P.round) {
      const long long nr = (n + 31) & ~31ll;
      const T ts = (T)scale;
      unsigned long long hs = 0ull;
      for (long long i = gtid; i < nr; i += nthreads) {
        bool bit = false;
        if (i < n) {
          const T x = (T)(A.yout[i] * ts) * (T)((double)A.sigma[i] * A.sqrt_c);
          bit = x >= T(0);
        }
        const unsigned int word = __ballot_sync(0xffffffffu, bit);
        if ((threadIdx.x & 31) == 0) {
          A.bits[i >> 5] = word;
          hs += word_mix(i >> 5, word);
        }
      }
      if ((threadIdx.x & 31) == 0 && hs) atomicAdd(&C->sig, hs);
    }
    block_store_partials<1>(v, A.part, A.pw, 0, sm, pol.block());
  }
  if (!pol.sync(&C->gs, [&] {
        reduce_partials(A.part, A.pw, pol.nblocks(), 1, sh);
        if (threadIdx.x == 0) {
          C->rr = sh[0];
          if (P.residual_check) { C->bytes += A.spmv_bytes; C->spmvs += 1; }
          if (P.round) C->bytes += (double)n * sizeof(T) + (double)n / 8.0;
          C->bytes += 2.0 * (double)n * sizeof(T);   // F3
        }
      })) return;
  mark(5);
  // F3: y <- scale * y (aligned, unit norm)
  {
    const T ts = (T)scale;
    for (long long i = gtid; i < n; i += nthreads) A.yout[i] = A.yout[i] * ts;
  }
  mark(5);
}

}  // namespace sa

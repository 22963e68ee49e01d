// Batched SpecAnn: many (instance, seed) problems of uneven size through ONE persistent cooperative
// launch (the reference's run_solver loop over instances and seeds, utils/core.py:103-105, each
// problem a full models/spectral_annealing.py:262-525 solve).
//
// The grid's CTAs are split into teams (contiguous CTA ranges); a team works through its own list
// of problems one after another, each problem with the whole sweep on the device:
//   per alpha: Gershgorin bound and shift (models/spectral_annealing.py:56-67, :579-581), start
//   mode (:589-612), the alpha solve of alpha_body.cuh under TeamPolicy, the breakdown checks and
//   the cold retry with a random start (:614-651), deduplication of the rounded spins by signature
//   plus an exact word comparison (:349-370), and the warm-start commit;
//   after the sweep: the batched local search of ls_body.cuh over the problem's distinct
//   candidates (or only their energies when the local search is off).
// A team of one CTA separates phases with __syncthreads; larger teams (for the large problems)
// use a barrier of their CTAs. Which problems form which team is the host's plan
// (sa_batch_plan: LPT on a cost model, with large problems split over several CTAs) and is an
// input of sa_batch_create, so a caller can measure and pick plans (the Python autotuner).
//
// Memory: the Lanczos and local-search working arrays belong to the team (sized for its largest
// problem, reused problem after problem); only the outputs (candidate stores, per-alpha records,
// summaries) are per problem. The only state that must be zero at launch, the teams' barrier
// blocks, is cleared by one memset that is part of the same (optionally graph-captured) launch.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "alpha_body.cuh"
#include "ls_body.cuh"

namespace sa {

size_t ls_workspace_bytes(long long n, long long nnz, int k, int integer);

constexpr int kBatchThreads = 128;
constexpr int kBatchWarps = kBatchThreads / 32;
constexpr int kBatchPartWidth = 2 * kNcvMax + kDotBatch + 8;
constexpr double kPlanStepFloor = 4.0e5;   // latency floor of a Lanczos step, in bytes-equivalent

// One instance (matrix + prelude of its handle), shared by its seeds.
struct BInstance {
  const void* rowptr;
  const int* col;
  const void* val;
  const WorkItem* items;
  long long n_items;
  const long long* mc_base;
  const double* ld;
  long long n, nnz, W, ldv;
  double c, dmin, dmax, half_log2_c, sqrt_c;
  int integer_J, rp64;
  const int* scol;   // packed signed columns (one coupling magnitude wmag) or null
  double wmag;
};

// Sweep state of the problem a team is running (written in barrier epilogues).
struct BSweep {
  double lam_prev, alpha_prev;
  double pred_residual0;
  int pred_accepted0, first_ok;
  int warm, iy_out, iy_last, iy_prev, has_last, has_prev;
  int ncand, skipped, retried, decision, status, pad;
  unsigned long long t0;
};

// Working arrays of a team.
struct BTeam {
  int b0, nb, first, count;     // CTAs [b0, b0 + nb); problems order[first, first + count)
  void* sigma;
  void* V;
  void* w;
  void* u;
  void* y[3];
  double* part;
  double* dense;
  AlphaCtrl* actrl;
  int* mc_count;
  void* long_part;
  uint32_t* bits;
  char* ls_ws;
  BSweep* sweep;
};

// Outputs of a problem.
struct BProblem {
  int inst, pad;
  unsigned long long seed;
  uint32_t* cand;
  uint32_t* refined;
  unsigned long long* sigs;
  sa_batch_alpha_record* rec;
  sa_batch_summary* sum;
};

struct BatchArgs {
  const BInstance* inst;
  const BTeam* teams;
  int n_teams, pad;
  const BProblem* probs;
  const int* order;
  GridSync* team_gs;
  const sa_batch_config* cfg;
  const double* alphas;
  int capacity, ncv_max;
};

__device__ __forceinline__ double gershgorin_dev(double dmin, double dmax, double alpha) {
  const double e = 1.0 - alpha;
  double r = -INFINITY;
  const double ds[2] = {dmin, dmax};
  for (int q = 0; q < 2; ++q) {
    const double d = ds[q];
    const double v = d > 0.0 ? pow(d, e) : (e > 0.0 ? 0.0 : (e == 0.0 ? 1.0 : INFINITY));
    r = fmax(r, v);
  }
  return r;
}

__device__ __forceinline__ double shift_rho_dev(double lam_prev, double g, double eps) {
  const double base = (!(lam_prev > 0.0) || !isfinite(lam_prev)) ? g : fmax(lam_prev, g);
  double rho = (1.0 + eps) * base;
  if (rho <= 0.0) rho = (1.0 + eps) * fmax(g, 1.0);
  return rho;
}

__device__ __forceinline__ void ls_geometry_dev(int k, int* kp, int* kw, int* cp) {
  const int p = k <= 8 ? 8 : (k <= 16 ? 16 : 32 * ((k + 31) / 32));
  *kp = p;
  *kw = p >= 32 ? p / 32 : 1;
  *cp = p >= 32 ? 32 : p;
}

// The local search (or only the energies) of the problem's k candidates on the team.
template <typename T, typename RP, typename GT>
__device__ bool batch_ls(const BatchArgs& B, const BTeam& tm, const BProblem& pr, const BInstance& I, int k,
                         const TeamPolicy& pol) {
  __shared__ LsArgs<T, RP, GT> L;
  const sa_batch_config& cfg = *B.cfg;
  if (threadIdx.x == 0) {
    int kp, kw, cp;
    ls_geometry_dev(k, &kp, &kw, &cp);
    const long long n = I.n;
    const long long wl_cap = n + I.nnz / kChunk + 2;
    char* ws = tm.ls_ws;
    Layout Ly;
    const size_t o_ctrl = Ly.off(sizeof(LsCtrl));
    const size_t o_eb = Ly.off(sizeof(double) * 128);
    const size_t o_ea = Ly.off(sizeof(double) * 128);
    const size_t o_sb = Ly.off(sizeof(uint32_t) * (size_t)n * kw);
    const size_t o_fm = Ly.off(sizeof(uint32_t) * (size_t)n * kw);
    const size_t o_h = Ly.off(sizeof(GT) * (size_t)n * kp);
    const size_t o_wl = Ly.off(sizeof(long long) * (size_t)wl_cap);
    const size_t o_wm = Ly.off(sizeof(uint32_t) * (size_t)n * kw);
    const size_t o_pr = Ly.off(sizeof(int) * (size_t)n);
    const size_t o_wq = Ly.off(sizeof(int) * (size_t)n);
    L.rowptr = (const RP*)I.rowptr;
    L.col = I.col;
    L.val = (const T*)I.val;
    L.items = I.items;
    L.n_items = I.n_items;
    L.n = n;
    L.k = k;
    L.kp = kp;
    L.kw = kw;
    L.cp = cp;
    L.sb = (uint32_t*)(ws + o_sb);
    L.h = (GT*)(ws + o_h);
    L.flipm = (uint32_t*)(ws + o_fm);
    L.wl = (long long*)(ws + o_wl);
    L.wl_cap = wl_cap;
    L.wm = (uint32_t*)(ws + o_wm);
    L.prio = (int*)(ws + o_pr);
    L.wq = (int*)(ws + o_wq);
    L.priority = cfg.ls_semantics == 0 ? 1 : 0;
    L.ctrl = (LsCtrl*)(ws + o_ctrl);
    L.ebefore = (typename LsArgs<T, RP, GT>::EAccPtr)(ws + o_eb);
    L.eafter = (typename LsArgs<T, RP, GT>::EAccPtr)(ws + o_ea);
    L.cand = pr.cand;
    L.refined = pr.refined;
    L.W = I.W;
    sa_ls_params p;
    p.k = k;
    p.first_slot = 0;
    p.max_iterations = cfg.use_local_search ? cfg.max_local_iterations : 0;
    p.subset_fraction = cfg.subset_fraction;
    p.final_sweep_fraction = cfg.final_sweep_fraction;
    p.final_sweep_iters = cfg.use_local_search ? cfg.final_sweep_iters : 0;
    p.num_rounds = cfg.use_local_search ? cfg.num_rounds : 0;
    p.seed = pr.seed;
    p.semantics = cfg.ls_semantics;
    p.reserved = 0;
    L.p = p;
    L.m_main = (long long)(p.subset_fraction * (double)n);
    if (L.m_main < 1) L.m_main = 1;
    L.m_final = (long long)(p.final_sweep_fraction * (double)n);
    if (L.m_final < 1) L.m_final = 1;
  }
  __syncthreads();
  ls_body<T, RP, GT>(L, pol);
  if (ld_volatile_i32(&pol.gs->error)) return false;
  return pol.sync(nullptr, [&] {
    if (threadIdx.x == 0) {
      const LsCtrl* C = L.ctrl;
      pr.sum->ls_iterations = C->it;
      pr.sum->ls_final_passes = C->final_passes;
      pr.sum->ls_total_flips = C->total_flips;
      pr.sum->integer_gains = std::is_same<GT, int>::value ? 1 : 0;
    }
    for (int q = threadIdx.x; q < k; q += blockDim.x) {
      double eb, ea;
      if (std::is_same<GT, int>::value) {
        eb = -0.5 * (double)((const long long*)L.ebefore)[q];
        ea = -0.5 * (double)((const long long*)L.eafter)[q];
      } else {
        eb = -0.5 * ((const double*)L.ebefore)[q];
        ea = -0.5 * ((const double*)L.eafter)[q];
      }
      pr.sum->energy_before[q] = eb;
      pr.sum->energy_after[q] = ea;
    }
  });
}

// The whole sweep of problem p on the team. Returns false when the team's barrier failed (the
// team then stops).
template <typename T, typename RP>
__device__ bool batch_problem(const BatchArgs& B, const BTeam& tm, int p, const TeamPolicy& pol) {
  __shared__ AlphaArgs<T, RP> A;
  __shared__ int s_dec, s_found;
  const BProblem& pr = B.probs[p];
  const BInstance& I = B.inst[pr.inst];
  const sa_batch_config& cfg = *B.cfg;
  BSweep* S = tm.sweep;
  const long long n = I.n;
  // CuPy's default basis min(33, n - 1) unless one is given, at least 2, at most the workspace's
  int ncv = cfg.ncv > 0 ? cfg.ncv : (int)(n - 1 < 33 ? n - 1 : 33);
  ncv = min(ncv, (int)(n > 2 ? (n < (long long)kNcvMax ? n : (long long)kNcvMax) : 2));
  ncv = max(2, min(ncv, B.ncv_max));
  const double eps = cfg.shift_eps;

  // problem start: sweep state, zero multi-chunk tickets (they reset themselves after every SpMV)
  if (pol.block() == 0 && threadIdx.x == 0) {
    S->lam_prev = nan("");
    S->alpha_prev = nan("");
    S->warm = 0;
    S->iy_out = 0; S->iy_last = 1; S->iy_prev = 2;
    S->has_last = 0; S->has_prev = 0;
    S->ncand = 0; S->skipped = 0; S->retried = 0;
    S->status = SA_OK;
    S->t0 = global_ns();
    for (int q = 0; q < 6; ++q) pr.sum->phase_ms[q] = 0.0;
  }
  for (long long i = pol.tid(); i < (long long)(I.nnz / (kChunk + 1) + 1); i += pol.nthr()) tm.mc_count[i] = 0;
  if (!pol.sync(nullptr)) return false;

  for (int a = 0; a < cfg.num_alphas; ++a) {
    const double alpha = B.alphas[a];
    for (int att = 0; att < 2; ++att) {
      const double lam_prev = *((volatile double*)&S->lam_prev);
      const double alpha_prev = *((volatile double*)&S->alpha_prev);
      const int warm = ld_volatile_i32(&S->warm);
      const double g = gershgorin_dev(I.dmin, I.dmax, alpha);
      const double rho = shift_rho_dev(lam_prev, g, eps);
      int mode;
      if (att == 1 || a == 0 || !cfg.warm_start || !warm) mode = SA_START_RANDOM;
      else mode = cfg.pred_mode;
      if (threadIdx.x == 0) {
        A.S.rowptr = (const RP*)I.rowptr;
        A.S.col = I.col;
        A.S.val = (const T*)I.val;
        A.S.items = I.items;
        A.S.n_items = I.n_items;
        A.S.mc_base = I.mc_base;
        A.S.mc_count = tm.mc_count;
        A.S.long_part = (T*)tm.long_part;
        A.S.scol = I.scol;
        A.S.wmag = (T)I.wmag;
        A.use_panel = 0;
        A.n_splits = 0;
        A.n = n;
        A.ldv = I.ldv;
        A.sigma = (T*)tm.sigma;
        A.ld = I.ld;
        A.aoff = nullptr;
        A.V = (T*)tm.V;
        A.w = (T*)tm.w;
        A.u = (T*)tm.u;
        A.ylast = (const T*)tm.y[ld_volatile_i32(&S->iy_last)];
        A.yprev = (const T*)tm.y[ld_volatile_i32(&S->iy_prev)];
        A.yout = (T*)tm.y[ld_volatile_i32(&S->iy_out)];
        A.v0 = nullptr;
        A.part = tm.part;
        A.pw = kBatchPartWidth;
        A.ctrl = tm.actrl;
        A.bits = tm.bits;
        A.W = I.W;
        sa_alpha_params q;
        memset(&q, 0, sizeof(q));
        q.alpha = alpha;
        q.alpha_prev = isfinite(alpha_prev) ? alpha_prev : alpha;
        q.rho = rho;
        q.gershgorin = g;
        q.tol = cfg.eigsh_tol;
        q.pred_tol = cfg.pred_tol;
        q.secant_gamma = cfg.secant_gamma;
        q.maxiter = cfg.maxiter;
        q.ncv = ncv;
        q.start_mode = mode;
        q.align = 1;
        q.seed = pr.seed;
        q.stream_id = 4 * a + att;
        q.v0 = nullptr;
        q.round = 1;
        q.residual_check = cfg.residual_check;
        A.p = q;
        A.has_last = ld_volatile_i32(&S->has_last);
        A.has_prev = ld_volatile_i32(&S->has_prev);
        A.half_log2_c = I.half_log2_c;
        A.sqrt_c = I.sqrt_c;
        A.group = 8;
        A.spmv_bytes = (double)I.nnz * (4.0 + sizeof(T)) + (double)(n + 1) * sizeof(RP) + 3.0 * (double)n * sizeof(T);
        A.dense = tm.dense;
      }
      __syncthreads();
      alpha_body<T, RP, TeamPolicy, kBatchWarps, false>(A, pol);
      if (ld_volatile_i32(&pol.gs->error)) return false;
      if (pol.block() == 0 && threadIdx.x == 0)
        for (int q = 0; q < 6; ++q) pr.sum->phase_ms[q] += (double)tm.actrl->tph[q] * 1e-6;
      // decision (models/spectral_annealing.py:614-651): accept, retry cold, or skip the alpha
      if (!pol.sync(nullptr, [&] {
            if (threadIdx.x == 0) {
              const AlphaCtrl* C = tm.actrl;
              int st = C->status;
              if (C->nonfinite && st == SA_OK) st = SA_ERR_NONFINITE;
              bool breakdown = false, error = false;
              if (st == SA_ERR_BREAKDOWN || st == SA_ERR_NONFINITE) breakdown = true;
              else if (st != SA_OK && st != SA_ERR_NOT_CONVERGED) error = true;
              else if (!isfinite(C->theta)) breakdown = true;
              else if (rho - C->theta > g * (1.0 + fmax(0.5 * eps, 1e-5))) breakdown = true;
              if (att == 0) {
                S->pred_residual0 = C->pred_residual;
                S->pred_accepted0 = C->pred_accepted;
                S->first_ok = (breakdown || error) ? 0 : 1;
              }
              S->status = st;
              S->decision = breakdown ? (att == 0 ? 1 : 2) : (error ? 2 : 0);
              s_dec = S->decision;
              s_found = -1;
            }
            __syncthreads();
            const int dec = s_dec;
            sa_batch_alpha_record* R = pr.rec + a;
            if (dec == 1) return;      // cold retry next
            const AlphaCtrl* C = tm.actrl;
            if (dec == 2) {            // skipped alpha
              if (threadIdx.x == 0) {
                memset(R, 0, sizeof(*R));
                R->alpha = alpha;
                R->lambda1 = nan("");
                R->rho = rho;
                R->gershgorin = g;
                R->residual = nan("");
                R->pred_residual = nan("");
                R->degree_scale = nan("");
                R->status = S->status;
                R->pred_accepted = -1;
                R->retry = att;
                R->candidate = -1;
                S->skipped += 1;
              }
              return;
            }
            // accepted: deduplicate (signature, then the packed words), commit, record
            const unsigned long long sig = C->sig;
            const int nc = S->ncand;
            for (int c = 0; c < nc; ++c) {
              if (__ldcg(pr.sigs + c) != sig) continue;
              int diff = 0;
              const uint32_t* cw = pr.cand + (size_t)c * I.W;
              for (long long w = threadIdx.x; w < I.W; w += blockDim.x) diff |= (__ldcg(cw + w) != __ldcg(tm.bits + w));
              if (!__syncthreads_or(diff)) { s_found = c; break; }
            }
            __syncthreads();
            int slot = s_found;
            if (slot < 0) {
              slot = nc;
              uint32_t* dst = pr.cand + (size_t)slot * I.W;
              for (long long w = threadIdx.x; w < I.W; w += blockDim.x) dst[w] = __ldcg(tm.bits + w);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
              if (slot == nc) { pr.sigs[slot] = sig; S->ncand = nc + 1; }
              const double lam = rho - C->theta;
              const double resid = cfg.residual_check ? (C->nrm_y > 0.0 ? sqrt(C->rr) / C->nrm_y : nan("")) : nan("");
              R->alpha = alpha;
              R->lambda1 = lam;
              R->rho = rho;
              R->gershgorin = g;
              R->residual = resid;
              R->pred_residual = S->first_ok ? S->pred_residual0 : C->pred_residual;
              R->degree_scale = C->degree_scale;
              R->signature = sig;
              R->status = S->status;
              R->iterations = C->iters;
              R->restarts = C->restarts;
              R->spmv_count = C->spmvs;
              R->pred_accepted = S->first_ok ? S->pred_accepted0 : C->pred_accepted;
              R->retry = att;
              R->converged = (S->status == SA_OK || (isfinite(resid) && resid <= cfg.eigsh_tol)) ? 1 : 0;
              R->candidate = slot;
              S->retried += att;
              if (cfg.warm_start) {
                const int old_prev = S->iy_prev;
                S->iy_prev = S->iy_last;
                S->iy_last = S->iy_out;
                S->iy_out = old_prev;
                S->has_prev = S->has_last;
                S->has_last = 1;
                S->lam_prev = lam;
                S->alpha_prev = alpha;
                S->warm = 1;
              }
            }
          })) return false;
      if (ld_volatile_i32(&S->decision) != 1) break;
    }
  }

  // the local search of the distinct candidates (energies only when it is off)
  const int k = ld_volatile_i32(&S->ncand);
  if (pol.block() == 0 && threadIdx.x == 0) {
    sa_batch_summary* Z = pr.sum;
    Z->num_candidates = k;
    Z->alphas_skipped = S->skipped;
    Z->alphas_retried = S->retried;
    Z->team_first_block = tm.b0;
    Z->team_blocks = tm.nb;
    Z->ls_iterations = 0;
    Z->ls_final_passes = 0;
    Z->ls_total_flips = 0;
    Z->integer_gains = I.integer_J;
    Z->status = k > 0 ? SA_OK : SA_ERR_BREAKDOWN;
  }
  const unsigned long long t_ls = global_ns();
  if (k > 0) {
    const bool ok = I.integer_J ? batch_ls<T, RP, int>(B, tm, pr, I, k, pol) : batch_ls<T, RP, double>(B, tm, pr, I, k, pol);
    if (!ok) return false;
  }
  if (pol.block() == 0 && threadIdx.x == 0) {
    const unsigned long long t1 = global_ns();
    pr.sum->device_ms = (double)(t1 - S->t0) * 1e-6;
    pr.sum->ls_ms = (double)(t1 - t_ls) * 1e-6;
  }
  return true;
}

template <typename T, typename RP>
__global__ void __launch_bounds__(kBatchThreads, 4) batch_kernel(BatchArgs B) {
  __shared__ int s_team;
  if (threadIdx.x == 0) {
    s_team = -1;
    for (int t = 0; t < B.n_teams; ++t) {
      const int b0 = B.teams[t].b0, nb = B.teams[t].nb;
      if ((int)blockIdx.x >= b0 && (int)blockIdx.x < b0 + nb) { s_team = t; break; }
    }
  }
  __syncthreads();
  if (s_team < 0) return;
  const BTeam& tm = B.teams[s_team];
  const TeamPolicy pol{tm.b0, tm.nb, B.team_gs + s_team};
  for (int q = 0; q < tm.count; ++q) {
    const int p = B.order[tm.first + q];
    if (!batch_problem<T, RP>(B, tm, p, pol)) {
      if (pol.block() == 0 && threadIdx.x == 0) B.probs[p].sum->status = SA_ERR_BARRIER_TIMEOUT;
      return;
    }
  }
}

void count_launches(int k);

}  // namespace sa

using namespace sa;

struct sa_batch {
  int n_inst = 0, seeds = 0, n_prob = 0, n_teams = 0, prec = 32, rp64 = 0, capacity = 128, ncv_max = 33;
  int grid = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  char* ws = nullptr;
  size_t ws_bytes = 0;
  BatchArgs args;
  GridSync* team_gs = nullptr;
  sa_batch_config* d_cfg = nullptr;
  double* d_alphas = nullptr;
  sa_batch_alpha_record* d_rec = nullptr;
  sa_batch_summary* d_sum = nullptr;
  std::vector<BProblem> probs;
  std::vector<BTeam> teams;
  std::vector<long long> prob_n;
};

namespace {

struct BatchSizes {
  size_t header, team_total, prob_total, total;
};

// Bytes of the working arrays of a team whose problems have at most (n, nnz, ...) of each kind.
size_t team_bytes(long long n, long long nnz, long long n_long_part, int nb, int prec, int ncv_max, int capacity,
                  int integer_all) {
  const size_t T = prec == 32 ? 4 : 8;
  const long long ldv = (n + 63) & ~63ll;
  const long long W = (n + 31) / 32;
  Layout L;
  L.off(T * n);                                  // sigma
  L.off(T * (size_t)ldv * ncv_max);              // V
  L.off(T * n);                                  // w
  L.off(T * n);                                  // u
  for (int q = 0; q < 3; ++q) L.off(T * n);      // y
  L.off(8 * (size_t)nb * kBatchPartWidth);       // part
  L.off(8 * 2 * (size_t)kNcvMax * kNcvMax);      // dense
  L.off(sizeof(AlphaCtrl));
  L.off(4 * (size_t)(nnz / (kChunk + 1) + 1));   // mc_count
  L.off(T * (size_t)std::max(1ll, n_long_part)); // long_part
  L.off(4 * (size_t)W);                          // bits
  L.off(ls_workspace_bytes(n, nnz, capacity, integer_all));
  L.off(sizeof(BSweep));
  return L.total;
}

size_t prob_bytes(long long n, int capacity, int num_alphas_max) {
  const long long W = (n + 31) / 32;
  Layout L;
  L.off(4 * (size_t)W * capacity);       // cand
  L.off(4 * (size_t)W * capacity);       // refined
  L.off(8 * (size_t)capacity);           // sigs
  L.off(sizeof(sa_batch_alpha_record) * (size_t)num_alphas_max);
  L.off(sizeof(sa_batch_summary));
  return L.total;
}

int check_plan(int n_prob, int n_teams, const int32_t* team_b0, const int32_t* team_nb, const int32_t* team_of,
               int grid) {
  if (n_teams < 1 || !team_b0 || !team_nb || !team_of) return SA_ERR_INVALID_ARG;
  int end = 0;
  for (int t = 0; t < n_teams; ++t) {
    if (team_nb[t] < 1 || team_b0[t] != end) return SA_ERR_INVALID_ARG;   // contiguous, in order
    end = team_b0[t] + team_nb[t];
  }
  if (grid > 0 && end > grid) return SA_ERR_INVALID_ARG;
  for (int p = 0; p < n_prob; ++p)
    if (team_of[p] < 0 || team_of[p] >= n_teams) return SA_ERR_INVALID_ARG;
  return SA_OK;
}

int inst_ok(int n_inst, sa_handle* const* inst, int* prec, int* rp64) {
  if (n_inst < 1 || !inst) return SA_ERR_INVALID_ARG;
  for (int i = 0; i < n_inst; ++i) {
    if (!inst[i] || !inst[i]->bound) return SA_ERR_INVALID_ARG;
    if (inst[i]->prec != inst[0]->prec || inst[i]->rp64 != inst[0]->rp64) return SA_ERR_INVALID_ARG;
  }
  *prec = inst[0]->prec;
  *rp64 = inst[0]->rp64;
  return SA_OK;
}

BatchSizes sizes(int n_inst, sa_handle* const* inst, int seeds, int ncv_max, int capacity, int n_teams,
                 const int32_t* team_nb, const int32_t* team_of) {
  BatchSizes s{0, 0, 0, 0};
  const int n_prob = n_inst * seeds;
  Layout H;
  H.off(sizeof(BInstance) * (size_t)n_inst);
  H.off(sizeof(BTeam) * (size_t)n_teams);
  H.off(sizeof(BProblem) * (size_t)n_prob);
  H.off(sizeof(int) * (size_t)n_prob);
  H.off(sizeof(GridSync) * (size_t)n_teams);
  H.off(sizeof(sa_batch_config));
  H.off(sizeof(double) * 128);
  s.header = H.total;
  const int prec = inst[0]->prec;
  for (int t = 0; t < n_teams; ++t) {
    long long n = 1, nnz = 0, nlp = 0;
    int integer_all = 1;
    for (int p = 0; p < n_prob; ++p) {
      if (team_of[p] != t) continue;
      const sa_handle* h = inst[p / seeds];
      n = std::max(n, h->n);
      nnz = std::max(nnz, h->nnz);
      nlp = std::max(nlp, h->n_long_part);
      integer_all &= h->integer_J;
    }
    s.team_total += team_bytes(n, nnz, nlp, team_nb[t], prec, ncv_max, capacity, integer_all);
  }
  for (int p = 0; p < n_prob; ++p) s.prob_total += prob_bytes(inst[p / seeds]->n, capacity, 128);
  s.total = s.header + s.team_total + s.prob_total;
  return s;
}

}  // namespace

extern "C" {

int sa_batch_grid(int32_t precision, int32_t rowptr64, int32_t* blocks) {
  // batched instances are small (n <= 2^31 stored entries): 32-bit row pointers only
  if (!blocks || (precision != 32 && precision != 64) || rowptr64) return SA_ERR_INVALID_ARG;
  int dev = 0, sms = 0, occ = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return SA_ERR_CUDA;
  const void* fn = precision == 32 ? (const void*)batch_kernel<float, int> : (const void*)batch_kernel<double, int>;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kBatchThreads, 0) != cudaSuccess) return SA_ERR_CUDA;
  *blocks = sms * occ;
  return *blocks > 0 ? SA_OK : SA_ERR_CUDA;
}

int sa_batch_plan(int32_t n_prob, const int64_t* n, const int64_t* nnz, const double* measured_cost, int32_t blocks,
                  double split, double barrier_cost, int32_t* team_of, int32_t* team_b0, int32_t* team_nb,
                  int32_t* n_teams) {
  if (n_prob < 1 || !n || !nnz || blocks < 1 || !(split > 0.0) || !(barrier_cost >= 0.0) || !team_of || !team_b0 ||
      !team_nb || !n_teams)
    return SA_ERR_INVALID_ARG;
  // cost of a problem on one CTA: measured (CTA-time of an earlier run), else the model of one
  // Lanczos step in bytes moved (SpMV stream, ~24 basis-vector passes) plus a latency floor that
  // dominates for small problems (a step of a few tiles per warp still pays its phases' latency)
  std::vector<double> cost(n_prob);
  double total = 0.0;
  for (int p = 0; p < n_prob; ++p) {
    if (n[p] < 1 || nnz[p] < 0) return SA_ERR_INVALID_ARG;
    if (measured_cost) {
      if (!(measured_cost[p] > 0.0) || !std::isfinite(measured_cost[p])) return SA_ERR_INVALID_ARG;
      cost[p] = measured_cost[p];
    } else {
      cost[p] = 8.0 * (double)nnz[p] + 100.0 * (double)n[p] + kPlanStepFloor;
    }
    total += cost[p];
  }
  std::vector<int> ord(n_prob);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  // Finish time M of the plan: a problem whose cost exceeds M gets its own team of
  // nb = ceil(split c (1 + barrier_cost) / M) CTAs when that is 2 or more; the others share
  // single-CTA teams, as many as their total cost needs at M. The smallest M whose plan fits in
  // `blocks` CTAs is found by bisection (the CTA count needed falls as M grows).
  const double b1 = 1.0 + barrier_cost;
  auto team_size = [&](int p, double M) -> long long {
    if (cost[p] <= M) return 1;
    return (long long)std::ceil(split * cost[p] * b1 / M);
  };
  auto ctas_for = [&](double M, int* n_small_ctas) {
    long long need = 0;
    double small = 0.0;
    for (int p = 0; p < n_prob; ++p) {
      const long long nb = team_size(p, M);
      if (nb >= 2) need += nb;
      else small += cost[p];
    }
    const int ns = small > 0.0 ? (int)std::max(1.0, std::ceil(small / M)) : 0;
    if (n_small_ctas) *n_small_ctas = ns;
    return need + ns;
  };
  double lo = total / (double)blocks * 0.5, hi = total * b1 * 2.0 + 1.0;
  for (int it = 0; it < 200 && hi - lo > 1e-9 * hi; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (ctas_for(mid, nullptr) <= blocks) hi = mid;
    else lo = mid;
  }
  const double M = hi;
  int n_small_ctas = 0;
  ctas_for(M, &n_small_ctas);
  struct Team { int nb; double load; };
  std::vector<Team> teams;
  for (int p = 0; p < n_prob; ++p) team_of[p] = -1;
  auto t_on = [&](int p, int nb) { return cost[p] / (double)nb * (nb > 1 ? b1 : 1.0); };
  for (int p : ord) {                                    // own teams for the large problems
    const int nb = (int)team_size(p, M);
    if (nb < 2) continue;
    team_of[p] = (int)teams.size();
    teams.push_back({nb, t_on(p, nb)});
  }
  const int first_small = (int)teams.size();
  for (int q = 0; q < n_small_ctas; ++q) teams.push_back({1, 0.0});
  for (int p : ord) {                                    // LPT over the single-CTA teams
    if (team_of[p] >= 0) continue;
    int best = first_small;
    for (int t = first_small; t < (int)teams.size(); ++t)
      if (teams[t].load < teams[best].load) best = t;
    team_of[p] = best;
    teams[best].load += cost[p];
  }
  // drop empty teams, renumber contiguously
  std::vector<int> remap(teams.size(), -1);
  int nt = 0, b0 = 0;
  for (int t = 0; t < (int)teams.size(); ++t) {
    bool any = false;
    for (int p = 0; p < n_prob && !any; ++p) any = team_of[p] == t;
    if (!any) continue;
    remap[t] = nt;
    team_b0[nt] = b0;
    team_nb[nt] = teams[t].nb;
    b0 += teams[t].nb;
    ++nt;
  }
  for (int p = 0; p < n_prob; ++p) team_of[p] = remap[team_of[p]];
  *n_teams = nt;
  return SA_OK;
}

int sa_batch_workspace_size(int32_t n_inst, sa_handle* const* inst, int32_t seeds_per_instance, int32_t ncv_max,
                            int32_t capacity, int32_t n_teams, const int32_t* team_b0, const int32_t* team_nb,
                            const int32_t* team_of, size_t* bytes) {
  int prec = 0, rp64 = 0;
  if (!bytes || seeds_per_instance < 1 || ncv_max < 2 || ncv_max > kNcvMax || capacity < 1 || capacity > 128)
    return SA_ERR_INVALID_ARG;
  int st = inst_ok(n_inst, inst, &prec, &rp64);
  if (st != SA_OK) return st;
  if (rp64) return SA_ERR_INVALID_ARG;
  st = check_plan(n_inst * seeds_per_instance, n_teams, team_b0, team_nb, team_of, 0);
  if (st != SA_OK) return st;
  *bytes = sizes(n_inst, inst, seeds_per_instance, ncv_max, capacity, n_teams, team_nb, team_of).total;
  return SA_OK;
}

int sa_batch_create(sa_batch** out, int32_t n_inst, sa_handle* const* inst, int32_t seeds_per_instance,
                    const uint64_t* seeds, int32_t ncv_max, int32_t capacity, int32_t n_teams, const int32_t* team_b0,
                    const int32_t* team_nb, const int32_t* team_of, void* workspace, size_t bytes, void* stream) {
  if (!out || !seeds) return SA_ERR_INVALID_ARG;
  *out = nullptr;
  size_t need = 0;
  int st = sa_batch_workspace_size(n_inst, inst, seeds_per_instance, ncv_max, capacity, n_teams, team_b0, team_nb,
                                   team_of, &need);
  if (st != SA_OK) return st;
  if (!workspace || bytes < need) return SA_ERR_OOM;
  if (((uintptr_t)workspace) & 255) return SA_ERR_INVALID_ARG;
  int prec = 0, rp64 = 0;
  inst_ok(n_inst, inst, &prec, &rp64);
  int grid = 0;
  st = sa_batch_grid(prec, rp64, &grid);
  if (st != SA_OK) return st;
  const int n_prob = n_inst * seeds_per_instance;
  st = check_plan(n_prob, n_teams, team_b0, team_nb, team_of, grid);
  if (st != SA_OK) return st;

  sa_batch* b = new sa_batch();
  b->n_inst = n_inst;
  b->seeds = seeds_per_instance;
  b->n_prob = n_prob;
  b->n_teams = n_teams;
  b->prec = prec;
  b->rp64 = rp64;
  b->capacity = capacity;
  b->ncv_max = ncv_max;
  b->grid = grid;
  b->stream = (cudaStream_t)stream;
  b->ws = (char*)workspace;
  b->ws_bytes = bytes;
  const BatchSizes sz = sizes(n_inst, inst, seeds_per_instance, ncv_max, capacity, n_teams, team_nb, team_of);
  const size_t T = prec == 32 ? 4 : 8;

  // header
  Layout H;
  const size_t o_inst = H.off(sizeof(BInstance) * (size_t)n_inst);
  const size_t o_team = H.off(sizeof(BTeam) * (size_t)n_teams);
  const size_t o_prob = H.off(sizeof(BProblem) * (size_t)n_prob);
  const size_t o_ord = H.off(sizeof(int) * (size_t)n_prob);
  const size_t o_gs = H.off(sizeof(GridSync) * (size_t)n_teams);
  const size_t o_cfg = H.off(sizeof(sa_batch_config));
  const size_t o_alp = H.off(sizeof(double) * 128);
  std::vector<BInstance> hi(n_inst);
  for (int i = 0; i < n_inst; ++i) {
    const sa_handle* h = inst[i];
    BInstance& I = hi[i];
    I.rowptr = h->rowptr;
    I.col = h->col;
    I.val = h->val;
    I.items = h->items;
    I.n_items = h->n_items;
    I.mc_base = h->mc_base;
    I.ld = h->ld;
    I.n = h->n;
    I.nnz = h->nnz;
    I.W = h->W;
    I.ldv = h->ldv;
    I.c = h->c;
    I.dmin = h->dmin;
    I.dmax = h->dmax;
    I.half_log2_c = 0.5 * std::log2(h->c);
    I.sqrt_c = std::sqrt(h->c);
    I.integer_J = h->integer_J;
    I.rp64 = h->rp64;
    I.scol = h->packed ? h->scol : nullptr;
    I.wmag = h->wmag;
  }
  // teams: working arrays
  char* base = b->ws + sz.header;
  std::vector<int> order;
  b->teams.resize(n_teams);
  size_t off = 0;
  for (int t = 0; t < n_teams; ++t) {
    long long n = 1, nnz = 0, nlp = 0;
    int integer_all = 1;
    BTeam& tm = b->teams[t];
    tm.b0 = team_b0[t];
    tm.nb = team_nb[t];
    tm.first = (int)order.size();
    for (int p = 0; p < n_prob; ++p) {
      if (team_of[p] != t) continue;
      order.push_back(p);
      const sa_handle* h = inst[p / seeds_per_instance];
      n = std::max(n, h->n);
      nnz = std::max(nnz, h->nnz);
      nlp = std::max(nlp, h->n_long_part);
      integer_all &= h->integer_J;
    }
    tm.count = (int)order.size() - tm.first;
    const long long ldv = (n + 63) & ~63ll;
    const long long W = (n + 31) / 32;
    char* tb = base + off;
    Layout L;
    tm.sigma = tb + L.off(T * n);
    tm.V = tb + L.off(T * (size_t)ldv * ncv_max);
    tm.w = tb + L.off(T * n);
    tm.u = tb + L.off(T * n);
    for (int q = 0; q < 3; ++q) tm.y[q] = tb + L.off(T * n);
    tm.part = (double*)(tb + L.off(8 * (size_t)tm.nb * kBatchPartWidth));
    tm.dense = (double*)(tb + L.off(8 * 2 * (size_t)kNcvMax * kNcvMax));
    tm.actrl = (AlphaCtrl*)(tb + L.off(sizeof(AlphaCtrl)));
    tm.mc_count = (int*)(tb + L.off(4 * (size_t)(nnz / (kChunk + 1) + 1)));
    tm.long_part = tb + L.off(T * (size_t)std::max(1ll, nlp));
    tm.bits = (uint32_t*)(tb + L.off(4 * (size_t)W));
    tm.ls_ws = tb + L.off(ls_workspace_bytes(n, nnz, capacity, integer_all));
    tm.sweep = (BSweep*)(tb + L.off(sizeof(BSweep)));
    off += L.total;
  }
  // problems: outputs
  char* pbase = base + sz.team_total;
  b->probs.resize(n_prob);
  b->prob_n.resize(n_prob);
  off = 0;
  for (int p = 0; p < n_prob; ++p) {
    const sa_handle* h = inst[p / seeds_per_instance];
    const long long W = h->W;
    BProblem& pr = b->probs[p];
    char* pb = pbase + off;
    Layout L;
    pr.inst = p / seeds_per_instance;
    pr.pad = 0;
    pr.seed = seeds[p];
    pr.cand = (uint32_t*)(pb + L.off(4 * (size_t)W * capacity));
    pr.refined = (uint32_t*)(pb + L.off(4 * (size_t)W * capacity));
    pr.sigs = (unsigned long long*)(pb + L.off(8 * (size_t)capacity));
    pr.rec = (sa_batch_alpha_record*)(pb + L.off(sizeof(sa_batch_alpha_record) * 128));
    pr.sum = (sa_batch_summary*)(pb + L.off(sizeof(sa_batch_summary)));
    off += L.total;
    b->prob_n[p] = h->n;
  }
  b->team_gs = (GridSync*)(b->ws + o_gs);
  b->d_cfg = (sa_batch_config*)(b->ws + o_cfg);
  b->d_alphas = (double*)(b->ws + o_alp);
  BatchArgs& A = b->args;
  A.inst = (const BInstance*)(b->ws + o_inst);
  A.teams = (const BTeam*)(b->ws + o_team);
  A.n_teams = n_teams;
  A.pad = 0;
  A.probs = (const BProblem*)(b->ws + o_prob);
  A.order = (const int*)(b->ws + o_ord);
  A.team_gs = b->team_gs;
  A.cfg = b->d_cfg;
  A.alphas = b->d_alphas;
  A.capacity = capacity;
  A.ncv_max = ncv_max;
  cudaStream_t s = b->stream;
  bool ok = cudaMemcpyAsync(b->ws + o_inst, hi.data(), sizeof(BInstance) * n_inst, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(b->ws + o_team, b->teams.data(), sizeof(BTeam) * n_teams, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(b->ws + o_prob, b->probs.data(), sizeof(BProblem) * n_prob, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemcpyAsync(b->ws + o_ord, order.data(), sizeof(int) * n_prob, cudaMemcpyHostToDevice, s) == cudaSuccess &&
            cudaMemsetAsync(pbase, 0, sz.prob_total, s) == cudaSuccess &&
            cudaStreamSynchronize(s) == cudaSuccess;
  if (!ok) { delete b; return SA_ERR_CUDA; }
  *out = b;
  return SA_OK;
}

static int batch_launch(sa_batch* b, cudaStream_t s) {
  if (cudaMemsetAsync(b->team_gs, 0, sizeof(GridSync) * b->n_teams, s) != cudaSuccess) return SA_ERR_CUDA;
  void* args[] = {&b->args};
  const void* fn = b->prec == 32 ? (const void*)batch_kernel<float, int> : (const void*)batch_kernel<double, int>;
  if (cudaLaunchCooperativeKernel(fn, dim3(b->grid), dim3(kBatchThreads), args, 0, s) != cudaSuccess) return SA_ERR_CUDA;
  return SA_OK;
}

int sa_batch_sweep(sa_batch* b, const sa_batch_config* cfg, const double* alphas, int32_t use_graph) {
  if (!b || !cfg || !alphas || cfg->num_alphas < 1 || cfg->num_alphas > 128 || cfg->num_alphas > b->capacity ||
      cfg->ncv > b->ncv_max || cfg->maxiter < 1 || cfg->ls_semantics < 0 || cfg->ls_semantics > 1 ||
      (cfg->pred_mode != SA_START_DIAGONAL && cfg->pred_mode != SA_START_SECANT && cfg->pred_mode != SA_START_PREV))
    return SA_ERR_INVALID_ARG;
  cudaStream_t s = b->stream;
  if (cudaMemcpyAsync(b->d_cfg, cfg, sizeof(*cfg), cudaMemcpyHostToDevice, s) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaMemcpyAsync(b->d_alphas, alphas, sizeof(double) * cfg->num_alphas, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return SA_ERR_CUDA;
  int st;
  if (use_graph) {
    if (!b->graph) {
      // capture the memset and the launch once on a private stream; later sweeps replay it
      if (!b->cap_stream && cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
        return SA_ERR_CUDA;
      cudaGraph_t g = nullptr;
      if (cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SA_ERR_CUDA;
      const int lst = batch_launch(b, b->cap_stream);
      const cudaError_t ec = cudaStreamEndCapture(b->cap_stream, &g);
      if (lst != SA_OK || ec != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return SA_ERR_CUDA;
      }
      const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
      cudaGraphDestroy(g);
      if (ei != cudaSuccess) { b->graph = nullptr; return SA_ERR_CUDA; }
    }
    st = cudaGraphLaunch(b->graph, s) == cudaSuccess ? SA_OK : SA_ERR_CUDA;
  } else {
    st = batch_launch(b, s);
  }
  count_launches(1);
  return st;
}

int sa_batch_results(sa_batch* b, sa_batch_alpha_record* records, sa_batch_summary* summaries) {
  if (!b) return SA_ERR_INVALID_ARG;
  cudaStream_t s = b->stream;
  for (int p = 0; p < b->n_prob; ++p) {
    if (records && cudaMemcpyAsync(records + (size_t)p * 128, b->probs[p].rec, sizeof(sa_batch_alpha_record) * 128,
                                   cudaMemcpyDeviceToHost, s) != cudaSuccess)
      return SA_ERR_CUDA;
    if (summaries && cudaMemcpyAsync(summaries + p, b->probs[p].sum, sizeof(sa_batch_summary), cudaMemcpyDeviceToHost,
                                     s) != cudaSuccess)
      return SA_ERR_CUDA;
  }
  return cudaStreamSynchronize(s) == cudaSuccess ? SA_OK : SA_ERR_CUDA;
}

int sa_batch_candidate(sa_batch* b, int32_t problem, int32_t slot, int32_t refined, uint32_t* packed_device) {
  if (!b || !packed_device || problem < 0 || problem >= b->n_prob || slot < 0 || slot >= b->capacity)
    return SA_ERR_INVALID_ARG;
  const BProblem& pr = b->probs[problem];
  const long long W = (b->prob_n[problem] + 31) / 32;
  const uint32_t* src = (refined ? pr.refined : pr.cand) + (size_t)slot * W;
  return cudaMemcpyAsync(packed_device, src, 4 * W, cudaMemcpyDeviceToDevice, b->stream) == cudaSuccess ? SA_OK
                                                                                                        : SA_ERR_CUDA;
}

int sa_batch_destroy(sa_batch* b) {
  if (!b) return SA_ERR_INVALID_ARG;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
  delete b;
  return SA_OK;
}

}  // extern "C"

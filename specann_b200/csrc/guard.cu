// Guarded local-search policies (ls_policy other than "default"): the refiners of
// models/local_search_guards/ (policies.py:13-69) on the device.
//
//   fixed guard / adaptive guard (safe_flip_refinement, models/spectral_annealing_safe.py:1035-1335):
//     rounds of a Jacobi proposal from the current spins over the selected nodes of every active
//     candidate, kept only if its exact energy change is a strict drop (models/safe_update_policy.py:
//     4-29); the adaptive guard shrinks a rejected candidate's batch fraction and grows an accepted
//     one's (:68-95); a candidate retires after 3 rounds without acceptance; a main phase (subset
//     0.9, max_iterations rounds) then a final phase (subset 1.0, 25 x 25 rounds);
//   independent set (models/local_search_guards/conflict_free.py:80-367): each update flips, in
//     every active candidate, the nodes of one colour class whose gain is negative; classes in a
//     random order per sweep (computed on the host); a candidate retires after a sweep without flips;
//   sequential oracle (models/local_search_guards/sequential_oracle.py:26-219): exact one-flip
//     steepest descent, one CTA per candidate.
//
// One persistent cooperative kernel runs the first three with the node-major field cache of the
// default search (ls_body.cuh): per round (R1) every selected node decides for every candidate from
// the current state; (R2, guards) the exact energy change of each candidate's proposal,
//   dE = sum_{i in F} 2 s_i h_i - 2 sum_{i, j in F} s_i J_ij s_j,
// is summed from the flipping nodes' rows (int64 for integer couplings: exact and order-free);
// (epilogue) acceptance, adaptation and retirement per candidate; (R3) the accepted flips are applied
// and (U) their field changes scattered. Energies are tracked in units of J; the acceptance
// tolerance 1e-10 + 1e-12 max(1, |E / c|) applies to E / c as in the reference (whose energies are
// those of J / c).
#include <cmath>
#include <cstring>

#include "ls_body.cuh"

namespace sa {

namespace {

constexpr double kGuardAbsTol = 1e-10, kGuardRelTol = 1e-12;   // models/local_search_guards/policies.py:28-29
constexpr int kGuardPatience = 3;                                // :32
constexpr double kGuardMinFrac = 0.01, kGuardShrink = 0.5, kGuardGrowth = 1.25;   // :33-35

struct GuardCtrl {
  GridSync gs;
  int phase;                  // 0 main, 1 final (guards) / the updates (independent set), 2 done
  int round;                  // rounds of the current phase
  int rounds_main, rounds_final;
  int accepted, rejected;
  long long wq_count, wl_count;
  long long total_flips;
  unsigned int active[4];
  unsigned int accept[4];
  int streak[128];
  double frac[128];
  long long sel[128];         // nodes selected for each candidate this round (rank < sel)
  long long want[128];        // proposed flips per candidate this round
  long long dE_i[128];        // proposal energy change (integer couplings)
  double dE_d[128];
  long long E_i[128];         // current energies, units of J
  double E_d[128];
  long long sweep_flips[128];
};

template <typename VT, typename RP, typename GT>
struct GuardArgs {
  LsArgs<VT, RP, GT> L;       // fields, spins, work lists, energies (the default search's layout)
  GuardCtrl* G;
  int mode;                   // SA_GUARD_FIXED, SA_GUARD_ADAPTIVE, SA_GUARD_INDEPENDENT_SET
  int num_colors;
  const int* colors;
  const int* color_seq;
  int limit_main, limit_final;   // rounds of the phases (independent set: updates in limit_main)
  double c;                   // normalisation factor (max absolute degree)
};

// Fields of the control block that other CTAs write are read past L1 (it is not coherent with them).
__device__ __forceinline__ long long gld(const long long* p) { return __ldcg(p); }
__device__ __forceinline__ double gld(const double* p) { return __ldcg(p); }
__device__ __forceinline__ int gld(const int* p) { return __ldcg(p); }
__device__ __forceinline__ unsigned int gld(const unsigned int* p) { return __ldcg(p); }

__device__ __forceinline__ double guard_tol(double E_norm) {
  return kGuardAbsTol + kGuardRelTol * fmax(1.0, fabs(E_norm));
}

template <typename GT>
__device__ __forceinline__ double dE_of(const GuardCtrl* G, int q) {
  return std::is_same<GT, int>::value ? (double)gld(&G->dE_i[q]) : gld(&G->dE_d[q]);
}
template <typename GT>
__device__ __forceinline__ double E_of(const GuardCtrl* G, int q) {
  return std::is_same<GT, int>::value ? (double)gld(&G->E_i[q]) : gld(&G->E_d[q]);
}

// Selection counts of the next round: max(1, (int)(fraction * n)) per active candidate.
template <typename VT, typename RP, typename GT>
__device__ void guard_set_selection(const GuardArgs<VT, RP, GT>& A, double fraction) {
  GuardCtrl* G = A.G;
  const long long n = A.L.n;
  for (int q = threadIdx.x; q < A.L.k; q += blockDim.x) {
    const bool act = (gld(&G->active[q >> 5]) >> (q & 31)) & 1u;
    const double f = (A.mode == SA_GUARD_ADAPTIVE) ? gld(&G->frac[q]) : fraction;
    long long m = (long long)(f * (double)n);
    if (m < 1) m = 1;
    G->sel[q] = act ? m : 0;
  }
}

template <typename VT, typename RP, typename GT>
__device__ void guard_start_phase(const GuardArgs<VT, RP, GT>& A, int phase) {
  GuardCtrl* G = A.G;
  const double fraction = phase == 0 ? A.L.p.subset_fraction : A.L.p.final_sweep_fraction;
  if (threadIdx.x == 0) {
    G->phase = phase;
    G->round = 0;
    for (int w = 0; w < 4; ++w) G->active[w] = 0u;
    for (int q = 0; q < A.L.k; ++q) G->active[q >> 5] |= 1u << (q & 31);
  }
  for (int q = threadIdx.x; q < 128; q += blockDim.x) {
    G->streak[q] = 0;
    G->frac[q] = fraction;
    G->sweep_flips[q] = 0;
  }
  __syncthreads();
  guard_set_selection(A, fraction);
}

template <typename VT, typename RP, typename GT>
__global__ void __launch_bounds__(kThreads, 2) guard_kernel(GuardArgs<VT, RP, GT> A) {
  using E = EAcc<GT>;
  const LsArgs<VT, RP, GT>& L = A.L;
  GuardCtrl* G = A.G;
  LsCtrl* C = L.ctrl;               // its GridSync separates the phases
  GridPolicy pol;
  __shared__ E s_acc[128];
  __shared__ long long s_cnt[128];
  __shared__ E s_dE[128];
  __shared__ long long s_sel[128];
  __shared__ unsigned int s_act[4], s_acc_mask[4];
  __shared__ double s_tolc[128];    // independent set: tolerance x c per candidate (non-integer gains)
  const int lane = threadIdx.x & 31;
  const long long gtid = pol.tid(), nthreads = pol.nthr();
  const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const long long n = L.n;
  const int cp = L.cp, ne = 32 / cp, slot = lane / cp, c = lane % cp;
  const bool indep = A.mode == SA_GUARD_INDEPENDENT_SET;

  // ---- set-up: node-major bits, fields, energies -----------------------------------------------
  for (long long i = gtid; i < n; i += nthreads) {
    for (int t = 0; t < L.kw; ++t) {
      uint32_t word = 0u;
      const int c1 = min(L.k, 32 * t + 32);
      for (int q = 32 * t; q < c1; ++q) {
        const uint32_t cw = __ldg(L.cand + (long long)q * L.W + (i >> 5));
        word |= ((cw >> (i & 31)) & 1u) << (q - 32 * t);
      }
      L.sb[i * L.kw + t] = word;
    }
    for (int q = 0; q < L.kp; ++q) L.h[i * L.kp + q] = GT(0);
  }
  for (long long q = gtid; q < L.kp; q += nthreads) { L.ebefore[q] = 0; L.eafter[q] = 0; }
  if (!pol.sync(&C->gs)) return;
  for (long long itm = gwarp; itm < L.n_items; itm += nwarps) {
    const long long e0 = __ldg(&L.items[itm].e0);
    const int irow = __ldg(&L.items[itm].row);
    const int meta = __ldg(&L.items[itm].meta);
    if (irow >= 0) {
      const long long r1 = irow + item_nrows(meta);
      for (long long r = irow; r < r1; ++r) {
        const long long rs = rp_load(L.rowptr, r), re = rp_load(L.rowptr, r + 1);
        for (int t = 0; t < L.kw; ++t) {
          const GT f = row_field(L, rs, re, t);
          if (slot == 0 && 32 * t + c < L.kp) L.h[r * L.kp + 32 * t + c] = f;
        }
      }
    } else {
      const long long row = -((long long)irow + 1);
      for (int t = 0; t < L.kw; ++t) {
        const GT f = row_field(L, e0, e0 + item_len(meta), t);
        if (slot == 0 && 32 * t + c < L.kp) atomicAdd(&L.h[row * L.kp + 32 * t + c], f);
      }
    }
  }
  if (!pol.sync(&C->gs)) return;
  energy_phase(L, L.ebefore, s_acc, gwarp, nwarps);
  if (!pol.sync(&C->gs, [&] {
        for (int q = threadIdx.x; q < L.k; q += blockDim.x) {
          if (std::is_same<GT, int>::value) G->E_i[q] = -(long long)__ldcg((const long long*)L.ebefore + q) / 2;
          else G->E_d[q] = -0.5 * __ldcg((const double*)L.ebefore + q);
          G->want[q] = 0;
          G->dE_i[q] = 0;
          G->dE_d[q] = 0.0;
        }
        if (threadIdx.x == 0) {
          G->rounds_main = G->rounds_final = 0;
          G->accepted = G->rejected = 0;
          G->wq_count = G->wl_count = 0;
          G->total_flips = 0;
        }
        __syncthreads();
        if (indep) {
          guard_start_phase(A, 0);
          if (A.limit_main < 1 && threadIdx.x == 0) G->phase = 2;
        } else if (A.limit_main > 0) {
          guard_start_phase(A, 0);
        } else if (A.limit_final > 0) {
          guard_start_phase(A, 1);
        } else if (threadIdx.x == 0) {
          G->phase = 2;
        }
      })) return;

  // ---- rounds --------------------------------------------------------------------------------
  while (ld_volatile_i32(&G->phase) != 2) {
    const int phase = gld(&G->phase), round = gld(&G->round);
    for (int q = threadIdx.x; q < 128; q += blockDim.x) {
      s_cnt[q] = 0;
      s_dE[q] = E(0);
      s_sel[q] = (q < L.k) ? gld(&G->sel[q]) : 0;
      if (indep && q < L.k) {
        const double Ec = E_of<GT>(G, q);
        s_tolc[q] = guard_tol(Ec / A.c) * A.c;
      }
    }
    if (threadIdx.x < 4) s_act[threadIdx.x] = gld(&G->active[threadIdx.x]);
    __syncthreads();
    const long long stream = phase == 0 ? (long long)round : kFinalStreamBase + round;
    const SelKeys keys = make_sel_keys(L.p.seed, stream, n);
    const int color = indep ? __ldg(A.color_seq + round) : 0;

    // R1: proposals from the current state (wanting masks; the independent set also sums its
    // energy change here, its flips being independent)
    for (long long tile = gwarp * 32; tile < n; tile += nwarps * 32) {
      long long rk = 0x7fffffffffffll;
      bool member = false;
      if (tile + lane < n) {
        if (indep) member = __ldg(A.colors + tile + lane) == color;
        else rk = sel_rank(tile + lane, keys, n);
      }
      uint32_t tile_want = 0u;   // bit l set if node tile + l proposes a flip
      for (int sub = 0; sub < 32; sub += ne) {
        const long long i = tile + sub + slot;
        const long long rki = __shfl_sync(0xffffffffu, rk, (sub + slot) & 31);
        const bool mem = __shfl_sync(0xffffffffu, member, (sub + slot) & 31);
        uint32_t fl[4] = {0u, 0u, 0u, 0u};
        for (int t = 0; t < L.kw; ++t) {
          const int q = 32 * t + c;
          bool f = false;
          if (i < n && q < L.k && ((s_act[t] >> c) & 1u)) {
            const bool allowed = indep ? mem : (rki < s_sel[q]);
            if (allowed) {
              const uint32_t word = __ldcg(L.sb + i * L.kw + t);
              const GT hv = __ldcg(L.h + i * L.kp + q);
              const GT gain = ((word >> c) & 1u) ? GT(2) * hv : GT(-2) * hv;   // 2 s_i h_i
              if (indep) {
                f = std::is_same<GT, int>::value ? (gain < GT(0)) : ((double)gain < -s_tolc[q]);
                if (f) acc_add(&s_dE[q], (E)gain);
              } else {
                f = gain < GT(0);
              }
            }
          }
          const uint32_t bal = __ballot_sync(0xffffffffu, f);
          fl[t] = (cp == 32) ? bal : ((bal >> (slot * cp)) & ((1u << cp) - 1u));
          if (f) atomicAdd((unsigned long long*)&s_cnt[q], 1ull);
        }
        uint32_t any = 0u;
        for (int t = 0; t < L.kw; ++t) any |= fl[t];
        if (c == 0 && i < n)
          for (int t = 0; t < L.kw; ++t) L.wm[i * L.kw + t] = fl[t];
        const uint32_t wb = __ballot_sync(0xffffffffu, c == 0 && i < n && any != 0u);
        for (int sl = 0; sl < ne; ++sl)
          if ((wb >> (sl * cp)) & 1u) tile_want |= 1u << (sub + sl);
      }
      if (tile_want) {
        // one queue reservation per tile of 32 nodes
        long long pos = 0;
        if (lane == 0) pos = (long long)atomicAdd((unsigned long long*)&G->wq_count, (unsigned long long)__popc(tile_want));
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if ((tile_want >> lane) & 1u) L.wq[pos + __popc(tile_want & ((1u << lane) - 1u))] = (int)(tile + lane);
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < L.k; q += blockDim.x) {
      if (s_cnt[q]) atomicAdd((unsigned long long*)&G->want[q], (unsigned long long)s_cnt[q]);
      if (indep && s_dE[q] != E(0)) {
        if (std::is_same<GT, int>::value) acc_add(&G->dE_i[q], (long long)s_dE[q]);
        else acc_add(&G->dE_d[q], (double)s_dE[q]);
      }
      s_dE[q] = E(0);
    }
    if (!pol.sync(&C->gs)) return;

    // R2 (guards): dE of each candidate's proposal from the rows of its flipping nodes
    const long long nwq = *((volatile long long*)&G->wq_count);
    if (!indep) {
      for (long long e = gwarp; e < nwq; e += nwarps) {
        const long long i = (long long)__ldcg(L.wq + e);
        const long long rs = rp_load(L.rowptr, i), re = rp_load(L.rowptr, i + 1);
        for (int t = 0; t < L.kw; ++t) {
          const uint32_t Wi = __ldcg(L.wm + i * L.kw + t);
          if (!Wi) continue;
          GT acc = GT(0);   // sum over flipping neighbours j of J_ij s_j (candidate 32 t + c)
          for (long long p = rs + slot; p < re; p += ne) {
            const int j = __ldg(L.col + p);
            const uint32_t Wj = __ldcg(L.wm + (long long)j * L.kw + t);
            if ((Wj >> c) & 1u) {
              const GT v = coupling_as<GT>(__ldg(L.val + p));
              acc += ((__ldcg(L.sb + (long long)j * L.kw + t) >> c) & 1u) ? v : -v;
            }
          }
          acc = xor_sum_above(acc, cp);
          const int q = 32 * t + c;
          if (slot == 0 && ((Wi >> c) & 1u)) {
            const bool si = (__ldcg(L.sb + i * L.kw + t) >> c) & 1u;
            const GT hv = __ldcg(L.h + i * L.kp + q);
            const GT term = si ? GT(2) * (hv - acc) : GT(-2) * (hv - acc);   // 2 s_i h_i - 2 s_i acc
            acc_add(&s_dE[q], (E)term);
          }
        }
      }
      __syncthreads();
      for (int q = threadIdx.x; q < L.k; q += blockDim.x)
        if (s_dE[q] != E(0)) {
          if (std::is_same<GT, int>::value) acc_add(&G->dE_i[q], (long long)s_dE[q]);
          else acc_add(&G->dE_d[q], (double)s_dE[q]);
        }
    }
    if (!pol.sync(&C->gs, [&] {
          // acceptance, energies, adaptation and retirement (models/spectral_annealing_safe.py:502-688)
          if (threadIdx.x < 4) G->accept[threadIdx.x] = 0u;
          __syncthreads();
          for (int q = threadIdx.x; q < L.k; q += blockDim.x) {
            const bool act = (gld(&G->active[q >> 5]) >> (q & 31)) & 1u;
            const long long want = gld(&G->want[q]);
            const bool has = act && want > 0;
            const double dE = dE_of<GT>(G, q), Ec = E_of<GT>(G, q);
            bool accepted, rejected = false;
            if (indep) {
              accepted = has;
              G->sweep_flips[q] = gld(&G->sweep_flips[q]) + want;
            } else {
              accepted = has && (dE / A.c < -guard_tol(Ec / A.c));
              rejected = has && !accepted;
            }
            if (accepted) {
              atomicOr(&G->accept[q >> 5], 1u << (q & 31));
              if (std::is_same<GT, int>::value) G->E_i[q] = gld(&G->E_i[q]) + gld(&G->dE_i[q]);
              else G->E_d[q] = gld(&G->E_d[q]) + gld(&G->dE_d[q]);
              atomicAdd(&G->accepted, 1);
            }
            if (rejected) atomicAdd(&G->rejected, 1);
            if (!indep && act) {
              bool stalled;
              if (A.mode == SA_GUARD_ADAPTIVE) {     // models/safe_update_policy.py:68-95
                const double initial = phase == 0 ? L.p.subset_fraction : L.p.final_sweep_fraction;
                const double f = gld(&G->frac[q]);
                double nf = f;
                if (rejected) nf = fmax(kGuardMinFrac, f * kGuardShrink);
                if (accepted) nf = fmin(initial, f * kGuardGrowth);
                const bool shrunk = rejected && nf < f;
                G->frac[q] = nf;
                stalled = (act && !has) || (rejected && !shrunk);
              } else {
                stalled = !accepted;
              }
              G->streak[q] = accepted ? 0 : (stalled ? gld(&G->streak[q]) + 1 : 0);
            }
            G->want[q] = 0;
            G->dE_i[q] = 0;
            G->dE_d[q] = 0.0;
          }
        })) return;

    // R3: apply the accepted proposals
    for (int q = threadIdx.x; q < 4; q += blockDim.x) s_acc_mask[q] = gld(&G->accept[q]);
    __syncthreads();
    for (long long e = gwarp; e < nwq; e += nwarps) {
      if (lane != 0) continue;
      const long long i = (long long)__ldcg(L.wq + e);
      uint32_t any = 0u;
      for (int t = 0; t < L.kw; ++t) {
        const uint32_t F = __ldcg(L.wm + i * L.kw + t) & s_acc_mask[t];
        L.flipm[i * L.kw + t] = F;
        if (F) L.sb[i * L.kw + t] = __ldcg(L.sb + i * L.kw + t) ^ F;
        any |= F;
      }
      if (any) {
        const long long deg = rp_load(L.rowptr, i + 1) - rp_load(L.rowptr, i);
        const long long nch = deg > kChunk ? (deg + kChunk - 1) / kChunk : 1;
        const long long pos = (long long)atomicAdd((unsigned long long*)&G->wl_count, (unsigned long long)nch);
        for (long long q = 0; q < nch && pos + q < L.wl_cap; ++q) L.wl[pos + q] = (i << 22) | q;
      }
    }
    if (!pol.sync(&C->gs)) return;

    // U: field changes of the applied flips (as the default search)
    const long long nwl = min(*((volatile long long*)&G->wl_count), L.wl_cap);
    for (long long e = gwarp; e < nwl; e += nwarps) {
      const long long ent = __ldcg(L.wl + e);
      const long long i = ent >> 22;
      const long long q = ent & ((1ll << 22) - 1);
      const long long rs = rp_load(L.rowptr, i), re = rp_load(L.rowptr, i + 1);
      const long long cb = rs + q * kChunk;
      const long long ce = (cb + kChunk < re) ? cb + kChunk : re;
      for (int t = 0; t < L.kw; ++t) {
        const uint32_t F = __ldcg(L.flipm + i * L.kw + t);
        if (!((F >> c) & 1u)) continue;
        const bool up = (__ldcg(L.sb + i * L.kw + t) >> c) & 1u;
        for (long long p = cb + slot; p < ce; p += ne) {
          const int j = __ldg(L.col + p);
          const GT v = coupling_as<GT>(__ldg(L.val + p));
          atomicAdd(&L.h[(long long)j * L.kp + 32 * t + c], up ? GT(2) * v : GT(-2) * v);
        }
      }
    }
    if (!pol.sync(&C->gs, [&] {
          // round bookkeeping, retirement and the next phase
          if (threadIdx.x == 0) {
            G->total_flips = gld(&G->total_flips) + gld(&G->wl_count);
            G->wq_count = 0;
            G->wl_count = 0;
            G->round = gld(&G->round) + 1;
            if (indep) {
              G->rounds_main = gld(&G->rounds_main) + 1;
              if (G->round % A.num_colors == 0) {       // end of a sweep
                for (int q = 0; q < L.k; ++q)
                  if (((gld(&G->active[q >> 5]) >> (q & 31)) & 1u) && gld(&G->sweep_flips[q]) == 0)
                    G->active[q >> 5] = gld(&G->active[q >> 5]) & ~(1u << (q & 31));
                for (int q = 0; q < L.k; ++q) G->sweep_flips[q] = 0;
              }
              const bool any = (gld(&G->active[0]) | gld(&G->active[1]) | gld(&G->active[2]) | gld(&G->active[3])) != 0u;
              if (!any || G->round >= A.limit_main) G->phase = 2;
            } else {
              for (int q = 0; q < L.k; ++q)
                if (gld(&G->streak[q]) >= kGuardPatience) G->active[q >> 5] = gld(&G->active[q >> 5]) & ~(1u << (q & 31));
              if (gld(&G->phase) == 0) G->rounds_main = gld(&G->rounds_main) + 1;
              else G->rounds_final = gld(&G->rounds_final) + 1;
              const bool any = (gld(&G->active[0]) | gld(&G->active[1]) | gld(&G->active[2]) | gld(&G->active[3])) != 0u;
              const int limit = gld(&G->phase) == 0 ? A.limit_main : A.limit_final;
              if (!any || G->round >= limit) G->phase = (gld(&G->phase) == 0 && A.limit_final > 0) ? 3 : 2;
            }
          }
          __syncthreads();
          const int ph = gld(&G->phase);
          if (ph == 3) {
            guard_start_phase(A, 1);
          } else if (ph != 2) {
            guard_set_selection(A, ph == 0 ? L.p.subset_fraction : L.p.final_sweep_fraction);
          }
        })) return;
  }

  // ---- energies after; refined candidates back to candidate-major -----------------------------
  energy_phase(L, L.eafter, s_acc, gwarp, nwarps);
  const long long pairs = (long long)L.k * L.W;
  for (long long pr = gwarp; pr < pairs; pr += nwarps) {
    const long long cq = pr / L.W, wd = pr % L.W;
    const long long i = wd * 32 + lane;
    bool bit = false;
    if (i < n) bit = (__ldcg(L.sb + i * L.kw + (cq >> 5)) >> (cq & 31)) & 1u;
    const uint32_t word = __ballot_sync(0xffffffffu, bit);
    if (lane == 0) L.refined[cq * L.W + wd] = word;
  }
}

// Sequential oracle: one CTA per candidate; candidate-major spins (int8) and fields in the
// workspace. Each step flips the node of least energy change 2 s_i h_i (first on ties) if the
// change is a strict drop beyond the tolerance, until none is or max_steps.
template <typename VT, typename RP, typename GT>
__global__ void __launch_bounds__(kThreads) oracle_kernel(const RP* rowptr, const int* col, const VT* val, long long n,
                                                         const uint32_t* cand, uint32_t* refined, long long W,
                                                         int8_t* spins, GT* field, long long max_steps, double cnorm,
                                                         long long* steps_out, double* e_before, double* e_after) {
  using E = EAcc<GT>;
  const int q = blockIdx.x;
  int8_t* s = spins + (long long)q * n;
  GT* h = field + (long long)q * n;
  const uint32_t* cw = cand + (long long)q * W;
  __shared__ E red[kWarps];
  __shared__ GT bg[kWarps];
  __shared__ long long bi[kWarps];
  __shared__ E s_E;
  __shared__ GT s_best;
  __shared__ long long s_idx;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) s[i] = ((__ldg(cw + (i >> 5)) >> (i & 31)) & 1u) ? 1 : -1;
  __syncthreads();
  E e = E(0);
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    GT acc = GT(0);
    for (long long p = rp_load(rowptr, i); p < rp_load(rowptr, i + 1); ++p)
      acc += coupling_as<GT>(__ldg(val + p)) * (GT)s[__ldg(col + p)];
    h[i] = acc;
    e += (E)s[i] * (E)acc;
  }
  e = warp_sum(e);
  if (lane == 0) red[wid] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    E t = E(0);
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    s_E = -t / 2;
    e_before[q] = (double)s_E;
  }
  __syncthreads();
  long long steps = 0;
  for (; steps < max_steps; ++steps) {
    GT best = GT(0);
    long long idx = -1;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) {
      const GT g = (GT)(2 * s[i]) * h[i];
      if (idx < 0 || g < best) { best = g; idx = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const GT ob = __shfl_xor_sync(0xffffffffu, best, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, idx, o);
      if (oi >= 0 && (idx < 0 || ob < best || (ob == best && oi < idx))) { best = ob; idx = oi; }
    }
    if (lane == 0) { bg[wid] = best; bi[wid] = idx; }
    __syncthreads();
    if (threadIdx.x == 0) {
      GT b = GT(0);
      long long ib = -1;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
        if (bi[w] >= 0 && (ib < 0 || bg[w] < b || (bg[w] == b && bi[w] < ib))) { b = bg[w]; ib = bi[w]; }
      const double tol = (kGuardAbsTol + kGuardRelTol * fmax(1.0, fabs((double)s_E / cnorm))) * cnorm;
      const bool improve = ib >= 0 && (std::is_same<GT, int>::value ? (b < GT(0)) : ((double)b < -tol));
      s_best = b;
      s_idx = improve ? ib : -1;
      if (improve) s_E += (E)b;
    }
    __syncthreads();
    const long long b = s_idx;
    if (b < 0) break;
    const int8_t old = s[b];
    for (long long p = rp_load(rowptr, b) + threadIdx.x; p < rp_load(rowptr, b + 1); p += blockDim.x)
      h[__ldg(col + p)] -= GT(2 * old) * coupling_as<GT>(__ldg(val + p));
    __syncthreads();
    if (threadIdx.x == 0) s[b] = (int8_t)(-old);
    __syncthreads();
  }
  for (long long wd = wid; wd < W; wd += blockDim.x >> 5) {
    const long long i = wd * 32 + lane;
    const uint32_t word = __ballot_sync(0xffffffffu, i < n && s[i] > 0);
    if (lane == 0) refined[(long long)q * W + wd] = word;
  }
  if (threadIdx.x == 0) {
    steps_out[q] = steps;
    e_after[q] = (double)s_E;
  }
}

}  // namespace

void ls_geometry(int k, int* kp, int* kw, int* cp);
size_t ls_workspace_bytes(long long n, long long nnz, int k, int integer);

size_t guard_workspace_bytes(long long n, long long nnz, int k, int integer) {
  Layout L;
  L.off(ls_workspace_bytes(n, nnz, k, integer));
  L.off(sizeof(GuardCtrl));
  L.off((size_t)k * (size_t)n);                                       // oracle spins
  L.off((integer ? sizeof(int) : sizeof(double)) * (size_t)k * (size_t)n);   // oracle fields
  L.off(sizeof(long long) * 128 + sizeof(double) * 256);
  return L.total;
}

template <typename VT, typename RP, typename GT>
static int launch_guard(sa_handle* h, const sa_guard_params* p, char* ws, sa_guard_result* res, double* eb, double* ea) {
  int kp, kw, cp;
  ls_geometry(p->k, &kp, &kw, &cp);
  const long long wl_cap = h->n + h->nnz / kChunk + 2;
  Layout Lo;
  const size_t o_ls = Lo.off(ls_workspace_bytes(h->n, h->nnz, p->k, h->integer_J));
  const size_t o_g = Lo.off(sizeof(GuardCtrl));
  const size_t o_os = Lo.off((size_t)p->k * (size_t)h->n);
  const size_t o_of = Lo.off(sizeof(GT) * (size_t)p->k * (size_t)h->n);
  const size_t o_or = Lo.off(sizeof(long long) * 128 + sizeof(double) * 256);
  (void)o_ls;
  const uint32_t* cand = h->cand + (size_t)p->first_slot * h->W;
  uint32_t* refined = h->refined + (size_t)p->first_slot * h->W;
  if (p->policy == SA_GUARD_SEQUENTIAL) {
    long long* steps = (long long*)(ws + o_or);
    double* e_b = (double*)(ws + o_or + sizeof(long long) * 128);
    double* e_a = e_b + 128;
    const long long max_steps = 100ll * h->n;    // models/local_search_guards/policies.py:37
    oracle_kernel<VT, RP, GT><<<p->k, kThreads, 0, h->stream>>>(
        (const RP*)h->rowptr, h->col, (const VT*)h->val, h->n, cand, refined, h->W, (int8_t*)(ws + o_os),
        (GT*)(ws + o_of), max_steps, h->c, steps, e_b, e_a);
    count_launches(1);
    if (cudaGetLastError() != cudaSuccess) return SA_ERR_CUDA;
    long long hs[128];
    double hb[128], ha[128];
    if (cudaMemcpyAsync(hs, steps, sizeof(long long) * p->k, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(hb, e_b, sizeof(double) * p->k, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(ha, e_a, sizeof(double) * p->k, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
      return SA_ERR_CUDA;
    long long mx = 0, tot = 0;
    for (int q = 0; q < p->k; ++q) {
      mx = hs[q] > mx ? hs[q] : mx;
      tot += hs[q];
      if (eb) eb[q] = hb[q];
      if (ea) ea[q] = ha[q];
    }
    res->status = (mx >= max_steps) ? SA_ERR_NOT_CONVERGED : SA_OK;
    res->rounds = (int)mx;
    res->final_rounds = 0;
    res->accepted = (int)tot;
    res->rejected = 0;
    res->integer_gains = std::is_same<GT, int>::value ? 1 : 0;
    res->flips = tot;
    return SA_OK;
  }
  GuardArgs<VT, RP, GT> A;
  LsArgs<VT, RP, GT>& L = A.L;
  L.rowptr = (const RP*)h->rowptr;
  L.col = h->col;
  L.val = (const VT*)h->val;
  L.items = h->items;
  L.n_items = h->n_items;
  L.n = h->n;
  L.k = p->k;
  L.kp = kp;
  L.kw = kw;
  L.cp = cp;
  Layout Ll;
  const size_t o_ctrl = Ll.off(sizeof(LsCtrl));
  const size_t o_eb = Ll.off(sizeof(double) * 128);
  const size_t o_ea = Ll.off(sizeof(double) * 128);
  const size_t o_sb = Ll.off(sizeof(uint32_t) * (size_t)h->n * kw);
  const size_t o_fm = Ll.off(sizeof(uint32_t) * (size_t)h->n * kw);
  const size_t o_h = Ll.off(sizeof(GT) * (size_t)h->n * kp);
  const size_t o_wl = Ll.off(sizeof(long long) * (size_t)wl_cap);
  const size_t o_wm = Ll.off(sizeof(uint32_t) * (size_t)h->n * kw);
  const size_t o_pr = Ll.off(sizeof(int) * (size_t)h->n);
  const size_t o_wq = Ll.off(sizeof(int) * (size_t)h->n);
  (void)o_pr;
  L.ctrl = (LsCtrl*)(ws + o_ctrl);
  L.ebefore = (typename LsArgs<VT, RP, GT>::EAccPtr)(ws + o_eb);
  L.eafter = (typename LsArgs<VT, RP, GT>::EAccPtr)(ws + o_ea);
  L.sb = (uint32_t*)(ws + o_sb);
  L.flipm = (uint32_t*)(ws + o_fm);
  L.h = (GT*)(ws + o_h);
  L.wl = (long long*)(ws + o_wl);
  L.wl_cap = wl_cap;
  L.wm = (uint32_t*)(ws + o_wm);
  L.prio = nullptr;
  L.wq = (int*)(ws + o_wq);
  L.priority = 0;
  L.cand = cand;
  L.refined = refined;
  L.W = h->W;
  sa_ls_params lp;
  memset(&lp, 0, sizeof(lp));
  lp.k = p->k;
  lp.subset_fraction = p->subset_fraction;
  lp.final_sweep_fraction = p->final_sweep_fraction;
  lp.seed = p->seed;
  L.p = lp;
  L.m_main = L.m_final = 0;
  A.G = (GuardCtrl*)(ws + o_g);
  A.mode = p->policy;
  A.num_colors = p->num_colors;
  A.colors = p->colors;
  A.color_seq = p->color_seq;
  A.c = h->c;
  if (p->policy == SA_GUARD_INDEPENDENT_SET) {
    A.limit_main = p->max_iterations + p->final_sweep_iters * p->num_rounds;
    A.limit_final = 0;
  } else {
    A.limit_main = p->max_iterations;
    A.limit_final = p->final_sweep_iters * p->num_rounds;
  }
  if (cudaMemsetAsync(L.ctrl, 0, sizeof(GridSync), h->stream) != cudaSuccess) return SA_ERR_CUDA;
  if (cudaMemsetAsync(A.G, 0, sizeof(GuardCtrl), h->stream) != cudaSuccess) return SA_ERR_CUDA;
  void* args[] = {&A};
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)guard_kernel<VT, RP, GT>, dim3(h->blocks), dim3(kThreads),
                                              args, 0, h->stream);
  count_launches(1);
  if (e != cudaSuccess) return SA_ERR_CUDA;
  GuardCtrl g;
  LsCtrl lc;
  long long sb_raw[128], sa_raw[128];
  if (cudaMemcpyAsync(&g, A.G, sizeof(GuardCtrl), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaMemcpyAsync(&lc, L.ctrl, sizeof(LsCtrl), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaMemcpyAsync(sb_raw, ws + o_eb, sizeof(long long) * 128, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaMemcpyAsync(sa_raw, ws + o_ea, sizeof(long long) * 128, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess)
    return SA_ERR_CUDA;
  if (lc.gs.error) return lc.gs.error;
  const bool integer = std::is_same<GT, int>::value;
  for (int q = 0; q < p->k; ++q) {
    double x, y;
    if (integer) {
      x = (double)sb_raw[q];
      y = (double)sa_raw[q];
    } else {
      memcpy(&x, &sb_raw[q], 8);
      memcpy(&y, &sa_raw[q], 8);
    }
    if (eb) eb[q] = -0.5 * x;
    if (ea) ea[q] = -0.5 * y;
  }
  res->status = SA_OK;
  res->rounds = g.rounds_main;
  res->final_rounds = g.rounds_final;
  res->accepted = g.accepted;
  res->rejected = g.rejected;
  res->integer_gains = integer ? 1 : 0;
  res->flips = g.total_flips;
  return SA_OK;
}

}  // namespace sa

extern "C" {

int sa_guard_workspace_size(sa_handle* h, int32_t k, size_t* bytes) {
  if (!h || !bytes || k < 1 || k > 128) return SA_ERR_INVALID_ARG;
  *bytes = sa::guard_workspace_bytes(h->n, h->nnz, k, h->integer_J);
  return SA_OK;
}

int sa_guard_search(sa_handle* h, const sa_guard_params* p, void* ws, size_t bytes, double* energies_before,
                    double* energies_after, sa_guard_result* result) {
  if (!h || !h->bound || !p || !ws || !result || p->k < 1 || p->k > 128 || p->first_slot < 0 ||
      p->first_slot + p->k > h->max_cand || p->policy < SA_GUARD_FIXED || p->policy > SA_GUARD_SEQUENTIAL ||
      p->max_iterations < 0 || p->final_sweep_iters < 0 || p->num_rounds < 0 || ((uintptr_t)ws & 255))
    return SA_ERR_INVALID_ARG;
  if (p->policy != SA_GUARD_SEQUENTIAL &&
      !(p->subset_fraction > 0.0 && p->subset_fraction <= 1.0 && p->final_sweep_fraction > 0.0 &&
        p->final_sweep_fraction <= 1.0))
    return SA_ERR_INVALID_ARG;
  if (p->policy == SA_GUARD_INDEPENDENT_SET && (!p->colors || !p->color_seq || p->num_colors < 1))
    return SA_ERR_INVALID_ARG;
  if (bytes < sa::guard_workspace_bytes(h->n, h->nnz, p->k, h->integer_J)) return SA_ERR_OOM;
  memset(result, 0, sizeof(*result));
  char* w = (char*)ws;
  const bool integer = h->integer_J != 0;
  if (h->prec == 32) {
    if (h->rp64) return integer ? sa::launch_guard<float, long long, int>(h, p, w, result, energies_before, energies_after)
                                : sa::launch_guard<float, long long, double>(h, p, w, result, energies_before, energies_after);
    return integer ? sa::launch_guard<float, int, int>(h, p, w, result, energies_before, energies_after)
                   : sa::launch_guard<float, int, double>(h, p, w, result, energies_before, energies_after);
  }
  if (h->rp64) return integer ? sa::launch_guard<double, long long, int>(h, p, w, result, energies_before, energies_after)
                              : sa::launch_guard<double, long long, double>(h, p, w, result, energies_before, energies_after);
  return integer ? sa::launch_guard<double, int, int>(h, p, w, result, energies_before, energies_after)
                 : sa::launch_guard<double, int, double>(h, p, w, result, energies_before, energies_after);
}

}  // extern "C"

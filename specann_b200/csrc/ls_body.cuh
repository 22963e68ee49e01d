// Batched single-flip local search over all distinct candidates as one persistent cooperative
// kernel, with a cache of the local fields h_ic = sum_j J_ij s_cj and snapshot passes.
//
// Pass semantics (both decided from the pass-start state; bit-exact with oracle/specann_oracle.py):
//   priority (default): a wanting node flips unless a wanting neighbour has a lower rank in the
//     pass's permutation, so the flips form an independent set and every flip lowers the energy
//     by its gain (phases D1: wanting masks and ranks, D2: blocking check, U);
//   snapshot: every wanting node flips (phases D, U).
// Layout (node-major, so one read of a CSR row serves every candidate):
//   sb[i * kw + t]     bit c of word t: spin of candidate 32 t + c at node i is +1
//   h[i * kp + c]      local field of node i in candidate c (int32 for integer couplings, which
//                      makes every gain and energy exact; double otherwise)
//   flipm[i * kw + t]  candidates flipping at node i in the current pass
// A pass: (D) every selected node decides for every candidate from the pass-start state, flips
// its own spin bits and appends (node, chunk) entries to a work list; (U) one warp per entry
// scatters the field changes 2 J_ij s_i(new) to the neighbours of the chunk for the flipped
// candidates (integer atomics: exact and order-independent). Arrays that other CTAs change during
// the kernel (h, sb, flipm, the work list) are read with ld.global.cg: the per-SM L1 is not
// coherent with their writes. The last CTA at each barrier runs
// the stopping rules of flip_refinement / gpu_final_sweep (models/spectral_annealing.py:983-1112).
#pragma once
#include <cmath>
#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "handle.cuh"
#include "spmv.cuh"
#include "policy.cuh"

namespace sa {

void count_launches(int k);

template <typename GT>
struct EAccOf { using type = typename std::conditional<std::is_same<GT, int>::value, long long, double>::type; };

template <typename VT, typename RP, typename GT>
struct LsArgs {
  using EAccPtr = typename EAccOf<GT>::type*;
  const RP* rowptr;
  const int* col;
  const VT* val;
  const WorkItem* items;
  long long n_items;
  long long n;
  int k, kp, kw, cp;
  uint32_t* sb;
  GT* h;
  uint32_t* flipm;
  long long* wl;
  long long wl_cap;
  uint32_t* wm;          // wanting masks of the pass (priority passes), n x kw
  int* prio;             // rank of the node in the pass's permutation (INT_MAX if not selected)
  int* wq;               // wanting nodes of the pass
  int priority;          // 1: priority passes, 0: snapshot passes
  LsCtrl* ctrl;
  EAccPtr ebefore;      // kp sums of s_i h_i (energy = -sum / 2): int64 or double
  EAccPtr eafter;
  const uint32_t* cand;
  uint32_t* refined;
  long long W;
  sa_ls_params p;
  long long m_main, m_final;
};

template <typename GT>
__device__ __forceinline__ GT coupling_as(float v);
template <>
__device__ __forceinline__ int coupling_as<int>(float v) { return __float2int_rn(v); }
template <>
__device__ __forceinline__ double coupling_as<double>(float v) { return (double)v; }
template <typename GT>
__device__ __forceinline__ GT coupling_as(double v);
template <>
__device__ __forceinline__ int coupling_as<int>(double v) { return __double2int_rn(v); }
template <>
__device__ __forceinline__ double coupling_as<double>(double v) { return v; }

template <typename GT>
__device__ __forceinline__ GT xor_sum_above(GT v, int cp) {
  for (int o = cp; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Local fields of the candidate word t for entries [e0, e1) of a row (lanes: element slot
// lane / cp, candidate lane % cp). Returns the sum for candidate 32 t + lane % cp in every lane.
template <typename VT, typename RP, typename GT>
__device__ __forceinline__ GT row_field(const LsArgs<VT, RP, GT>& A, long long e0, long long e1, int t) {
  const int lane = threadIdx.x & 31;
  const int ne = 32 / A.cp, es = lane / A.cp, c = lane % A.cp;
  GT acc = GT(0);
  for (long long e = e0 + es; e < e1; e += ne) {
    const int j = __ldg(A.col + e);
    const GT v = coupling_as<GT>(__ldg(A.val + e));
    const uint32_t word = A.sb[(long long)j * A.kw + t];
    acc += ((word >> c) & 1u) ? v : -v;
  }
  return xor_sum_above(acc, A.cp);
}

// Per-candidate sums of s_i h_i over all nodes into out[kp] (64-bit integer sums for int32 fields:
// exact and order-independent; FP64 sums otherwise).
template <typename GT>
using EAcc = typename std::conditional<std::is_same<GT, int>::value, long long, double>::type;

__device__ __forceinline__ void acc_add(long long* p, long long v) {
  atomicAdd((unsigned long long*)p, (unsigned long long)v);
}
__device__ __forceinline__ void acc_add(double* p, double v) { atomicAdd(p, v); }

template <typename VT, typename RP, typename GT>
__device__ void energy_phase(const LsArgs<VT, RP, GT>& A, EAcc<GT>* out, EAcc<GT>* sacc, long long gwarp,
                             long long nwarps) {
  using E = EAcc<GT>;
  const int lane = threadIdx.x & 31;
  const int ne = 32 / A.cp, slot = lane / A.cp, c = lane % A.cp;
  for (int q = threadIdx.x; q < A.kp; q += blockDim.x) sacc[q] = E(0);
  __syncthreads();
  for (int t = 0; t < A.kw; ++t) {
    E acc = E(0);
    for (long long base = gwarp * ne; base < A.n; base += nwarps * ne) {
      const long long i = base + slot;
      if (i < A.n) {
        const uint32_t word = __ldcg(A.sb + i * A.kw + t);
        const GT hv = __ldcg(A.h + i * A.kp + 32 * t + c);
        acc += ((word >> c) & 1u) ? (E)hv : -(E)hv;
      }
    }
    for (int o = A.cp; o < 32; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (slot == 0 && 32 * t + c < A.kp) acc_add(&sacc[32 * t + c], acc);
  }
  __syncthreads();
  for (int q = threadIdx.x; q < A.kp; q += blockDim.x) acc_add(&out[q], sacc[q]);
  __syncthreads();
}

template <typename VT, typename RP, typename GT, class Pol>
__device__ __forceinline__ void ls_body(const LsArgs<VT, RP, GT>& A, const Pol& pol) {
  __shared__ EAcc<GT> s_acc[128];           // per-CTA energy sums
  __shared__ long long s_cnt[128];
  LsCtrl* C = A.ctrl;
  const int lane = threadIdx.x & 31;
  const long long gtid = pol.tid();
  const long long nthreads = pol.nthr();
  const long long gwarp = gtid >> 5, nwarps = nthreads >> 5;
  const long long n = A.n;
  const int cp = A.cp, ne = 32 / cp, slot = lane / cp, c = lane % cp;
  // phase timer: the first CTA's thread 0 charges the time since its previous mark to a phase
  const bool timer = pol.block() == 0 && threadIdx.x == 0;
  unsigned long long t_mark = timer ? global_ns() : 0ull;
  auto mark = [&](int ph) {
    if (timer) {
      const unsigned long long t = global_ns();
      C->tph[ph] += t - t_mark;
      t_mark = t;
    }
  };

  // ---- L0: candidate-major packed spins -> node-major bits; zero the fields -----------------
  if (pol.block() == 0 && threadIdx.x == 0) {
    C->it = 0; C->round = 0; C->sub = 0; C->final_passes = 0; C->total_flips = 0; C->wl_count = 0;
    C->wq_count = 0;
    for (int q = 0; q < 4; ++q) C->active[q] = 0u;
    for (int q = 0; q < A.k; ++q) C->active[q >> 5] |= 1u << (q & 31);
    for (int q = 0; q < 128; ++q) C->counts[q] = 0;
    for (int q = 0; q < 4; ++q) C->tph[q] = 0ull;
    const bool main_loop = A.p.max_iterations > 0;
    const bool final_sweep = A.p.num_rounds > 0 && A.p.final_sweep_iters > 0;
    C->phase = main_loop ? 0 : (final_sweep ? 1 : 2);
    C->stream = main_loop ? 0 : kFinalStreamBase;
    C->m = main_loop ? A.m_main : A.m_final;
  }
  for (long long i = gtid; i < n; i += nthreads) {
    for (int t = 0; t < A.kw; ++t) {
      uint32_t word = 0u;
      const int c1 = min(A.k, 32 * t + 32);
      for (int q = 32 * t; q < c1; ++q) {
        const uint32_t cw = __ldg(A.cand + (long long)q * A.W + (i >> 5));
        word |= ((cw >> (i & 31)) & 1u) << (q - 32 * t);
      }
      A.sb[i * A.kw + t] = word;
    }
    for (int q = 0; q < A.kp; ++q) A.h[i * A.kp + q] = GT(0);
  }
  for (long long q = gtid; q < A.kp; q += nthreads) { A.ebefore[q] = 0; A.eafter[q] = 0; }
  if (!pol.sync(&C->gs)) return;

  // ---- L1: local fields h = J s for all candidates (work-list balanced) ---------------------
  for (long long itm = gwarp; itm < A.n_items; itm += nwarps) {
    const long long e0 = __ldg(&A.items[itm].e0);
    const int irow = __ldg(&A.items[itm].row);
    const int meta = __ldg(&A.items[itm].meta);
    if (irow >= 0) {
      const long long r1 = irow + item_nrows(meta);
      for (long long r = irow; r < r1; ++r) {
        const long long rs = rp_load(A.rowptr, r), re = rp_load(A.rowptr, r + 1);
        for (int t = 0; t < A.kw; ++t) {
          const GT f = row_field(A, rs, re, t);
          if (slot == 0 && 32 * t + c < A.kp) A.h[r * A.kp + 32 * t + c] = f;
        }
      }
    } else {
      const long long row = -((long long)irow + 1);
      const long long cb = e0;
      const long long ce = e0 + item_len(meta);
      for (int t = 0; t < A.kw; ++t) {
        const GT f = row_field(A, cb, ce, t);
        if (slot == 0 && 32 * t + c < A.kp) atomicAdd(&A.h[row * A.kp + 32 * t + c], f);
      }
    }
  }
  if (!pol.sync(&C->gs)) return;
  energy_phase(A, A.ebefore, s_acc, gwarp, nwarps);
  if (!pol.sync(&C->gs)) return;
  mark(0);

  // ---- passes ------------------------------------------------------------------------------
  while (ld_volatile_i32(&C->phase) != 2) {
    const long long m = *((volatile long long*)&C->m);
    const long long stream = *((volatile long long*)&C->stream);
    const bool all_sel = m >= n;
    const SelKeys keys = make_sel_keys(A.p.seed, stream, n);
    for (int q = threadIdx.x; q < 128; q += blockDim.x) s_cnt[q] = 0;
    __syncthreads();
    // D1: every selected node decides for every candidate from the pass-start state. Snapshot
    // passes flip the wanting pairs here; priority passes record the wanting masks and ranks.
    int cnt[4] = {0, 0, 0, 0};
    for (long long tile = gwarp * 32; tile < n; tile += nwarps * 32) {
      bool selb = false;
      int rk = 0x7fffffff;
      if (tile + lane < n) {
        if (all_sel && !A.priority) {
          selb = true;
        } else {
          const long long r = sel_rank(tile + lane, keys, n);
          selb = r < m;
          rk = (int)r;
        }
        if (A.priority) A.prio[tile + lane] = selb ? rk : 0x7fffffff;
      }
      const uint32_t selmask = __ballot_sync(0xffffffffu, selb);
      for (int sub = 0; sub < 32; sub += ne) {
        const long long i = tile + sub + slot;
        const bool valid = i < n && ((selmask >> (sub + slot)) & 1u);
        uint32_t fl[4] = {0u, 0u, 0u, 0u};
        for (int t = 0; t < A.kw; ++t) {
          bool f = false;
          uint32_t word = 0u;
          if (valid) {
            word = __ldcg(A.sb + i * A.kw + t);
            const GT hv = __ldcg(A.h + i * A.kp + 32 * t + c);
            const bool sp = (word >> c) & 1u;
            f = (32 * t + c < A.k) && (sp ? (hv < GT(0)) : (hv > GT(0)));
          }
          const uint32_t bal = __ballot_sync(0xffffffffu, f);
          const uint32_t bits = (cp == 32) ? bal : ((bal >> (slot * cp)) & ((1u << cp) - 1u));
          fl[t] = bits;
          if (!A.priority) {
            cnt[t] += f ? 1 : 0;
            if (c == 0 && bits) A.sb[i * A.kw + t] = word ^ bits;
          }
        }
        if (c == 0 && i < n) {
          uint32_t any = 0u;
          for (int t = 0; t < A.kw; ++t) any |= fl[t];
          if (A.priority) {
            for (int t = 0; t < A.kw; ++t) A.wm[i * A.kw + t] = fl[t];
            if (any) {
              const long long pos = (long long)atomicAdd((unsigned long long*)&C->wq_count, 1ull);
              A.wq[pos] = (int)i;
            }
          } else if (any) {
            for (int t = 0; t < A.kw; ++t) A.flipm[i * A.kw + t] = fl[t];
            const long long deg = rp_load(A.rowptr, i + 1) - rp_load(A.rowptr, i);
            const long long nch = deg > kChunk ? (deg + kChunk - 1) / kChunk : 1;
            const long long pos = (long long)atomicAdd((unsigned long long*)&C->wl_count, (unsigned long long)nch);
            for (long long q = 0; q < nch && pos + q < A.wl_cap; ++q) A.wl[pos + q] = (i << 22) | q;
          }
        }
      }
    }
    if (!A.priority) {
      for (int t = 0; t < A.kw; ++t) {
        int v = cnt[t];
        for (int o = cp; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (slot == 0 && v) atomicAdd((unsigned long long*)&s_cnt[32 * t + c], (unsigned long long)v);
      }
    } else {
      if (!pol.sync(&C->gs)) return;
      // D2: a wanting node flips the candidates for which no wanting neighbour has a lower rank
      // (one warp per wanting node; the blocking masks are OR-reduced over the row)
      const long long nwq = *((volatile long long*)&C->wq_count);
      int cnt2[4] = {0, 0, 0, 0};
      for (long long e = gwarp; e < nwq; e += nwarps) {
        const long long i = (long long)__ldcg(A.wq + e);
        const int pi = __ldcg(A.prio + i);
        uint32_t W[4] = {0u, 0u, 0u, 0u}, B[4] = {0u, 0u, 0u, 0u};
        for (int t = 0; t < A.kw; ++t) W[t] = __ldcg(A.wm + i * A.kw + t);
        const long long rs = rp_load(A.rowptr, i), re = rp_load(A.rowptr, i + 1);
        for (long long p = rs + lane; p < re; p += 32) {
          const int j = __ldg(A.col + p);
          if (__ldcg(A.prio + j) < pi)
            for (int t = 0; t < A.kw; ++t) B[t] |= __ldcg(A.wm + (long long)j * A.kw + t);
        }
        uint32_t any = 0u;
        for (int t = 0; t < A.kw; ++t) {
          B[t] = __reduce_or_sync(0xffffffffu, B[t]);
          W[t] &= ~B[t];
          any |= W[t];
          cnt2[t] += (W[t] >> lane) & 1u;
        }
        if (lane == 0 && any) {
          for (int t = 0; t < A.kw; ++t) {
            A.flipm[i * A.kw + t] = W[t];
            if (W[t]) A.sb[i * A.kw + t] = __ldcg(A.sb + i * A.kw + t) ^ W[t];
          }
          const long long deg = re - rs;
          const long long nch = deg > kChunk ? (deg + kChunk - 1) / kChunk : 1;
          const long long pos = (long long)atomicAdd((unsigned long long*)&C->wl_count, (unsigned long long)nch);
          for (long long q = 0; q < nch && pos + q < A.wl_cap; ++q) A.wl[pos + q] = (i << 22) | q;
        }
      }
      for (int t = 0; t < A.kw; ++t)
        if (cnt2[t]) atomicAdd((unsigned long long*)&s_cnt[32 * t + lane], (unsigned long long)cnt2[t]);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < A.k; q += blockDim.x)
      if (s_cnt[q]) atomicAdd((unsigned long long*)&C->counts[q], (unsigned long long)s_cnt[q]);
    if (!pol.sync(&C->gs)) return;
    mark(1);

    // U: scatter field changes of the flipped (node, candidate) pairs
    const long long nwl = min(*((volatile long long*)&C->wl_count), A.wl_cap);
    for (long long e = gwarp; e < nwl; e += nwarps) {
      const long long ent = __ldcg(A.wl + e);
      const long long i = ent >> 22;
      const long long q = ent & ((1ll << 22) - 1);
      const long long rs = rp_load(A.rowptr, i), re = rp_load(A.rowptr, i + 1);
      const long long cb = rs + q * kChunk;
      const long long ce = (cb + kChunk < re) ? cb + kChunk : re;
      for (int t = 0; t < A.kw; ++t) {
        const uint32_t F = __ldcg(A.flipm + i * A.kw + t);
        if (!F) continue;
        const uint32_t S = __ldcg(A.sb + i * A.kw + t);
        const bool mine = (F >> c) & 1u;
        const bool up = (S >> c) & 1u;
        if (!mine) continue;
        for (long long p = cb + slot; p < ce; p += ne) {
          const int j = __ldg(A.col + p);
          const GT v = coupling_as<GT>(__ldg(A.val + p));
          atomicAdd(&A.h[(long long)j * A.kp + 32 * t + c], up ? GT(2) * v : GT(-2) * v);
        }
      }
    }
    if (!pol.sync(&C->gs, [&] {
          if (threadIdx.x == 0) {
            long long tot = 0;
            bool any = false;
            for (int q = 0; q < A.k; ++q) {
              const long long cq = C->counts[q];
              tot += cq;
              any |= cq > 0;
              if (C->phase == 0 && cq == 0) C->active[q >> 5] &= ~(1u << (q & 31));
              C->counts[q] = 0;
            }
            C->total_flips += tot;
            C->wl_count = 0;
            C->wq_count = 0;
            if (C->phase == 0) {
              C->it += 1;
              const bool any_active = (C->active[0] | C->active[1] | C->active[2] | C->active[3]) != 0u;
              if (!any_active || C->it >= A.p.max_iterations) {
                const bool final_sweep = A.p.num_rounds > 0 && A.p.final_sweep_iters > 0;
                C->phase = final_sweep ? 1 : 2;
                C->round = 0;
                C->sub = 0;
              }
            } else {
              C->sub += 1;
              C->final_passes += 1;
              if (!any || C->sub >= A.p.final_sweep_iters) {
                C->round += 1;
                C->sub = 0;
                if (C->round >= A.p.num_rounds) C->phase = 2;
              }
            }
            if (C->phase == 0) { C->stream = C->it; C->m = A.m_main; }
            else if (C->phase == 1) { C->stream = kFinalStreamBase + C->round; C->m = A.m_final; }
          }
        })) return;
    mark(2);
  }

  // ---- energies after, refined candidates back to candidate-major ---------------------------
  energy_phase(A, A.eafter, s_acc, gwarp, nwarps);
  const long long pairs = (long long)A.k * A.W;
  for (long long pr = gwarp; pr < pairs; pr += nwarps) {
    const long long cq = pr / A.W, wd = pr % A.W;
    const long long i = wd * 32 + lane;
    bool bit = false;
    if (i < n) bit = (__ldcg(A.sb + i * A.kw + (cq >> 5)) >> (cq & 31)) & 1u;
    const uint32_t word = __ballot_sync(0xffffffffu, bit);
    if (lane == 0) A.refined[cq * A.W + wd] = word;
  }
  mark(3);
}

}  // namespace sa

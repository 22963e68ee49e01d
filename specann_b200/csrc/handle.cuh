// Host-side handle of the SpecAnn engine and the device control blocks of its kernels.
#pragma once
#include <vector>
#include <cstdint>
#include <cstddef>
#include <cuda_runtime.h>

#include "common.cuh"

namespace sa {

// Control block of the alpha-solve kernel (device memory, part of the workspace).
struct AlphaCtrl {
  GridSync gs;
  double a[kNcvMax];        // diagonal of the projected tridiagonal T
  double b[kNcvMax];        // off-diagonal (b[i] couples basis vectors i and i + 1)
  double h[kNcvMax];        // reorthogonalisation coefficients of the current step
  double s[kNcvMax];        // Ritz coefficients (restart / final vector)
  double theta;             // current smallest Ritz value
  double inv_b;             // 1 / norm of the pending (unnormalised) vector w
  double ww;                // ||w||^2 before the update of the current step
  double scale;             // final normalisation and sign of y
  double nrm_y;
  double rr;                // squared true residual
  int j;                    // index of the basis vector the next step creates
  int action;               // next action of every CTA (see alpha kernel)
  int iters;
  int restarts;
  int mode;                 // start mode in use
  int test_pred;            // the next step is the predictor's residual test
  int pass2;                // second reorthogonalisation pass in progress
  int nonfinite;
  int secant_sign;
  int pad0;
  double pred_residual;
  int pred_accepted;
  int status;
  unsigned long long sig;   // order-independent hash of the packed spins
  double degree_scale;
  double align_dot;
  double res_est;
  double bytes;             // algorithmic DRAM bytes of this launch
  int spmvs;                // fused SpMVs run by this launch
  int irl_k;                // basis vectors kept by the last implicit restart
  double irl_beta;          // T+[k][k-1] of the last implicit restart
  double irl_sigma;         // Q[m-1][k-1] of the last implicit restart
  unsigned long long tph[6];  // ns by phase (set-up, SpMV, dots, update+Ritz, restart, final)
  int ritz_ok;              // theta / res_est hold the previous step's Ritz value and residual estimate
};

// Control block of the local-search kernel.
struct LsCtrl {
  GridSync gs;
  int phase;                // 0 main loop, 1 final sweep, 2 done
  int it;                   // main-loop passes used
  int round, sub;
  int final_passes;
  int pad;
  long long stream;         // selection stream of the current pass
  long long m;              // nodes selected in the current pass
  long long wl_count;       // work-list entries of the current pass
  long long wq_count;       // wanting nodes of the current pass (priority passes)
  long long total_flips;
  unsigned int active[4];   // candidates that have not yet had a pass without a flip
  long long counts[128];    // flips per candidate in the current pass
  unsigned long long tph[4];  // ns by phase (set-up, decide, scatter, final)
};

struct Layout {
  size_t total = 0;
  __host__ __device__ size_t off(size_t bytes) {
    size_t o = total;
    total += (bytes + 255) & ~size_t(255);
    return o;
  }
};

// Upper bound of the SpMV work list for a matrix of n rows and nnz entries: a short segment is
// closed when it has kSegRows rows or the next row would take it past kSegMax entries (so it
// holds more than kSegMax - kShortMax entries, or kSegRows rows, unless a long row or the end
// follows it); a long row gives at most nnz_row / kChunk + 1 chunks.
inline long long max_items(long long n, long long nnz) {
  return n / kSegRows + nnz / (kSegMax - kShortMax) + 2 * (nnz / (kShortMax + 1)) + nnz / kChunk + 8;
}
inline long long max_multichunk_rows(long long nnz) { return nnz / (kChunk + 1) + 1; }
inline long long max_long_partials(long long nnz) { return nnz / kChunk + max_multichunk_rows(nnz) + 1; }

// The SpMV work list of a CSR given its host row pointers (capi.cu): items, the partial-sum base of
// every multi-chunk row, the partial sums they need and the mean length of the short rows.
void build_items(const std::vector<long long>& rp, long long n, std::vector<WorkItem>& items,
                 std::vector<long long>& mc_base, long long* n_long_part, double* mean_short);

}  // namespace sa

struct sa_handle {
  long long n = 0, nnz = 0;
  int rp64 = 0, prec = 32, ncv_max = 33, max_cand = 128;
  cudaStream_t stream = nullptr;
  char* ws = nullptr;
  size_t ws_bytes = 0;
  // bound matrix (caller-owned device memory)
  const void* rowptr = nullptr;
  const int32_t* col = nullptr;
  const void* val = nullptr;
  bool bound = false;
  double c = 0.0, dmin = 0.0, dmax = 0.0;
  int integer_J = 0;
  // SpMV stream of couplings of one magnitude: packed signed columns (workspace, nnz int32)
  int32_t* scol = nullptr;
  double wmag = 0.0;        // the common |J_ij| when every coupling has it, else 0
  int packed = 0;           // scol holds the bound matrix and the SpMV streams it
  int packed_allowed = 1;   // sa_set_spmv_policy
  // L2 column splits (sa_split_build): per split a CSR of the columns in one range and its work list
  int split_ready = 0, split_on = 0, n_splits = 0;
  struct Split {
    const void* rowptr = nullptr;    // n + 1, the handle's row pointer type
    const int32_t* col = nullptr;    // packed signed columns when the couplings have one magnitude
    const void* val = nullptr;       // values (null with packed columns)
    sa::WorkItem* items = nullptr;
    long long n_items = 0, nnz = 0;
    long long* mc_base = nullptr;
    int* mc_count = nullptr;
    void* long_part = nullptr;
  } split[sa::kMaxSplits];
  void* split_part = nullptr;        // partial row sums between the passes (n, working precision)
  double split_bytes = 0.0;          // algorithmic bytes of one split SpMV's matrix stream
  // column-panel SpMV (sa_panel_build): layout in the caller's panel workspace
  int panel_ready = 0, panel_on = 0;
  int panel_blocks = 0, panel_count = 0, panel_width = 0;
  long long panel_slots = 0;   // entry slots of the layout (padding included)
  const unsigned int* panel_ent = nullptr;
  const void* panel_val = nullptr;
  const long long* panel_chunk = nullptr;
  const int* panel_row0 = nullptr;
  // workspace carve-out
  long long ldv = 0;            // leading dimension of basis vectors (n rounded up to 64)
  void* sigma = nullptr;        // D^{-1/2} / sqrt(c) for the current alpha (T)
  double* ld = nullptr;         // log2 d (double)
  const double* aoff = nullptr; // per-vertex exponent offsets of the solves (caller's device array) or null
  double* deg = nullptr;        // absolute degrees (double)
  void* V = nullptr;            // Lanczos basis, ncv_max x ldv (T)
  void* w = nullptr;
  void* u = nullptr;
  void* yv[3] = {nullptr, nullptr, nullptr};
  int iy_out = 0, iy_last = 1, iy_prev = 2;
  bool has_last = false, has_prev = false;
  sa::WorkItem* items = nullptr;
  long long n_items = 0, cap_items = 0;
  long long* mc_base = nullptr;
  int* mc_count = nullptr;
  long long n_mc = 0, cap_mc = 0;
  void* long_part = nullptr;
  long long cap_long_part = 0;
  long long n_long_part = 0;    // partial sums the bound matrix's multi-chunk rows use
  double* blk_part = nullptr;
  int blk_part_width = 0;
  sa::AlphaCtrl* actrl = nullptr;
  double* dense = nullptr;      // implicit-restart scratch: dense T and Q (2 x kNcvMax^2 doubles)
  double* red = nullptr;        // small reduction scratch (set-up kernels)
  uint32_t* cand = nullptr;     // candidate store, max_cand x W
  uint32_t* refined = nullptr;  // refined candidates, max_cand x W
  uint32_t* scratch = nullptr;  // rounded spins of the last solve, W words
  long long W = 0;              // words per packed candidate
  int group = 8;                // lanes per short row in the SpMV
  int sm_count = 0;
  int max_blocks = 0;           // cooperative grid size cap for this device
  int blocks = 0;               // grid size used by the persistent kernels
};

namespace sa {
// Sticky status word of the asynchronous standalone operator (sa_spmv_scaled on the panel layout):
// a timed-out panel wait records SA_ERR_BARRIER_TIMEOUT here; sa_operator_status reads and clears it.
inline int* operator_status_word(sa_handle* h) { return (int*)(h->red + 20); }
}  // namespace sa

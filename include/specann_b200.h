/* C-ABI of the B200 SpecAnn engine (libspecann_b200.so).
 *
 * Plain pointers and sizes only. Device buffers are allocated by the caller (the Python host uses
 * torch) and passed as raw device pointers together with a cudaStream_t (as void*). Every entry
 * point returns an int status (sa_status below); none of them allocates device memory.
 *
 * Each declaration names the reference interface it replaces (paths inside the reference
 * repository Vgueca/SpecAnn).
 */
#ifndef SPECANN_B200_H
#define SPECANN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. The Python host maps them onto the reference's exceptions
 * (models/spectral_annealing.py:70-77 EigensolverBreakdown, utils/failures.py:4-25
 * NumericalFailure / out-of-memory). */
typedef enum {
  SA_OK = 0,
  SA_ERR_BREAKDOWN = 1,        /* Lanczos breakdown: non-finite or impossible Ritz matrix entry */
  SA_ERR_NONFINITE = 2,        /* non-finite eigenvalue or eigenvector */
  SA_ERR_NOT_CONVERGED = 3,    /* stopped at maxiter above tol (the pair is still returned) */
  SA_ERR_OOM = 4,              /* workspace too small */
  SA_ERR_INVALID_ARG = 5,
  SA_ERR_CUDA = 6,             /* a CUDA runtime call failed */
  SA_ERR_BARRIER_TIMEOUT = 7   /* a bounded grid-barrier wait ran out (kernel returned early) */
} sa_status;

/* Start vector of an alpha solve (models/spectral_annealing.py:589-612). */
typedef enum {
  SA_START_RANDOM = 0,     /* cold start: a seeded standard-normal vector */
  SA_START_PREV = 1,       /* the previous eigenvector y_last as is (pred_mode "prev") */
  SA_START_DIAGONAL = 2,   /* utils/predictors.py:6-26, then the residual acceptance test */
  SA_START_SECANT = 3,     /* utils/predictors.py:29-56, then the residual acceptance test */
  SA_START_GIVEN = 4,      /* the device vector passed in sa_alpha_params.v0 */
  SA_START_TANGENT = 5     /* y_last + (alpha - alpha_prev) v0 with v0 the eigenvector tangent dy/dalpha
                              at alpha_prev (sa_adjoint, SA_ADJ_TANGENT), then the residual acceptance test; no
                              counterpart in the reference (a third predictor beside diagonal/secant) */
} sa_start_mode;

typedef struct sa_handle sa_handle;

typedef struct {
  double alpha;          /* normalisation exponent of this solve */
  double alpha_prev;     /* alpha of y_last (diagonal predictor step) */
  double rho;            /* shift: S_rho = rho I - N_alpha */
  double gershgorin;     /* g = max d^(1 - alpha): bound used by the Ritz-matrix guard */
  double tol;            /* Lanczos residual-estimate tolerance (eigsh_tol) */
  double pred_tol;       /* predictor acceptance tolerance */
  double secant_gamma;   /* secant step (1.0 in the reference) */
  int32_t maxiter;       /* maximum Lanczos matvecs (eigsh_maxiter) */
  int32_t ncv;           /* Lanczos basis size (<= the handle's ncv_max) */
  int32_t start_mode;    /* sa_start_mode */
  int32_t align;         /* 1: sign-align the result with y_last (when a y_last exists) */
  uint64_t seed;         /* seed of the random start stream */
  int64_t stream_id;     /* random stream id (alpha index and attempt) */
  const void* v0;        /* device start vector (SA_START_GIVEN) or tangent (SA_START_TANGENT), else NULL */
  int32_t round;         /* 1: round x = D^{-1/2} y to packed spins and hash them */
  int32_t residual_check;/* 1: true residual ||S y - mu y|| with one more SpMV */
  int32_t restart_keep;  /* Ritz vectors kept by an implicit restart (0: 8; at most 16 and ncv / 2) */
  int32_t reserved;
} sa_alpha_params;

typedef struct {
  int32_t status;        /* sa_status of this solve */
  int32_t iterations;    /* Lanczos matvecs (the predictor test matvec not counted) */
  int32_t restarts;      /* thick restarts */
  int32_t pred_accepted; /* -1 no predictor ran, 0 rejected (restarted from y_last), 1 accepted */
  double mu;             /* smallest eigenvalue of S_rho (Ritz value) */
  double lambda1;        /* rho - mu: leading eigenvalue of N_alpha */
  double residual;       /* ||S y - mu y|| / ||y|| with FP64 accumulation (NaN if not checked) */
  double res_estimate;   /* Lanczos estimate |b_j s_j| */
  double pred_residual;  /* ||N y0 - (y0.N y0) y0|| of the predicted start (NaN if none) */
  double degree_scale;   /* sum_i d_i^alpha (the per-alpha CSV column degree_scale) */
  double align_dot;      /* y . y_last before the sign alignment (0 without y_last) */
  uint64_t signature;    /* 64-bit hash of the packed rounded spins */
  int32_t nonfinite;     /* 1 if the eigenvector had a non-finite entry */
  int32_t basis_used;    /* basis vectors in use at the end */
  int32_t spmv_count;    /* fused SpMVs the launch ran (Lanczos steps, predictor test, residual) */
  int32_t reserved;
  double alg_bytes;      /* algorithmic DRAM bytes of the launch: SpMVs + basis/vector passes */
  double phase_ms[6];    /* device time by phase: set-up, SpMV, dots, update+Ritz, restart, final */
} sa_alpha_record;

typedef struct {
  int32_t k;                    /* candidates (slots first_slot .. first_slot + k - 1) */
  int32_t first_slot;           /* first candidate slot (0 for the batched search) */
  int32_t max_iterations;       /* main-loop passes (max_local_iterations) */
  double subset_fraction;       /* 0.9 */
  double final_sweep_fraction;  /* 1.0 */
  int32_t final_sweep_iters;    /* 25 */
  int32_t num_rounds;           /* 25 */
  uint64_t seed;                /* node-selection stream seed */
  int32_t semantics;            /* 0: priority passes (default), 1: snapshot (Jacobi) passes */
  int32_t reserved;
} sa_ls_params;

typedef struct {
  int32_t status;
  int32_t iterations;           /* main-loop passes used (flip_refinement's max_iters_used) */
  int32_t final_passes;         /* passes run by the final sweep */
  int32_t integer_gains;        /* 1: int32 gains (bit-exact); 0: FP64 gains */
  int64_t total_flips;
  double phase_ms[4];           /* device time by phase: set-up (fields, energies), decide (passes'
                                   selection, decisions and blocking check), scatter (field updates and
                                   the stopping rules), final (energies after, refined spins) */
} sa_ls_result;

/* ---- workspace and handle ------------------------------------------------------------------ */

/* Bytes of device workspace for a handle (no reference counterpart: CuPy's memory pool,
 * models/spectral_annealing.py:493-496, is replaced by one caller-owned buffer). */
int sa_workspace_size(int64_t n, int64_t nnz, int32_t rowptr64, int32_t precision,
                      int32_t ncv_max, int32_t max_candidates, size_t* bytes);

/* Create a solver handle over a caller-owned workspace (replaces the per-solve CuPy setup of
 * SpectralAnnealing.solve, models/spectral_annealing.py:262-288). precision: 32 or 64. */
int sa_create(sa_handle** out, int64_t n, int64_t nnz, int32_t rowptr64, int32_t precision,
              int32_t ncv_max, int32_t max_candidates, void* workspace, size_t workspace_bytes,
              void* stream);
int sa_destroy(sa_handle* h);

/* Bind the device CSR (rowptr: int32 or int64 per rowptr64; col: int32; val: float or double per
 * precision; symmetric, zero diagonal) and run the prelude of models/spectral_annealing.py:270-288:
 * absolute degrees, c = max degree, d = deg / c, log2 d; build the SpMV work list. Reports c,
 * min/max of d and whether every coupling is an integer (int32 gains in the local search). */
int sa_set_matrix(sa_handle* h, const void* rowptr, const int32_t* col, const void* val,
                  double* norm_c, double* d_min, double* d_max, int32_t* integer_couplings);

/* y = rho x - N_alpha x with N_alpha = D^{-1/2} (J/c) D^{-1/2}, D = max(d^alpha, 1e-12): the
 * fused operator of NAlphaOperator/SRhoOperator (models/spectral_annealing.py:29-53). x, y are
 * device vectors of the handle's precision. */
int sa_spmv_scaled(sa_handle* h, double alpha, double rho, const void* x, void* y);

/* Status of the asynchronous standalone operator since the last query: sa_spmv_scaled on the
 * column-panel layout waits (bounded) for each staged panel, and a wait that runs out leaves y
 * partly written and records SA_ERR_BARRIER_TIMEOUT in a sticky word of the handle. This call
 * synchronises the handle's stream, returns that word in *status (SA_OK when every application since
 * the last query completed) and clears it. The work-list and split layouts have no waits and always
 * report SA_OK. No reference counterpart (CuPy's SpMV, models/spectral_annealing.py:38-41, has no
 * device-side waits). */
int sa_operator_status(sa_handle* h, int32_t* status);

/* SpMV stream policy (every kernel that applies the operator). packed_columns = 1 (the default):
 * when every coupling of the bound matrix has the same magnitude w, the work-list SpMV streams one
 * int32 per entry (the column with the coupling's sign in bit 31) instead of the column and the
 * value; the products are unchanged. Takes effect at the next launch and survives sa_set_matrix. */
int sa_set_spmv_policy(sa_handle* h, int32_t packed_columns);
/* The policy in effect: packed (1 when the packed stream is used) and the common coupling magnitude
 * (0 when the magnitudes differ). Any pointer may be NULL. */
int sa_get_spmv_policy(sa_handle* h, int32_t* packed_columns, double* magnitude);

/* Column-panel SpMV. Every CTA keeps the row sums of a block of rows in shared memory and gathers
 * the scaled input from panels of it staged in shared memory, instead of from L2: it pays when
 * rows average more than ~20 entries and the row blocks (at most 16384 rows in FP32, 8192 in
 * FP64, about equal entries) are no more than the SMs. sa_panel_workspace_size gives the bytes of
 * the layout for the bound matrix and its number of row blocks (row_blocks may be NULL);
 * sa_panel_build lays the matrix out in that caller-owned device workspace
 * (256-byte aligned, kept until the next sa_set_matrix) and switches the operator kernels to it;
 * sa_panel_enable(h, 0 / 1) switches back and forth. sa_set_matrix drops the layout. */
int sa_panel_workspace_size(sa_handle* h, size_t* bytes, int32_t* row_blocks);
int sa_panel_build(sa_handle* h, void* workspace, size_t bytes);
int sa_panel_enable(sa_handle* h, int32_t on);
/* L2 column splits, for operators whose gathered vector is larger than L2 (n > ~8 M in FP32): the
 * columns are cut into `splits` ranges (2..8; 0: one per 48 MB of the vector) and the operator is
 * applied as one work-list pass per range, so every pass gathers from an L2-resident slice.
 * sa_split_workspace_size gives the bytes of the layout (and the split count used);
 * sa_split_build builds it in a caller-owned device workspace (256-byte aligned, kept until the
 * next sa_set_matrix) and switches the operator kernels to it (the panel layout, if any, off);
 * sa_split_enable switches back and forth; sa_split_count reports the splits in use (0: off) and the
 * algorithmic bytes of one split SpMV's matrix stream and partial sums (matrix_bytes may be NULL). */
int sa_split_workspace_size(sa_handle* h, int32_t splits, size_t* bytes, int32_t* splits_used);
int sa_split_build(sa_handle* h, int32_t splits, void* workspace, size_t bytes);
int sa_split_enable(sa_handle* h, int32_t on);
int sa_split_count(sa_handle* h, int32_t* splits, double* matrix_bytes);

/* The built layout: entry slots (padding included), row blocks, panels, columns per panel and the
 * algorithmic DRAM bytes of one panel SpMV's matrix stream (entries, values when they differ in
 * magnitude, chunk bounds). Any pointer may be NULL; INVALID_ARG when no layout is built. */
int sa_panel_info(sa_handle* h, int64_t* slots, int32_t* row_blocks, int32_t* panels, int32_t* width,
                  double* alg_bytes);
/* Device pointers to the built layout's tables (diagnostics; no reference counterpart): the padded
 * entry stream (uint32 per slot: row in block << 16 | sign << 15 | column in panel; padding
 * 0xFFFF0000), the chunk starts (int64, [(block * panels + panel) * 16 + warp], one extra end entry)
 * and the block first rows (int32, row_blocks + 1). Any pointer may be NULL; valid until the next
 * sa_set_matrix. */
int sa_panel_tables(sa_handle* h, const void** entries, const void** chunk_starts, const void** block_rows);

/* One alpha of the sweep (models/spectral_annealing.py:568-669 with utils/eigsh.py:10-17 and
 * utils/predictors.py): start vector / predictor with its residual test, warm-started
 * thick-restart Lanczos for the smallest eigenpair of S_rho with the Ritz-matrix guard
 * (:85-120), sign alignment with y_last and normalisation (:653-663), optional true residual
 * (:636-647), and the rounding s = sign(x >= 0) of x = D^{-1/2} y (:345) packed into the scratch
 * candidate with its signature (:557-561). One cooperative launch. */
int sa_alpha_solve(sa_handle* h, const sa_alpha_params* p, sa_alpha_record* rec);

/* The last solved eigenvector y (unit norm, aligned) as a device pointer valid until the next
 * sa_alpha_solve or sa_commit_alpha. */
int sa_result_vector(sa_handle* h, const void** y);

/* Accept the last solve as the new warm start: y_prev <- y_last <- y
 * (models/spectral_annealing.py:330-342). */
int sa_commit_alpha(sa_handle* h);

/* Set y_last (and clear y_prev) from a device vector (tests, external warm starts). */
int sa_set_last_vector(sa_handle* h, const void* y);

/* Rounding only: align a given device eigenvector with y_last (if align), normalise it, form
 * x = D^{-1/2} y for this alpha and round it into the scratch candidate
 * (models/spectral_annealing.py:345, :557-561). */
int sa_round_vector(sa_handle* h, double alpha, const void* y, int32_t align, uint64_t* signature);

/* Candidate store (the dict of models/spectral_annealing.py:362-370): copy the scratch
 * candidate into slot; compare it with a slot; copy packed words in or out; unpack to int8. */
int sa_candidate_keep(sa_handle* h, int32_t slot);
int sa_candidate_equal(sa_handle* h, int32_t slot, int32_t* equal);
int sa_candidate_set(sa_handle* h, int32_t slot, const uint32_t* packed_device);
int sa_candidate_get(sa_handle* h, int32_t slot, int32_t refined, uint32_t* packed_device);
int sa_candidate_unpack(sa_handle* h, int32_t slot, int32_t refined, int8_t* spins_device);

/* Bytes of device workspace for a local search over k candidates. */
int sa_ls_workspace_size(sa_handle* h, int32_t k, size_t* bytes);

/* Batched local search of candidate slots first_slot..first_slot+k-1 (flip_refinement + gpu_final_sweep,
 * models/spectral_annealing.py:983-1112) as one persistent kernel with snapshot passes and the
 * counter-based node selection; also the energies before and after
 * (models/spectral_annealing.py:693-720, :925-976). Refined spins go to the refined store.
 * energies_*: host arrays of k doubles (exact integers for integer couplings). */
int sa_local_search(sa_handle* h, const sa_ls_params* p, void* ls_workspace, size_t ls_bytes,
                    double* energies_before, double* energies_after, sa_ls_result* result);

/* Energies E = -1/2 s^T J s of candidate slots 0..k-1 (no local search): _batch_energies /
 * fp32_energies, models/spectral_annealing.py:693-707, :962-976. */
int sa_energies(sa_handle* h, int32_t k, void* ls_workspace, size_t ls_bytes, double* energies);

/* ---- guarded local-search policies (ls_policy other than "default") ------------------------------
 * The refiners of models/local_search_guards/ (policies.py:13-69, registry.py:8-13) over candidate
 * slots first_slot .. first_slot + k - 1; refined spins go to the refined store. Node selection uses
 * the same counter-based stream as sa_local_search; decisions use exact integer gains for integer
 * couplings. */
typedef enum {
  SA_GUARD_FIXED = 1,            /* Fixed Guard: safe_flip_refinement, models/spectral_annealing_safe.py:1035-1335,
                                    models/local_search_guards/safe_fixed.py */
  SA_GUARD_ADAPTIVE = 2,         /* Adaptive Guard: the same with per-candidate batch adaptation,
                                    models/local_search_guards/safe_adaptive.py, models/safe_update_policy.py:68-95 */
  SA_GUARD_INDEPENDENT_SET = 3,  /* Independent-Set: one colour class per update, models/local_search_guards/
                                    conflict_free.py:80-367 (colouring and class order from the host) */
  SA_GUARD_SEQUENTIAL = 4        /* Sequential-Oracle: exact one-flip steepest descent,
                                    models/local_search_guards/sequential_oracle.py:26-219 */
} sa_guard_policy;

typedef struct {
  int32_t k;                     /* candidates */
  int32_t first_slot;
  int32_t policy;                /* sa_guard_policy */
  int32_t max_iterations;        /* main-phase rounds (max_local_iterations) */
  double subset_fraction;        /* 0.9 */
  double final_sweep_fraction;   /* 1.0 */
  int32_t final_sweep_iters;     /* 25 */
  int32_t num_rounds;            /* 25 */
  uint64_t seed;                 /* node-selection stream seed */
  const int32_t* colors;         /* SA_GUARD_INDEPENDENT_SET: device colour of every node */
  const int32_t* color_seq;      /* SA_GUARD_INDEPENDENT_SET: device colour class of every update
                                    (max_iterations + final_sweep_iters * num_rounds entries) */
  int32_t num_colors;
  int32_t reserved;
} sa_guard_params;

typedef struct {
  int32_t status;                /* SA_OK; SA_ERR_NOT_CONVERGED when the oracle stopped at 100 n steps */
  int32_t rounds;                /* main-phase rounds (guards), updates (independent set) or steps (oracle):
                                    the iteration count the reference reports */
  int32_t final_rounds;          /* final-phase rounds (guards) */
  int32_t accepted, rejected;    /* guarded candidate updates accepted / rejected */
  int32_t integer_gains;         /* 1: exact integer arithmetic */
  int64_t flips;                 /* applied (node, chunk) updates; oracle: flips */
} sa_guard_result;

int sa_guard_workspace_size(sa_handle* h, int32_t k, size_t* bytes);
int sa_guard_search(sa_handle* h, const sa_guard_params* p, void* workspace, size_t bytes,
                    double* energies_before, double* energies_after, sa_guard_result* result);

/* ---- differentiation form: adjoint of the leading eigenvector ------------------------------------
 * No counterpart in the reference (it has no gradients). With per-vertex exponents a (a_i = alpha +
 * offset_i, offsets optional) the solves use N_a = D_a^{-1/2} (J/c) D_a^{-1/2}; the rounding vector
 * is x = D_a^{-1/2} y (models/spectral_annealing.py:663, :345) and the smoothed energy is
 * L = -1/2 tanh(beta x)^T J tanh(beta x). */

/* Per-vertex exponent offsets used by the following sa_alpha_solve and sa_adjoint calls (device
 * array of n doubles owned by the caller; NULL clears them). sa_spmv_scaled ignores them. */
int sa_set_exponent_offsets(sa_handle* h, const double* offsets_device);

typedef enum {
  SA_ADJ_GRADIENT = 0,   /* dL/da per vertex (and dL/dalpha = its sum) at the eigenpair (lambda1, y) */
  SA_ADJ_TANGENT = 1,    /* dy/dalpha at the eigenpair: the tangent predictor's direction */
  SA_ADJ_SOLVE = 2       /* (lambda1 I - N_a) out = (I - y y^T) rhs with out orthogonal to y */
} sa_adjoint_mode;

typedef struct {
  double alpha;          /* exponent of the eigenpair */
  double lambda1;        /* its leading eigenvalue */
  double beta;           /* tanh sharpness (SA_ADJ_GRADIENT) */
  double tol;            /* MINRES tolerance on the residual relative to the right-hand side */
  int32_t maxiter;       /* MINRES iterations at most */
  int32_t mode;          /* sa_adjoint_mode */
  const void* y;         /* unit leading eigenvector (device, the handle's precision) */
  const void* rhs;       /* SA_ADJ_SOLVE: right-hand side (device) */
  void* out;             /* SA_ADJ_TANGENT / SA_ADJ_SOLVE: the solution (device, n values) */
  double* grad;          /* SA_ADJ_GRADIENT: dL/da_i (device, n doubles) */
} sa_adjoint_params;

typedef struct {
  int32_t status;        /* SA_OK (tol reached, or the residual stalled below 1e-3 of the right-hand
                            side: the eigenpair's own error bounds what the solve can resolve),
                            SA_ERR_NOT_CONVERGED, SA_ERR_NONFINITE, ... */
  int32_t iterations;    /* MINRES iterations */
  int32_t spmv_count;    /* fused SpMVs of the call */
  int32_t reserved;
  double residual;       /* MINRES residual estimate relative to the projected right-hand side */
  double loss;           /* SA_ADJ_GRADIENT: L at the eigenpair */
  double dloss_dalpha;   /* SA_ADJ_GRADIENT: dL/dalpha = sum_i dL/da_i */
} sa_adjoint_result;

int sa_adjoint_workspace_size(sa_handle* h, size_t* bytes);

/* One persistent cooperative launch: right-hand side, MINRES on the projected operator (FP64
 * scalars and inner products), and for the gradient the products M w, M y and the assembly. */
int sa_adjoint(sa_handle* h, const sa_adjoint_params* p, void* work, size_t bytes, sa_adjoint_result* res);

/* ---- batched sweeps: many (instance, seed) problems in one launch ------------------------------
 * Replaces the reference's driver loop that builds one solver per (instance, seed) and calls
 * solve(J) on it (utils/core.py:103-105, models/spectral_annealing.py:262-525 per problem): every
 * problem runs the whole alpha sweep (shift, start mode, alpha solve, cold retry, checks,
 * deduplication, warm-start commit) and the local search of its distinct candidates inside one
 * persistent cooperative kernel. Instances are sa_handle objects with a bound matrix (their prelude
 * is reused); all must share the precision and use 32-bit row pointers. Problem p is instance
 * p / seeds_per_instance with seed seeds[p]. */
typedef struct sa_batch sa_batch;

typedef struct {
  double eigsh_tol, pred_tol, shift_eps, secant_gamma;
  double subset_fraction, final_sweep_fraction;
  int32_t num_alphas;            /* <= 128 and <= the batch's candidate capacity */
  int32_t maxiter;
  int32_t ncv;                   /* 0: min(33, n - 1) per instance */
  int32_t pred_mode;             /* SA_START_DIAGONAL, SA_START_SECANT or SA_START_PREV */
  int32_t warm_start;
  int32_t residual_check;
  int32_t use_local_search;
  int32_t max_local_iterations;
  int32_t final_sweep_iters;
  int32_t num_rounds;
  int32_t ls_semantics;          /* 0 priority, 1 snapshot */
  int32_t reserved;
} sa_batch_config;

/* One alpha of one problem: the columns of the reference's per-alpha rows. */
typedef struct {
  double alpha, lambda1, rho, gershgorin, residual, pred_residual, degree_scale;
  uint64_t signature;
  int32_t status, iterations, restarts, spmv_count;
  int32_t pred_accepted;         /* -1: no predictor test */
  int32_t retry, converged;
  int32_t candidate;             /* -1: the alpha was skipped */
} sa_batch_alpha_record;

/* One problem after the sweep. */
typedef struct {
  int32_t status, num_candidates, ls_iterations, ls_final_passes;
  int32_t alphas_skipped, alphas_retried, team_first_block, team_blocks;
  int32_t integer_gains, reserved;
  int64_t ls_total_flips;
  double device_ms;
  double phase_ms[6];            /* sweep time by phase as sa_alpha_record.phase_ms, summed over alphas */
  double ls_ms;                  /* local-search time */
  double energy_before[128];     /* per candidate slot, exact integers for integer couplings */
  double energy_after[128];
} sa_batch_summary;

/* CTAs of the batch kernel that fit on this device at once (the grid of every batch launch). */
int sa_batch_grid(int32_t precision, int32_t rowptr64, int32_t* blocks);

/* Host-only plan of problems onto teams of CTAs: the problems sorted by cost (measured_cost[p],
 * the CTA-time of an earlier run, or NULL for a model of sizes n, nnz), each large one given its
 * own team of about split x its share of `blocks` CTAs, the rest placed longest-first on the team
 * that finishes first (barrier_cost: relative overhead of a multi-CTA team). Outputs
 * team_of[n_prob] and the contiguous teams [team_b0, team_b0 + team_nb) (arrays of `blocks`
 * entries; *n_teams used). No counterpart in the reference. */
int sa_batch_plan(int32_t n_prob, const int64_t* n, const int64_t* nnz, const double* measured_cost,
                  int32_t blocks, double split, double barrier_cost, int32_t* team_of, int32_t* team_b0,
                  int32_t* team_nb, int32_t* n_teams);

int sa_batch_workspace_size(int32_t n_inst, sa_handle* const* inst, int32_t seeds_per_instance,
                            int32_t ncv_max, int32_t capacity, int32_t n_teams, const int32_t* team_b0,
                            const int32_t* team_nb, const int32_t* team_of, size_t* bytes);

int sa_batch_create(sa_batch** out, int32_t n_inst, sa_handle* const* inst, int32_t seeds_per_instance,
                    const uint64_t* seeds, int32_t ncv_max, int32_t capacity, int32_t n_teams,
                    const int32_t* team_b0, const int32_t* team_nb, const int32_t* team_of,
                    void* workspace, size_t bytes, void* stream);

/* Run every problem's sweep (alphas: host array of cfg->num_alphas values). With use_graph the
 * first call captures the launch (barrier reset + cooperative kernel) into a CUDA graph and later
 * calls replay it. Asynchronous on the batch's stream. */
int sa_batch_sweep(sa_batch* b, const sa_batch_config* cfg, const double* alphas, int32_t use_graph);

/* Per-problem results (host arrays: records n_prob x 128, summaries n_prob); synchronises. */
int sa_batch_results(sa_batch* b, sa_batch_alpha_record* records, sa_batch_summary* summaries);

/* Packed words of candidate slot of a problem (refined: after the local search). */
int sa_batch_candidate(sa_batch* b, int32_t problem, int32_t slot, int32_t refined, uint32_t* packed_device);

int sa_batch_destroy(sa_batch* b);

/* ---- instance matrix built on the device ------------------------------------------------------
 * The COO -> CSR step of the reference's loader (utils/data_loader.py:112-204: both triangles appended
 * edge by edge, coo_matrix(...).tocsr() summing duplicates, _remove_isolated_nodes) for an edge list
 * parsed on the host: a stable device radix sort of the 2 num_edges directed entries by (row, column),
 * duplicates summed in file order in FP64, rows whose entries are all zero removed (when any entry
 * exists) and the rest renumbered. ei, ej (int64) and ew (double) are device arrays of num_edges
 * undirected edges in file order; the outputs are device arrays sized for the worst case (row pointers
 * num_vertices + 1, columns and values 2 num_edges, node_ids num_vertices): the kept rows' original
 * indices go to node_ids, and *n_out, *nnz_out give the result's size. Synchronises `stream`. */
int sa_coo_workspace_size(int64_t num_edges, int64_t num_vertices, size_t* bytes);
int sa_coo_to_csr(int64_t num_edges, int64_t num_vertices, const int64_t* ei, const int64_t* ej, const double* ew,
                  void* workspace, size_t bytes, int64_t* rowptr, int32_t* col, double* val, int64_t* node_ids,
                  int64_t* n_out, int64_t* nnz_out, void* stream);

/* ---- allocation-free operator ------------------------------------------------------------- */

/* Largest n accepted by sa_spmv_scaled_noalloc. */
#define SA_NOALLOC_MAX_N (1 << 20)

/* y = rho x - N_alpha x (the operator of sa_spmv_scaled) for callers that cannot allocate device
 * memory and have no workspace to hand over, such as a host framework whose pool allocator owns the
 * whole device, or a latency-sensitive caller that must not pay for cudaMalloc's implicit device
 * synchronisation. No counterpart in the reference. It needs no handle: the CSR (int32 row pointers,
 * int32 columns, float couplings; symmetric, zero diagonal), x and y are the caller's device
 * buffers, and the degrees and scaling are computed on every call. Its scratch is a fixed device
 * array inside the library (8 MiB per GPU, held until the process exits), so it allocates nothing.
 * n > SA_NOALLOC_MAX_N is rejected with SA_ERR_INVALID_ARG. The first call on each device looks up
 * the array's device address; make that first call before any stream capture. All calls share the
 * array: calls that overlap on the GPU race, so serialise them. The row pointers must be a valid CSR
 * of nnz entries; a column outside [0, n) is skipped (its product counts as zero), and a matrix
 * whose couplings are all zero gives y = rho x. */
int sa_spmv_scaled_noalloc(int64_t n, int64_t nnz, const int32_t* rowptr, const int32_t* col,
                           const float* val, double alpha, double rho, const float* x, float* y,
                           void* stream);

/* Diagnostics of the bounded grid barrier that separates the phases of the persistent kernels (no
 * reference counterpart): one launch of `blocks` CTAs (1 .. the SM count) that meet at one barrier of
 * `expected` arrivals, each waiting at most spin_limit sleeps of ~64 ns (1 .. 2^25). scratch: a
 * caller-owned device buffer of at least 16 + 4 * blocks bytes, 16-byte aligned. Synchronises
 * `stream`. *status: the barrier's error word (SA_OK, or SA_ERR_BARRIER_TIMEOUT when a wait ran out,
 * e.g. with expected > blocks); *passed_blocks: CTAs whose barrier returned success; *epilogues:
 * CTAs that ran the last-arrival epilogue (1 on success, 0 when nobody arrives last). */
int sa_barrier_selftest(int32_t blocks, int32_t expected, uint64_t spin_limit, void* scratch, size_t scratch_bytes,
                        int32_t* status, int32_t* passed_blocks, int32_t* epilogues, void* stream);

/* Version string of the library. */
const char* sa_version(void);

/* Kernel launches this library has issued since it was loaded (diagnostics; no reference
 * counterpart). */
uint64_t sa_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* SPECANN_B200_H */

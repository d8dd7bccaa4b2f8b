/*
 * cy3q.h -- C ABI of the B200 (sm_100a) CY3 quintic metric solver.
 *
 * Drop-in boundary for the data-parallel hot path of the reference crate
 * `substrate_sm_derivation/cy3_solver` (Rust).  The reference exposes that path as the
 * in-process Rust workspace `QuinticSolver` (src/quintic.rs:117-165) plus free functions and the
 * GPU object `AdamGradientKernel` (src/gpu_adam.rs:1533-2195).  Each entry point below names the
 * reference interface it replaces.  All arrays are caller-owned HOST memory in the reference's
 * layouts, copied in and out; device state is owned by the handle.  Plain C types only.
 *
 * Layouts (reference conventions):
 *   points      [P x 10]  f64, (re, im) of z_0..z_4 interleaved            (quintic.rs:128)
 *   weights     [P]       f64, w_p = 1/|grad f|^2                          (quintic.rs:3507)
 *   log_omega   [P]       f64, log|Omega|^2                                (quintic.rs:4858)
 *   h_block     [2N x 2N] f64 row-major, [2a][2b] = Re h_ab, [2a][2b+1] = -Im h_ab,
 *                         [2a+1][2b] = Im h_ab, [2a+1][2b+1] = Re h_ab       (quintic.rs:4081-4085)
 *   grad        [2N^2]    f64, first N^2 = d/d Re h_ab, next N^2 = d/d Im h_ab (quintic.rs:2306-2308)
 *   monomials   [N x 5]   u32 exponents, lex order with e0 outermost       (quintic.rs:3192)
 *
 * Threading: a solver handle is single-threaded (the reference methods take &mut self).
 * The server handle (cy3q_server_*) is thread-safe.  No function throws or aborts across the
 * ABI; failures return a status and leave a message for cy3q_last_error().
 */
#ifndef CY3Q_H
#define CY3Q_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CY3Q_OK = 0,
  CY3Q_ERR_ARG = 1,          /* bad argument (null pointer, out-of-range value) */
  CY3Q_ERR_SHAPE = 2,        /* size mismatch or size beyond a stated limit */
  CY3Q_ERR_CUDA = 3,         /* CUDA runtime / library error */
  CY3Q_ERR_OOM = 4,          /* device allocation failed or HBM budget exceeded */
  CY3Q_ERR_SINGULAR = 5,     /* T-operator not invertible (the reference silently sets h = I, quintic.rs:1874) */
  CY3Q_ERR_NONFINITE = 6,    /* NaN / Inf in an input or a result */
  CY3Q_ERR_TIMEOUT = 7,      /* deadline passed (server wait, device watchdog) */
  CY3Q_ERR_CANCELLED = 8,    /* request cancelled */
  CY3Q_ERR_UNSUPPORTED = 9,  /* option not supported by this build */
  CY3Q_ERR_NOT_PD = 10,      /* FS Gram matrix not positive-definite (quintic.rs:3148-3149) */
  CY3Q_ERR_EMPTY = 11,       /* no sample points (the reference constructors return None, quintic.rs:204) */
  CY3Q_ERR_MISS = 12,        /* no usable cached metric for the key (metric cache) */
  CY3Q_ERR_STALE = 13        /* cached metric above the sigma quality threshold (MetricCacheError::StaleQuality,
                                route34/metric_cache.rs:75-79) */
} cy3q_status;

typedef enum {
  CY3Q_SAMPLER_NEWTON = 0,   /* SamplerKind::NewtonProjection (quintic.rs:3613) */
  CY3Q_SAMPLER_SZ = 1        /* SamplerKind::ShiffmanZelditch: line intersection (quintic.rs:3633, 3810) */
} cy3q_sampler;

typedef enum {
  CY3Q_PREC_FP64 = 0,        /* FP64 everywhere: the drop-in, parity 1e-10 with the FP64 reference path */
  CY3Q_PREC_FP16X3 = 1,      /* split-precision tcgen05 GEMMs: fp16 hi/lo operands, 3 products, FP32 TMEM
                                accumulation flushed to FP64; FP64 inverse, log-det and reductions */
  CY3Q_PREC_BF16X3 = 2       /* same with bf16 hi/lo operands */
} cy3q_precision;

typedef struct {
  uint32_t k;                /* section degree k (quintic.rs:120) */
  double psi_re, psi_im;     /* psi of f = sum z^5 - 5 psi prod z; the reference takes a real psi (quintic.rs:125) */
  uint64_t n_points;         /* requested sample points */
  uint64_t seed;             /* LCG seed (lib.rs:225) */
  int32_t sampler;           /* cy3q_sampler */
  int32_t fermat_variant;    /* 1: sample_quintic_points_sz (Fermat f, |f|<=1e-3, 4x lines, quintic.rs:3633);
                                0: sample_deformed_quintic_points_sz (psi f, |f|<=1e-2, 8x lines, quintic.rs:3810) */
  int32_t dk_iters;          /* Durand-Kerner sweeps per line (reference: 50, quintic.rs:250) */
  int32_t newton_polish;     /* FP64 Newton steps on each root after Durand-Kerner (0 = reference behaviour) */
  int32_t reduced_basis;     /* 1: drop monomials divisible by z0^5 (ideal-reduced basis, N_6 = 205, N_8 = 460) */
  int32_t precision;         /* cy3q_precision */
  int32_t with_derivs;       /* 1: keep section derivatives resident (needed for sigma / gradient / Laplacian) */
  int32_t device;            /* CUDA device ordinal */
  uint64_t hbm_budget_bytes; /* 0 = no limit; allocations beyond it fail with CY3Q_ERR_OOM */
  double newton_tol;         /* Newton-projection sampler tolerance (quintic.rs:174) */
} cy3q_config;

typedef struct cy3q_solver cy3q_solver;

/* ---- lifecycle: QuinticSolver::new / new_with_psi / new_with_psi_sz / new_with_sampler (quintic.rs:174-322) ---- */
cy3q_status cy3q_config_default(cy3q_config* cfg);
cy3q_status cy3q_solver_create(const cy3q_config* cfg, cy3q_solver** out);
void cy3q_solver_destroy(cy3q_solver* s);
/* Copies the last error message of the handle (or of the calling thread when s == NULL). */
cy3q_status cy3q_last_error(const cy3q_solver* s, char* buf, size_t len);
/* Use a caller-provided CUDA stream (cudaStream_t passed as void*); NULL restores the handle's own stream. */
cy3q_status cy3q_set_stream(cy3q_solver* s, void* cuda_stream);
cy3q_status cy3q_set_precision(cy3q_solver* s, int32_t precision);

/* ---- sample set ---- */
/* GPU line-intersection / Newton sampler + weights + log|Omega|^2 + section tables
   (sample_quintic_points_with quintic.rs:4006, cy_measure_weights quintic.rs:3507,
   finish_workspace_construction quintic.rs:328).  Resets h to identity. */
cy3q_status cy3q_sample(cy3q_solver* s);
/* Install caller points (identical-point parity runs).  w / log_omega may be NULL: then they are
   computed on the device from the points (quintic.rs:3507-3563, 4858). Resets h to identity. */
cy3q_status cy3q_set_points(cy3q_solver* s, const double* points, const double* weights, const double* log_omega,
                            uint64_t n_points);
cy3q_status cy3q_get_points(const cy3q_solver* s, double* points, double* weights, double* log_omega);
cy3q_status cy3q_n_points(const cy3q_solver* s, uint64_t* n);
cy3q_status cy3q_n_basis(const cy3q_solver* s, uint32_t* n);
cy3q_status cy3q_get_basis(const cy3q_solver* s, uint32_t* monomials);
/* Section values s [P x 2N] (evaluate_quintic_basis, quintic.rs:4021) in the current basis. */
cy3q_status cy3q_get_sections(const cy3q_solver* s, double* section_values);

/* ---- balancing: QuinticSolver::orthonormalise_basis_fs_gram / donaldson_step / donaldson_solve ---- */
cy3q_status cy3q_orthonormalise_fs_gram(cy3q_solver* s);                             /* quintic.rs:3140 */
cy3q_status cy3q_donaldson_step(cy3q_solver* s, double* residual);                   /* quintic.rs:428, 1734 */
/* quintic.rs:433; residual_trace may be NULL, else holds max_iter entries. */
cy3q_status cy3q_donaldson_solve(cy3q_solver* s, int32_t max_iter, double tol, int32_t* iters,
                                 double* residual_trace);
cy3q_status cy3q_get_h(const cy3q_solver* s, double* h_block);
cy3q_status cy3q_set_h(cy3q_solver* s, const double* h_block);

/* ---- sigma functional (compute_sigma_from_workspace quintic.rs:1301) ---- */
cy3q_status cy3q_sigma(cy3q_solver* s, double* sigma_l1);
/* Per-point eta (NaN for skipped points) of the last cy3q_sigma call, [P]. */
cy3q_status cy3q_get_eta(const cy3q_solver* s, double* eta);
/* sigma on other points with the current h (C1: fresh points, seed 0); w / log_omega may be NULL. */
cy3q_status cy3q_sigma_on_points(cy3q_solver* s, const double* points, const double* weights,
                                 const double* log_omega, uint64_t n_points, double* sigma_l1);
/* sigma_squared_and_gradient (quintic.rs:2714) / AdamGradientKernel::compute_sigma_grad_h_only
   (gpu_adam.rs:1769): sigma_L2^2, gradient [2N^2] and sigma_L1. */
cy3q_status cy3q_sigma_grad(cy3q_solver* s, double* sigma_l2sq, double* grad, double* sigma_l1);
/* QuinticSolver::sigma_refine_analytic (quintic.rs:453) with optional minibatching: minibatch == 0 or
   >= P uses every point (the reference behaviour); otherwise each step draws `minibatch` points by a
   seeded permutation.  history[steps] receives sigma_L1 before each update; *steps_done the count. */
cy3q_status cy3q_adam_refine(cy3q_solver* s, int32_t steps, double lr, uint64_t minibatch, uint64_t seed,
                             double* history, int32_t* steps_done);
/* QuinticSolver::sigma_refine_lbfgs_gpu_legacy (quintic.rs:678-890; sigma_refine_lbfgs_gpu, quintic.rs:901,
   follows the same trajectory): L-BFGS on [h_re ; h_im] minimising sigma_L2^2 with the analytic gradient,
   m_history pairs, backtracking Armijo search with a steepest-descent fallback, Hermitian projection and
   trace renormalisation of every trial h; the lowest-sigma h is kept.  history (n_iter + 1 entries) receives
   sigma_L1 at the start and after each accepted step; *n_history the count. */
cy3q_status cy3q_lbfgs_refine(cy3q_solver* s, int32_t n_iter, int32_t m_history, double* history,
                              int32_t* n_history);
/* QuinticSolver::sigma_refine_lbfgs_with_restarts_gpu (quintic.rs:1100-1139): one run, then n_restarts runs
   from the best h with a Hermitian uniform(-scale, scale) perturbation drawn from LCG(seed)
   (perturb_h_block_hermitian, quintic.rs:1195-1223).  history (n_restarts + 1 entries) receives sigma after
   each run; *best_sigma the lowest, whose h the handle keeps. */
cy3q_status cy3q_lbfgs_refine_restarts(cy3q_solver* s, int32_t n_restarts, int32_t n_iter, int32_t m_history,
                                       double perturb_scale, uint64_t seed, double* best_sigma, double* history);
/* Failure-detection hook, no reference counterpart: the handle's next split-precision balancing step starves
   its own tensor-core issuer (the point-tile producer skips its first load), so a bounded device wait expires
   after about 2 s, every role of the step's kernels winds down, and the step returns CY3Q_ERR_TIMEOUT with
   the previous h kept.  No fault reaches the GPU and the handle steps normally afterwards.  Needs a
   split-precision handle that has stepped once (CY3Q_ERR_UNSUPPORTED otherwise). */
cy3q_status cy3q_debug_stall_next_step(cy3q_solver* s);

/* ---- checkpoints and run manifest (no reference file format; the reference keeps this state in the public
        fields of QuinticSolver, quintic.rs:117-165) ---- */
/* Versioned checkpoint of the solve: h_block, Adam m, v and step count, and what identifies the problem (k,
   basis, N, psi, seed, point count, precision, FS-Gram transform, FNV-1a hash of the points).  Written to a
   temporary name and renamed, so an interrupted save leaves no partial file. */
cy3q_status cy3q_checkpoint_save(const cy3q_solver* s, const char* path);
/* Restores h_block and the Adam state into a handle holding the same points and basis; CY3Q_ERR_SHAPE when
   the checkpoint belongs to another solve. */
cy3q_status cy3q_checkpoint_load(cy3q_solver* s, const char* path);
/* JSON description of the handle: library version, device, configuration, basis and sample sizes, h version,
   launches, device bytes.  *needed receives the buffer size required (including the terminating zero). */
cy3q_status cy3q_manifest(const cy3q_solver* s, char* buf, size_t len, size_t* needed);

/* ---- Laplacian Galerkin spectrum + Yukawa overlap (templates: route34/metric_laplacian.rs:296-531,
        route34/yukawa_overlap_real.rs:298-372; the reference has no quintic version) ----
   Test functions f_ab = s_a conj(s_b) / (z^H z)^d, s the degree-d monomials (d = 1: 25 functions,
   d = 2: 225), indexed al = a * n_d + b in the monomial order of the basis.  Integration measure
   c_p = w_p eta_p (the volume form of the metric of the current h); points the sigma functional skips
   are left out.  Assembly uses the handle's precision: FP64, or the tensor cores with a 16-bit hi/lo
   split (four products); the per-point metric is always FP64. */
typedef struct {
  uint32_t test_degree;      /* d in f_ab above: 1 or 2 */
  uint32_t n_eigs;           /* lowest eigenvalues returned (by magnitude), 1 .. n_functions */
  double reg;                /* mass-matrix shift reg * |M|_F (metric_laplacian.rs:547-553 uses 1e-10) */
} cy3q_laplacian_config;
/* Lowest n_eigs magnitudes of the eigenvalues of K v = lambda (M + reg |M|_F I) v, ascending (FP64
   generalised Hermitian eigensolve on the device; metric_laplacian.rs:296-392).  eigs [n_eigs]. */
cy3q_status cy3q_laplacian(cy3q_solver* s, const cy3q_laplacian_config* cfg, double* eigs);
/* The assembled mass and stiffness matrices (no reference counterpart; exposes build_mass_matrix /
   build_stiffness_matrix, metric_laplacian.rs:424-531): M = sum c conj(f_al) f_be / sum c,
   K = sum c g^{ab~} conj(d_b f_al) d_a f_be / sum c, row-major n x n complex (interleaved re, im).
   *n_functions receives n; with mass == stiffness == NULL only n is returned. */
cy3q_status cy3q_laplacian_matrices(cy3q_solver* s, const cy3q_laplacian_config* cfg, double* mass,
                                    double* stiffness, uint32_t* n_functions);
/* Y_ijk = sum_p w_p psi_i psi_j psi_k conj(Omega_p) / sum_p w_p (yukawa_overlap_real.rs:298-349) with
   psi_i = sum_al c_{i,al} f_al over the sampler weights w_p; Omega_p = z_chart / (df/dz_elim)
   (quintic.rs:4894-4909).  coeffs [n_modes][n_functions] complex interleaved, n_modes 1..4;
   y [n_modes^3] complex interleaved, index (i n_modes + j) n_modes + k. */
cy3q_status cy3q_yukawa(cy3q_solver* s, const cy3q_laplacian_config* cfg, const double* coeffs, uint32_t n_modes,
                        double* y);

/* ---- grouped balancing: one Donaldson step of many solves of different (psi, k, P) with the same
        launches (no reference counterpart; each member's step is QuinticSolver::donaldson_step,
        quintic.rs:428 / 1734-1894) ----
   The tensor-core kernels of the step are persistent over a work list spanning all members and, with
   the rest of the step, replayed from two CUDA graphs captured once per group (a membership change only
   rewrites the group's tables).  Members are split-precision handles (fp16x3 / bf16x3) with points on
   the group's device; the FP64 Cholesky of each T-operator runs between the two graphs.  A group is
   used by one thread at a time (calls are serialised); its members must not be used elsewhere during a
   call.  Each member's result equals its own cy3q_donaldson_step bit for bit. */
typedef struct cy3q_group cy3q_group;
/* capacity: the largest number of members per step (1 .. 1024) */
cy3q_status cy3q_group_create(int32_t device, uint32_t capacity, cy3q_group** out);
void cy3q_group_destroy(cy3q_group* g);
/* One step of each of solvers[0 .. n): residuals[n] and statuses[n] (cy3q_status per member; a member
   whose step failed keeps its previous h) may be NULL.  Returns the first member failure, or OK. */
cy3q_status cy3q_group_step(cy3q_group* g, cy3q_solver* const* solvers, uint32_t n, double* residuals,
                            int32_t* statuses);

/* ---- serving: continuous batching of balancing solves on one GPU (no reference analogue; nearest is
        the toy crossbeam work queue, src/orchestrator.rs:1-120) ---- */
typedef struct cy3q_server cy3q_server;
typedef struct {
  uint32_t k;
  double psi_re, psi_im;
  uint64_t n_points;
  uint64_t seed;
  int32_t iterations;        /* balancing iterations */
  int32_t precision;         /* cy3q_precision */
  int32_t reduced_basis;
} cy3q_request;
typedef struct {
  cy3q_status status;
  double sigma_l1;           /* sigma after the last iteration (NaN when not requested) */
  double residual;           /* last balancing residual */
  int32_t iterations;
  uint32_t n_basis;
  double submit_ms, start_ms, finish_ms;   /* times on the server clock */
  int32_t cache_hit;         /* 1: h came from the server's metric cache and no iteration ran */
} cy3q_result;
typedef struct {
  uint64_t submitted, completed, failed, cancelled;
  double p50_ms, p99_ms;     /* solve latency (submit -> finish) over completed requests */
  double iters_per_s;        /* aggregate balancing iterations per second since server start */
  uint64_t hbm_in_use, hbm_peak;
} cy3q_server_stats;

/* hbm_budget_bytes: admission limit for the solves in flight (0: 85 % of the free device memory).  The server
   grows the device's default memory pool to the budget at creation, so that its solves allocate from memory
   already mapped; cy3q_server_destroy synchronises the device and trims the pool back. */
cy3q_status cy3q_server_create(int32_t device, uint64_t hbm_budget_bytes, int32_t max_active, cy3q_server** out);
void cy3q_server_destroy(cy3q_server* srv);
cy3q_status cy3q_submit(cy3q_server* srv, const cy3q_request* req, uint64_t* ticket);
cy3q_status cy3q_wait(cy3q_server* srv, uint64_t ticket, int64_t timeout_ms, cy3q_result* out);
cy3q_status cy3q_cancel(cy3q_server* srv, uint64_t ticket);
cy3q_status cy3q_server_stats_get(cy3q_server* srv, cy3q_server_stats* out);
/* h of a completed request, [2N x 2N] in the reference packing. */
cy3q_status cy3q_result_h(cy3q_server* srv, uint64_t ticket, double* h_block);
/* Warm starts from the metric cache (below) under `root`, NULL or "" to turn them off: a submitted request
   whose key (the request's fields with the server's sampler settings, max_iter = iterations, tol = 0) has a
   cached metric completes at once with that h (cache_hit = 1, no device work); every request solved
   afterwards is stored (by a writer thread, without the sample-cloud hash). */
cy3q_status cy3q_server_set_cache(cy3q_server* srv, const char* root);

/* ---- per-stage device timing (tracing; the reference's nearest analogue is
        AdamGradientKernel::compute_sigma_grad_h_only_profiled, gpu_adam.rs:1626-1767) ---- */
typedef enum {
  CY3Q_STAGE_BERGMAN = 0,     /* K_p = s^H h s: GEMM + row dot */
  CY3Q_STAGE_TOPERATOR = 1,   /* T = S^H diag(w/K) S contraction over the points */
  CY3Q_STAGE_TREDUCE = 2,     /* split reduction, /sum w, trace renormalisation */
  CY3Q_STAGE_INVERSE = 3,     /* FP64 Cholesky + inverse of T */
  CY3Q_STAGE_PACK = 4,        /* h_block packing + residual */
  CY3Q_STAGE_SIGMA_GEMM = 5,  /* h applied to s and d s */
  CY3Q_STAGE_SIGMA_POINT = 6, /* per-point metric algebra + reductions */
  CY3Q_STAGE_GRAD = 7,        /* gradient rows + contractions + assembly */
  CY3Q_STAGE_OPERANDS = 8,    /* split-precision operand preparation */
  CY3Q_STAGE_GALERKIN_ROWS = 9,   /* Laplacian test-function rows (mass + stiffness) */
  CY3Q_STAGE_GALERKIN_GRAM = 10,  /* mass / stiffness Gram contractions */
  CY3Q_STAGE_GALERKIN_EIGEN = 11, /* FP64 generalised Hermitian eigensolve */
  CY3Q_STAGE_YUKAWA = 12,         /* Yukawa overlap */
  CY3Q_STAGE_COUNT = 13
} cy3q_stage;
/* Records CUDA events around each stage (no extra synchronisation while enabled). */
cy3q_status cy3q_profile_enable(cy3q_solver* s, int32_t on);
/* Waits for the handle's stream and returns the accumulated device time and call count of a stage. */
cy3q_status cy3q_profile_read(cy3q_solver* s, int32_t stage, double* total_ms, uint64_t* calls, int32_t reset);

/* ---- sigma without device allocation (this entry point has no counterpart in the reference) ----
   For callers that must not have the library allocate device memory (a process that reserved its HBM
   in one arena at start-up, a fixed per-process memory budget on a shared GPU, or a loop in which a
   cudaMalloc / cudaFree -- which may synchronise the whole device -- is not acceptable).  Computes the
   same sigma_L1 and per-point eta as cy3q_sigma (monomial basis, no FS-Gram transform) for the
   h_block given in device memory; all inputs and the eta output are caller-owned DEVICE buffers.
   Intermediates live in one fixed device array inside the library (about 7 MiB, held on every GPU
   that loads the library until exit); its address is looked up by the first call on each device, so
   make that first call before any stream capture.  Calls share that array: calls that overlap on the
   GPU race.  Rejects bases of more than CY3Q_NOALLOC_MAX_BASIS sections with CY3Q_ERR_SHAPE.
   cuda_stream may be NULL (legacy default stream).  The call waits for its stream before returning. */
#define CY3Q_NOALLOC_MAX_BASIS 224
cy3q_status cy3q_sigma_noalloc(int32_t device, uint32_t k, int32_t reduced_basis, double psi_re, double psi_im,
                               const double* d_points, const double* d_weights, const double* d_log_omega,
                               uint64_t n_points, const double* d_h_block, double* d_eta, double* sigma_l1,
                               void* cuda_stream);

/* ---- content-addressed metric cache (route34/metric_cache.rs: ty_cache_path :175-193, load_or_solve_ty
        :247-281, check_sigma_quality :318-340) ----
   A balanced h_block is stored under a cache root in a file named by the key's readable fields and the first
   16 hex digits of the SHA-256 of its canonical text:  quintic_k{k}_n{P}_i{max_iter}_seed{seed}_{hash}.cy3m.
   The file holds the key text (checked on load, so a hash-prefix collision cannot alias), h_block, sigma_L1,
   the last residual, the SHA-256 of the sample cloud (points, weights, log|Omega|^2) and a SHA-256 of the
   whole file; it is written to a temporary name and renamed. */
typedef struct {
  uint32_t k;
  double psi_re, psi_im;
  uint64_t n_points;         /* requested points */
  uint64_t seed;
  int32_t sampler, fermat_variant, dk_iters, newton_polish, reduced_basis, precision;  /* as in cy3q_config */
  int32_t max_iter;          /* iteration cap of the solve */
  double tol;                /* its residual tolerance (0: a fixed iteration count) */
} cy3q_cache_key;
#define CY3Q_SIGMA_QUALITY_THRESHOLD 1.0e-3   /* SIGMA_QUALITY_THRESHOLD, route34/metric_cache.rs:65 */
/* The key of a handle's configuration (TyKeyMaterial, metric_cache.rs:131-142, for the quintic). */
cy3q_status cy3q_cache_key_of(const cy3q_solver* s, int32_t max_iter, double tol, cy3q_cache_key* key);
/* The cache file path of `key` under `root` (ty_cache_path); no device work, no file access. */
cy3q_status cy3q_cache_path(const char* root, const cy3q_cache_key* key, char* path, size_t len);
/* Stores the handle's h_block with sigma_l1 and residual (NaN allowed) and its sample-cloud hash. */
cy3q_status cy3q_cache_store(const char* root, const cy3q_cache_key* key, cy3q_solver* s, double sigma_l1,
                             double residual);
/* Hit: installs the cached h_block in the handle and returns OK with sigma_l1 and residual (either may be
   NULL).  CY3Q_ERR_MISS when there is no file, it is damaged, it belongs to another key or basis size, or the
   handle holds points whose cloud hash differs; with strict != 0, CY3Q_ERR_STALE when the cached sigma is not
   below CY3Q_SIGMA_QUALITY_THRESHOLD (the handle's h is then unchanged). */
cy3q_status cy3q_cache_load(const char* root, const cy3q_cache_key* key, cy3q_solver* s, int32_t strict,
                            double* sigma_l1, double* residual);
/* SHA-256 (FIPS 180-4) of n bytes as 64 hex digits and a terminating zero (hex65 holds 65 bytes). */
cy3q_status cy3q_sha256_hex(const void* data, uint64_t n, char* hex65);

/* ---- build / device information ---- */
const char* cy3q_version(void);
/* Number of this library's kernels launched by the handle since the last reset. */
cy3q_status cy3q_launch_count(const cy3q_solver* s, uint64_t* launches, int32_t reset);

#ifdef __cplusplus
}
#endif
#endif /* CY3Q_H */

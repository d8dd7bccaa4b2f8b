/*
 * cy3q_ty.h -- C ABI of the Tian-Yau metric solve on B200 (sm_100a).
 *
 * Drop-in for the reference's `solve_ty_metric(TyMetricConfig) -> TyMetricResult`
 * (substrate_sm_derivation/cy3_solver/src/route34/ty_metric.rs:461-760, reached through
 * `TianYauSolver::solve_metric`, src/route34/cy3_metric_unified.rs:232-270) and the pieces it is made
 * of.  The variety is the Z/3 quotient of the complete intersection
 *     f1 = sum z_i^3,  f2 = sum w_i^3,  f3 = sum z_i w_i   in CP^3 x CP^3
 * (`BicubicPair::z3_invariant_default`, src/cicy_sampler.rs:236-283).
 *
 * Layouts (reference conventions):
 *   coords   [P x 16] f64, (re, im) of z_0..z_3, w_0..w_3, each factor divided by its largest coordinate
 *                      (`SampledPoint` / `TyPoint`, cicy_sampler.rs:352-362, ty_metric.rs:478-490)
 *   omega_sq [P]      f64, |Omega|^2 with Omega = 1 / det J_elim (cicy_sampler.rs:488-500)
 *   weight   [P]      f64, |Omega|^2 / det g_pb normalised to sum 1, divided by 3 for the quotient
 *   basis    [N x 8]  int exponents of the Z/3-invariant, ideal-reduced (k, k) monomials (ty_metric.rs:870-888)
 *   h_re, h_im [N x N] f64 row-major: the upper-index metric G = h_re + i h_im of ty_metric.rs:404-424
 *
 * Host memory in and out, device state owned by the handle; status codes of cy3q.h; one thread per handle.
 * A handle holds one complete-intersection solve: Tian-Yau (cy3q_ty_create) or Schoen (cy3q_schoen_create,
 * at the end of this header).
 */
#ifndef CY3Q_TY_H
#define CY3Q_TY_H

#include "cy3q.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cy3q_ty cy3q_ty;

typedef struct {
  int k_degree;           /* bidegree (k, k) of the section basis (TyMetricConfig::k_degree) */
  long long n_sample;     /* points requested (TyMetricConfig::n_sample) */
  int max_iter;           /* Donaldson iteration cap (TyMetricConfig::max_iter) */
  double donaldson_tol;   /* stop once the residual is below (TyMetricConfig::donaldson_tol) */
  uint64_t seed;          /* ChaCha8Rng::seed_from_u64 seed of the sampler (TyMetricConfig::seed) */
  int apply_z3_quotient;  /* divide the weights by 3 (TyMetricConfig::apply_z3_quotient) */
  double damping;         /* <= 0: the reference's rule (static 1 for k < 4, adaptive 0.3 / 0.05 / 1.0 for
                             k >= 4, ty_metric.rs:247-264); otherwise a static alpha in (0, 1] */
  int sigma_every_iter;   /* 1: sigma after every iteration, as the reference's loop does (ty_metric.rs:686) */
  int device;             /* CUDA device ordinal */
  const char* checkpoint_path;  /* NULL, or a file rewritten after every iteration of cy3q_ty_solve in the
                                   reference's checkpoint JSON (write_checkpoint, ty_metric.rs:2603-2656:
                                   n_basis, iterations, h_re, h_im, donaldson_history, sigma_history; values
                                   as Rust's {:.17e}; temporary file renamed into place) */
} cy3q_ty_config;

typedef struct {
  long long n_points;
  int n_basis;
  int iterations_run;
  double sigma_fs_identity;         /* sigma at h = I before the first iteration (ty_metric.rs:557) */
  double sigma_final;               /* sigma after the last iteration (final_sigma_residual) */
  double final_donaldson_residual;  /* ||h_new - h_old||_F of the last iteration */
} cy3q_ty_result;

/* TyMetricConfig::default() with the Cy3MetricSpec::TianYau overrides (cy3_metric_unified.rs:249-261). */
cy3q_status cy3q_ty_config_default(cy3q_ty_config* cfg);
/* build_ty_invariant_reduced_basis (ty_metric.rs:870): writes min(cap, N) rows of 8 exponents, N to *n.
   The reduced Groebner basis of (f1, f2, f3) in the deg-lex order z0 > .. > z3 > w0 > .. > w3
   (ty_metric.rs:840-852, groebner.rs:470-656) is computed by the library. */
cy3q_status cy3q_ty_basis(int k, int* n, int* exps, int cap);
cy3q_status cy3q_ty_create(const cy3q_ty_config* cfg, cy3q_ty** out);
void cy3q_ty_destroy(cy3q_ty* t);
cy3q_status cy3q_ty_last_error(const cy3q_ty* t, char* buf, size_t len);
/* CicySampler::sample_batch + apply_z3_quotient (cicy_sampler.rs:600-763) on the device: the line inputs of
   the ChaCha8 / StandardNormal stream in the order sample_batch_gpu draws them (max(4n, 64) lines of one
   Newton attempt each, cicy_sampler.rs:640-740), the Newton steps of newton_solve_line (:771-850), the patch
   rescale, residue and weight of post_process_solved_point (:452-590), the first n accepted lines in order. */
cy3q_status cy3q_ty_sample(cy3q_ty* t, long long* n_out);
/* Caller-supplied points (e.g. the reference's own cloud): rescaled coords, |Omega|^2, weights. */
cy3q_status cy3q_ty_set_points(cy3q_ty* t, const double* coords, const double* omega_sq, const double* weight,
                               long long P);
cy3q_status cy3q_ty_get_points(cy3q_ty* t, double* coords, double* omega_sq, double* weight, long long cap,
                               long long* P);
cy3q_status cy3q_ty_n_basis(const cy3q_ty* t, int* n);
cy3q_status cy3q_ty_set_h(cy3q_ty* t, const double* h_re, const double* h_im);
cy3q_status cy3q_ty_get_h(cy3q_ty* t, double* h_re, double* h_im);
/* donaldson_iteration (ty_metric.rs:1062-1370) with damping alpha; h kept on CY3Q_ERR_SINGULAR. */
cy3q_status cy3q_ty_donaldson_step(cy3q_ty* t, double alpha, double* residual);
/* compute_sigma (ty_metric.rs:1402-1468); eta may be NULL, else cap >= P values (NaN where invalid). */
cy3q_status cy3q_ty_sigma(cy3q_ty* t, double* sigma, double* eta, long long cap);
/* The balancing loop of solve_ty_metric (ty_metric.rs:555-720) from h = I on the handle's points:
   damping rule, min-residual snapshot and catastrophe guard, tolerance stop.  Histories (sigma and
   residual per iteration) are written up to hist_cap entries each (may be NULL). */
cy3q_status cy3q_ty_solve(cy3q_ty* t, cy3q_ty_result* out, double* sigma_hist, double* res_hist, int hist_cap);
/* Kernel launches made by the handle so far. */
cy3q_status cy3q_ty_launch_count(const cy3q_ty* t, uint64_t* n);
/* adam_refine_sigma_ty (ty_metric.rs:1488-1583; AdamRefineConfig of schoen_metric.rs:115-136): Adam on
   sigma^2 with the finite-difference gradient over the 2 N^2 real parameters of h (step fd_step), from the
   handle's h, updated in place.  All N^2 perturbed sigmas of a step are evaluated in one pass (each form is
   linear in h; the frames do not depend on it).  hist gets the sigma history (the value before each step and
   after the last), *n_hist its length. */
cy3q_status cy3q_ty_adam_refine(cy3q_ty* t, int max_iters, double lr, double fd_step, double tol, double* hist,
                                int cap, int* n_hist);
/* Seed of the next cy3q_ty_sample (the handle, its device buffers and the sampler's scratch are reused, as a
   per-seed loop over one configuration does). */
cy3q_status cy3q_ty_set_seed(cy3q_ty* t, uint64_t seed);

/*
 * Schoen: the Z/3 x Z/3 quotient of the complete intersection in CP^2 x CP^2 x CP^1 with coordinates
 * x_0..x_2, y_0..y_2, t_0, t_1 (the coords layout above in this order),
 *     F1 = (x0^3 + x1^3 + x2^3) t0 + x0 x1 x2 t1,   F2 = (y0^3 + y1^3 + y2^3) t1 + y0 y1 y2 t0
 * (`SchoenPoly::z3xz3_invariant_default`, src/route34/schoen_sampler.rs:188-216), solved by
 * `solve_schoen_metric` (src/route34/schoen_metric.rs:766-1000) through the same handle type and entry points
 * (cy3q_ty_sample, _set_points, _donaldson_step, _sigma, _solve, _get_h ...).  The sampler draws one Newton
 * attempt per line (origin, two directions, t: 52 draws) and keeps the first n accepted lines; the weights are
 * normalised by the inverse of their sum and multiplied by 1/9 (schoen_sampler.rs:555-560, 1177-1185).
 */
typedef struct {
  int d_x, d_y, d_t;          /* tri-degree of the section basis (SchoenMetricConfig::d_x, d_y, d_t) */
  long long n_sample;
  int max_iter;
  double donaldson_tol;
  uint64_t seed;
  int apply_z3xz3_quotient;   /* divide the weights by 9 (SchoenMetricConfig::apply_z3xz3_quotient) */
  double damping;             /* <= 0: the reference's rule (static 1, adaptive when d_x + d_y + d_t >= 10,
                                 schoen_metric.rs:649-665); otherwise a static alpha */
  int sigma_every_iter;
  int device;
  const char* checkpoint_path;  /* as in cy3q_ty_config (schoen_metric.rs:1035-1037) */
} cy3q_schoen_config;

/* SchoenMetricConfig defaults with the Cy3MetricSpec::Schoen overrides (cy3_metric_unified.rs:289-320). */
cy3q_status cy3q_schoen_config_default(cy3q_schoen_config* cfg);
/* build_schoen_invariant_reduced_basis (schoen_metric.rs:1185): Gamma-invariant tri-degree monomials not in
   the leading-monomial ideal of the reduced deg-lex Groebner basis of schoen_generators (groebner.rs:705). */
cy3q_status cy3q_schoen_basis(int d_x, int d_y, int d_t, int* n, int* exps, int cap);
cy3q_status cy3q_schoen_create(const cy3q_schoen_config* cfg, cy3q_ty** out);

/*
 * Metric cache for both geometries (route34/metric_cache.rs, load_or_solve_ty / load_or_solve_schoen :242-310).
 * The file name is the reference's: ty_k{k}_n{n}_i{max_iter}_seed{seed}_{h} or
 * schoen_dx{..}_dy{..}_dt{..}_n{n}_i{max_iter}_seed{seed}_{h}, h = the first 16 hex digits of SHA-256 of the
 * reference's key JSON (TyKeyMaterial / SchoenKeyMaterial, metric_cache.rs:131-226), with the library's own
 * payload format (extension .cy3m: key JSON, basis size, sigma, residual, the SHA-256 of the sample cloud as
 * sha256_points computes it, h_re and h_im, a checksum), written under a temporary name and renamed.
 * Loading checks the key, the basis size, the checksum and, when the handle holds points, the cloud hash
 * (CY3Q_ERR_MISS otherwise); strict mode refuses sigma >= CY3Q_SIGMA_QUALITY_THRESHOLD (CY3Q_ERR_STALE).
 */
cy3q_status cy3q_ty_cache_file(const cy3q_ty_config* cfg, const char* root, char* path, size_t len);
cy3q_status cy3q_schoen_cache_file(const cy3q_schoen_config* cfg, const char* root, char* path, size_t len);
/* sha256_points (ty_metric.rs:2569, schoen_metric.rs:2630) of the handle's points, 64 hex digits + NUL. */
cy3q_status cy3q_ty_cloud_sha256(cy3q_ty* t, char* hex65);
cy3q_status cy3q_ty_cache_store(cy3q_ty* t, const char* root, double sigma_final, double residual);
cy3q_status cy3q_ty_cache_load(cy3q_ty* t, const char* root, int strict, double* sigma_final, double* residual);

#ifdef __cplusplus
}
#endif

#endif /* CY3Q_TY_H */

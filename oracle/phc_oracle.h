/*
 * phc_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C interface of the CPU restatement of polyhomocont's solve() path
 * (src/random.f90, src/linalg.f90, src/sparse.f90, src/homotopy.f90,
 * src/tracker.f90, src/endgame.f90, src/solve.f90 of the reference).
 * It is the checker for the CUDA path and the timed CPU baseline; the
 * product library never includes, links or calls it.
 *
 * Parity pin: the reference (Fortran 2008) cannot be compiled in this
 * environment (no Fortran compiler). The restatement is pinned against
 * the reference's own known-answer tests (test/*.f90) and against the
 * Katsura golden vectors produced by the reference's Python script
 * (reference/ref_katsura.py), re-expressed as pytest cases under tests/.
 *
 * Conventions: complex numbers are interleaved (re, im) doubles, like
 * Fortran complex(real64); matrices are column-major; indices exposed
 * through this interface are 0-based unless stated otherwise.
 */
#ifndef PHC_ORACLE_H
#define PHC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* tracker_options, src/tracker.f90:56-77 */
typedef struct {
  double step_init;
  double step_max;
  double step_min;
  double corrector_tol;
  int32_t corrector_maxit;
  int32_t grow_after;
  double contraction;
  int32_t max_steps;
  int32_t pad_;
} orc_tracker_options;

/* endgame_options, src/endgame.f90:73-101 */
typedef struct {
  double t_start;
  double radius_factor;
  double radius_min;
  double loop_radius;
  double winding_agreement;
  double tol;
  double residual_tol;
  double closure_factor;
  int32_t nsamples;
  int32_t max_winding;
} orc_endgame_options;

/* solve_options, src/solve.f90:57-84 */
typedef struct {
  orc_tracker_options tracker;
  orc_endgame_options endgame;
  int32_t use_endgame;
  int32_t seed;
  int32_t refine_maxit;
  int32_t pad_;
  double infinity_tol;
  double singular_cond;
  double real_tol;
  double dedup_tol;
  double singular_dedup_tol;
} orc_solve_options;

/* path_info, src/tracker.f90:95-110 */
typedef struct {
  int32_t status;
  int32_t naccepted;
  int32_t nrejected;
  int32_t pad_;
  double s;
  double t_re;
  double t_im;
  double step;
} orc_path_info;

/* endgame_result, src/endgame.f90:103-120 (z returned separately) */
typedef struct {
  int32_t status;
  int32_t winding_number;
  int32_t naccepted;
  int32_t nrejected;
  double error;
  double residual;
  double radius;
} orc_endgame_result;

/* path_result, src/solve.f90:86-119 (z, x returned separately).
 * Same field layout as phc_path_out of the product interface. The unit
 * counters are not in the reference; they count evaluate+LU(+solve)
 * units for the flop model. solution_index/singular_index are 1-based
 * like the reference (0 = none). */
typedef struct {
  int32_t status;
  int32_t winding_number;
  int32_t endgame_status;
  int32_t at_infinity;
  int32_t singular;
  int32_t is_real;
  int32_t naccepted;
  int32_t nrejected;
  int32_t solution_index;
  int32_t singular_index;
  int32_t n_tangent;   /* predictor units (evaluate + LU + solve)   */
  int32_t n_newton;    /* corrector units (evaluate + LU + solve)   */
  int32_t n_refine;    /* refine units (evaluate + LU + solve)      */
  int32_t n_eval;      /* evaluate-only units (backward error, ...) */
  int32_t n_cond;      /* cond1 calls (LU + N solves)               */
  int32_t n_fp64_retry;/* mixed mode only; always 0 here            */
  double t;
  double endgame_error;
  double cond;
  double residual;
} orc_path_out;

/* Aggregate counts of solve_result, src/solve.f90:121-150 */
typedef struct {
  int32_t n;
  int32_t npaths;
  int32_t nsolutions;
  int32_t nreal;
  int32_t nsingular;
  int32_t ninfinite;
  int32_t nfailed;
  int32_t nduplicates;
} orc_solve_counts;

void orc_default_solve_options(orc_solve_options* o);

/* ---- random.f90 ---- */
void* orc_rng_new(void);
void orc_rng_free(void* g);
void orc_rng_seed(void* g, int32_t seed);
double orc_rng_uniform(void* g);
void orc_rng_unit_complex(void* g, double* z);
void orc_rng_normal_complex(void* g, double* z);

/* ---- linalg.f90 (ipiv 1-based, as the reference) ---- */
int32_t orc_lu_factor(int32_t n, double* a, int32_t* ipiv);
void orc_lu_solve(int32_t n, const double* a, const int32_t* ipiv, double* b);
int32_t orc_solve_linear(int32_t n, const double* a, const double* b, double* x);
double orc_cond1(int32_t n, const double* a);
double orc_norm_inf(int32_t n, const double* z);

/* ---- sparse.f90 ---- */
void* orc_sparse_new(void);
void orc_sparse_free(void* s);
void orc_sparse_init(void* s, int32_t n);
/* exps: rows x cols column-major (the Fortran exponent matrix) */
int32_t orc_sparse_add_equation(void* s, int32_t ncoefs, const double* coefs,
                                int32_t rows, int32_t cols, const int32_t* exps);
int32_t orc_sparse_nvars(void* s);
int32_t orc_sparse_nequations(void* s);
int32_t orc_sparse_nterms(void* s, int32_t i); /* i 1-based */
int32_t orc_sparse_total_terms(void* s);
int32_t orc_sparse_maxexp(void* s);
void orc_sparse_degrees(void* s, int32_t* d);
/* packed table: first[neq+1] 0-based, hexps[(n+1)*T], coefs[2T] */
void orc_sparse_table(void* s, int32_t* first, int32_t* hexps, double* coefs);
void orc_sparse_evaluate(void* s, const double* x, double* f, double* jac);
void orc_sparse_evaluate_homogeneous(void* s, const double* z, double* f,
                                     double* jac);
/* A user system (class(poly_system), src/system.f90:27-67): evaluate(x, f,
 * jac) as a callback (x, f interleaved complex [n]; jac n x n column-major),
 * exact degrees[n]. The object then evaluates F^h by the reference's default
 * homogenization (src/system.f90:71-119) and solves like any system. */
typedef int32_t (*orc_user_evaluator)(void* ctx, int32_t n, const double* x, double* f,
                                      double* jac);
void orc_sparse_set_user(void* s, int32_t n, const int32_t* degrees, orc_user_evaluator fn,
                         void* ctx);

/* ---- homotopy.f90 ---- */
void* orc_hom_new(void);
void orc_hom_free(void* h);
int32_t orc_hom_init(void* h, void* sys, void* gen);
int32_t orc_hom_nstart(void* h);
void orc_hom_constants(void* h, double* gamma, double* b, double* patch);
void orc_hom_start_solution(void* h, int32_t k, double* z); /* k 1-based */
void orc_hom_evaluate(void* h, const double* z, const double* t, double* hv,
                      double* hz, double* ht);

/* ---- tracker.f90 ---- */
void orc_track_path(void* h, double* z, double t_start, double t_end,
                    const orc_tracker_options* o, orc_path_info* info);
void orc_track_line(void* h, double* z, const double* t0, const double* t1,
                    const orc_tracker_options* o, orc_path_info* info);
void orc_track_arc(void* h, double* z, double radius, double theta0,
                   double dtheta, const orc_tracker_options* o,
                   orc_path_info* info);

/* ---- endgame.f90 ---- */
void orc_cauchy_endgame(void* h, double* z, const orc_endgame_options* eo,
                        const orc_tracker_options* to, orc_endgame_result* r,
                        double* zres);

/* ---- solve.f90 ----
 * orc_solve_paths: per-path numerics (start_solution, endpoint,
 * classify) for 1-based paths [k0, k0+count) with nthreads host
 * threads; z_out[count*(n+1)], x_out[count*n] (zero where not finite).
 * orc_solve: the whole solve() including the order-dependent host
 * bookkeeping; per-path arrays sized npaths = Bezout number (query
 * with orc_bezout); sols/ssols sized n*npaths, realsols n*npaths,
 * mult npaths. Returns the solve status. */
int64_t orc_bezout(void* sys);
int32_t orc_solve_paths(void* sys, const orc_solve_options* o, int64_t k0,
                        int64_t count, int32_t nthreads, orc_path_out* paths,
                        double* z_out, double* x_out);
int32_t orc_solve(void* sys, const orc_solve_options* o, int32_t nthreads,
                  orc_path_out* paths, double* z_out, double* x_out,
                  orc_solve_counts* counts, double* sols, double* realsols,
                  double* ssols, int32_t* mult);

#ifdef __cplusplus
}
#endif

#endif

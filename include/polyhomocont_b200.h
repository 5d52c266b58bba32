/*
 * polyhomocont_b200.h -- C ABI of the B200 path tracker for polyhomocont.
 *
 * Drop-in for the per-path work behind polyhomocont's
 *   subroutine solve(sys, res, status, options)       src/solve.f90:154-215
 * on type(sparse_system) inputs (src/sparse.f90:31-61). The Fortran side
 * keeps its API; a bind(C) interface module on the Fortran side packs the
 * sparse table and calls phc_solve_sparse, which:
 *   - seeds the reference generator and draws gamma, b, patch exactly as
 *     hom%init (src/homotopy.f90:104-149);
 *   - runs start_solution + endpoint + classify for every path on the GPU
 *     (src/solve.f90:190-198, :217-328), one warp per path;
 *   - runs the order-dependent bookkeeping (add_solution, add_singular,
 *     find, collect_real; src/solve.f90:330-426) on the host in path order,
 *     path by path as the GPU finishes them (the kernel writes its results
 *     into page-locked host memory that the library keeps per device).
 *
 * Conventions (all entry points):
 *   - plain C types; complex values are interleaved (re, im) doubles, like
 *     Fortran complex(real64); matrices column-major;
 *   - the caller owns every input and output array; the library owns
 *     device memory, streams and server objects;
 *   - return codes: 0 ok; 1..3 mirror src/config.f90:16-23
 *     (err_invalid_input, err_singular_matrix, err_numerical); negative
 *     codes are device/runtime errors (PHC_ERR_*). Per-path failures are
 *     reported in the path records, never as a return code, as in the
 *     reference.
 *   - N = n + 1 unknowns (projective coordinates, w last) must be <= 32.
 */
#ifndef POLYHOMOCONT_B200_H
#define POLYHOMOCONT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PHC_OK 0
#define PHC_ERR_INVALID_INPUT 1   /* err_invalid_input,   src/config.f90:17 */
#define PHC_ERR_SINGULAR_MATRIX 2 /* err_singular_matrix, src/config.f90:19 */
#define PHC_ERR_NUMERICAL 3       /* err_numerical,       src/config.f90:21 */
#define PHC_ERR_CUDA (-1)         /* a CUDA runtime call failed */
#define PHC_ERR_UNSUPPORTED (-2)  /* N > 32 or a table too large for a block */
#define PHC_ERR_NO_DEVICE (-3)    /* no CUDA device / extension unusable */
#define PHC_ERR_OOM (-4)          /* device allocation failed */
#define PHC_ERR_ADMISSION (-5)    /* server: request larger than its budget */
#define PHC_ERR_DEADLINE (-6)     /* server: deadline passed before done */
#define PHC_ERR_ABORTED (-7)      /* server shut down / request cancelled */
#define PHC_ERR_BAD_HANDLE (-8)   /* unknown ticket or null handle */
#define PHC_ERR_NOT_READY (-9)    /* server: result not available yet */

/* path status (res%paths(k)%status), src/tracker.f90:46-51, src/solve.f90:53 */
#define PHC_PATH_SUCCESS 0
#define PHC_PATH_FAILED_MIN_STEP 1
#define PHC_PATH_FAILED_MAX_STEPS 2
#define PHC_PATH_ENDGAME_FAILED 3
/* end game status, src/endgame.f90:65-70 */
#define PHC_ENDGAME_CONVERGED 0
#define PHC_ENDGAME_NOT_CONVERGED 1
#define PHC_ENDGAME_FAILED 2

#define PHC_MAX_UNKNOWNS 32

/* ---- options: POD mirrors of the reference's derived types ------------- */
/* type(tracker_options), src/tracker.f90:56-77 */
typedef struct {
  double step_init;       /* 0.05   */
  double step_max;        /* 0.1    */
  double step_min;        /* 1e-14  */
  double corrector_tol;   /* 1e-10  */
  int32_t corrector_maxit;/* 3      */
  int32_t grow_after;     /* 5      */
  double contraction;     /* 0.5    */
  int32_t max_steps;      /* 20000  */
  int32_t pad_;
} phc_tracker_options;

/* type(endgame_options), src/endgame.f90:73-101 */
typedef struct {
  double t_start;           /* 0.1    */
  double radius_factor;     /* 0.25   */
  double radius_min;        /* 1e-13  */
  double loop_radius;       /* 1e-5   */
  double winding_agreement; /* 0.2    */
  double tol;               /* 1e-11  */
  double residual_tol;      /* 1e-8   */
  double closure_factor;    /* 0.1    */
  int32_t nsamples;         /* 8      */
  int32_t max_winding;      /* 16     */
} phc_endgame_options;

/* type(solve_options), src/solve.f90:57-84 */
typedef struct {
  phc_tracker_options tracker;
  phc_endgame_options endgame;
  int32_t use_endgame;      /* .true. */
  int32_t seed;             /* 1      */
  int32_t refine_maxit;     /* 5      */
  int32_t pad_;
  double infinity_tol;      /* 1e-8   */
  double singular_cond;     /* 1e10   */
  double real_tol;          /* 1e-8   */
  double dedup_tol;         /* 1e-8   */
  double singular_dedup_tol;/* 1e-6   */
} phc_solve_options;

/* GPU-only knobs, kept out of phc_solve_options so that it stays a POD
 * mirror of solve_options. A NULL pointer means all defaults. */
#define PHC_PREC_FP64 0  /* all-FP64 tracker */
#define PHC_PREC_MIXED 1 /* complex FP32 eliminations for the predictor and the
                            corrector (and an FP32 evaluation of the predictor
                            for n <= 7); FP64 evaluation, residual, update,
                            norms, end game decisions, refine, cond1 */
#define PHC_SCHED_GRID 0       /* one warp per path, one launch, no refill */
#define PHC_SCHED_PERSISTENT 1 /* persistent warps, atomic path queue refill */
typedef struct {
  int32_t precision;       /* PHC_PREC_*                               */
  int32_t schedule;        /* PHC_SCHED_*                              */
  int32_t device;          /* CUDA device ordinal                      */
  int32_t warps_per_block; /* 0 = the value phc_autotune chose for this
                              device, precision, schedule and row width,
                              else 4                                    */
  int32_t blocks_per_sm;   /* persistent grid: 0 = max resident        */
  int32_t chunk;           /* persistent refill granularity (paths), 0 = the
                              tuned value, else 1                        */
  int32_t fp64_sticky;     /* mixed: FP64 steps after an FP32 failure, -1 = default */
  int32_t unit_budget_log2; /* per-path safety budget of 2^k units (evaluations
                               with eliminations); a path that exhausts it ends
                               with PHC_PATH_FAILED_MAX_STEPS. 0 = 2^24, far
                               above any path tracked in practice; at most 40 */
} phc_gpu_options;

/* ---- per-path record: fields of type(path_result), src/solve.f90:86-119 -- */
/* z (N complex) and x (n complex, zero if at infinity or failed) are
 * returned in separate arrays. solution_index and singular_index are
 * 1-based like the reference (0 = none). The n_* counters are not in the
 * reference: they count executed units for the flop model. */
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
  int32_t n_tangent;    /* predictor units: evaluate + LU + solve         */
  int32_t n_newton;     /* corrector units: evaluate + LU + solve         */
  int32_t n_refine;     /* refine units: evaluate + LU + solve            */
  int32_t n_eval;       /* evaluate-only units (backward error, classify) */
  int32_t n_cond;       /* cond1: LU + N solves                           */
  int32_t n_fp64_retry; /* mixed: predictor/corrector units run in FP64   */
  double t;
  double endgame_error;
  double cond;
  double residual;
} phc_path_out;

/* aggregate counts of type(solve_result), src/solve.f90:121-150 */
typedef struct {
  int32_t n;
  int32_t npaths;
  int32_t nsolutions;
  int32_t nreal;
  int32_t nsingular;
  int32_t ninfinite;
  int32_t nfailed;
  int32_t nduplicates;
} phc_solve_counts;

/* caller-allocated result arrays of one solve; capacities in rows of n:
 * paths/z/x hold npaths rows, solutions/singular_solutions/real_solutions
 * and multiplicities at most npaths rows (the Bezout number). */
typedef struct {
  phc_solve_counts counts;
  phc_path_out* paths;          /* [npaths]                         */
  double* z;                    /* [npaths][n+1][2]                 */
  double* x;                    /* [npaths][n][2]                   */
  double* solutions;            /* [npaths][n][2]  (rows used: nsolutions) */
  double* real_solutions;       /* [npaths][n]     (rows used: nreal)      */
  double* singular_solutions;   /* [npaths][n][2]  (rows used: nsingular)  */
  int32_t* multiplicities;      /* [npaths]        (used: nsingular)       */
} phc_solve_result;

/* ---- packed sparse table: the private components of type(sparse_system)
 * (src/sparse.f90:31-48) as the Fortran wrapper passes them ------------- */
typedef struct {
  int32_t n;               /* variables = equations                        */
  int32_t nterms;          /* total number of (nonzero) terms              */
  const int32_t* first;    /* [n+1] 0-based term offsets per equation      */
  const int32_t* deg;      /* [n] total degrees d_i                         */
  const int32_t* hexps;    /* [nterms][n+1] homogenized exponents, w last   */
  const double* coefs;     /* [nterms][2]                                   */
} phc_system;

/* the random constants of type(total_degree_homotopy), src/homotopy.f90:45-68 */
typedef struct {
  double gamma[2];
  const double* b;         /* [n][2]   */
  const double* patch;     /* [n+1][2] */
} phc_homotopy;

/* ---- type(sparse_system) builder (src/sparse.f90:65-195) --------------- */
typedef struct phc_sparse phc_sparse;
phc_sparse* phc_sparse_create(void);
void phc_sparse_destroy(phc_sparse* s);
/* sys%init(n), src/sparse.f90:65-81 */
int32_t phc_sparse_init(phc_sparse* s, int32_t n);
/* sys%add_equation(coefs, exps, status), src/sparse.f90:83-141; exps is the
 * rows x cols column-major exponent matrix; returns the status */
int32_t phc_sparse_add_equation(phc_sparse* s, int32_t ncoefs, const double* coefs,
                                int32_t rows, int32_t cols, const int32_t* exps);
int32_t phc_sparse_nvars(const phc_sparse* s);       /* :177-184 */
int32_t phc_sparse_nequations(const phc_sparse* s);  /* :156-164 */
int32_t phc_sparse_nterms(const phc_sparse* s, int32_t i); /* :166-175, i 1-based */
int32_t phc_sparse_total_terms(const phc_sparse* s);
void phc_sparse_degrees(const phc_sparse* s, int32_t* d);  /* :186-195 */
/* view of the packed table; valid until the builder changes */
int32_t phc_sparse_table(const phc_sparse* s, phc_system* out);
/* sys%evaluate(x, f, jac), src/sparse.f90:197-207, on the host: x[2n] and
 * f[2n] interleaved complex, jac[2 n n] with dF_i/dx_j at complex index
 * i + j*n (column-major, Fortran's layout) */
int32_t phc_sparse_evaluate(const phc_sparse* s, const double* x, double* f, double* jac);
/* sys%evaluate_homogeneous(z, f, jac), src/sparse.f90:209-221: z[2(n+1)]
 * with w = z_(n+1) last, f[2n], jac[2 n (n+1)]; exact also at w = 0 */
int32_t phc_sparse_evaluate_homogeneous(const phc_sparse* s, const double* z, double* f,
                                        double* jac);

/* ---- user-evaluator systems (class(poly_system), src/system.f90:27-67) -- */
/* sys%evaluate(x, f, jac): x[2n], f[2n] interleaved complex; jac[2 n n] is
 * the n x n Jacobian column-major, jac(i, j) = dF_i/dx_j at complex index
 * i + j*n (Fortran's layout). Returns 0, or nonzero to abort sampling. */
typedef int32_t (*phc_evaluator)(void* ctx, int32_t n, const double* x, double* f,
                                 double* jac);
/* Replaces the builder's content (sys%init(n) + n add_equation calls) with
 * the sparse table of the polynomial system that eval computes, whose
 * equation i has the exact total degree degrees[i]: F is sampled at
 * 2 C(n+d, d) generic points per degree d and interpolated by least
 * squares, and the table is checked against F and the Jacobian at fresh
 * points (worst relative error in *max_error, may be NULL). Returns
 * err_invalid_input when eval is not a polynomial of those degrees or its
 * Jacobian disagrees, PHC_ERR_UNSUPPORTED above 1500 monomials of degree
 * <= d_i, PHC_ERR_ABORTED when eval returned nonzero. */
int32_t phc_sparse_sample(phc_sparse* s, int32_t n, const int32_t* degrees, phc_evaluator eval,
                          void* ctx, int32_t seed, double* max_error);

/* ---- homotopy set-up: gen%seed(seed); hom%init(sys, gen, status) ------- */
/* src/random.f90:43-62, src/homotopy.f90:104-149. gamma[2], b[2n],
 * patch[2(n+1)] are caller-allocated; nstart = Bezout number. */
int32_t phc_homotopy_init(const phc_system* sys, int32_t seed, double* gamma,
                          double* b, double* patch, int64_t* nstart);

void phc_default_solve_options(phc_solve_options* o);
void phc_default_gpu_options(phc_gpu_options* g);

/* ---- the drop-in: solve(sys, res, status, options) ---------------------- */
/* Bezout number of the system (0 if the system is invalid) */
int64_t phc_bezout(const phc_system* sys);
/* Whole solve: host set-up, GPU path numerics, host bookkeeping. Arrays in
 * *res are caller-allocated with capacity phc_bezout(sys) rows. opts or
 * gpu may be NULL (defaults). Returns the solve status. The bookkeeping of
 * each path runs on the calling thread while later paths are tracked;
 * calls on one device are serialized. */
int32_t phc_solve_sparse(const phc_system* sys, const phc_solve_options* opts,
                         const phc_gpu_options* gpu, phc_solve_result* res);

/* The host half of solve() on per-path records produced elsewhere (e.g. by
 * several GPUs on contiguous path ranges, gathered in path order):
 * add_solution / add_singular / find / collect_real, src/solve.f90:193-213,
 * :330-426. paths[npaths] gets its solution/singular indices; res arrays as
 * for phc_solve_sparse (res->paths/z/x are not touched). */
int32_t phc_finish_solve(int32_t n, int64_t npaths, const phc_solve_options* opts,
                         phc_path_out* paths, const double* x, phc_solve_result* res);

/* Per-path numerics only (start_solution + endpoint + classify) for the
 * 1-based paths k0 .. k0+count-1 of the homotopy hom; host buffers:
 * out[count], z_out[count][n+1][2], x_out[count][n][2] (x may be NULL). */
int32_t phc_solve_paths(const phc_system* sys, const phc_homotopy* hom,
                        const phc_solve_options* opts, const phc_gpu_options* gpu,
                        int64_t k0, int64_t count, phc_path_out* out,
                        double* z_out, double* x_out);

/* Per-path numerics without any device allocation. No counterpart in the
 * reference. For callers that cannot call cudaMalloc -- services whose
 * device memory is reserved and accounted for up front, and hosts that
 * forbid device allocations after start-up because an allocation can block
 * or fail at an unpredictable moment. The caller passes the host table and
 * constants and its own device output buffers (d_out[count],
 * d_z[count][n+1][2], d_x[count][n][2] or NULL); the compiled table and the
 * path-queue counter go into one fixed 256 KiB array in device memory that
 * every GPU loading the library holds until exit. Tables larger than that
 * are rejected with PHC_ERR_UNSUPPORTED. The call only enqueues work on
 * `stream`; it calls no cudaMalloc, cudaFree or other allocating routine.
 * Its first call on a device looks up the array's address on that device
 * and caches it (make that first call before any stream capture; a
 * cudaDeviceReset invalidates the cached address, so do not use the entry
 * point on a device after one). All calls share the array, and each call
 * rewrites the table and clears the queue counter it holds: calls that
 * overlap on the GPU (different streams, no ordering) race on it; calls on
 * one stream are ordered. */
int32_t phc_solve_paths_noalloc(const phc_system* sys, const phc_homotopy* hom,
                                const phc_solve_options* opts, const phc_gpu_options* gpu,
                                int64_t k0, int64_t count, phc_path_out* d_out, double* d_z,
                                double* d_x, void* stream);

/* ---- device-resident plan (inputs already in device memory) ------------ */
typedef struct phc_plan phc_plan;
int32_t phc_plan_create(const phc_system* sys, const phc_homotopy* hom,
                        const phc_solve_options* opts, const phc_gpu_options* gpu,
                        phc_plan** plan);
/* Launches the tracker for paths k0 .. k0+count-1 on a CUDA stream (0 =
 * default); d_out and d_z are device buffers of count records / count*(n+1)
 * complex values. Asynchronous: returns after the launch. */
int32_t phc_plan_launch(phc_plan* plan, int64_t k0, int64_t count,
                        phc_path_out* d_out, double* d_z, void* stream);
/* number of kernel launches phc_plan_launch issues */
int32_t phc_plan_launch_count(const phc_plan* plan);
int32_t phc_plan_destroy(phc_plan* plan);
/* resolved launch configuration of a plan and the size of its device table */
int32_t phc_plan_config(const phc_plan* plan, int32_t* warps_per_block,
                        int32_t* grid, int32_t* smem_bytes, int32_t* unknowns_cap,
                        int32_t* table_bytes);

/* ---- CUDA graphs of plan launches ------------------------------------- */
/* Captures what phc_plan_launch(plan, k0, count, d_out, d_z, stream) issues
 * -- the reset of the persistent queue and the tracker kernel -- into a
 * CUDA graph and instantiates it; phc_graph_launch replays it on a stream
 * with one call. The plan and the device buffers must outlive the graph.
 * For a batch of paths that is solved repeatedly, or as a piece of a
 * larger application graph. The reference has no counterpart. */
typedef struct phc_graph phc_graph;
int32_t phc_graph_create(phc_plan* plan, int64_t k0, int64_t count, phc_path_out* d_out,
                         double* d_z, phc_graph** graph);
int32_t phc_graph_launch(phc_graph* graph, void* stream);
int32_t phc_graph_destroy(phc_graph* graph);

/* ---- autotuner -------------------------------------------------------- */
/* Picks the launch configuration -- schedule (persistent refill or one path
 * per warp), warps per block and refill chunk -- by timing the tracker on
 * the first sample_paths paths of sys (0 = four paths per resident warp of
 * the device) for each candidate, on gpu->device in gpu->precision. Writes
 * the fastest into gpu->schedule, warps_per_block and chunk, and remembers
 * it for this process: later plans and solves on the same device with the
 * same precision, schedule and row width that pass warps_per_block = 0 or
 * chunk = 0 get the tuned values. Allocates its own device buffers for the
 * sample. The reference has no counterpart (its tracker is serial). */
#define PHC_TUNE_MAX 32
typedef struct {
  int32_t ncand;                       /* candidates timed                 */
  int32_t best;                        /* index of the chosen candidate    */
  int32_t schedule[PHC_TUNE_MAX];
  int32_t warps_per_block[PHC_TUNE_MAX];
  int32_t chunk[PHC_TUNE_MAX];
  double ms[PHC_TUNE_MAX];             /* best of the timed launches       */
  int64_t sample_paths;
} phc_tune_report;
int32_t phc_autotune(const phc_system* sys, const phc_solve_options* opts,
                     phc_gpu_options* gpu, int64_t sample_paths, phc_tune_report* report);

/* ---- compact request format (serving ingest) ---------------------------- */
/* A system and optional solve_options as one byte string: a 24-byte header
 * ("PHCR", version 1, n, total terms, flags), the options if flagged, the
 * term count of each equation, then per term its coefficient (two float64)
 * and its nonzero affine exponents as uint16 (variable, exponent) pairs.
 * The packed counterpart of sparse_system%add_equation's input
 * (src/sparse.f90:83-141); the reference itself has no wire format. */
int64_t phc_request_size(const phc_system* sys, int32_t with_options);
/* opts may be NULL (the request then carries none); *len = bytes written,
 * or the bytes needed when cap is too small */
int32_t phc_request_encode(const phc_system* sys, const phc_solve_options* opts, void* buf,
                           int64_t cap, int64_t* len);
/* Fills a fresh builder through phc_sparse_add_equation (the reference's
 * validation and degree rules) and *opts (defaults when the request has
 * none). Malformed input returns PHC_ERR_INVALID_INPUT. */
int32_t phc_request_decode(const void* buf, int64_t len, phc_sparse* builder,
                           phc_solve_options* opts);

/* ---- serving loop: continuous batching of whole systems ---------------- */
typedef struct phc_server phc_server;
typedef struct {
  int32_t device;
  int32_t nslots;            /* concurrent batches in flight (streams)      */
  int32_t max_batch_systems; /* systems packed into one batch launch        */
  int32_t max_batch_paths;   /* paths packed into one batch launch          */
  int64_t mem_budget_bytes;  /* device memory the server may hold, 0 = 1 GiB */
  phc_gpu_options gpu;
} phc_server_config;

int32_t phc_server_create(const phc_server_config* cfg, phc_server** srv);
/* Copies the system and options; the request is admitted to the GPU as
 * soon as a slot and enough of the memory budget are free. */
int32_t phc_server_submit(phc_server* srv, const phc_system* sys,
                          const phc_solve_options* opts, uint64_t* ticket);
/* *done = 1 once the result is ready; returns PHC_ERR_BAD_HANDLE for an
 * unknown ticket */
/* phc_server_submit for a request in the compact format */
int32_t phc_server_submit_request(phc_server* srv, const void* buf, int64_t len,
                                  uint64_t* ticket);
int32_t phc_server_poll(phc_server* srv, uint64_t ticket, int32_t* done);
/* blocks until done or timeout_ms passed (PHC_ERR_NOT_READY); < 0 waits */
int32_t phc_server_wait(phc_server* srv, uint64_t ticket, int64_t timeout_ms);
/* copies the result into caller arrays (capacity npaths rows) and releases
 * the ticket; latency_s = completion - submission time; returns the solve
 * status of the request */
int32_t phc_server_result(phc_server* srv, uint64_t ticket, phc_solve_result* res,
                          double* latency_s);
/* number of paths (Bezout number) of a submitted request */
int64_t phc_server_npaths(phc_server* srv, uint64_t ticket);
int32_t phc_server_stats(phc_server* srv, int64_t* submitted, int64_t* completed,
                         int64_t* batches, int64_t* in_flight);
int32_t phc_server_destroy(phc_server* srv);

/* ---- misc ---------------------------------------------------------------- */
const char* phc_version(void);
/* last CUDA error text of this thread (after a PHC_ERR_CUDA return) */
const char* phc_last_error(void);
/* Measures the CUDA-core FP64 and FP32 FMA throughput of a device (TFLOP/s),
 * the denominators of the tracker's roofline. Not part of the reference. */
int32_t phc_measure_fma_peaks(int32_t device, double* fp64_tflops, double* fp32_tflops);

#ifdef __cplusplus
}
#endif

#endif /* POLYHOMOCONT_B200_H */

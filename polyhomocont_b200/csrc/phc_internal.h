// phc_internal.h -- layout of the device-side system table ("plan") and
// of the kernel parameters, shared by the host plan builder
// (phc_plan.cpp) and the CUDA kernels (phc_track.cuh, phc_launch.cu).
//
// The reference evaluates F^h and its Jacobian per term with prefix and
// suffix products over all N variables (eval_terms, src/sparse.f90:223-280).
// Here the table is compiled once per system into "contributions": one
// record per (output entry, term) pair, i.e. the value c*z^a of a term for
// f_i and the partial derivative c*e_j*z_j^(e_j-1)*prod_{l!=j} z_l^(e_l) for
// J(i,j), each as a coefficient times a short list of power-table factors.
// Output entries are assigned to the 32 lanes of a warp by a
// longest-processing-time schedule; each lane sums the contributions of
// its entries in the reference's term order and writes the sum once, so
// no two lanes touch the same entry and the result is deterministic.
#pragma once

#include <cstdint>

#include "polyhomocont_b200.h"

#if defined(__CUDACC__)
#define PHC_HD __host__ __device__
#else
#define PHC_HD
#endif

namespace phc {

constexpr int kMaxN = 32;      // unknowns N = n + 1 (one lane per row)
constexpr int kMaxFac = 3;     // power-table factors per record (longer products chain)
constexpr int kMaxPw = 1024;   // power-table entries (maxexp + 1) * N, 10-bit indices
constexpr int kWarp = 32;

// Record metadata, packed into 64 bits:
//   bits  0- 9  dest   i*S + j: Jacobian entry (row-major, odd stride S)
//   bits 12-14  flags  kRecLast: last contribution of its entry
//   bits 15-44  fac    three 10-bit offsets into the extended power table
// A record contributes coef * pw[fac_0] * pw[fac_1] * pw[fac_2]; unused
// factor slots point at pw[0] = z_0^0 = 1. Extended entries pw[pw_size + e]
// hold products of three earlier entries (terms with more than three
// nonzero exponents), computed level by level before the records run.
enum : unsigned {
  kRecLast = 1,
};
constexpr int kMaxLevels = 8;

// Records are stored lane-interleaved: record i of lane l sits in slot
// i * 32 + l of three arrays (FP64 coefficient, FP32 coefficient, metadata),
// so the 32 lanes of a warp read consecutive 16-, 8- and 8-byte words
// without shared-memory bank conflicts. The FP32 coefficient arrays are the
// table's last bytes, so that kernels that evaluate only in FP64 stage the
// first bytes_fp64 bytes and leave them out.
struct alignas(16) PlanHeader {
  int32_t n;            // variables / equations
  int32_t N;            // unknowns n + 1
  int32_t S;            // row stride of the Jacobian buffer (odd)
  int32_t maxexp;       // largest homogenized exponent
  int32_t pw_size;      // (maxexp + 1) * N, plus n_pre extended entries in the table
  int32_t len_f;        // slots per lane of the f schedule
  int32_t len_j;        // slots per lane of the Jacobian schedule
  int32_t total_bytes;  // header + arrays (multiple of 16)
  int32_t off_fd, off_ff, off_fm;  // byte offsets of the f schedule arrays
  int32_t off_jd, off_jf, off_jm;  // byte offsets of the Jacobian schedule arrays
  int32_t nrec;         // records of both schedules
  int32_t n_pre;        // extended power-table entries (products of three)
  int32_t off_pre;      // byte offset of their packed factor triples (uint32)
  int32_t n_levels;
  int32_t level_off[kMaxLevels + 1];  // word ranges per level (2 words per entry)
  int32_t pw_total;     // pw_size + n_pre: entries of the per-warp table
  int32_t max_fac;      // most power-table factors of any Jacobian record (0..3)
  int32_t bytes_fp64;   // bytes before the FP32 coefficient arrays (which come last):
                        // what a kernel without an FP32 evaluation stages
  int32_t cnt_f[kWarp]; // records of each lane
  int32_t cnt_j[kWarp];
  int32_t deg[kMaxN];
  double inv_deg[kMaxN];    // 1/d_i (Euler's relation for F^h_i)
  int64_t radix[kMaxN];     // prod_{l < i} d_l (mixed-radix start index)
  int64_t nstart;           // Bezout number
  int64_t pad1_;
  double argb[kMaxN];       // atan2(Im b_i, Re b_i), host libm
  double gamma[2];
  double b[kMaxN][2];
  double patch[kMaxN][2];
  // the patch row eliminated first (evaluate_rows_of; reduce = 1 for
  // n = 16): pivot column c, the largest |a_c| (first maximum),
  // rho_j = a_j / a_c, 1/a_c, and the patch row's absolute sum sum_j |a_j|
  int32_t reduce;
  int32_t red_c;
  int32_t pad2_[2];
  double rho[kMaxN][2];
  double inv_ac[2];
  double patch_abs_sum;
  double pad3_;
};

// Per-kernel options: the POD mirror of solve_options plus GPU knobs.
struct KOpts {
  phc_solve_options so;
  int32_t precision;     // PHC_PREC_*
  int32_t fp64_sticky;   // mixed: FP64 step attempts after an FP32 failure
  int64_t max_units;     // safety budget of units per path
};

struct KParams {
  const unsigned char* plan;  // device copy of header + records
  int32_t plan_bytes;
  int32_t ws_bytes;           // per-warp workspace bytes
  int32_t warps;              // warps per block
  int32_t persistent;         // 1: atomic queue, 0: one path per warp
  int32_t chunk;              // paths per queue grab
  int32_t pad_;
  int64_t k0;                 // first path (1-based)
  int64_t count;              // number of paths
  unsigned long long* counter;  // persistent queue head (device)
  phc_path_out* out;          // [count]
  double* z;                  // [count][N][2]
  double* x;                  // [count][n][2] or null
  // [count] or null: set to 1 (system scope) once path q's record, z and x
  // are visible to the host; outputs in mapped host memory are then read
  // while the launch runs
  unsigned int* done;
  KOpts opts;
};

// One request of a batch (device memory): where its table, options and
// outputs are (byte offsets into the batch buffer), and which global path
// indices of the batch are its paths.
struct alignas(16) BatchSys {
  int64_t table_off;
  int64_t path_begin;   // global index (0-based) of its first path in the batch
  int64_t npaths;
  int64_t out_off;      // phc_path_out[npaths]
  int64_t z_off;        // double[npaths][N][2]
  int64_t x_off;        // double[npaths][n][2], or -1
  int32_t table_bytes;  // multiple of 16
  int32_t pad_;
  KOpts opts;
};

// Parameters of the batched kernel: persistent warps pull global path
// indices of the whole batch from one queue; each warp stages the table and
// options of the request it is working on into its own shared-memory slice
// [table_cap | ws_cap | KOpts].
struct KParamsBatch {
  unsigned char* base;        // batch buffer: descriptors, tables, outputs
  const BatchSys* sys;        // [nsys], sorted by path_begin
  int32_t nsys;
  int32_t chunk;              // paths per queue grab
  int32_t table_cap;          // multiple of 16
  int32_t ws_cap;             // multiple of 16
  int32_t slice_bytes;        // table_cap + ws_cap + KOpts, multiple of 16
  int32_t pad_;
  int64_t total_paths;
  unsigned long long* counter;
  // finished paths per request, in host memory mapped into the device (may
  // be null): the host finishes a request as soon as its count is complete,
  // while the rest of the batch is still running
  unsigned int* done;
};

// Cold per-path state of the tracker state machine, kept in shared memory
// (one per warp) so that registers stay free for the evaluation and the LU.
// Scalars are warp-uniform; the vectors hold component j in slot j.
struct alignas(16) WarpState {
  // the path: its current point z, the segment's start point zs, the
  // corrector's point zp, the RK4 sum, the pending unit's input point zin
  double z[kWarp][2], zs[kWarp][2], zp[kWarp][2], ksum[kWarp][2], zin[kWarp][2];
  double zold[kWarp][2];   // end game: z before a radial segment
  double est[kWarp][2];    // current Cauchy estimate
  double prev[kWarp][2];   // previous estimate
  double resz[kWarp][2];   // best estimate so far (res%z)
  double zprev[kWarp][2];  // loops: point before the last arc
  double zsum[kWarp][2];   // loops: sum of the samples
  double hsave[kWarp][2];  // classify: H(z, 0) of the last evaluation
  double xv[kWarp][2];     // classify: affine endpoint z(1:n)/w
  double seg_t0[2], seg_t1[2];
  double seg_r, seg_th0, seg_dth;
  double o_step_init, o_step_max;
  double p_t, p_ege, p_cond, p_resid;
  double r, rnew, best_resid, dprev, cest, cest_prev, eg_segstep, eg_error, eg_residual,
      eg_radius, rec_err;
  double lp_spacing, lp_floor, lp_dth;
  double cond_anorm, cond_ainv;  // cond1 accumulated over right-hand-side chunks
  // segment stepper (track_segment's s, step, ds, s + ds, Newton's last
  // squared update norm) and the pending unit's t and dt/ds
  double s, step, ds, sn, dnorm_prev;
  double tin[2], dtin[2];
  long long units;
  long long kpath;               // the path (1-based)
  phc_path_out* rec;             // its outputs
  double* zo;
  double* xo;
  int nsucc, sacc, srej, sstat;  // segment: accepted since the last growth, counts, status
  int stage, att64, uk, pc_after, u_prec;  // RK4 stage / Newton iteration; pending unit
  int seg_arc, o_grow, seg_cont;
  int p_status, p_wind, p_egs, p_nacc, p_nrej, p_atinf, p_sing, p_real;
  int c_tan, c_new, c_ref, c_eval, c_cond, c_retry;
  int max_loops, eg_status, eg_wind, eg_nacc, eg_nrej, cw, rec_cont, have_prev, gate;
  int lp_c, lp_j, lp_max, lp_nsamp, lp_cont, lp_ok;
  int rf_it, sticky;
  int cond_c0, cond_ret;  // cond1: first column of the current chunk, state to return to
};

// Per-warp shared-memory workspace layout (byte offsets from the warp's
// base), shared by host (sizing) and device (addressing).
struct WsLayout {
  int pwd, pwf, jd, jf, piv, st, bytes;
};

PHC_HD inline int align16(int x) { return (x + 15) & ~15; }

// eval32: the kernel carries the FP32 evaluation (FP32 power table and
// Jacobian buffer).
PHC_HD inline WsLayout ws_layout(int n, int S, int pw_size, bool eval32) {
  WsLayout L;
  int off = 0;
  L.pwd = off; off += align16(pw_size * 16);
  L.pwf = off; off += eval32 ? align16(pw_size * 8) : 0;
  L.jd = off; off += align16((n + 1) * S * 16);  // rows 0..n-1: dF^h, row n: patch
  L.jf = off; off += eval32 ? align16((n + 1) * S * 8) : 0;
  L.piv = off; off += kWarp * 4;
  L.st = off; off += align16((int)sizeof(WarpState));
  L.bytes = off;
  return L;
}

// Supported register-row widths: the compile-time capacity NM of the N =
// n + 1 rows of the eliminated system.
constexpr int kNMs[] = {6, 8, 12, 16, 18, 24, 32};
inline int pick_nm(int rows) {
  for (int v : kNMs)
    if (rows <= v) return v;
  return 0;
}
// The kernel family of n = 16 with the patch row eliminated first: 16 rows
// of 16 columns (RowLayout), its own width id so that the reduction is
// compiled into these kernels only and no kernel carries both forms.
constexpr int kNmReduced16 = 17;
// The patch row is eliminated first where that moves the system into a
// layout with more lanes per row: 17 unknowns have 16 equation rows, which
// fit the two-lane layout (rows of up to 16). (For 9 unknowns the same would
// give the four-lane layout, but on one serving-stream system it turned a
// path that the other form fails in 14,000 units into one that fails in the
// end game after 3.2 million, so n = 8 keeps the patch as a row.)
PHC_HD constexpr bool reduce_patch_row(int n) { return n == 16; }
// The kernel width for a system of n equations.
inline int kernel_nm(int n) { return reduce_patch_row(n) ? kNmReduced16 : pick_nm(n + 1); }
// The single-system kernels of rows up to 8 columns carry an FP32
// evaluation for the mixed predictor; every other kernel evaluates in FP64.
PHC_HD constexpr bool kernel_eval32(int nm, int precision) {
  return precision == PHC_PREC_MIXED && nm <= 8;
}
// Most warps per block of the tracking kernels. The lean form (the path
// state out of registers across a unit, see track_one) is compiled for
// larger blocks, so that more warps share one staged copy of the table:
// rows of up to 17 columns for 16 warps (65,536 / 512 = 128 registers per
// thread; the n = 16 family spills a few bytes at that bound, the narrower
// ones need no more), rows of 18 for 12 warps (170 registers). The other
// kernels are compiled for blocks of up to 8 warps (255 registers).
PHC_HD constexpr int max_warps_per_block(int nm, bool lean) {
  return lean ? (nm <= 17 ? 16 : (nm <= 18 ? 12 : 8)) : 8;
}
constexpr int kMaxWarpsPerBlock = 16;  // over all kernels
// Resident warps per SM below which a launch is latency-bound: the form
// that keeps the path state in registers is used for launches of at most
// twice that many paths per SM, the lean form above.
constexpr int kLeanPathsPerSm = 16;

}  // namespace phc

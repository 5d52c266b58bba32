// phc_track.cuh -- the path-tracking kernel: one warp tracks one path
// through start_solution, the predictor-corrector tracker, the Cauchy end
// game and the classification numerics (src/solve.f90:190-198, :217-328).
//
// The reference's nested procedures (track_segment inside loops inside
// cauchy_endgame inside endpoint) are flattened into one warp-uniform
// state machine whose every step either changes control state or runs
// exactly one "unit": an evaluation of H(z,t) (and H_z, H_t), optionally
// followed by a Gauss-Jordan solve (one right-hand side, or four columns
// of the inverse for cond1). The unit has a single call site and chooses
// its precision at run time, so each evaluation and elimination exists
// once in the kernel binary, and the same machine serves the predictor,
// the corrector, the end game's backward errors, refine and cond1.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cstdint>
#include <type_traits>

#include "phc_device.cuh"
#include "phc_internal.h"

namespace phc {

enum UnitKind : int { UK_TANGENT = 0, UK_NEWTON = 1, UK_BACKERR = 2, UK_COND = 3,
                      UK_REFINE = 4 };

struct UnitRes {
  cd x;       // solution component of this lane
  cd h;       // residual component of this lane (UK_COND)
  double a1;  // UK_BACKERR: ||h||_inf; UK_COND: ||A||_1 (first chunk)
  double a2;  // UK_BACKERR: max row sum of |H_z|; UK_COND: max column sum of the chunk of A^-1
  bool ok;    // LU nonsingular
};

// Columns of A^-1 per cond1 unit.
constexpr int kCondChunk = 4;

// One unit: an evaluation of H, H_z and H_t followed by one elimination.
// prec selects the arithmetic (only the FP64 form exists when MIXED is
// false):
//   0: FP64 evaluation and elimination (FP64 tracker, FP64 retries, the
//      end game's backward errors, refine, cond1)
//   1: FP64 evaluation, FP32 elimination (mixed corrector: the residual in
//      FP64, the update in FP32; mixed predictor unless EVAL32)
//   2: FP32 evaluation and elimination (mixed predictor when EVAL32)
// EVAL32 compiles the FP32 evaluation into the kernel. It pays where one
// path's latency sets the time and the kernel is small: the single-system
// kernels for rows of up to 8 columns (n <= 7), whose paths run nearly
// alone. Elsewhere the second evaluation body costs more in instruction
// fetch than it saves: the batch kernels, throughput-bound, and the wider
// rows, whose bodies are long. Measured on one B200: n=4 systems 1.00 ms
// with an FP64 evaluation against 0.85 ms with an FP32 one; 17 unknowns,
// 65,536 paths, 342.6 ms against 358.3 ms; the serving stream's capacity
// about 2,200 against 1,800 systems/s.
// Every piece of code -- each evaluation, the FP32 and the FP64
// elimination -- appears once in the kernel.
// UK_COND eliminates against the unit vectors e_c0 .. e_c0+3 (cond1,
// src/linalg.f90:135-174); the state machine runs one such unit per chunk.
// Rows of up to 16 columns use the split layout (two lanes per row, half
// a row each: evaluate_rows_of, gauss_jordan_split); wider rows one lane per
// row.
// Workspace pointers of a warp inside its shared-memory region. The FP32
// power table and Jacobian buffer exist only in kernels that carry the FP32
// evaluation (EVAL32).
template <bool EVAL32>
__device__ __forceinline__ WarpWS warp_workspace(const PlanHeader& P, unsigned char* wbase) {
  const WsLayout L = ws_layout(P.n, P.S, P.pw_total, EVAL32);
  WarpWS ws;
  ws.pwd = reinterpret_cast<cd*>(wbase + L.pwd);
  ws.pwf = reinterpret_cast<cf*>(wbase + L.pwf);
  ws.jd = reinterpret_cast<cd*>(wbase + L.jd);
  ws.jf = reinterpret_cast<cf*>(wbase + L.jf);
  ws.piv = reinterpret_cast<int*>(wbase + L.piv);
  return ws;
}
template <bool EVAL32>
__device__ __forceinline__ WarpState* warp_state(const PlanHeader& P, unsigned char* wbase) {
  return reinterpret_cast<WarpState*>(wbase + ws_layout(P.n, P.S, P.pw_total, EVAL32).st);
}

template <int NM>
struct RowLayout {
  // the kernels of width kNmReduced16 hold 16 rows of 16 columns, the
  // reduced system of n = 16 with the patch row eliminated first
  static constexpr bool kReduce = NM == kNmReduced16;
  static constexpr int kCols = kReduce ? 16 : NM;
  static constexpr int kLanes = kCols <= 8 ? 4 : (kCols <= 16 ? 2 : 1);  // lanes per row
  static constexpr bool kSplit = kLanes > 1;
  static constexpr int kRegs = kLanes == 4 ? 2 : (kLanes == 2 ? kCols / 2 : kCols);  // per lane
  static constexpr int kRows = 32 / kLanes;  // rows per warp
};

template <int NM, typename T, int F>
__device__ __forceinline__ void evaluate_rows(const WarpConst& C, const WarpWS& ws, cd z, cd t,
                                              int lane, bool reduce,
                                              cpx<T> (&a)[RowLayout<NM>::kRegs], cpx<T>& aic,
                                              cd& h, cd& ht) {
  evaluate_rows_of<RowLayout<NM>::kRegs, RowLayout<NM>::kLanes, T, F>(C, ws, z, t, lane, reduce,
                                                                      a, aic, h, ht);
}

template <int NM, int R, typename T>
__device__ __forceinline__ bool eliminate(cpx<T> (&a)[RowLayout<NM>::kRegs], cpx<T> (&r)[R],
                                          int rows, int lane, int* piv) {
  if constexpr (RowLayout<NM>::kSplit)
    return gauss_jordan_split<RowLayout<NM>::kRegs, RowLayout<NM>::kLanes, R, T>(a, r, rows, lane,
                                                                                piv);
  else
    return gauss_jordan<NM, R, T>(a, r, rows, lane, piv);
}

// h_n = a . z - 1, the patch row of H (src/homotopy.f90:228-230), on every
// lane (lane j holds z_j).
__device__ __forceinline__ cd patch_residual(const WarpConst& C, cd z, int lane) {
  const cd pz = (lane < C.N) ? mkc<double>(C.patch[lane][0], C.patch[lane][1]) * z
                             : czero<double>();
  const cd s = warp_csum(pz);
  return mkc<double>(s.re - 1.0, s.im);
}

// The solution x of the full system (lane j receives x_j) from the
// eliminated right-hand side y (component r of the eliminated system in
// lane piv[r]). With the patch row eliminated first (see
// evaluate_rows_of), rn is its right-hand side and x_c follows from the
// others.
template <typename T>
__device__ __forceinline__ cd full_solution(const PlanHeader& P, const WarpConst& C,
                                            const WarpWS& ws, bool reduce, cpx<T> y, cd rn,
                                            int lane) {
  const int n = C.n, N = C.N, c = C.red_c;
  if (!reduce) {
    const cpx<T> yj = shfl(y, ws.piv[lane < N ? lane : 0]);
    return (lane < N) ? ccast<double>(yj) : czero<double>();
  }
  const bool own = lane < N && lane != c;
  const int src = (lane == n) ? c : lane;  // reduced column of unknown `lane`
  const cpx<T> yj = shfl(y, ws.piv[own ? src : 0]);
  const cd x = own ? ccast<double>(yj) : czero<double>();
  const cd rho = own ? mkc<double>(C.rho[lane][0], C.rho[lane][1]) : czero<double>();
  const cd s = warp_csum(rho * x);
  const cd xc = rn * mkc<double>(P.inv_ac[0], P.inv_ac[1]) - s;
  return (lane == c) ? xc : x;
}

// One unit on the staged table tbl with the system's constants C and the
// warp's workspace ws. With the patch row eliminated first (the header's
// `reduce`) it works on the n x n reduced system and returns the solution
// of the full one.
template <int NM, bool MIXED, bool EVAL32, int F>
__device__ __forceinline__ void run_unit(const unsigned char* tbl, const WarpConst& C,
                                         const WarpWS& ws, int kind, int prec, int c0, cd zin,
                                         cd t, cd dt, int lane, UnitRes& u) {
  using L = RowLayout<NM>;
  constexpr int RW = L::kRegs;
  constexpr int S = L::kLanes;
  const PlanHeader& P = *reinterpret_cast<const PlanHeader*>(tbl);
  const int n = C.n, N = C.N, c = C.red_c;
  constexpr bool reduce = L::kReduce;
  const int rows = reduce ? n : N;  // rows of the eliminated system
  // the row this lane works on (rows >= `rows` hold zeros), and whether it
  // reports the row (part 0)
  const int row = lane & (L::kRows - 1);
  const bool owner = lane < L::kRows;
  cd h, ht;
  cpx<float> as[RW];
  cpx<float> rs32;
  cd rn = czero<double>();  // the patch row's right-hand side (reduced system)
  if (!MIXED || !EVAL32 || prec != 2) {
    cpx<double> a[RW];
    cd aic;
    evaluate_rows<NM, double, F>(C, ws, zin, t, lane, reduce, a, aic, h, ht);
    if (kind == UK_BACKERR) {
      // backward_error, src/endgame.f90:269-285: ||H(z,0)|| and the maximum
      // absolute row sum of H_z, over the n equation rows and the patch row
      double rsum = 0.0;
#pragma unroll
      for (int j = 0; j < RW; ++j) rsum += cabs(a[j]);
      rsum = row_sum<S>(rsum);
      if (reduce) {
        rsum += cabs(aic);
        const double hn = cabs(patch_residual(C, zin, lane));
        u.a1 = fmax(warp_max_nonneg(row < n ? cabs(h) : 0.0), hn);
        u.a2 = fmax(warp_max_nonneg(row < n ? rsum : 0.0), P.patch_abs_sum);
      } else {
        u.a1 = warp_max_nonneg(row < N ? cabs(h) : 0.0);
        u.a2 = warp_max_nonneg(row < N ? rsum : 0.0);
      }
      u.ok = true;
      return;
    }
    if (kind == UK_COND) {
      u.h = h;
      if (c0 == 0) {
        // ||A||_1: the largest column sum over all N rows
        if (reduce) {
          // every column but c is one of the lane's columns; the patch row
          // adds |a_o|
          const int j0 = (lane / L::kRows) * RW;
          double anorm = 0.0;
#pragma unroll
          for (int jj = 0; jj < RW; ++jj) {
            const int r = j0 + jj;
            const double cs = part_sum<S>(row < n ? cabs(a[jj]) : 0.0);
            if (r < n) {
              const int o = reduced_col(r, c, n);
              anorm = fmax(anorm, cs + hypot(C.patch[o][0], C.patch[o][1]));
            }
          }
          const double csc = part_sum<S>(row < n ? cabs(aic) : 0.0);
          anorm = fmax(anorm, csc + hypot(C.patch[c][0], C.patch[c][1]));
          u.a1 = warp_max_nonneg(anorm);
        } else {
          double anorm = 0.0;
#pragma unroll
          for (int j = 0; j < RW; ++j) {
            if constexpr (L::kSplit)
              anorm = fmax(anorm, part_sum<S>(row < N ? cabs(a[j]) : 0.0));
            else if (j < N)
              anorm = fmax(anorm, warp_sum(row < N ? cabs(a[j]) : 0.0));
          }
          if constexpr (L::kSplit) anorm = warp_max_nonneg(anorm);
          u.a1 = anorm;
        }
      }
      // right-hand sides e_col, col = c0 .. c0+3 (unknowns 0..N-1); in the
      // reduced system the patch row's is 1 for col = n
      cd r[kCondChunk];
      if (reduce) {
        fold_patch<RW, S, double>(C, lane, a, aic);
        const cd inv_ac = mkc<double>(P.inv_ac[0], P.inv_ac[1]);
#pragma unroll
        for (int q = 0; q < kCondChunk; ++q) {
          const cd rq = (row == c0 + q && row < n) ? cone<double>() : czero<double>();
          r[q] = (c0 + q == n) ? rq - aic * inv_ac : rq;
        }
      } else {
#pragma unroll
        for (int q = 0; q < kCondChunk; ++q)
          r[q] = (row == c0 + q) ? cone<double>() : czero<double>();
      }
      if (!eliminate<NM, kCondChunk, double>(a, r, rows, lane, ws.piv)) {
        u.ok = false;  // cond1 of an exactly singular matrix
        return;
      }
      double ainv = 0.0;
#pragma unroll
      for (int q = 0; q < kCondChunk; ++q) {
        if (c0 + q < N) {
          if (reduce) {
            const cd rnq = (c0 + q == n) ? cone<double>() : czero<double>();
            const cd x = full_solution<double>(P, C, ws, true, r[q], rnq, lane);
            ainv = fmax(ainv, warp_sum(lane < N ? cabs(x) : 0.0));
          } else {
            // the column sum is the same in pivot order
            ainv = fmax(ainv, warp_sum(owner && row < N ? cabs(r[q]) : 0.0));
          }
        }
      }
      u.a2 = ainv;
      u.ok = true;
      return;
    }
    cd r0 = (kind == UK_TANGENT) ? -(ht * dt) : -h;
    if (reduce) {
      fold_patch<RW, S, double>(C, lane, a, aic);
      if (kind != UK_TANGENT) {  // H_t of the patch row is zero
        rn = -patch_residual(C, zin, lane);
        r0 = r0 - aic * (rn * mkc<double>(P.inv_ac[0], P.inv_ac[1]));
      }
    }
    if (!MIXED || prec == 0) {
      cd r[1] = {r0};
      u.ok = eliminate<NM, 1, double>(a, r, rows, lane, ws.piv);
      if (!u.ok) return;
      u.x = full_solution<double>(P, C, ws, reduce, r[0], rn, lane);
      return;
    }
    // FP64 evaluation, FP32 elimination
    if constexpr (MIXED) {
#pragma unroll
      for (int j = 0; j < RW; ++j) as[j] = ccast<float>(a[j]);
      rs32 = ccast<float>(r0);
    }
  } else if constexpr (MIXED && EVAL32) {
    // FP32 evaluation (the predictor: the patch row's right-hand side is
    // zero)
    cpx<float> aic;
    evaluate_rows<NM, float, F>(C, ws, zin, t, lane, reduce, as, aic, h, ht);
    if (reduce) fold_patch<RW, S, float>(C, lane, as, aic);
    rs32 = ccast<float>(-(ht * dt));
  }
  if constexpr (MIXED) {
    cpx<float> r[1] = {rs32};
    u.ok = eliminate<NM, 1, float>(as, r, rows, lane, ws.piv);
    if (!u.ok) return;
    u.x = full_solution<float>(P, C, ws, reduce, r[0], rn, lane);
  }
}

enum Pc : int {
  PC_START,
  PC_SEG_BEGIN,
  PC_SEG_ATTEMPT,
  PC_SEG_AFTER_UNIT,
  PC_SEG_END,
  PC_MAIN_DONE,
  PC_EG_INIT,
  PC_EG_TOP,
  PC_EG_AFTER_LOOPS,
  PC_EG_AFTER_RECORD_MAIN,
  PC_EG_RADIAL,
  PC_EG_AFTER_RADIAL,
  PC_EG_AFTER_FALLBACK,
  PC_LOOPS_BEGIN,
  PC_LOOP_ARC,
  PC_LOOP_AFTER_ARC,
  PC_RECORD,
  PC_RECORD_AFTER,
  PC_EG_DONE,
  PC_CL_START,
  PC_CL_AFTER_COND1,
  PC_CL_AFTER_REFINE,
  PC_CL_COND2,
  PC_CL_AFTER_COND2,
  PC_CL_FINAL,
  PC_COND_STEP,
  PC_FINISH,
};

constexpr double kPi = 3.14159265358979323846;
constexpr double kEps = DBL_EPSILON;
constexpr double kTiny = DBL_MIN;
constexpr double kHuge = DBL_MAX;

__device__ __forceinline__ double vnorm(cd v, int lane, int N) {
  return warp_max_nonneg(lane < N ? cabs(v) : 0.0);
}

// better(), src/endgame.f90:287-311
__device__ __forceinline__ bool better(double resid, double err, double best_resid,
                                       double best_err, double residual_tol) {
  const bool valid = resid <= residual_tol;
  const bool best_valid = best_resid <= residual_tol;
  if (valid != best_valid) return valid;
  return err < best_err;
}

// Segment t(s) and dt/ds of the segment stored in the warp state.
__device__ __forceinline__ cd seg_t(const WarpState& st, double s) {  // :142-162
  if (!st.seg_arc) {
    const cd t0 = mkc<double>(st.seg_t0[0], st.seg_t0[1]);
    const cd t1 = mkc<double>(st.seg_t1[0], st.seg_t1[1]);
    if (s >= 1.0) return t1;
    return t0 + s * (t1 - t0);
  }
  double sn, cs;
  sincos(st.seg_th0 + s * st.seg_dth, &sn, &cs);
  return st.seg_r * mkc<double>(cs, sn);
}
__device__ __forceinline__ cd seg_dt(const WarpState& st, double s) {  // :164-177
  if (!st.seg_arc)
    return mkc<double>(st.seg_t1[0] - st.seg_t0[0], st.seg_t1[1] - st.seg_t0[1]);
  return mkc<double>(0.0, st.seg_dth) * seg_t(st, s);
}

// t(s) and dt/ds together, with one sincos on arcs.
__device__ __forceinline__ void seg_tdt(const WarpState& st, double s, cd& t, cd& dt) {
  if (!st.seg_arc) {
    t = seg_t(st, s);
    dt = mkc<double>(st.seg_t1[0] - st.seg_t0[0], st.seg_t1[1] - st.seg_t0[1]);
    return;
  }
  double sn, cs;
  sincos(st.seg_th0 + s * st.seg_dth, &sn, &cs);
  t = st.seg_r * mkc<double>(cs, sn);
  dt = mkc<double>(0.0, st.seg_dth) * t;
}

// t(s) and dt/ds into the warp state (the pending unit's t and dt)
__device__ __forceinline__ void seg_tdt_store(WarpState& st, double s) {
  cd t, dt;
  seg_tdt(st, s, t, dt);
  st.tin[0] = t.re;
  st.tin[1] = t.im;
  st.dtin[0] = dt.re;
  st.dtin[1] = dt.im;
}

// max_j |v_j|^2 over the warp (squared moduli compare like the moduli of
// the reference's norm_inf, without a hypot per lane)
__device__ __forceinline__ double vnorm2(cd v, int lane, int N) {
  return warp_max_nonneg(lane < N ? v.re * v.re + v.im * v.im : 0.0);
}

#define LV(f) (reinterpret_cast<cd*>(st.f)[lane])
#define LDV(f) lds(&LV(f))
#define STV(f, v) sts(&LV(f), (v))

// Tracks path k (1-based) and writes its record, z and x.
//
// The hot state of the path (z, the segment's start point zs, the corrector's
// point zp, the RK4 sum, the segment stepper's scalars) lives in registers
// while the state machine runs. LEAN selects what happens across a unit:
//   LEAN = false: the state and the system's constants (WarpConst, the
//     workspace pointers, loaded once) stay in registers. Fewest
//     instructions and dependent shared-memory round trips per unit: the
//     form for launches in which one path's latency sets the time.
//   LEAN = true: the state is stored to the warp's WarpState before the unit
//     and loaded back after it (independent stores and loads, issued
//     together), and the unit loads the constants itself, so that neither
//     occupies registers while the unit runs. About 70 registers fewer per
//     thread (134 against 210 for 16-column rows), hence more resident warps:
//     the form for launches with many more paths than resident warps.
template <int NM, int PREC, bool EVAL32, int F, bool LEAN>
__device__ __forceinline__ void track_one(const unsigned char* tbl, unsigned char* wbase,
                                          WarpState& st, const KOpts& O, int64_t k, int lane,
                                          phc_path_out* rec, double* zo, double* xo) {
  const phc_tracker_options& TO = O.so.tracker;
  const phc_endgame_options& EO = O.so.endgame;
  const PlanHeader& P = *reinterpret_cast<const PlanHeader*>(tbl);
  // the constants the unit reads, held for the whole path (not LEAN)
  const WarpConst C0 = load_warp_const(P, tbl, lane);
  const WarpWS ws0 = warp_workspace<EVAL32>(P, wbase);
  constexpr bool kMixed = (PREC == PHC_PREC_MIXED);

  // hot lane vectors (component j in lane j)
  cd z = czero<double>(), zs = z, zp = z, ksum = z, zin = z;
  // hot uniform state of the segment being tracked
  double s = 0.0, step = 0.0, ds = 0.0, sn = 0.0, dnorm_prev = kHuge;
  int nsucc = 0, sacc = 0, srej = 0, sstat = PHC_PATH_SUCCESS, stage = 0;
  bool att64 = true;
  // pending unit
  int uk = UK_TANGENT, pc_after = PC_FINISH;
  int u_prec = 0;  // 0: FP64, 1: FP64 evaluation + FP32 elimination, 2: FP32 evaluation + elimination
  cd tin = z, dtin = z;
  UnitRes U;
  U.x = U.h = czero<double>();
  U.a1 = U.a2 = 0.0;
  U.ok = true;

  // path result defaults (type(path_result), src/solve.f90:86-119)
  st.p_status = PHC_PATH_SUCCESS;
  st.p_wind = st.p_egs = st.p_nacc = st.p_nrej = 0;
  st.p_t = 1.0;
  st.p_ege = st.p_cond = st.p_resid = 0.0;
  st.p_atinf = st.p_sing = st.p_real = 0;
  st.c_tan = st.c_new = st.c_ref = st.c_eval = st.c_cond = st.c_retry = 0;
  st.units = 0;
  st.sticky = 0;
  st.cond_c0 = 0;
  st.kpath = k;
  st.rec = rec;
  st.zo = zo;
  st.xo = xo;
  STV(xv, czero<double>());

  int pc = PC_START;
  for (;;) {
    bool want = false;
    const int n = P.n, N = P.N;
    while (!want) {
      switch (pc) {
        case PC_START: {
          // tdh_start_solution, src/homotopy.f90:151-177
          if (lane < n) {
            const int d = P.deg[lane];
            const int64_t digit = ((st.kpath - 1) / P.radix[lane]) % d;
            const double phi = (P.argb[lane] + 2.0 * kPi * (double)digit) / (double)d;
            double sp, cp;
            sincos(phi, &sp, &cp);
            z = mkc<double>(cp, sp);
          } else if (lane == n) {
            z = cone<double>();
          }
          const cd pz = (lane < N) ? mkc<double>(P.patch[lane][0], P.patch[lane][1]) * z
                                   : czero<double>();
          const cd sum = warp_csum(pz);
          if (lane < N) z = cdiv(z, sum);
          // track_path(hom, z, 1, t_end), src/solve.f90:230-232
          st.seg_arc = 0;
          st.seg_t0[0] = 1.0;
          st.seg_t0[1] = 0.0;
          st.seg_t1[0] = O.so.use_endgame ? EO.t_start : 0.0;
          st.seg_t1[1] = 0.0;
          st.o_step_init = TO.step_init;
          st.o_step_max = TO.step_max;
          st.o_grow = TO.grow_after;
          zs = z;
          st.seg_cont = PC_MAIN_DONE;
          pc = PC_SEG_BEGIN;
          break;
        }

        // ---------------- track_segment, src/tracker.f90:196-264 -------------
        case PC_SEG_BEGIN:
          s = 0.0;
          step = fmin(st.o_step_init, st.o_step_max);
          nsucc = 0;
          sacc = 0;
          srej = 0;
          sstat = PHC_PATH_SUCCESS;
          pc = PC_SEG_ATTEMPT;
          break;

        case PC_SEG_ATTEMPT: {
          if (!(s < 1.0)) {
            pc = PC_SEG_END;
            break;
          }
          if (sacc + srej >= TO.max_steps || st.units > O.max_units) {
            sstat = PHC_PATH_FAILED_MAX_STEPS;
            pc = PC_SEG_END;
            break;
          }
          ds = fmin(step, 1.0 - s);
          sn = s + ds;
          if (1.0 - sn <= 1.0e-3 * step) {
            sn = 1.0;
            ds = 1.0 - s;
          }
          const int sticky = st.sticky;
          att64 = !kMixed || sticky > 0;
          if (sticky > 0) st.sticky = sticky - 1;
          // predict_rk4 stage 1: tangent at (z, s), src/tracker.f90:283
          stage = 0;
          uk = UK_TANGENT;
          u_prec = att64 ? 0 : (EVAL32 ? 2 : 1);
          zin = zs;
          seg_tdt(st, s, tin, dtin);
          pc_after = PC_SEG_AFTER_UNIT;
          want = true;
          break;
        }

        case PC_SEG_AFTER_UNIT: {
          int outcome = 0;  // 1 accept, 2 reject
          if (stage < 4) {
            ++st.c_tan;
            if (!U.ok) {
              outcome = 2;
            } else {
              // predict_rk4, src/tracker.f90:266-293
              const cd kk = U.x;
              double s_in = s;
              if (stage == 0) {
                ksum = kk;
                zin = zs + (0.5 * ds) * kk;
                s_in = s + 0.5 * ds;
              } else if (stage == 1) {
                ksum = ksum + 2.0 * kk;
                zin = zs + (0.5 * ds) * kk;
                s_in = s + 0.5 * ds;
              } else if (stage == 2) {
                ksum = ksum + 2.0 * kk;
                zin = zs + ds * kk;
                s_in = s + ds;
              } else {
                ksum = ksum + kk;
                zp = zs + (ds / 6.0) * ksum;
              }
              if (stage < 3) {
                ++stage;
                uk = UK_TANGENT;
                // stages 1 and 2 share s + ds/2: t and dt/ds are reused
                if (stage != 2) seg_tdt(st, s_in, tin, dtin);
              } else {
                // newton_correct at t(sn), src/tracker.f90:319-360
                stage = 4;
                dnorm_prev = kHuge;
                uk = UK_NEWTON;
                u_prec = att64 ? 0 : 1;
                zin = zp;
                if (sn != s + ds) tin = seg_t(st, sn);  // else t(s + ds) of stage 3
              }
              pc_after = PC_SEG_AFTER_UNIT;
              want = true;
              break;
            }
          } else {
            ++st.c_new;
            const int it = stage - 3;
            if (!U.ok) {
              outcome = 2;
            } else {
              zp = zp + U.x;
              // ||dz|| <= tol ||z|| and the contraction test on squared norms
              const double d2 = vnorm2(U.x, lane, N);
              const double z2 = vnorm2(zp, lane, N);
              if (d2 <= (TO.corrector_tol * TO.corrector_tol) * z2) {
                outcome = 1;
              } else if (it > 1 && d2 > (TO.contraction * TO.contraction) * dnorm_prev) {
                outcome = 2;
              } else {
                dnorm_prev = d2;
                if (it >= TO.corrector_maxit) {
                  outcome = 2;
                } else {
                  ++stage;
                  uk = UK_NEWTON;
                  zin = zp;
                  pc_after = PC_SEG_AFTER_UNIT;
                  want = true;
                  break;
                }
              }
            }
          }
          if (outcome == 1) {
            zs = zp;
            s = sn;
            ++sacc;
            ++nsucc;
            if (nsucc >= st.o_grow) {
              step = fmin(2.0 * step, st.o_step_max);
              nsucc = 0;
            }
            pc = PC_SEG_ATTEMPT;
          } else {
            if (kMixed && !att64) {
              // the FP32 attempt failed: redo the same step in FP64 before
              // counting a rejection, and stay in FP64 for a few steps
              att64 = true;
              st.sticky = O.fp64_sticky;
              stage = 0;
              uk = UK_TANGENT;
              u_prec = 0;
              zin = zs;
              seg_tdt(st, s, tin, dtin);
              pc_after = PC_SEG_AFTER_UNIT;
              want = true;
              break;
            }
            ++srej;
            nsucc = 0;
            step = 0.5 * step;
            if (step < TO.step_min) {
              sstat = PHC_PATH_FAILED_MIN_STEP;
              pc = PC_SEG_END;
            } else {
              pc = PC_SEG_ATTEMPT;
            }
          }
          break;
        }

        case PC_SEG_END:
          pc = st.seg_cont;
          break;

        // ---------------- endpoint, src/solve.f90:217-252 ----------------------
        case PC_MAIN_DONE:
          z = zs;
          st.p_status = sstat;
          st.p_t = seg_t(st, s).re;
          st.p_nacc = sacc;
          st.p_nrej = srej;
          if (sstat != PHC_PATH_SUCCESS)
            pc = PC_FINISH;
          else if (!O.so.use_endgame)
            pc = PC_CL_START;
          else
            pc = PC_EG_INIT;
          break;

        // ---------------- cauchy_endgame, src/endgame.f90:124-267 --------------
        case PC_EG_INIT:
          st.eg_segstep = 1.0;  // segopts: step_init = step_max = 1, grow_after = 2
          st.eg_status = PHC_ENDGAME_FAILED;
          STV(resz, z);
          st.r = EO.t_start;
          st.have_prev = 0;
          st.best_resid = kHuge;
          st.gate = 0;
          st.dprev = -1.0;
          st.cest = -1.0;
          st.cest_prev = -1.0;
          st.max_loops = EO.max_winding;
          st.eg_wind = 0;
          st.eg_error = kHuge;
          st.eg_residual = kHuge;
          st.eg_radius = 0.0;
          st.eg_nacc = 0;
          st.eg_nrej = 0;
          pc = PC_EG_TOP;
          break;

        case PC_EG_TOP:
          if (st.gate || st.r < EO.loop_radius) {
            if (!st.gate) st.max_loops = EO.max_winding;
            st.lp_max = st.max_loops;
            st.lp_cont = PC_EG_AFTER_LOOPS;
            pc = PC_LOOPS_BEGIN;
          } else {
            st.lp_ok = 0;
            pc = PC_EG_AFTER_LOOPS;
          }
          break;

        case PC_EG_AFTER_LOOPS:
          if (!st.lp_ok) {
            st.have_prev = 0;
            st.gate = 0;
            pc = PC_EG_RADIAL;
          } else {
            st.rec_cont = PC_EG_AFTER_RECORD_MAIN;
            pc = PC_RECORD;
          }
          break;

        case PC_EG_AFTER_RECORD_MAIN:
          if (st.eg_status == PHC_ENDGAME_CONVERGED) {
            pc = PC_EG_DONE;
          } else {
            STV(prev, LDV(est));
            st.have_prev = 1;
            pc = PC_EG_RADIAL;
          }
          break;

        case PC_EG_RADIAL: {
          const double rnew = EO.radius_factor * st.r;
          st.rnew = rnew;
          if (rnew < EO.radius_min) {
            pc = PC_EG_DONE;
            break;
          }
          STV(zold, z);
          zs = z;
          st.seg_arc = 0;
          st.seg_t0[0] = st.r;
          st.seg_t0[1] = 0.0;
          st.seg_t1[0] = rnew;
          st.seg_t1[1] = 0.0;
          st.o_step_init = st.eg_segstep;
          st.o_step_max = 1.0;
          st.o_grow = 2;
          st.seg_cont = PC_EG_AFTER_RADIAL;
          pc = PC_SEG_BEGIN;
          break;
        }

        case PC_EG_AFTER_RADIAL: {
          z = zs;
          st.eg_segstep = fmin(fmax(step, TO.step_min), 1.0);
          st.eg_nacc += sacc;
          st.eg_nrej += srej;
          const cd zold = LDV(zold);
          if (sstat != PHC_PATH_SUCCESS) {
            z = zold;
            if (!(st.gate || st.r < EO.loop_radius)) {
              st.lp_max = EO.max_winding;
              st.lp_cont = PC_EG_AFTER_FALLBACK;
              pc = PC_LOOPS_BEGIN;
            } else {
              pc = PC_EG_DONE;
            }
            break;
          }
          st.r = st.rnew;
          // winding number estimate from the radial differences
          const double d = vnorm(z - zold, lane, N);
          const double dprev = st.dprev;
          if (!st.gate && dprev > 0.0 && d > 0.0) {
            const double cest_prev = st.cest;
            double cest = -1.0;
            if (dprev > d) cest = log(1.0 / EO.radius_factor) / log(dprev / d);
            st.cest_prev = cest_prev;
            st.cest = cest;
            if (cest >= 0.5 && cest <= (double)EO.max_winding + 0.5 && cest_prev > 0.0) {
              if (fabs(cest - cest_prev) <= EO.winding_agreement * fmax(1.0, cest)) {
                st.gate = 1;
                st.max_loops = min(EO.max_winding, 2 * (int)llround(cest) + 2);
              }
            }
          }
          st.dprev = d;
          pc = PC_EG_TOP;
          break;
        }

        case PC_EG_AFTER_FALLBACK:
          st.have_prev = 0;
          if (st.lp_ok) {
            st.rec_cont = PC_EG_DONE;
            pc = PC_RECORD;
          } else {
            pc = PC_EG_DONE;
          }
          break;

        case PC_LOOPS_BEGIN:
          st.lp_dth = 2.0 * kPi / (double)EO.nsamples;
          st.lp_floor = 10.0 * TO.corrector_tol * vnorm(z, lane, N);
          zs = z;
          STV(zsum, czero<double>());
          st.lp_nsamp = 0;
          st.lp_spacing = kHuge;
          st.lp_c = 1;
          st.lp_j = 1;
          pc = PC_LOOP_ARC;
          break;

        case PC_LOOP_ARC:
          STV(zsum, LDV(zsum) + zs);
          ++st.lp_nsamp;
          STV(zprev, zs);
          st.seg_arc = 1;
          st.seg_r = st.r;
          st.seg_th0 = (double)(st.lp_j - 1) * st.lp_dth;
          st.seg_dth = st.lp_dth;
          st.o_step_init = st.eg_segstep;
          st.o_step_max = 1.0;
          st.o_grow = 2;
          st.seg_cont = PC_LOOP_AFTER_ARC;
          pc = PC_SEG_BEGIN;
          break;

        case PC_LOOP_AFTER_ARC: {
          st.eg_segstep = fmin(fmax(step, TO.step_min), 1.0);
          st.eg_nacc += sacc;
          st.eg_nrej += srej;
          if (sstat != PHC_PATH_SUCCESS) {
            st.lp_ok = 0;
            pc = st.lp_cont;
            break;
          }
          st.lp_spacing = fmin(st.lp_spacing, vnorm(zs - LDV(zprev), lane, N));
          const int j = st.lp_j + 1;
          st.lp_j = j;
          if (j <= EO.nsamples) {
            pc = PC_LOOP_ARC;
            break;
          }
          if (vnorm(zs - z, lane, N) <= fmax(EO.closure_factor * st.lp_spacing, st.lp_floor)) {
            const double inv = (double)st.lp_nsamp;
            const cd zsum = LDV(zsum);
            STV(est, mkc<double>(zsum.re / inv, zsum.im / inv));
            st.cw = st.lp_c;
            st.lp_ok = 1;
            pc = st.lp_cont;
            break;
          }
          const int c = st.lp_c + 1;
          st.lp_c = c;
          st.lp_j = 1;
          if (c <= st.lp_max) {
            pc = PC_LOOP_ARC;
          } else {
            st.lp_ok = 0;
            pc = st.lp_cont;
          }
          break;
        }

        case PC_RECORD: {  // record(), src/endgame.f90:240-265
          const cd est = LDV(est);
          double err = kHuge;
          if (st.have_prev)
            err = vnorm(est - LDV(prev), lane, N) / fmax(vnorm(est, lane, N), kTiny);
          st.rec_err = err;
          uk = UK_BACKERR;
          u_prec = 0;
          zin = est;
          tin = czero<double>();
          dtin = czero<double>();
          pc_after = PC_RECORD_AFTER;
          want = true;
          break;
        }

        case PC_RECORD_AFTER: {
          ++st.c_eval;
          const double err = st.rec_err;
          const double resid = U.a1 / fmax(U.a2 * vnorm(zin, lane, N), kTiny);
          if (st.eg_status == PHC_ENDGAME_FAILED ||
              better(resid, err, st.best_resid, st.eg_error, EO.residual_tol)) {
            st.eg_status = PHC_ENDGAME_NOT_CONVERGED;
            STV(resz, zin);
            st.eg_wind = st.cw;
            st.eg_error = err;
            st.eg_residual = resid;
            st.eg_radius = st.r;
            st.best_resid = resid;
          }
          if (err <= EO.tol && resid <= EO.residual_tol) st.eg_status = PHC_ENDGAME_CONVERGED;
          pc = st.rec_cont;
          break;
        }

        case PC_EG_DONE:
          st.p_nacc += st.eg_nacc;
          st.p_nrej += st.eg_nrej;
          if (st.eg_status == PHC_ENDGAME_FAILED) {
            st.p_status = PHC_PATH_ENDGAME_FAILED;
            pc = PC_FINISH;
          } else {
            z = LDV(resz);
            st.p_t = 0.0;
            st.p_wind = st.eg_wind;
            st.p_egs = st.eg_status;
            st.p_ege = st.eg_error;
            pc = PC_CL_START;
          }
          break;

        // ---------------- classify, src/solve.f90:288-328 ---------------------
        case PC_CL_START:
          uk = UK_COND;
          u_prec = 0;
          zin = z;
          tin = czero<double>();
          dtin = czero<double>();
          st.cond_c0 = 0;
          st.cond_ret = PC_CL_AFTER_COND1;
          pc_after = PC_COND_STEP;
          want = true;
          break;

        // cond1 (src/linalg.f90:135-174) chunk by chunk: ||A||_1 from the
        // first unit, the largest column sum of A^-1 over all chunks
        case PC_COND_STEP: {
          const int c0 = st.cond_c0;
          if (c0 == 0) st.cond_anorm = U.a1;
          if (!U.ok) {
            U.a1 = kHuge;  // huge(1.0_wp) for an exactly singular matrix
            pc = st.cond_ret;
            break;
          }
          const double ainv = (c0 == 0) ? U.a2 : fmax(st.cond_ainv, U.a2);
          st.cond_ainv = ainv;
          if (c0 + kCondChunk < N) {
            st.cond_c0 = c0 + kCondChunk;
            uk = UK_COND;
            pc_after = PC_COND_STEP;
            want = true;
            break;
          }
          U.a1 = st.cond_anorm * ainv;
          U.ok = true;
          pc = st.cond_ret;
          break;
        }

        case PC_CL_AFTER_COND1: {
          ++st.c_eval;
          ++st.c_cond;
          st.p_cond = U.a1;
          STV(hsave, U.h);
          const bool sing = st.p_wind > 1 || U.a1 > O.so.singular_cond;
          st.p_sing = sing ? 1 : 0;
          if (!sing && O.so.refine_maxit >= 1) {
            // refine, src/solve.f90:254-286
            st.rf_it = 1;
            dnorm_prev = kHuge;
            uk = UK_REFINE;
            zin = z;
            pc_after = PC_CL_AFTER_REFINE;
            want = true;
          } else {
            pc = sing ? PC_CL_FINAL : PC_CL_COND2;
          }
          break;
        }

        case PC_CL_AFTER_REFINE: {
          ++st.c_ref;
          if (!U.ok) {
            pc = PC_CL_COND2;
            break;
          }
          const double dnorm = vnorm(U.x, lane, N);
          if (dnorm > dnorm_prev) {
            pc = PC_CL_COND2;
            break;
          }
          z = z + U.x;
          if (dnorm <= 4.0 * kEps * vnorm(z, lane, N)) {
            pc = PC_CL_COND2;
            break;
          }
          dnorm_prev = dnorm;
          const int it = st.rf_it + 1;
          st.rf_it = it;
          if (it > O.so.refine_maxit) {
            pc = PC_CL_COND2;
            break;
          }
          uk = UK_REFINE;
          zin = z;
          pc_after = PC_CL_AFTER_REFINE;
          want = true;
          break;
        }

        case PC_CL_COND2:
          uk = UK_COND;
          u_prec = 0;
          zin = z;
          st.cond_c0 = 0;
          st.cond_ret = PC_CL_AFTER_COND2;
          pc_after = PC_COND_STEP;
          want = true;
          break;

        case PC_CL_AFTER_COND2:
          ++st.c_eval;
          ++st.c_cond;
          st.p_cond = U.a1;
          STV(hsave, U.h);
          pc = PC_CL_FINAL;
          break;

        case PC_CL_FINAL: {
          const double znorm = vnorm(z, lane, N);
          const double ri =
              (lane < n) ? cabs(LDV(hsave)) / rpowi(znorm, P.deg[lane]) : 0.0;
          st.p_resid = warp_max_nonneg(ri);
          const cd w = shfl(z, n);
          const bool atinf =
              cabs(w) <= fmax(O.so.infinity_tol, 10.0 * fmin(st.p_ege, 1.0e-4)) * znorm;
          st.p_atinf = atinf ? 1 : 0;
          if (!atinf) {
            // x = z(1:n)/w, src/solve.f90:322-326
            const cd xv = (lane < n) ? cdiv(z, w) : czero<double>();
            STV(xv, xv);
            const double imax = warp_max_nonneg(lane < n ? fabs(xv.im) : 0.0);
            const double xnorm = vnorm(xv, lane, n);
            st.p_real = (imax <= O.so.real_tol * fmax(1.0, xnorm)) ? 1 : 0;
          }
          pc = PC_FINISH;
          break;
        }

        case PC_FINISH: {
          __syncwarp();
          if (lane == 0) {
            phc_path_out o;
            o.status = st.p_status;
            o.winding_number = st.p_wind;
            o.endgame_status = st.p_egs;
            o.at_infinity = st.p_atinf;
            o.singular = st.p_sing;
            o.is_real = st.p_real;
            o.naccepted = st.p_nacc;
            o.nrejected = st.p_nrej;
            o.solution_index = 0;
            o.singular_index = 0;
            o.n_tangent = st.c_tan;
            o.n_newton = st.c_new;
            o.n_refine = st.c_ref;
            o.n_eval = st.c_eval;
            o.n_cond = st.c_cond;
            o.n_fp64_retry = st.c_retry;
            o.t = st.p_t;
            o.endgame_error = st.p_ege;
            o.cond = st.p_cond;
            o.residual = st.p_resid;
            *st.rec = o;
          }
          double* zo_ = st.zo;
          double* xo_ = st.xo;
          if (lane < N) {
            zo_[2 * lane] = z.re;
            zo_[2 * lane + 1] = z.im;
          }
          if (xo_ != nullptr && lane < n) {
            const cd xv = LDV(xv);
            xo_[2 * lane] = xv.re;
            xo_[2 * lane + 1] = xv.im;
          }
          __syncwarp();
          return;
        }
      }
    }
    // ---- run the requested unit ----
    if constexpr (LEAN) {
      // the path's state goes to the warp state for the unit's duration
      STV(z, z);
      STV(zs, zs);
      STV(zp, zp);
      STV(ksum, ksum);
      st.s = s;
      st.step = step;
      st.ds = ds;
      st.sn = sn;
      st.dnorm_prev = dnorm_prev;
      st.tin[0] = tin.re;
      st.tin[1] = tin.im;
      st.dtin[0] = dtin.re;
      st.dtin[1] = dtin.im;
      st.nsucc = nsucc;
      st.sacc = sacc;
      st.srej = srej;
      st.sstat = sstat;
      st.stage = stage;
      st.att64 = att64 ? 1 : 0;
      st.uk = uk;
      st.pc_after = pc_after;
      st.u_prec = u_prec;
      {
        const WarpConst C = load_warp_const(P, tbl, lane);
        const WarpWS ws = warp_workspace<EVAL32>(P, wbase);
        run_unit<NM, kMixed, EVAL32, F>(tbl, C, ws, uk, kMixed ? u_prec : 0, st.cond_c0, zin,
                                        tin, dtin, lane, U);
      }
      z = LDV(z);
      zs = LDV(zs);
      zp = LDV(zp);
      ksum = LDV(ksum);
      s = st.s;
      step = st.step;
      ds = st.ds;
      sn = st.sn;
      dnorm_prev = st.dnorm_prev;
      tin = mkc<double>(st.tin[0], st.tin[1]);
      dtin = mkc<double>(st.dtin[0], st.dtin[1]);
      nsucc = st.nsucc;
      sacc = st.sacc;
      srej = st.srej;
      sstat = st.sstat;
      stage = st.stage;
      att64 = st.att64 != 0;
      uk = st.uk;
      u_prec = st.u_prec;
      pc_after = st.pc_after;
    } else {
      run_unit<NM, kMixed, EVAL32, F>(tbl, C0, ws0, uk, kMixed ? u_prec : 0, st.cond_c0, zin,
                                      tin, dtin, lane, U);
    }
    if (kMixed && u_prec == 0 && uk <= UK_NEWTON) ++st.c_retry;  // predictor/corrector unit in FP64
    ++st.units;
    pc = pc_after;
  }
}

#undef LV
#undef LDV
#undef STV

// Structural zeros of the Jacobian are never written by the schedule, so
// the buffer is cleared once per system; row n holds the patch a (the last
// row of H_z).
template <bool EVAL32>
__device__ __forceinline__ void init_jacobian_buffer(const PlanHeader& P, unsigned char* wbase,
                                                     int lane) {
  const WarpWS ws = warp_workspace<EVAL32>(P, wbase);
  for (int q = lane; q < (P.n + 1) * P.S; q += kWarp) {
    const int row = q / P.S, col = q - row * P.S;
    cd v = czero<double>();
    if (row == P.n && col < P.N) v = mkc<double>(P.patch[col][0], P.patch[col][1]);
    sts(&ws.jd[q], v);
    if (EVAL32) sts(&ws.jf[q], ccast<float>(v));
  }
  __syncwarp();
}

// Threads per block the kernels of a row width and form are compiled for.
template <int NM, bool LEAN>
constexpr int kMaxBlockThreads = max_warps_per_block(NM, LEAN) * kWarp;

// Single-system kernel: every block stages the table once for its warps.
template <int NM, int PREC, int F, bool LEAN>
__global__ void __launch_bounds__(kMaxBlockThreads<NM, LEAN>) track_kernel(const KParams kp) {
  extern __shared__ __align__(16) unsigned char smem[];
  // the single-system kernels of narrow rows carry the FP32 evaluation
  constexpr bool E32 = kernel_eval32(NM, PREC);
  const int tid = threadIdx.x;
  {
    const int4* src = reinterpret_cast<const int4*>(kp.plan);
    int4* dst = reinterpret_cast<int4*>(smem);
    const int nv = kp.plan_bytes >> 4;
    for (int q = tid; q < nv; q += blockDim.x) dst[q] = src[q];
  }
  __syncthreads();
  const PlanHeader& P = *reinterpret_cast<const PlanHeader*>(smem);
  const int warp = tid >> 5, lane = tid & 31;
  unsigned char* wbase = smem + kp.plan_bytes + warp * kp.ws_bytes;
  WarpState* stp = warp_state<E32>(P, wbase);
  init_jacobian_buffer<E32>(P, wbase, lane);
  // one call site of the path state machine: a persistent warp pulls paths
  // from the atomic queue, a grid warp takes exactly one
  long long q = -1, qend = 0;
  for (;;) {
    if (q + 1 < qend) {
      ++q;
    } else if (kp.persistent) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(kp.counter, (unsigned long long)kp.chunk);
      base = __shfl_sync(kFull, base, 0);
      if (base >= (unsigned long long)kp.count) break;
      q = (long long)base;
      qend = min((long long)base + kp.chunk, (long long)kp.count);
    } else {
      if (qend != 0) break;
      q = (long long)blockIdx.x * kp.warps + warp;
      qend = q + 1;
      if (q >= kp.count) break;
    }
    const int n = P.n, N = P.N;
    track_one<NM, PREC, E32, F, LEAN>(smem, wbase, *stp, kp.opts, kp.k0 + q, lane, kp.out + q,
                                      kp.z + 2 * q * N, kp.x ? kp.x + 2 * q * n : nullptr);
    if (kp.done != nullptr) {
      // every lane's result stores are made visible system-wide before the
      // path is flagged
      __threadfence_system();
      __syncwarp();
      if (lane == 0) atomicExch_system(&kp.done[q], 1u);
    }
  }
}

// Batched kernel: the paths of many systems (different n, degrees and
// options) in one launch. Persistent warps pull global path indices from
// one queue; a warp that moves on to another system stages that system's
// table and options into its own shared-memory slice.
template <int NM, int PREC, int F, bool LEAN>
__global__ void __launch_bounds__(kMaxBlockThreads<NM, LEAN>)
    track_batch_kernel(const KParamsBatch kb) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* slice = smem + warp * kb.slice_bytes;
  unsigned char* tbl = slice;
  unsigned char* wbase = slice + kb.table_cap;
  KOpts* opts = reinterpret_cast<KOpts*>(wbase + kb.ws_cap);
  int cur = -1;
  long long q = -1, qend = 0;
  for (;;) {
    if (q + 1 < qend) {
      ++q;
    } else {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(kb.counter, (unsigned long long)kb.chunk);
      base = __shfl_sync(kFull, base, 0);
      if (base >= (unsigned long long)kb.total_paths) break;
      q = (long long)base;
      qend = min((long long)base + kb.chunk, (long long)kb.total_paths);
    }
    // the request owning global path q (uniform binary search)
    int lo = 0, hi = kb.nsys - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (kb.sys[mid].path_begin <= q)
        lo = mid;
      else
        hi = mid - 1;
    }
    const BatchSys& S = kb.sys[lo];
    if (lo != cur) {
      cur = lo;
      __syncwarp();
      const int4* src = reinterpret_cast<const int4*>(kb.base + S.table_off);
      int4* dst = reinterpret_cast<int4*>(tbl);
      for (int v = lane; v < (S.table_bytes >> 4); v += kWarp) dst[v] = src[v];
      static_assert(sizeof(KOpts) % 8 == 0, "KOpts is copied in 8-byte words");
      const unsigned long long* osrc = reinterpret_cast<const unsigned long long*>(&S.opts);
      unsigned long long* odst = reinterpret_cast<unsigned long long*>(opts);
      for (int v = lane; v < (int)(sizeof(KOpts) >> 3); v += kWarp) odst[v] = osrc[v];
      __syncwarp();
      init_jacobian_buffer<false>(*reinterpret_cast<const PlanHeader*>(tbl), wbase, lane);
    }
    const PlanHeader& P = *reinterpret_cast<const PlanHeader*>(tbl);
    WarpState* stp = warp_state<false>(P, wbase);
    const long long kl = q - S.path_begin;  // 0-based path of the request
    const int n = P.n, N = P.N;
    phc_path_out* out = reinterpret_cast<phc_path_out*>(kb.base + S.out_off) + kl;
    double* z = reinterpret_cast<double*>(kb.base + S.z_off) + 2 * kl * N;
    double* x = S.x_off >= 0 ? reinterpret_cast<double*>(kb.base + S.x_off) + 2 * kl * n : nullptr;
    track_one<NM, PREC, false, F, LEAN>(tbl, wbase, *stp, *opts, kl + 1, lane, out, z, x);
    if (kb.done != nullptr) {
      // every lane's result stores are made visible system-wide before the
      // path is counted as finished
      __threadfence_system();
      __syncwarp();
      if (lane == 0) atomicAdd_system(&kb.done[lo], 1u);
    }
  }
}

}  // namespace phc

// Host-side launch and occupancy helpers of one register-row width NM,
// defined in the instantiation units track_nm*.cu.
// mode: bit 0 the precision (PHC_PREC_*), (mode / 2) % 3 + 1 the schedule
// form, mode / 6 the lean form (kernel_mode in phc_host.h)
#define PHC_FOR_MODES(MACRO, NMV, ...)                                            \
  switch (mode) {                                                                 \
    case 0: MACRO(NMV, PHC_PREC_FP64, 1, false, __VA_ARGS__); break;              \
    case 1: MACRO(NMV, PHC_PREC_MIXED, 1, false, __VA_ARGS__); break;             \
    case 2: MACRO(NMV, PHC_PREC_FP64, 2, false, __VA_ARGS__); break;              \
    case 3: MACRO(NMV, PHC_PREC_MIXED, 2, false, __VA_ARGS__); break;             \
    case 4: MACRO(NMV, PHC_PREC_FP64, 3, false, __VA_ARGS__); break;              \
    case 5: MACRO(NMV, PHC_PREC_MIXED, 3, false, __VA_ARGS__); break;             \
    case 6: MACRO(NMV, PHC_PREC_FP64, 1, true, __VA_ARGS__); break;               \
    case 7: MACRO(NMV, PHC_PREC_MIXED, 1, true, __VA_ARGS__); break;              \
    case 8: MACRO(NMV, PHC_PREC_FP64, 2, true, __VA_ARGS__); break;               \
    case 9: MACRO(NMV, PHC_PREC_MIXED, 2, true, __VA_ARGS__); break;              \
    case 10: MACRO(NMV, PHC_PREC_FP64, 3, true, __VA_ARGS__); break;              \
    default: MACRO(NMV, PHC_PREC_MIXED, 3, true, __VA_ARGS__); break;             \
  }
#define PHC_SET_ATTR(NMV, PR, FF, LN, smax)                                        \
  cudaFuncSetAttribute(track_kernel<NMV, PR, FF, LN>,                             \
                       cudaFuncAttributeMaxDynamicSharedMemorySize, smax);        \
  cudaFuncSetAttribute(track_batch_kernel<NMV, PR, FF, LN>,                       \
                       cudaFuncAttributeMaxDynamicSharedMemorySize, smax)
#define PHC_LAUNCH(NMV, PR, FF, LN, K, P)                                          \
  K<NMV, PR, FF, LN><<<grid, block, smem, s>>>(P)
#define PHC_OCC(NMV, PR, FF, LN, K)                                                \
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, K<NMV, PR, FF, LN>, block, smem)

#define PHC_DEFINE_NM(NMV)                                                        \
  namespace phc {                                                                 \
  static void set_smem_attr_##NMV() {                                             \
    static int done[64] = {0};                                                    \
    int dev = 0;                                                                  \
    cudaGetDevice(&dev);                                                          \
    if (dev >= 0 && dev < 64 && !done[dev]) {                                     \
      int smax = 0;                                                               \
      cudaDeviceGetAttribute(&smax, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev); \
      for (int mode = 0; mode < 12; ++mode) {                                     \
        PHC_FOR_MODES(PHC_SET_ATTR, NMV, smax)                                    \
      }                                                                           \
      done[dev] = 1;                                                              \
    }                                                                             \
  }                                                                               \
  cudaError_t launch_nm_##NMV(int mode, const KParams& kp, int grid, int block,   \
                              int smem, cudaStream_t s) {                         \
    set_smem_attr_##NMV();                                                        \
    PHC_FOR_MODES(PHC_LAUNCH, NMV, track_kernel, kp)                              \
    return cudaGetLastError();                                                    \
  }                                                                               \
  cudaError_t launch_batch_nm_##NMV(int mode, const KParamsBatch& kb, int grid,   \
                                    int block, int smem, cudaStream_t s) {       \
    set_smem_attr_##NMV();                                                        \
    PHC_FOR_MODES(PHC_LAUNCH, NMV, track_batch_kernel, kb)                        \
    return cudaGetLastError();                                                    \
  }                                                                               \
  int occupancy_batch_nm_##NMV(int mode, int block, int smem) {                   \
    set_smem_attr_##NMV();                                                        \
    int nb = 0;                                                                   \
    cudaError_t e = cudaSuccess;                                                  \
    PHC_FOR_MODES(PHC_OCC, NMV, track_batch_kernel)                               \
    return e == cudaSuccess ? nb : 0;                                             \
  }                                                                               \
  int occupancy_nm_##NMV(int mode, int block, int smem) {                         \
    set_smem_attr_##NMV();                                                        \
    int nb = 0;                                                                   \
    cudaError_t e = cudaSuccess;                                                  \
    PHC_FOR_MODES(PHC_OCC, NMV, track_kernel)                                     \
    return e == cudaSuccess ? nb : 0;                                             \
  }                                                                               \
  }


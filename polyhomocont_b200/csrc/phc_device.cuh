// phc_device.cuh -- warp-level building blocks of the B200 path tracker:
// complex arithmetic, warp reductions, the sparse evaluation of the
// homotopy H(z,t) and its Jacobian, and a complex LU with partial
// pivoting in which lane i owns row i.
//
// Layout in a warp (N = n + 1 <= 32 unknowns, projective coordinates with
// w last): vector component j lives in lane j; row i of the N x N matrix
// H_z lives in the registers of lane i (a[0..NM-1], NM = compile-time
// capacity >= N). Lanes >= N hold zeros and take part in all collective
// operations, so control flow stays warp-uniform.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "phc_internal.h"

namespace phc {

constexpr unsigned kFull = 0xffffffffu;

// Compile-time loop: calls f(std::integral_constant<int, K>) for K = B..E-1,
// so that register arrays are always indexed by constants.
template <int B, int E>
struct StaticFor {
  template <typename F>
  __device__ __forceinline__ static void run(F&& f) {
    if constexpr (B < E) {
      f(std::integral_constant<int, B>{});
      StaticFor<B + 1, E>::run(f);
    }
  }
};

template <typename T>
struct cpx {
  T re;
  T im;
};
using cd = cpx<double>;
using cf = cpx<float>;

template <typename T>
__device__ __forceinline__ cpx<T> mkc(T r, T i) {
  cpx<T> c;
  c.re = r;
  c.im = i;
  return c;
}
template <typename T>
__device__ __forceinline__ cpx<T> czero() {
  return mkc<T>(T(0), T(0));
}
template <typename T>
__device__ __forceinline__ cpx<T> cone() {
  return mkc<T>(T(1), T(0));
}
template <typename T>
__device__ __forceinline__ cpx<T> operator+(cpx<T> a, cpx<T> b) {
  return mkc<T>(a.re + b.re, a.im + b.im);
}
template <typename T>
__device__ __forceinline__ cpx<T> operator-(cpx<T> a, cpx<T> b) {
  return mkc<T>(a.re - b.re, a.im - b.im);
}
template <typename T>
__device__ __forceinline__ cpx<T> operator-(cpx<T> a) {
  return mkc<T>(-a.re, -a.im);
}
template <typename T>
__device__ __forceinline__ cpx<T> operator*(cpx<T> a, cpx<T> b) {
  return mkc<T>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename T>
__device__ __forceinline__ cpx<T> operator*(T s, cpx<T> a) {
  return mkc<T>(s * a.re, s * a.im);
}
// Complex division by Smith's method (R. L. Smith, CACM 5 (1962) 435),
// the range-reducing division of Fortran compilers.
template <typename T>
__device__ __forceinline__ cpx<T> cdiv(cpx<T> a, cpx<T> b) {
  if (fabs(b.re) < fabs(b.im)) {
    T ratio = b.re / b.im;
    T den = b.re * ratio + b.im;
    return mkc<T>((a.re * ratio + a.im) / den, (a.im * ratio - a.re) / den);
  }
  T ratio = b.im / b.re;
  T den = b.im * ratio + b.re;
  return mkc<T>((a.im * ratio + a.re) / den, (a.im - a.re * ratio) / den);
}
__device__ __forceinline__ double cabs(cd a) { return hypot(a.re, a.im); }
__device__ __forceinline__ float cabs(cf a) { return hypotf(a.re, a.im); }

template <typename T, typename U>
__device__ __forceinline__ cpx<T> ccast(cpx<U> a) {
  return mkc<T>((T)a.re, (T)a.im);
}

// z**k, k >= 0, by square and multiply
template <typename T>
__device__ __forceinline__ cpx<T> cpowi(cpx<T> x, int k) {
  cpx<T> p = cone<T>();
  unsigned u = (unsigned)k;
  while (u) {
    if (u & 1u) p = p * x;
    u >>= 1;
    if (u) x = x * x;
  }
  return p;
}
// real**m, m >= 0, by square and multiply (low bit first)
__device__ __forceinline__ double rpowi(double x, int m) {
  unsigned n = (unsigned)m;
  double y = (n & 1u) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n & 1u) y = y * x;
  }
  return y;
}

// ---- shared-memory typed access -------------------------------------------
__device__ __forceinline__ cd lds(const cd* p) {
  double2 v = *reinterpret_cast<const double2*>(p);
  return mkc<double>(v.x, v.y);
}
__device__ __forceinline__ cf lds(const cf* p) {
  float2 v = *reinterpret_cast<const float2*>(p);
  return mkc<float>(v.x, v.y);
}
__device__ __forceinline__ void sts(cd* p, cd v) {
  *reinterpret_cast<double2*>(p) = make_double2(v.re, v.im);
}
__device__ __forceinline__ void sts(cf* p, cf v) {
  *reinterpret_cast<float2*>(p) = make_float2(v.re, v.im);
}

// ---- warp collectives -----------------------------------------------------
template <typename T>
__device__ __forceinline__ cpx<T> shfl(cpx<T> v, int src) {
  return mkc<T>(__shfl_sync(kFull, v.re, src), __shfl_sync(kFull, v.im, src));
}

// Maximum over the warp of a value v >= +0 (moduli). The bit patterns of
// non-negative doubles order like the values, so the maximum is taken on
// the high and then the low 32 bits with redux.sync; every lane gets the
// same result.
__device__ __forceinline__ double warp_max_nonneg(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  unsigned hi = (unsigned)(b >> 32), lo = (unsigned)b;
  unsigned mhi = __reduce_max_sync(kFull, hi);
  unsigned mlo = __reduce_max_sync(kFull, hi == mhi ? lo : 0u);
  return __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
}
__device__ __forceinline__ float warp_max_nonneg(float v) {
  return __uint_as_float(__reduce_max_sync(kFull, __float_as_uint(v)));
}
// Sum over the warp; the tree result of lane 0 is broadcast so that every
// lane holds bit-identical values (control decisions stay uniform).
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
  return __shfl_sync(kFull, v, 0);
}
template <typename T>
__device__ __forceinline__ cpx<T> warp_csum(cpx<T> v) {
  return mkc<T>(warp_sum(v.re), warp_sum(v.im));
}

// First lane (lowest index) among the candidates with the largest key
// (key >= 0); kmax receives the largest key. Mirrors the strict '>' scan of
// lu_factor (src/linalg.f90:51-58), which keeps the first maximum.
__device__ __forceinline__ int warp_argmax_first(double key, bool cand, double& kmax) {
  unsigned long long b = cand ? (unsigned long long)__double_as_longlong(key) : 0ull;
  unsigned hi = (unsigned)(b >> 32), lo = (unsigned)b;
  unsigned mhi = __reduce_max_sync(kFull, hi);
  bool c1 = cand && hi == mhi;
  unsigned mlo = __reduce_max_sync(kFull, c1 ? lo : 0u);
  unsigned m = __ballot_sync(kFull, c1 && lo == mlo);
  kmax = __longlong_as_double((long long)(((unsigned long long)mhi << 32) | mlo));
  return m ? __ffs(m) - 1 : -1;
}
__device__ __forceinline__ int warp_argmax_first(float key, bool cand, float& kmax) {
  unsigned b = cand ? __float_as_uint(key) : 0u;
  unsigned mx = __reduce_max_sync(kFull, b);
  unsigned m = __ballot_sync(kFull, cand && b == mx);
  kmax = __uint_as_float(mx);
  return m ? __ffs(m) - 1 : -1;
}

// ---- per-warp workspace -------------------------------------------------------
struct WarpWS {
  cd* pwd;   // power table z_j^e, FP64
  cf* pwf;   // power table, FP32 (mixed precision only)
  cd* fvd;   // F^h values
  cf* fvf;
  cd* jd;    // Jacobian of F^h, row-major, stride S
  cf* jf;
  cd* prow;  // pivot-row broadcast buffer (FP32 rows use it as cf*)
};

template <typename T> __device__ __forceinline__ cpx<T>* ws_pw(const WarpWS& w);
template <> __device__ __forceinline__ cd* ws_pw<double>(const WarpWS& w) { return w.pwd; }
template <> __device__ __forceinline__ cf* ws_pw<float>(const WarpWS& w) { return w.pwf; }
template <typename T> __device__ __forceinline__ cpx<T>* ws_fv(const WarpWS& w);
template <> __device__ __forceinline__ cd* ws_fv<double>(const WarpWS& w) { return w.fvd; }
template <> __device__ __forceinline__ cf* ws_fv<float>(const WarpWS& w) { return w.fvf; }
template <typename T> __device__ __forceinline__ cpx<T>* ws_j(const WarpWS& w);
template <> __device__ __forceinline__ cd* ws_j<double>(const WarpWS& w) { return w.jd; }
template <> __device__ __forceinline__ cf* ws_j<float>(const WarpWS& w) { return w.jf; }

// ---- sparse evaluation ----------------------------------------------------
// Power table of lane j's coordinate: pw[e*N + j] = z_j^e, e = 0..maxexp,
// by repeated multiplication (src/sparse.f90:251-255).
template <typename T>
__device__ __forceinline__ void power_table(const PlanHeader& P, cpx<T>* pw, cpx<T> zj,
                                            int lane) {
  if (lane < P.N) {
    cpx<T> p = cone<T>();
    sts(&pw[lane], p);
    for (int e = 1; e <= P.maxexp; ++e) {
      p = p * zj;
      sts(&pw[e * P.N + lane], p);
    }
  }
}

// Runs one schedule: lane sums the contributions of its entries and stores
// each sum once into out[dest].
template <typename T>
__device__ __forceinline__ void run_schedule(const Rec* recs, int rbeg, int rend,
                                             const cpx<T>* pw, cpx<T>* out) {
  cpx<T> acc = czero<T>();
  cpx<T> carry = czero<T>();
  for (int r = rbeg; r < rend; ++r) {
    const Rec& R = recs[r];
    const uint4 meta = *reinterpret_cast<const uint4*>(&R.dest);  // dest..fac[5]
    const unsigned flags = (meta.x >> 24) & 0xffu;
    const unsigned nf = (meta.x >> 16) & 0xffu;
    const unsigned dest = meta.x & 0xffffu;
    cpx<T> v = (flags & kRecContIn) ? carry : mkc<T>((T)R.cre, (T)R.cim);
    const unsigned f01 = meta.y, f23 = meta.z, f45 = meta.w;
    if (nf > 0) v = v * lds(&pw[f01 & 0xffffu]);
    if (nf > 1) v = v * lds(&pw[f01 >> 16]);
    if (nf > 2) v = v * lds(&pw[f23 & 0xffffu]);
    if (nf > 3) v = v * lds(&pw[f23 >> 16]);
    if (nf > 4) v = v * lds(&pw[f45 & 0xffffu]);
    if (nf > 5) v = v * lds(&pw[f45 >> 16]);
    if (flags & kRecContOut) {
      carry = v;
      continue;
    }
    acc = acc + v;
    if (flags & kRecLast) {
      sts(&out[dest], acc);
      acc = czero<T>();
    }
  }
}

// Homotopy H(z,t) = gamma t G(z) + (1 - t) F^h(z) plus the patch row
// (tdh_evaluate, src/homotopy.f90:188-231). Input: lane j holds z_j.
// Output: lane i holds row i of H_z in a[], and h_i, ht_i.
// TJ is the type of the Jacobian and of the row; f is evaluated in double
// when f64 is set (Newton residuals), else in TJ.
template <int NM, typename TJ>
__device__ __forceinline__ void evaluate(const PlanHeader& P, const Rec* recs,
                                         const WarpWS& ws, cd zl, cd t, int lane,
                                         bool f64, cpx<TJ> (&a)[NM], cd& h, cd& ht) {
  const int n = P.n, N = P.N, S = P.S;
  // power tables
  if (f64 || sizeof(TJ) == 8) power_table<double>(P, ws.pwd, zl, lane);
  if (sizeof(TJ) == 4) power_table<TJ>(P, ws_pw<TJ>(ws), ccast<TJ>(zl), lane);
  __syncwarp();
  const Rec* rf = recs;
  const Rec* rj = recs + P.nrec_f;
  if (f64) {
    run_schedule<double>(rf, P.lane_f[lane], P.lane_f[lane + 1], ws.pwd, ws.fvd);
  } else {
    run_schedule<TJ>(rf, P.lane_f[lane], P.lane_f[lane + 1], ws_pw<TJ>(ws),
                     ws_fv<TJ>(ws));
  }
  run_schedule<TJ>(rj, P.lane_j[lane], P.lane_j[lane + 1], ws_pw<TJ>(ws), ws_j<TJ>(ws));
  __syncwarp();

  const cd gamma = mkc<double>(P.gamma[0], P.gamma[1]);
  const cd gt = gamma * t;
  const cd omt = mkc<double>(1.0 - t.re, -t.im);
  const cd w = shfl(zl, n);
  h = czero<double>();
  ht = czero<double>();
  if (lane < n) {
    const int i = lane;
    const int d = P.deg[i];
    const cd bi = mkc<double>(P.b[i][0], P.b[i][1]);
    const cpx<TJ> omtT = ccast<TJ>(omt);
    const cpx<TJ>* J = ws_j<TJ>(ws) + i * S;
#pragma unroll
    for (int j = 0; j < NM; ++j) a[j] = (j < N) ? omtT * lds(&J[j]) : czero<TJ>();
    if (f64 || sizeof(TJ) == 8) {
      const cd zi = zl;
      const cd zd1 = cpowi(zi, d - 1);
      const cd wd1 = cpowi(w, d - 1);
      const cd g = zd1 * zi - (bi * wd1) * w;
      const cd f = lds(&ws.fvd[i]);
      h = gt * g + omt * f;
      ht = gamma * g - f;
      const cpx<TJ> dg = ccast<TJ>(((double)d * gt) * zd1);
      const cpx<TJ> dw = ccast<TJ>(((double)d * (gt * bi)) * wd1);
#pragma unroll
      for (int j = 0; j < NM; ++j) {
        if (j == i) a[j] = a[j] + dg;
        if (j == n) a[j] = a[j] - dw;
      }
    } else {
      const cpx<TJ> zi = ccast<TJ>(zl);
      const cpx<TJ> wT = ccast<TJ>(w);
      const cpx<TJ> biT = ccast<TJ>(bi);
      const cpx<TJ> gtT = ccast<TJ>(gt);
      const cpx<TJ> zd1 = cpowi(zi, d - 1);
      const cpx<TJ> wd1 = cpowi(wT, d - 1);
      const cpx<TJ> g = zd1 * zi - (biT * wd1) * wT;
      const cpx<TJ> f = lds(&ws_fv<TJ>(ws)[i]);
      h = ccast<double>(gtT * g + omtT * f);
      ht = ccast<double>(ccast<TJ>(gamma) * g - f);
      const cpx<TJ> dg = ((TJ)d * gtT) * zd1;
      const cpx<TJ> dw = ((TJ)d * (gtT * biT)) * wd1;
#pragma unroll
      for (int j = 0; j < NM; ++j) {
        if (j == i) a[j] = a[j] + dg;
        if (j == n) a[j] = a[j] - dw;
      }
    }
  } else if (lane == n) {
#pragma unroll
    for (int j = 0; j < NM; ++j)
      a[j] = (j < N) ? mkc<TJ>((TJ)P.patch[j][0], (TJ)P.patch[j][1]) : czero<TJ>();
  } else {
#pragma unroll
    for (int j = 0; j < NM; ++j) a[j] = czero<TJ>();
  }
  // patch row residual h_n = a . z - 1 (src/homotopy.f90:228)
  cd pz = (lane < N) ? mkc<double>(P.patch[lane][0], P.patch[lane][1]) * zl
                     : czero<double>();
  const cd s = warp_csum(pz);
  if (lane == n) h = mkc<double>(s.re - 1.0, s.im);
}

// ---- LU with partial pivoting, lane i owns row i --------------------------
// Factorizes the N x N matrix held row-wise in a[] (lu_factor,
// src/linalg.f90:26-78) without moving rows: pstep records the step at
// which a lane's row was chosen as pivot row (NM if never), piv packs the
// pivot lane of each step (4 steps per word). Multipliers overwrite a[k] of
// the eliminated rows, U stays in the pivot rows. Returns false for an
// exactly zero pivot column (err_singular_matrix).
template <int NM, typename T>
__device__ __forceinline__ bool lu_rows(cpx<T> (&a)[NM], int N, int lane, int& pstep,
                                        unsigned (&piv)[(NM + 3) / 4], cpx<T>* prow) {
  pstep = NM;
#pragma unroll
  for (int q = 0; q < (NM + 3) / 4; ++q) piv[q] = 0u;
  bool ok = true;
  StaticFor<0, NM>::run([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if (!ok || k >= N) return;
    const bool cand = lane < N && pstep == NM;
    T key = a[k].re * a[k].re + a[k].im * a[k].im;
    T kmax;
    int p = warp_argmax_first(key, cand, kmax);
    if (!(kmax > T(0))) {
      // zero or underflowed squares: decide with the modulus itself
      T m = cand ? cabs(a[k]) : T(0);
      p = warp_argmax_first(m, cand, kmax);
      if (!(kmax > T(0))) {
        ok = false;
        return;
      }
    }
    piv[k >> 2] |= (unsigned)p << (8 * (k & 3));
    if (lane == p) {
      pstep = k;
#pragma unroll
      for (int j = k; j < NM; ++j)
        if (j < N) sts(&prow[j], a[j]);
    }
    __syncwarp();
    if (cand && lane != p) {
      const cpx<T> l = cdiv(a[k], lds(&prow[k]));
      a[k] = l;
#pragma unroll
      for (int j = k + 1; j < NM; ++j)
        if (j < N) a[j] = a[j] - l * lds(&prow[j]);
    }
    __syncwarp();
  });
  return ok;
}

// Solves A x = b with the factors from lu_rows (lu_solve,
// src/linalg.f90:80-114). Lane i passes b_i; lane j returns x_j.
template <int NM, typename T>
__device__ __forceinline__ cpx<T> solve_rows(const cpx<T> (&a)[NM], int N, int lane,
                                             int pstep, const unsigned (&piv)[(NM + 3) / 4],
                                             cpx<T> b) {
  // forward substitution in pivot order (unit lower triangle)
  StaticFor<0, NM>::run([&](auto kc) {
    constexpr int k = decltype(kc)::value;
    if (k >= N) return;
    const int p = (piv[k >> 2] >> (8 * (k & 3))) & 0xff;
    const cpx<T> bp = shfl(b, p);
    if (pstep > k && lane < N) b = b - a[k] * bp;
  });
  // back substitution with U, last pivot first
  cpx<T> x = czero<T>();
  StaticFor<0, NM>::run([&](auto kc) {
    constexpr int k = NM - 1 - decltype(kc)::value;
    if (k >= N) return;
    const int p = (piv[k >> 2] >> (8 * (k & 3))) & 0xff;
    cpx<T> xk = czero<T>();
    if (lane == p) xk = cdiv(b, a[k]);
    xk = shfl(xk, p);
    if (pstep < k) b = b - a[k] * xk;
    if (lane == k) x = xk;
  });
  return x;
}

}  // namespace phc

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
// a - l*b as four fused multiply-adds, two deep per component (the
// separate product and subtraction take six operations, three deep).
__device__ __forceinline__ double fma_(double x, double y, double z) { return fma(x, y, z); }
__device__ __forceinline__ float fma_(float x, float y, float z) { return fmaf(x, y, z); }
template <typename T>
__device__ __forceinline__ cpx<T> cfms(cpx<T> a, cpx<T> l, cpx<T> b) {
  return mkc<T>(fma_(-l.re, b.re, fma_(l.im, b.im, a.re)),
                fma_(-l.re, b.im, fma_(-l.im, b.re, a.im)));
}
// acc + x*y as four fused multiply-adds
template <typename T>
__device__ __forceinline__ cpx<T> cfma(cpx<T> acc, cpx<T> x, cpx<T> y) {
  return mkc<T>(fma_(x.re, y.re, fma_(-x.im, y.im, acc.re)),
                fma_(x.re, y.im, fma_(x.im, y.re, acc.im)));
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
// Real reciprocal for the pivots: the hardware approximation (rcp.approx,
// about 23 correct bits in double) refined by two Newton-Raphson steps
// r <- r + r (1 - d r), which square the relative error each time
// (Newton's method for f(r) = 1/r - d), leaving an error of about one unit
// in the last place for d in [1e-290, 1e290].
__device__ __forceinline__ double rcp_nr(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}
__device__ __forceinline__ float rcp_nr(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  const float e = fmaf(-d, r, 1.0f);
  return fmaf(r, e, r);
}
// 1/a = conj(a)/|a|^2; Smith's division where |a|^2 would underflow or
// overflow.
__device__ __forceinline__ cd crcp(cd a) {
  const double d = a.re * a.re + a.im * a.im;
  if (d >= 1e-290 && d <= 1e290) {
    const double r = rcp_nr(d);
    return mkc<double>(a.re * r, -a.im * r);
  }
  return cdiv(cone<double>(), a);
}
__device__ __forceinline__ cf crcp(cf a) {
  const float d = a.re * a.re + a.im * a.im;
  if (d >= 1e-36f && d <= 1e36f) {
    const float r = rcp_nr(d);
    return mkc<float>(a.re * r, -a.im * r);
  }
  return cdiv(cone<float>(), a);
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

template <typename T>
__device__ __forceinline__ cpx<T> shfl_xor(cpx<T> v, int m) {
  return mkc<T>(__shfl_xor_sync(kFull, v.re, m), __shfl_xor_sync(kFull, v.im, m));
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
// Pivot search in one reduction: the high word of |a|^2 (|a|^2 >= 0, so its
// bit pattern orders like the value) with its low 5 bits replaced by
// 31 - lane; the maximum is the largest key and, among keys equal in the
// leading 15 mantissa bits, the lowest lane (the reference scans rows in
// order and keeps the first maximum). kmax is the key part of the winner
// (0 when every candidate is zero or tiny).
__device__ __forceinline__ int pivot_lane(double key, bool cand, int lane, unsigned& kmax) {
  const unsigned hi = (unsigned)((unsigned long long)__double_as_longlong(key) >> 32);
  const unsigned v = cand ? ((hi & ~31u) | (31u - (unsigned)lane)) : 0u;
  const unsigned m = __reduce_max_sync(kFull, v);
  kmax = m & ~31u;
  return 31 - (int)(m & 31u);
}
__device__ __forceinline__ int pivot_lane(float key, bool cand, int lane, unsigned& kmax) {
  const unsigned b = __float_as_uint(key);
  const unsigned v = cand ? ((b & ~31u) | (31u - (unsigned)lane)) : 0u;
  const unsigned m = __reduce_max_sync(kFull, v);
  kmax = m & ~31u;
  return 31 - (int)(m & 31u);
}
// Coarse variant for pivoting: the key is the high word of |a|^2, so
// candidates that agree in their leading 20 mantissa bits tie and the
// lowest lane wins. Returns -1 with kmax = 0 when every candidate key is 0.
__device__ __forceinline__ int warp_argmax_hi(double key, bool cand, unsigned& kmax) {
  const unsigned hi = cand ? (unsigned)((unsigned long long)__double_as_longlong(key) >> 32) : 0u;
  kmax = __reduce_max_sync(kFull, hi);
  const unsigned m = __ballot_sync(kFull, cand && hi == kmax);
  return m ? __ffs(m) - 1 : -1;
}
__device__ __forceinline__ int warp_argmax_hi(float key, bool cand, unsigned& kmax) {
  const unsigned b = cand ? __float_as_uint(key) : 0u;
  kmax = __reduce_max_sync(kFull, b);
  const unsigned m = __ballot_sync(kFull, cand && b == kmax);
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
  cd* pwd;    // power table z_j^e, FP64
  cf* pwf;    // power table, FP32 (mixed precision only)
  cd* jd;     // Jacobian of F^h, row-major, stride S
  cf* jf;
  int* piv;   // pivot row (lane) of each column
};

template <typename T> __device__ __forceinline__ cpx<T>* ws_pw(const WarpWS& w);
template <> __device__ __forceinline__ cd* ws_pw<double>(const WarpWS& w) { return w.pwd; }
template <> __device__ __forceinline__ cf* ws_pw<float>(const WarpWS& w) { return w.pwf; }
template <typename T> __device__ __forceinline__ cpx<T>* ws_j(const WarpWS& w);
template <> __device__ __forceinline__ cd* ws_j<double>(const WarpWS& w) { return w.jd; }
template <> __device__ __forceinline__ cf* ws_j<float>(const WarpWS& w) { return w.jf; }

// Constants of the system held in registers for the lifetime of a warp. The
// shared-memory table could alias the workspace that the evaluation writes,
// so reading its fields inside the hot loops would reload them after every
// store; these copies are loaded once.
struct WarpConst {
  int n, N, S, maxexp, len_j;
  int max_fac;                 // most factors of any Jacobian record
  int n_levels;                // levels of extended power-table entries
  const int32_t* level_off;    // shared memory: word ranges per level
  const uint32_t* pre;         // shared memory: (triple, destination) words
  int deg;          // d_lane (lane < n)
  double inv_deg;   // 1/d_lane
  cd b;             // b_lane
  cd gamma;
  const cd* coefd;  // Jacobian schedule arrays (shared memory)
  const cf* coeff;
  const uint2* meta;
  const double (*patch)[2];
  int red_c;                   // pivot column of the patch row (see evaluate_rows_of)
  const double (*rho)[2];      // rho_j = a_j / a_c
};

__device__ __forceinline__ WarpConst load_warp_const(const PlanHeader& P,
                                                     const unsigned char* pb, int lane) {
  WarpConst C;
  C.n = P.n;
  C.N = P.N;
  C.S = P.S;
  C.maxexp = P.maxexp;
  C.len_j = P.len_j;
  C.max_fac = P.max_fac;
  C.n_levels = P.n_levels;
  C.level_off = P.level_off;
  C.pre = reinterpret_cast<const uint32_t*>(pb + P.off_pre);
  C.deg = lane < P.n ? P.deg[lane] : 1;
  C.inv_deg = lane < P.n ? P.inv_deg[lane] : 1.0;  // lane n: patch row, no scaling
  C.b = lane < P.n ? mkc<double>(P.b[lane][0], P.b[lane][1]) : czero<double>();
  C.gamma = mkc<double>(P.gamma[0], P.gamma[1]);
  C.coefd = reinterpret_cast<const cd*>(pb + P.off_jd);
  C.coeff = reinterpret_cast<const cf*>(pb + P.off_jf);
  C.meta = reinterpret_cast<const uint2*>(pb + P.off_jm);
  C.patch = P.patch;
  C.red_c = P.red_c;
  C.rho = P.rho;
  return C;
}

template <typename T> __device__ __forceinline__ const cpx<T>* wc_coef(const WarpConst& C);
template <> __device__ __forceinline__ const cd* wc_coef<double>(const WarpConst& C) {
  return C.coefd;
}
template <> __device__ __forceinline__ const cf* wc_coef<float>(const WarpConst& C) {
  return C.coeff;
}

// ---- sparse evaluation ----------------------------------------------------
// Power table of lane j's coordinate: pw[e*N + j] = z_j^e, e = 0..maxexp,
// by repeated multiplication (src/sparse.f90:251-255).
template <typename T>
__device__ __forceinline__ void power_table(const WarpConst& C, cpx<T>* pw, cpx<T> zj,
                                            int lane) {
  const bool own = lane < C.N;
  cpx<T> p = cone<T>();
  if (own) sts(&pw[lane], p);
  for (int e = 1; e <= C.maxexp; ++e) {
    p = p * zj;
    if (own) sts(&pw[e * C.N + lane], p);
  }
  // extended entries: products of three earlier entries, level by level
  for (int L = 0; L < C.n_levels; ++L) {
    __syncwarp();
    const int w1 = C.level_off[L + 1];
    for (int w = C.level_off[L] + 2 * lane; w < w1; w += 2 * kWarp) {
      const uint32_t t = C.pre[w];
      const cpx<T> v = lds(&pw[t & 0x3ffu]) * lds(&pw[(t >> 10) & 0x3ffu]) *
                       lds(&pw[(t >> 20) & 0x3ffu]);
      sts(&pw[C.pre[w + 1]], v);
    }
  }
}

// Runs the Jacobian schedule: the lane sums the contributions of its
// entries and stores each sum once into out[dest]. Record i of the lane is
// slot i*32 + lane of the coefficient and metadata arrays (layout in
// phc_internal.h). A record multiplies its coefficient by up to three table
// entries; F is the most any record of the system uses (an unused factor
// is pw[0] = 1, exact), so a quadratic system (at most one factor per
// record) runs the one-factor form and a cubic one the two-factor form,
// which load and multiply only the factors they can have. Records do not depend on
// each other except through the running sum, so consecutive records
// overlap in the pipeline.
template <typename T, int F>
__device__ __forceinline__ void run_schedule(const cpx<T>* __restrict__ coef,
                                             const uint2* __restrict__ meta, int len, int lane,
                                             const cpx<T>* __restrict__ pw,
                                             cpx<T>* __restrict__ out) {
  // All lanes run len (the longest lane's count, a multiple of 4: shorter
  // lanes read zero padding records). Records are processed four at a time:
  // the loads of a batch are issued together, then the products, then the
  // running sums. The sum is stored (a predicated store, not a branch) when
  // the record is the entry's last contribution.
  static_assert(F >= 1 && F <= 3, "one-, two- and three-factor schedules");
  cpx<T> acc = czero<T>();
  for (int i0 = 0; i0 < len; i0 += 4) {
    uint2 m[4];
    cpx<T> c[4], p0[4], p1[4], p2[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int slot = (i0 + u) * kWarp + lane;
      if constexpr (F == 1) {
        m[u].x = reinterpret_cast<const unsigned*>(meta)[2 * slot];
        m[u].y = 0u;
      } else {
        m[u] = meta[slot];
      }
      c[u] = lds(&coef[slot]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const unsigned lo = m[u].x, hi = m[u].y;
      p0[u] = lds(&pw[(lo >> 15) & 0x3ffu]);
      if constexpr (F >= 2) p1[u] = lds(&pw[(lo >> 25) | ((hi & 7u) << 7)]);
      if constexpr (F == 3) p2[u] = lds(&pw[(hi >> 3) & 0x3ffu]);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      cpx<T> v;
      if constexpr (F == 1)
        v = c[u] * p0[u];
      else if constexpr (F == 2)
        v = (c[u] * p0[u]) * p1[u];
      else
        v = (c[u] * p0[u]) * (p1[u] * p2[u]);
      const unsigned lo = m[u].x;
      const bool last = (lo >> 12) & kRecLast;
      acc = acc + v;
      if (last) sts(&out[lo & 0x3ffu], acc);
      acc = last ? czero<T>() : acc;
    }
  }
}

template <typename T> __device__ __forceinline__ const cpx<T>* plan_coef(
    const unsigned char* pb, int off_d, int off_f);
template <> __device__ __forceinline__ const cd* plan_coef<double>(const unsigned char* pb,
                                                                   int off_d, int) {
  return reinterpret_cast<const cd*>(pb + off_d);
}
template <> __device__ __forceinline__ const cf* plan_coef<float>(const unsigned char* pb, int,
                                                                  int off_f) {
  return reinterpret_cast<const cf*>(pb + off_f);
}

// ---- rows of the system, and the reduced system -----------------------------
// The last row of H_z is the patch a (h_n = a . z - 1, src/homotopy.f90:228-230),
// the same for every unit of a path. Normally it is one of the N rows the
// elimination pivots over, as in the reference's LU. For n = 16 (the table
// header's `reduce`) it is eliminated first instead, with a
// fixed pivot: the column c of the largest |a_c| (the first such column;
// the header holds c, rho_j = a_j / a_c, |rho_j| <= 1, and 1/a_c). For
// A x = r that leaves the n x n system of the equation rows over the
// columns j != c,
//   sum_{j != c} (A_ij - A_ic rho_j) x_j = r_i - A_ic r_n / a_c,
// and x_c = r_n / a_c - sum_{j != c} rho_j x_j. Column c's place in the
// reduced system is taken by column n (w) when c != n. 16 rows instead of
// 17 put n = 16 into the split layout with two lanes per row. Its pivoting
// differs from the reference's partial pivoting over all n + 1 rows, which
// changes rounding; for the other sizes the patch stays a row.

// The S lanes that share a row (lanes i, i + RPW, ...) and the rows of a
// part: sums over them.
template <int S, typename T>
__device__ __forceinline__ T row_sum(T v) {
  if constexpr (S >= 4) v += __shfl_xor_sync(kFull, v, 8);
  if constexpr (S >= 2) v += __shfl_xor_sync(kFull, v, 16);
  return v;
}
template <int S, typename T>
__device__ __forceinline__ cpx<T> row_csum(cpx<T> v) {
  return mkc<T>(row_sum<S>(v.re), row_sum<S>(v.im));
}
// Sum over the RPW lanes of one part (a column of the matrix).
template <int S, typename T>
__device__ __forceinline__ T part_sum(T v) {
#pragma unroll
  for (int o = 16 / S; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Original column of reduced column r (r < n): r itself, except that the
// pivot column c is replaced by column n.
__device__ __forceinline__ int reduced_col(int r, int c, int n) { return r == c ? n : r; }

// Evaluation of H(z,t) = gamma t G(z) + (1 - t) F^h(z) and its Jacobian
// (tdh_evaluate, src/homotopy.f90:188-231) in precision T, with S lanes per
// row and HS columns each (S = 1: one lane per row, all columns). Input:
// lane j holds z_j. Output, for lane L of row i = L % RPW and part
// q = L / RPW:
//   reduce = 0: rows i <= n of H_z (row n the patch) over the N columns:
//     a[jj] = H_z(i, q HS + jj), h = h_i, ht = (H_t)_i;
//   reduce = 1: the n equation rows over the reduced columns, before the
//     patch elimination: a[jj] = H_z(i, reduced_col(q HS + jj)),
//     aic = H_z(i, c);
// zero beyond the rows and columns. F^h_i is obtained from row i of its
// Jacobian by Euler's relation for homogeneous polynomials,
// F^h_i = (1/d_i) sum_j z_j dF^h_i/dz_j, which needs no evaluation of its
// own; the patch row's h_n = a . z - 1 follows the same way (its buffer
// row holds a, "degree" 1). F: the schedule form of the kernel (the most
// power-table factors of any record: 1, 2 or 3).
template <int HS, int S, typename T, int F>
__device__ __forceinline__ void evaluate_rows_of(const WarpConst& C, const WarpWS& ws, cd zl,
                                                 cd t, int lane, bool reduce, cpx<T> (&a)[HS],
                                                 cpx<T>& aic, cd& h, cd& ht) {
  constexpr int RPW = 32 / S;
  const int n = C.n, N = C.N, S_ = C.S, c = C.red_c;
  cpx<T>* pw = ws_pw<T>(ws);
  power_table<T>(C, pw, ccast<T>(zl), lane);
  __syncwarp();
  run_schedule<T, F>(wc_coef<T>(C), C.meta, C.len_j, lane, pw, ws_j<T>(ws));
  __syncwarp();

  const cpx<T> gamma = ccast<T>(C.gamma);
  const cpx<T> tt = ccast<T>(t);
  const cpx<T> gt = gamma * tt;
  const cpx<T> omt = mkc<T>(T(1) - tt.re, -tt.im);
  const cpx<T>* zrow = pw + N;  // z_j = pw[1*N + j]
  const int i = lane & (RPW - 1), part = lane / RPW, j0 = part * HS;
  const bool eq = i < n;
  const bool patch = !reduce && i == n;
  const int row = eq ? i : n;  // rows beyond the system read the patch row (scale 0)
  const int ncols = reduce ? n : N;
  const cpx<T>* Jr = ws_j<T>(ws) + row * S_;
  // the row's constants are held by lane i (WarpConst is per lane; lane n
  // has degree 1 and 1/d = 1, for the patch row)
  const int deg = (S == 1) ? C.deg : __shfl_sync(kFull, C.deg, i);
  const double inv_deg = (S == 1) ? C.inv_deg : __shfl_sync(kFull, C.inv_deg, i);
  const cpx<T> bi = ccast<T>((S == 1) ? C.b : shfl(C.b, i));
  // start system G_i = z_i^d - b_i w^d from the power table, and its
  // derivatives d_i gamma t z_i^(d-1) (column i) and -d_i gamma t b_i w^(d-1)
  // (column n)
  const int dm1 = eq ? deg - 1 : 0;
  const cpx<T> zd1 = lds(&pw[dm1 * N + row]);
  const cpx<T> wd1 = lds(&pw[dm1 * N + n]);
  const cpx<T> zi = lds(&zrow[row]);
  const cpx<T> w = lds(&zrow[n]);
  const cpx<T> g = zd1 * zi - (bi * wd1) * w;
  const T dd = (T)deg;
  const cpx<T> dg = eq ? (dd * gt) * zd1 : czero<T>();
  const cpx<T> dw = eq ? (dd * (gt * bi)) * wd1 : czero<T>();
  // row scale: (1 - t) for an equation row, 1 for the patch row, 0 beyond
  const cpx<T> sc = eq ? omt : (patch ? cone<T>() : czero<T>());
  const bool live = eq || patch;
  // Euler sum over the lane's columns; in the reduced system part 0 adds
  // column c
  cpx<T> f0 = czero<T>(), f1 = czero<T>();
#pragma unroll
  for (int jj = 0; jj < HS; ++jj) {
    const int r = j0 + jj;
    if (r < ncols) {
      const int o = reduce ? reduced_col(r, c, n) : r;
      const cpx<T> jio = lds(&Jr[o]);
      if (jj & 1)
        f1 = cfma(f1, jio, lds(&zrow[o]));
      else
        f0 = cfma(f0, jio, lds(&zrow[o]));
      cpx<T> v = sc * jio;
      if (o == i) v = v + dg;
      if (o == n) v = v - dw;
      a[jj] = live ? v : czero<T>();
    } else {
      a[jj] = czero<T>();
    }
  }
  aic = czero<T>();
  if (reduce) {
    const cpx<T> jic = lds(&Jr[c]);
    if (part == 0) f0 = cfma(f0, jic, lds(&zrow[c]));
    cpx<T> v = sc * jic;
    if (c == i) v = v + dg;
    if (c == n) v = v - dw;
    aic = eq ? v : czero<T>();
  }
  const cpx<T> f = (T)inv_deg * row_csum<S>(f0 + f1);
  const cpx<T> hh = eq ? gt * g + omt * f : (patch ? mkc<T>(f.re - T(1), f.im) : czero<T>());
  const cpx<T> hht = eq ? gamma * g - f : czero<T>();
  h = ccast<double>(hh);
  ht = ccast<double>(hht);
}

// The patch elimination of a row: a[jj] -= aic rho_o (o = reduced_col of the
// lane's column jj; rows >= n hold zeros and stay zero).
template <int HS, int S, typename T>
__device__ __forceinline__ void fold_patch(const WarpConst& C, int lane, cpx<T> (&a)[HS],
                                           cpx<T> aic) {
  constexpr int RPW = 32 / S;
  const int n = C.n, c = C.red_c;
  const int j0 = (lane / RPW) * HS;
#pragma unroll
  for (int jj = 0; jj < HS; ++jj) {
    const int r = j0 + jj;
    if (r < n) {
      const int o = reduced_col(r, c, n);
      const cpx<T> rho = mkc<T>((T)C.rho[o][0], (T)C.rho[o][1]);
      a[jj] = cfms(a[jj], aic, rho);
    }
  }
}

// ---- Gauss-Jordan elimination with partial pivoting -----------------------
// Solves A X = B for the N x N matrix A held row-wise (lane i owns row i)
// and R right-hand-side columns (lane i holds row i of B in r[]). Rows are
// never moved: at step k every lane's row is shifted left by one column, so
// the column being eliminated is always a[0]. The pivot is the row of
// largest |a_ik|^2 among the rows not pivoted yet (pivot_lane; ties go to
// the lowest row as in the reference's first-maximum scan,
// src/linalg.f90:51-58). Every lane computes the reciprocal of its own
// candidate while the reduction runs; the pivot row, its right-hand side
// and its reciprocal are broadcast with shuffles, and every other row,
// pivoted before or not, subtracts m * (1/p) times it (Gauss-Jordan: no
// back substitution). Pivot rows are never rescaled: at the end each lane
// multiplies its right-hand side by the reciprocal of its own pivot, and
// piv[k] is the lane that then holds row k of X. Returns false for an
// exactly zero pivot column (err_singular_matrix of lu_factor).
constexpr int kGjGroup = 4;  // columns per uniform branch of the row update (NM > 8)

template <int NM, int R, typename T>
__device__ __forceinline__ bool gauss_jordan(cpx<T> (&a)[NM], cpx<T> (&r)[R], int N, int lane,
                                             int* piv) {
  bool done = false;
  int mystep = -1;
  cpx<T> myrinv = czero<T>();
  cpx<T> m0 = a[0];
  // The pivot search and the speculative reciprocal of step k+1 need only
  // column 0 after step k, so they are issued as soon as that column is
  // updated and run while the rest of step k's row update (shuffle-bound)
  // is issued.
  T d2 = m0.re * m0.re + m0.im * m0.im;
  unsigned kmax;
  int p = pivot_lane(d2, lane < N, lane, kmax);
  T rd = rcp_nr(d2);
  for (int k = 0; k < N; ++k) {
    const bool cand = lane < N && !done;
    cpx<T> rinv = mkc<T>(m0.re * rd, -m0.im * rd);
    if (kmax == 0u) {
      // zero or tiny squares: decide with the modulus itself
      T km;
      p = warp_argmax_first(cand ? cabs(m0) : T(0), cand, km);
      if (!(km > T(0))) return false;
    }
    const bool isp = (lane == p);
    if (isp && !(d2 >= T(1e-36) && d2 <= T(1e36))) rinv = crcp(m0);  // |p|^2 out of range
    if (isp) {
      done = true;
      mystep = k;
      myrinv = rinv;
    }
    const cpx<T> rp = shfl(rinv, p);
    // multiplier; the pivot row only shifts (l = 0)
    const cpx<T> l = isp ? czero<T>() : m0 * rp;
    // next pivot column, then the next step's search
    a[0] = (NM > 1) ? cfms(a[1], l, shfl(a[1], p)) : czero<T>();
    m0 = a[0];
    d2 = m0.re * m0.re + m0.im * m0.im;
    const int pn = pivot_lane(d2, lane < N && !done, lane, kmax);
    rd = rcp_nr(d2);
    // Columns N-1-k and beyond are zero after this step; the rest of the
    // update runs over groups of kGjGroup columns and skips (uniform
    // branch) the groups that hold only zeros before and after it.
    const int live = N - 1 - k;  // last column that is nonzero before the step
    constexpr int G = (NM <= 8) ? NM : kGjGroup;  // narrow rows: one group
    StaticFor<0, (NM + G - 1) / G>::run([&](auto gc) {
      constexpr int g = decltype(gc)::value;
      if (g == 0 || G * g <= live) {
#pragma unroll
        for (int j = (G * g > 1 ? G * g : 1); j < G * (g + 1) && j < NM; ++j) {
          if (j + 1 < NM)
            a[j] = cfms(a[j + 1], l, shfl(a[j + 1], p));
          else
            a[j] = czero<T>();
        }
      }
    });
#pragma unroll
    for (int q = 0; q < R; ++q) r[q] = cfms(r[q], l, shfl(r[q], p));
    p = pn;
  }
#pragma unroll
  for (int q = 0; q < R; ++q) r[q] = r[q] * myrinv;
  if (mystep >= 0) piv[mystep] = lane;
  __syncwarp();
  return true;
}

// Gauss-Jordan for the split layout (S lanes per row, HS columns each;
// every lane of a row keeps the right-hand sides). Same pivoting,
// multipliers and order of operations per element as gauss_jordan. Each
// step shifts the row left by one column across the parts: a part's last
// column receives the next part's first column. The pivot search runs on
// the lanes of part 0; piv[] receives their indices.
template <int HS, int S, int R, typename T>
__device__ __forceinline__ bool gauss_jordan_split(cpx<T> (&a)[HS], cpx<T> (&r)[R], int N,
                                                   int lane, int* piv) {
  static_assert(HS >= 2, "split rows need at least two columns per part");
  constexpr int RPW = 32 / S;
  const int i = lane & (RPW - 1);
  const int part = lane / RPW;
  const bool first = part == 0;
  const bool last = part == S - 1;
  bool done = false;
  int mystep = -1;
  cpx<T> myrinv = czero<T>();
  // m0: the row's column 0 (part 0's first column); bnd: the next part's
  // first column (this part's next column after the shift)
  auto exchange = [&](cpx<T>& m0, cpx<T>& bnd) {
    if constexpr (S == 2) {
      const cpx<T> x = shfl_xor(a[0], 16);
      m0 = first ? a[0] : x;
      bnd = first ? x : czero<T>();
    } else {
      m0 = shfl(a[0], i);
      const cpx<T> x = shfl(a[0], (lane + RPW) & 31);
      bnd = last ? czero<T>() : x;
    }
  };
  // The pivot search and the reciprocal run on the lanes of part 0, which
  // hold the pivot column themselves; the exchange only feeds the other
  // parts' multipliers and stays off that chain. (The other parts' rinv,
  // myrinv and right-hand sides are never read: results come from part 0.)
  cpx<T> m0, bnd;
  exchange(m0, bnd);
  T d2 = first ? a[0].re * a[0].re + a[0].im * a[0].im : T(0);
  unsigned kmax;
  int p = pivot_lane(d2, first && i < N, lane, kmax);
  T rd = rcp_nr(d2);
  for (int k = 0; k < N; ++k) {
    const bool cand = first && i < N && !done;
    cpx<T> rinv = mkc<T>(m0.re * rd, -m0.im * rd);
    if (kmax == 0u) {
      T km;
      p = warp_argmax_first(cand ? cabs(m0) : T(0), cand, km);
      if (!(km > T(0))) return false;
    }
    const bool isrow = (i == p);  // p is a lane of part 0: row p
    if (isrow && first && !(d2 >= T(1e-36) && d2 <= T(1e36))) rinv = crcp(m0);  // |p|^2 out of range
    if (isrow) {
      done = true;
      mystep = k;
      myrinv = rinv;
    }
    const cpx<T> rp = shfl(rinv, p);
    // multiplier; the pivot row only shifts (l = 0)
    const cpx<T> l = isrow ? czero<T>() : m0 * rp;
    // the pivot row's part, and its next part's first column, before the step
    const int src = p + part * RPW;
    const cpx<T> pb = shfl(a[0], (src + RPW) & 31);
    // next pivot column first, then the exchange and the next search
    a[0] = cfms(a[1], l, shfl(a[1], src));
    d2 = first ? a[0].re * a[0].re + a[0].im * a[0].im : T(0);
    const int pn = pivot_lane(d2, first && i < N && !done, lane, kmax);
    rd = rcp_nr(d2);
    cpx<T> m0n, bndn;
    exchange(m0n, bndn);
#pragma unroll
    for (int jj = 1; jj + 1 < HS; ++jj) a[jj] = cfms(a[jj + 1], l, shfl(a[jj + 1], src));
    // the part's last column comes from the next part; the last part's
    // (beyond the row) is zero
    a[HS - 1] = last ? czero<T>() : cfms(bnd, l, pb);
#pragma unroll
    for (int q = 0; q < R; ++q) r[q] = cfms(r[q], l, shfl(r[q], p));
    m0 = m0n;
    bnd = bndn;
    p = pn;
  }
#pragma unroll
  for (int q = 0; q < R; ++q) r[q] = r[q] * myrinv;
  if (mystep >= 0 && first) piv[mystep] = lane;
  __syncwarp();
  return true;
}

}  // namespace phc

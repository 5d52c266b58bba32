/*
 * phc_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the per-path numerics behind polyhomocont's solve()
 * and of its host bookkeeping. Each function names the reference
 * procedure (file:line) it follows; loop orders, tie-breaks and operation
 * orders are kept, with Fortran's complex arithmetic restated explicitly
 * (multiplication without fused operations, Smith's division as used by
 * gfortran's default -fcx-fortran-rules, abs = hypot, integer powers by
 * square-and-multiply). Used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py only; the product never links it.
 *
 * Parity pin: see phc_oracle.h.
 */
#include "phc_oracle.h"

#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace orc {

/* ---------------------------------------------------------------------
 * complex(wp) arithmetic
 * ------------------------------------------------------------------- */
struct cx {
  double re;
  double im;
};

static inline cx C(double r, double i = 0.0) { return cx{r, i}; }
static inline cx operator+(cx a, cx b) { return cx{a.re + b.re, a.im + b.im}; }
static inline cx operator-(cx a, cx b) { return cx{a.re - b.re, a.im - b.im}; }
static inline cx operator-(cx a) { return cx{-a.re, -a.im}; }
static inline cx operator*(cx a, cx b) {
  return cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
/* real * complex: Fortran promotes the real to (s, 0); the products with
 * the zero imaginary part vanish exactly, leaving a scaling. */
static inline cx operator*(double s, cx a) { return cx{s * a.re, s * a.im}; }
static inline bool operator==(cx a, cx b) { return a.re == b.re && a.im == b.im; }
static inline bool operator!=(cx a, cx b) { return !(a == b); }

/* Complex division by Smith's method (R. L. Smith, CACM 5 (1962) 435),
 * the range-reducing division gfortran emits by default. */
static inline cx operator/(cx a, cx b) {
  if (std::fabs(b.re) < std::fabs(b.im)) {
    double ratio = b.re / b.im;
    double div = b.re * ratio + b.im;
    return cx{(a.re * ratio + a.im) / div, (a.im * ratio - a.re) / div};
  }
  double ratio = b.im / b.re;
  double div = b.im * ratio + b.re;
  return cx{(a.im * ratio + a.re) / div, (a.im - a.re * ratio) / div};
}
static inline cx operator/(cx a, double s) { return a / C(s); }
static inline double cabs_(cx a) { return std::hypot(a.re, a.im); }

/* z**k for integer k >= 0 (square and multiply, as libgfortran's
 * pow_c8_i4) */
static inline cx cpowi(cx x, int k) {
  cx pw = C(1.0);
  if (k == 0) return pw;
  unsigned u = (unsigned)k;
  for (;;) {
    if (u & 1u) pw = pw * x;
    u >>= 1;
    if (u) x = x * x;
    else break;
  }
  return pw;
}
/* real**k for integer k >= 0 (square and multiply, libgcc __powidf2) */
static inline double rpowi(double x, int m) {
  unsigned n = (unsigned)m;
  double y = (n % 2) ? x : 1.0;
  while (n >>= 1) {
    x = x * x;
    if (n % 2) y = y * x;
  }
  return y;
}

static const double kPi = 3.14159265358979323846;
static const double kHuge = DBL_MAX;
static const double kTiny = DBL_MIN;
static const double kEps = DBL_EPSILON;

/* status codes, src/config.f90:16-23 */
enum { status_ok = 0, err_invalid_input = 1, err_singular_matrix = 2 };
/* path status, src/tracker.f90:46-51, src/solve.f90:53 */
enum { path_success = 0, path_failed_min_step = 1, path_failed_max_steps = 2,
       path_endgame_failed = 3 };
/* end game status, src/endgame.f90:65-70 */
enum { endgame_converged = 0, endgame_not_converged = 1, endgame_failed = 2 };

typedef std::vector<cx> cvec;

static double norm_inf(const cx* z, int n) {  // src/linalg.f90:176-189
  double r = 0.0;
  for (int i = 0; i < n; ++i) r = std::max(r, cabs_(z[i]));
  return r;
}
static double norm_inf(const cvec& z) { return norm_inf(z.data(), (int)z.size()); }

/* ---------------------------------------------------------------------
 * random.f90: L'Ecuyer combined MLCG
 * ------------------------------------------------------------------- */
static const int64_t m1 = 2147483563LL, m2 = 2147483399LL;
static const int64_t a1 = 40014LL, a2 = 40692LL;

struct rng {
  int64_t s1 = 1234567LL;
  int64_t s2 = 7654321LL;
};

static double rng_uniform(rng& g) {  // src/random.f90:64-78
  g.s1 = (a1 * g.s1) % m1;
  g.s2 = (a2 * g.s2) % m2;
  int64_t z = g.s1 - g.s2;
  if (z < 1) z = z + m1 - 1;
  return (double)z / (double)m1;
}
static void rng_seed(rng& g, int seed) {  // src/random.f90:43-62
  int64_t s = std::llabs((int64_t)seed);
  g.s1 = s % (m1 - 1) + 1;
  g.s2 = (s * 7919LL + 104729LL) % (m2 - 1) + 1;
  for (int i = 0; i < 16; ++i) (void)rng_uniform(g);
}
static cx rng_unit_complex(rng& g) {  // src/random.f90:80-91
  double phi = 2.0 * kPi * rng_uniform(g);
  return C(std::cos(phi), std::sin(phi));
}
static cx rng_normal_complex(rng& g) {  // src/random.f90:93-109
  double r = std::sqrt(-std::log(rng_uniform(g)));
  double phi = 2.0 * kPi * rng_uniform(g);
  return C(r * std::cos(phi), r * std::sin(phi));
}

/* ---------------------------------------------------------------------
 * linalg.f90 (column-major a(i,j) = a[i + j*n], 0-based here)
 * ------------------------------------------------------------------- */
static int lu_factor(int n, cx* a, int* ipiv) {  // src/linalg.f90:26-78
#define A(i, j) a[(i) + (size_t)(j) * n]
  for (int k = 0; k < n; ++k) {
    int p = k;
    double amax = cabs_(A(k, k));
    for (int i = k + 1; i < n; ++i) {
      if (cabs_(A(i, k)) > amax) {
        amax = cabs_(A(i, k));
        p = i;
      }
    }
    ipiv[k] = p;
    if (amax == 0.0) return err_singular_matrix;
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        cx tmp = A(k, j);
        A(k, j) = A(p, j);
        A(p, j) = tmp;
      }
    }
    cx piv = A(k, k);
    for (int i = k + 1; i < n; ++i) {
      A(i, k) = A(i, k) / piv;
      cx l = A(i, k);
      for (int j = k + 1; j < n; ++j) A(i, j) = A(i, j) - l * A(k, j);
    }
  }
  return status_ok;
}

static void lu_solve(int n, const cx* a, const int* ipiv, cx* b) {
  // src/linalg.f90:80-114
  for (int k = 0; k < n; ++k) {
    if (ipiv[k] != k) {
      cx tmp = b[k];
      b[k] = b[ipiv[k]];
      b[ipiv[k]] = tmp;
    }
  }
  for (int i = 1; i < n; ++i) {
    cx s = C(0.0);
    for (int j = 0; j < i; ++j) s = s + A(i, j) * b[j];
    b[i] = b[i] - s;
  }
  for (int i = n - 1; i >= 0; --i) {
    cx s = C(0.0);
    for (int j = i + 1; j < n; ++j) s = s + A(i, j) * b[j];
    b[i] = (b[i] - s) / A(i, i);
  }
}

static double cond1(int n, const cx* a0) {  // src/linalg.f90:135-174
  double anorm = 0.0;
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += cabs_(a0[i + (size_t)j * n]);
    anorm = std::max(anorm, s);
  }
  cvec lu(a0, a0 + (size_t)n * n);
  std::vector<int> ipiv(n);
  if (lu_factor(n, lu.data(), ipiv.data()) != status_ok) return kHuge;
  double ainvnorm = 0.0;
  cvec col(n);
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < n; ++i) col[i] = C(0.0);
    col[j] = C(1.0);
    lu_solve(n, lu.data(), ipiv.data(), col.data());
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += cabs_(col[i]);
    ainvnorm = std::max(ainvnorm, s);
  }
  return anorm * ainvnorm;
}
#undef A

/* ---------------------------------------------------------------------
 * sparse.f90
 * ------------------------------------------------------------------- */
struct sparse_system {
  int n = 0;
  int neq = 0;
  int maxexp = 0;
  bool initialized = false;
  std::vector<int> first;  // 0-based offsets, size neq+1
  std::vector<int> deg;
  std::vector<int> exps;   // n x nt column-major
  std::vector<int> hexps;  // (n+1) x nt column-major
  cvec coefs;
  // a user system (class(poly_system) other than sparse_system): F and
  // dF/dx from a callback, homogenized by poly_system_evaluate_homogeneous
  orc_user_evaluator user = nullptr;
  void* user_ctx = nullptr;
  int nt() const { return (int)coefs.size(); }
};

static void sparse_init(sparse_system& s, int n) {  // src/sparse.f90:65-81
  s.n = n;
  s.neq = 0;
  s.maxexp = 0;
  s.initialized = true;
  s.first.assign(1, 0);
  s.deg.clear();
  s.exps.clear();
  s.hexps.clear();
  s.coefs.clear();
}

static int sparse_add_equation(sparse_system& s, int ncoefs, const cx* coefs,
                               int rows, int cols, const int* exps) {
  // src/sparse.f90:83-141
  if (!s.initialized) return err_invalid_input;
  if (s.neq >= s.n) return err_invalid_input;
  if (rows != s.n) return err_invalid_input;
  if (cols != ncoefs) return err_invalid_input;
  for (int q = 0; q < rows * cols; ++q)
    if (exps[q] < 0) return err_invalid_input;
  int d = 0;
  int nkeep = 0;
  for (int k = 0; k < ncoefs; ++k) {
    if (coefs[k] != C(0.0)) {
      ++nkeep;
      int sum = 0;
      for (int j = 0; j < s.n; ++j) sum += exps[j + k * rows];
      d = std::max(d, sum);
    }
  }
  if (d < 1) return err_invalid_input;
  for (int k = 0; k < ncoefs; ++k) {
    if (coefs[k] == C(0.0)) continue;
    int sum = 0;
    for (int j = 0; j < s.n; ++j) {
      s.exps.push_back(exps[j + k * rows]);
      s.hexps.push_back(exps[j + k * rows]);
      s.maxexp = std::max(s.maxexp, exps[j + k * rows]);
      sum += exps[j + k * rows];
    }
    s.hexps.push_back(d - sum);
    s.maxexp = std::max(s.maxexp, d - sum);
    s.coefs.push_back(coefs[k]);
  }
  s.neq += 1;
  s.first.push_back(s.first[s.neq - 1] + nkeep);
  s.deg.push_back(d);
  return status_ok;
}

/* eval_terms, src/sparse.f90:223-280: f(i) and jac(i,j) (column-major,
 * neq rows) for m variables, prefix/suffix products per term. */
struct eval_scratch {
  cvec pw, pre, suf;
};

static void eval_terms(int neq, const int* first, const int* exps, int m,
                       const cx* coefs, int maxexp, const cx* v, cx* f, cx* jac,
                       eval_scratch& sc) {
  cvec& pw = sc.pw;
  cvec& pre = sc.pre;
  cvec& suf = sc.suf;
  pw.resize((size_t)(maxexp + 1) * m);
  pre.resize(m + 1);
  suf.resize(m + 2);
#define PW(e, j) pw[(size_t)(e) + (size_t)(j) * (maxexp + 1)]
  for (int j = 0; j < m; ++j) PW(0, j) = C(1.0);
  for (int e = 1; e <= maxexp; ++e)
    for (int j = 0; j < m; ++j) PW(e, j) = PW(e - 1, j) * v[j];
  for (int i = 0; i < neq; ++i) f[i] = C(0.0);
  for (int q = 0; q < neq * m; ++q) jac[q] = C(0.0);
  for (int i = 0; i < neq; ++i) {
    for (int k = first[i]; k < first[i + 1]; ++k) {
      cx c = coefs[k];
      const int* e = exps + (size_t)k * m;
      // pre[j] = product over variables 0..j-1 (pre(j) of the reference)
      pre[0] = C(1.0);
      for (int j = 1; j <= m; ++j) pre[j] = pre[j - 1] * PW(e[j - 1], j - 1);
      // suf[j] = product over variables j-1..m-1 (suf(j) of the reference)
      suf[m + 1] = C(1.0);
      for (int j = m; j >= 1; --j) suf[j] = PW(e[j - 1], j - 1) * suf[j + 1];
      f[i] = f[i] + c * pre[m];
      for (int j = 1; j <= m; ++j) {
        int ej = e[j - 1];
        if (ej > 0) {
          cx term = (double)ej * c;
          term = term * PW(ej - 1, j - 1);
          term = term * pre[j - 1];
          term = term * suf[j + 1];
          jac[i + (size_t)(j - 1) * neq] = jac[i + (size_t)(j - 1) * neq] + term;
        }
      }
    }
  }
#undef PW
}

/* poly_system_evaluate_homogeneous, src/system.f90:71-119: the default
 * homogenization of a user system, through x = z(1:n)/w and the affine
 * evaluator; jac is n x (n+1) column-major. */
static void user_evaluate_homogeneous(const sparse_system& s, const cx* z, cx* f, cx* jac,
                                      eval_scratch& sc) {
  const int n = s.n;
  cvec& x = sc.pre;
  cvec& fa = sc.suf;
  cvec& ja = sc.pw;
  x.resize(n);
  fa.resize(n);
  ja.resize((size_t)n * n);
  cx w = z[n];
  if (w == C(0.0))
    w = C(std::numeric_limits<double>::epsilon() *
          std::max(norm_inf(z, n + 1), std::numeric_limits<double>::min()));
  for (int j = 0; j < n; ++j) x[j] = z[j] / w;
  s.user(s.user_ctx, n, reinterpret_cast<const double*>(x.data()),
         reinterpret_cast<double*>(fa.data()), reinterpret_cast<double*>(ja.data()));
  for (int i = 0; i < n; ++i) {
    const cx wd1 = cpowi(w, s.deg[i] - 1);
    f[i] = wd1 * w * fa[i];
    for (int j = 0; j < n; ++j) jac[i + (size_t)j * n] = wd1 * ja[i + (size_t)j * n];
    cx acc = C(0.0);
    for (int j = 0; j < n; ++j) acc = acc + x[j] * ja[i + (size_t)j * n];
    jac[i + (size_t)n * n] = wd1 * (C((double)s.deg[i]) * fa[i] - acc);
  }
}

static void sparse_evaluate_homogeneous(const sparse_system& s, const cx* z,
                                        cx* f, cx* jac, eval_scratch& sc) {
  if (s.user) {
    user_evaluate_homogeneous(s, z, f, jac, sc);
    return;
  }
  // src/sparse.f90:209-221
  eval_terms(s.neq, s.first.data(), s.hexps.data(), s.n + 1, s.coefs.data(),
             s.maxexp, z, f, jac, sc);
}

/* ---------------------------------------------------------------------
 * homotopy.f90: total_degree_homotopy
 * ------------------------------------------------------------------- */
struct total_degree_homotopy {
  const sparse_system* sys = nullptr;
  int n = 0;
  std::vector<int> deg;
  cx gamma = C(1.0);
  cvec b;
  cvec patch;
  int nstart = 0;
};

static int tdh_init(total_degree_homotopy& h, const sparse_system& sys, rng& gen) {
  // src/homotopy.f90:104-149
  h.sys = &sys;
  h.n = sys.n;
  h.deg = sys.deg;
  if (h.n < 1) return err_invalid_input;
  if ((int)h.deg.size() != h.n) return err_invalid_input;
  for (int d : h.deg)
    if (d < 1) return err_invalid_input;
  int64_t nstart = 1;
  for (int i = 0; i < h.n; ++i) {
    nstart *= (int64_t)h.deg[i];
    if (nstart > (int64_t)INT32_MAX) return err_invalid_input;
  }
  h.nstart = (int)nstart;
  h.gamma = rng_unit_complex(gen);
  h.b.assign(h.n, C(0.0));
  for (int i = 0; i < h.n; ++i) h.b[i] = rng_unit_complex(gen);
  h.patch.assign(h.n + 1, C(0.0));
  for (int i = 0; i < h.n + 1; ++i) h.patch[i] = rng_normal_complex(gen);
  double ss = 0.0;
  for (int i = 0; i < h.n + 1; ++i) {
    double a = cabs_(h.patch[i]);
    ss += a * a;
  }
  double nrm = std::sqrt(ss);
  for (int i = 0; i < h.n + 1; ++i) h.patch[i] = h.patch[i] / nrm;
  return status_ok;
}

static void tdh_start_solution(const total_degree_homotopy& h, int k, cx* z) {
  // src/homotopy.f90:151-177 (k 1-based)
  int rest = k - 1;
  for (int i = 0; i < h.n; ++i) {
    int digit = rest % h.deg[i];
    rest = rest / h.deg[i];
    double phi = (std::atan2(h.b[i].im, h.b[i].re) + 2.0 * kPi * (double)digit) /
                 (double)h.deg[i];
    z[i] = C(std::cos(phi), std::sin(phi));
  }
  z[h.n] = C(1.0);
  cx s = C(0.0);
  for (int i = 0; i < h.n + 1; ++i) s = s + h.patch[i] * z[i];
  for (int i = 0; i < h.n + 1; ++i) z[i] = z[i] / s;
}

/* Scratch for one evaluation; reused to keep allocations out of the
 * step loop. */
struct work {
  cvec f, jf, h, hz, ht;
  eval_scratch sc;
  void resize(int n) {
    f.resize(n);
    jf.resize((size_t)n * (n + 1));
    h.resize(n + 1);
    hz.resize((size_t)(n + 1) * (n + 1));
    ht.resize(n + 1);
  }
};

static void tdh_evaluate(const total_degree_homotopy& H, const cx* z, cx t,
                         cx* h, cx* hz, cx* ht, work& w) {
  // src/homotopy.f90:188-231; hz column-major N x N
  const int n = H.n, N = n + 1;
  cx* f = w.f.data();
  cx* jf = w.jf.data();  // n x N column-major
  cx wv = z[n];
  sparse_evaluate_homogeneous(*H.sys, z, f, jf, w.sc);
  cx gt = H.gamma * t;
  cx omt = C(1.0) - t;
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < n; ++i) hz[i + (size_t)j * N] = omt * jf[i + (size_t)j * n];
  for (int i = 0; i < n; ++i) {
    int d = H.deg[i];
    cx zd1 = cpowi(z[i], d - 1);
    cx wd1 = cpowi(wv, d - 1);
    cx g = zd1 * z[i] - H.b[i] * wd1 * wv;
    h[i] = gt * g + omt * f[i];
    ht[i] = H.gamma * g - f[i];
    hz[i + (size_t)i * N] = hz[i + (size_t)i * N] + ((double)d * gt) * zd1;
    hz[i + (size_t)n * N] = hz[i + (size_t)n * N] - ((double)d * (gt * H.b[i])) * wd1;
  }
  cx s = C(0.0);
  for (int j = 0; j < N; ++j) s = s + H.patch[j] * z[j];
  h[n] = s - C(1.0);
  for (int j = 0; j < N; ++j) hz[n + (size_t)j * N] = H.patch[j];
  ht[n] = C(0.0);
}

/* ---------------------------------------------------------------------
 * tracker.f90
 * ------------------------------------------------------------------- */
struct tracker_options {
  double step_init = 0.05;
  double step_max = 0.1;
  double step_min = 1.0e-14;
  double corrector_tol = 1.0e-10;
  int corrector_maxit = 3;
  double contraction = 0.5;
  int grow_after = 5;
  int max_steps = 20000;
};

enum { kind_line = 1, kind_arc = 2 };
struct segment {
  int kind = kind_line;
  cx t0 = C(1.0);
  cx t1 = C(0.0);
  double radius = 0.0;
  double theta0 = 0.0;
  double dtheta = 0.0;
};

struct path_info {
  int status = path_success;
  double s = 0.0;
  cx t = C(0.0);
  int naccepted = 0;
  int nrejected = 0;
  double step = 0.0;
};

/* unit counters (not in the reference) */
struct counters {
  int tangent = 0, newton = 0, refine = 0, eval = 0, cond = 0;
};

static segment line_segment(cx t0, cx t1) {  // src/tracker.f90:114-125
  segment s;
  s.kind = kind_line;
  s.t0 = t0;
  s.t1 = t1;
  return s;
}
static segment arc_segment(double r, double th0, double dth) {  // :127-140
  segment s;
  s.kind = kind_arc;
  s.radius = r;
  s.theta0 = th0;
  s.dtheta = dth;
  return s;
}
static cx seg_t(const segment& seg, double s) {  // src/tracker.f90:142-162
  if (seg.kind == kind_line) {
    if (s >= 1.0) return seg.t1;
    return seg.t0 + s * (seg.t1 - seg.t0);
  }
  double theta = seg.theta0 + s * seg.dtheta;
  return seg.radius * C(std::cos(theta), std::sin(theta));
}
static cx seg_dt(const segment& seg, double s) {  // src/tracker.f90:164-177
  if (seg.kind == kind_line) return seg.t1 - seg.t0;
  return C(0.0, seg.dtheta) * seg_t(seg, s);
}

struct ctx {
  const total_degree_homotopy* H;
  work w;
  counters cnt;
  int N;
  cvec h, hz, ht;
  cvec k1, k2, k3, k4, zt;
  std::vector<int> ipiv;
  explicit ctx(const total_degree_homotopy& hom) : H(&hom), N(hom.n + 1) {
    w.resize(hom.n);
    k1.resize(N);
    k2.resize(N);
    k3.resize(N);
    k4.resize(N);
    zt.resize(N);
    h.resize(N);
    hz.resize((size_t)N * N);
    ht.resize(N);
    ipiv.resize(N);
  }
  void evaluate(const cx* z, cx t) {
    tdh_evaluate(*H, z, t, h.data(), hz.data(), ht.data(), w);
  }
};

static bool tangent(ctx& c, const segment& seg, const cx* z, double s,
                    cx* dzds) {  // src/tracker.f90:295-317
  c.cnt.tangent++;
  c.evaluate(z, seg_t(seg, s));
  for (int i = 0; i < c.N; ++i) dzds[i] = c.ht[i];
  if (lu_factor(c.N, c.hz.data(), c.ipiv.data()) != status_ok) return false;
  cx dt = seg_dt(seg, s);
  for (int i = 0; i < c.N; ++i) dzds[i] = (-dzds[i]) * dt;
  lu_solve(c.N, c.hz.data(), c.ipiv.data(), dzds);
  return true;
}

static bool predict_rk4(ctx& c, const segment& seg, const cvec& z, double s,
                        double ds, cvec& zp) {  // src/tracker.f90:266-293
  const int N = c.N;
  cvec &k1 = c.k1, &k2 = c.k2, &k3 = c.k3, &k4 = c.k4, &zt = c.zt;
  if (!tangent(c, seg, z.data(), s, k1.data())) return false;
  for (int i = 0; i < N; ++i) zt[i] = z[i] + (0.5 * ds) * k1[i];
  if (!tangent(c, seg, zt.data(), s + 0.5 * ds, k2.data())) return false;
  for (int i = 0; i < N; ++i) zt[i] = z[i] + (0.5 * ds) * k2[i];
  if (!tangent(c, seg, zt.data(), s + 0.5 * ds, k3.data())) return false;
  for (int i = 0; i < N; ++i) zt[i] = z[i] + ds * k3[i];
  if (!tangent(c, seg, zt.data(), s + ds, k4.data())) return false;
  for (int i = 0; i < N; ++i)
    zp[i] = z[i] + (ds / 6.0) * (k1[i] + 2.0 * k2[i] + 2.0 * k3[i] + k4[i]);
  return true;
}

static bool newton_correct(ctx& c, cvec& z, cx t, double tol, int maxit,
                           double contraction) {  // src/tracker.f90:319-360
  const int N = c.N;
  double dnorm_prev = kHuge;
  for (int it = 1; it <= maxit; ++it) {
    c.cnt.newton++;
    c.evaluate(z.data(), t);
    if (lu_factor(N, c.hz.data(), c.ipiv.data()) != status_ok) return false;
    for (int i = 0; i < N; ++i) c.h[i] = -c.h[i];
    lu_solve(N, c.hz.data(), c.ipiv.data(), c.h.data());
    for (int i = 0; i < N; ++i) z[i] = z[i] + c.h[i];
    double dnorm = norm_inf(c.h.data(), N);
    if (dnorm <= tol * norm_inf(z)) return true;
    if (it > 1 && dnorm > contraction * dnorm_prev) return false;
    dnorm_prev = dnorm;
  }
  return false;
}

static void track_segment(ctx& c, cvec& z, const segment& seg,
                          const tracker_options& o, path_info& info) {
  // src/tracker.f90:196-264
  const int N = c.N;
  cvec zp(N);
  double s = 0.0;
  double step = std::min(o.step_init, o.step_max);
  int nsuccess = 0;
  info.naccepted = 0;
  info.nrejected = 0;
  info.status = path_success;
  while (s < 1.0) {
    if (info.naccepted + info.nrejected >= o.max_steps) {
      info.status = path_failed_max_steps;
      break;
    }
    double ds = std::min(step, 1.0 - s);
    double sn = s + ds;
    if (1.0 - sn <= 1.0e-3 * step) {
      sn = 1.0;
      ds = 1.0 - s;
    }
    bool ok = predict_rk4(c, seg, z, s, ds, zp);
    if (ok)
      ok = newton_correct(c, zp, seg_t(seg, sn), o.corrector_tol,
                          o.corrector_maxit, o.contraction);
    if (ok) {
      z = zp;
      s = sn;
      info.naccepted++;
      nsuccess++;
      if (nsuccess >= o.grow_after) {
        step = std::min(2.0 * step, o.step_max);
        nsuccess = 0;
      }
    } else {
      info.nrejected++;
      nsuccess = 0;
      step = 0.5 * step;
      if (step < o.step_min) {
        info.status = path_failed_min_step;
        break;
      }
    }
  }
  info.s = s;
  info.t = seg_t(seg, s);
  info.step = step;
}

static void track_path(ctx& c, cvec& z, double t_start, double t_end,
                       const tracker_options& o, path_info& info) {
  // src/tracker.f90:179-194
  track_segment(c, z, line_segment(C(t_start), C(t_end)), o, info);
}

/* ---------------------------------------------------------------------
 * endgame.f90
 * ------------------------------------------------------------------- */
struct endgame_options {
  double t_start = 0.1;
  int nsamples = 8;
  double radius_factor = 0.25;
  double radius_min = 1.0e-13;
  int max_winding = 16;
  double loop_radius = 1.0e-5;
  double winding_agreement = 0.2;
  double tol = 1.0e-11;
  double residual_tol = 1.0e-8;
  double closure_factor = 0.1;
};

struct endgame_result {
  int status = endgame_failed;
  cvec z;
  int winding_number = 0;
  double error = kHuge;
  double residual = kHuge;
  double radius = 0.0;
  int naccepted = 0;
  int nrejected = 0;
};

static double backward_error(ctx& c, const cvec& z) {  // src/endgame.f90:269-285
  const int N = c.N;
  c.cnt.eval++;
  c.evaluate(z.data(), C(0.0));
  double rmax = 0.0;
  for (int i = 0; i < N; ++i) {
    double s = 0.0;
    for (int j = 0; j < N; ++j) s += cabs_(c.hz[i + (size_t)j * N]);
    rmax = std::max(rmax, s);
  }
  return norm_inf(c.h.data(), N) / std::max(rmax * norm_inf(z), kTiny);
}

static bool better(double resid, double err, double best_resid, double best_err,
                   double residual_tol) {  // src/endgame.f90:287-311
  bool valid = resid <= residual_tol;
  bool best_valid = best_resid <= residual_tol;
  if (valid != best_valid) return valid;
  return err < best_err;
}

static bool loops(ctx& c, const cvec& z, double r, const endgame_options& o,
                  int max_loops, tracker_options& segopts, cvec& est, int& cw,
                  endgame_result& res) {  // src/endgame.f90:313-378
  const int N = c.N;
  path_info info;
  double dtheta = 2.0 * kPi / (double)o.nsamples;
  double floor_ = 10.0 * segopts.corrector_tol * norm_inf(z);
  cvec zc = z, zprev(N), zsum(N, C(0.0)), diff(N);
  int nsamp = 0;
  double spacing = kHuge;
  for (cw = 1; cw <= max_loops; ++cw) {
    for (int j = 1; j <= o.nsamples; ++j) {
      for (int i = 0; i < N; ++i) zsum[i] = zsum[i] + zc[i];
      nsamp++;
      zprev = zc;
      track_segment(c, zc, arc_segment(r, (double)(j - 1) * dtheta, dtheta),
                    segopts, info);
      segopts.step_init = std::min(std::max(info.step, segopts.step_min), 1.0);
      res.naccepted += info.naccepted;
      res.nrejected += info.nrejected;
      if (info.status != path_success) return false;
      for (int i = 0; i < N; ++i) diff[i] = zc[i] - zprev[i];
      spacing = std::min(spacing, norm_inf(diff));
    }
    for (int i = 0; i < N; ++i) diff[i] = zc[i] - z[i];
    if (norm_inf(diff) <= std::max(o.closure_factor * spacing, floor_)) {
      for (int i = 0; i < N; ++i) est[i] = zsum[i] / (double)nsamp;
      return true;
    }
  }
  return false;
}

static void cauchy_endgame(ctx& c, cvec& z, const endgame_options& o,
                           const tracker_options& topts, endgame_result& res) {
  // src/endgame.f90:124-267
  const int N = c.N;
  tracker_options segopts = topts;
  segopts.step_init = 1.0;
  segopts.step_max = 1.0;
  segopts.grow_after = 2;
  path_info info;
  cvec est(N), prev(N), zold(N), diff(N);
  double r, rnew, err, resid, best_resid, d, dprev, cest, cest_prev;
  int cw = 0, max_loops;
  bool have_prev, gate, ok;

  res = endgame_result();
  res.status = endgame_failed;
  res.z = z;
  r = o.t_start;
  have_prev = false;
  best_resid = kHuge;
  gate = false;
  dprev = -1.0;
  cest = -1.0;
  cest_prev = -1.0;
  max_loops = o.max_winding;

  auto record = [&]() {  // src/endgame.f90:240-265
    err = kHuge;
    if (have_prev) {
      for (int i = 0; i < N; ++i) diff[i] = est[i] - prev[i];
      err = norm_inf(diff) / std::max(norm_inf(est), kTiny);
    }
    resid = backward_error(c, est);
    if (res.status == endgame_failed ||
        better(resid, err, best_resid, res.error, o.residual_tol)) {
      res.status = endgame_not_converged;
      res.z = est;
      res.winding_number = cw;
      res.error = err;
      res.residual = resid;
      res.radius = r;
      best_resid = resid;
    }
    if (err <= o.tol && resid <= o.residual_tol) res.status = endgame_converged;
  };

  for (;;) {
    if (gate || r < o.loop_radius) {
      if (!gate) max_loops = o.max_winding;
      ok = loops(c, z, r, o, max_loops, segopts, est, cw, res);
    } else {
      ok = false;
    }
    if (!ok) {
      have_prev = false;
      gate = false;
    }
    if (ok) {
      record();
      if (res.status == endgame_converged) return;
      prev = est;
      have_prev = true;
    }
    rnew = o.radius_factor * r;
    if (rnew < o.radius_min) return;
    zold = z;
    track_segment(c, z, line_segment(C(r), C(rnew)), segopts, info);
    segopts.step_init = std::min(std::max(info.step, segopts.step_min), 1.0);
    res.naccepted += info.naccepted;
    res.nrejected += info.nrejected;
    if (info.status != path_success) {
      z = zold;
      if (!(gate || r < o.loop_radius)) {
        ok = loops(c, z, r, o, o.max_winding, segopts, est, cw, res);
        have_prev = false;
        if (ok) record();
      }
      return;
    }
    r = rnew;
    for (int i = 0; i < N; ++i) diff[i] = z[i] - zold[i];
    d = norm_inf(diff);
    if (!gate && dprev > 0.0 && d > 0.0) {
      cest_prev = cest;
      cest = -1.0;
      if (dprev > d) cest = std::log(1.0 / o.radius_factor) / std::log(dprev / d);
      if (cest >= 0.5 && cest <= (double)o.max_winding + 0.5 && cest_prev > 0.0) {
        if (std::fabs(cest - cest_prev) <=
            o.winding_agreement * std::max(1.0, cest)) {
          gate = true;
          max_loops = std::min(o.max_winding, 2 * (int)std::lround(cest) + 2);
        }
      }
    }
    dprev = d;
  }
}

/* ---------------------------------------------------------------------
 * solve.f90
 * ------------------------------------------------------------------- */
struct solve_options {
  tracker_options tracker;
  endgame_options endgame;
  bool use_endgame = true;
  int seed = 1;
  int refine_maxit = 5;
  double infinity_tol = 1.0e-8;
  double singular_cond = 1.0e10;
  double real_tol = 1.0e-8;
  double dedup_tol = 1.0e-8;
  double singular_dedup_tol = 1.0e-6;
};

struct path_result {
  int status = path_success;
  double t = 1.0;
  cvec z;
  cvec x;  // empty if not finite
  bool at_infinity = false;
  bool singular = false;
  bool is_real = false;
  int winding_number = 0;
  int endgame_status = 0;
  double endgame_error = 0.0;
  double cond = 0.0;
  double residual = 0.0;
  int solution_index = 0;
  int singular_index = 0;
  int naccepted = 0;
  int nrejected = 0;
  counters cnt;
};

static void endpoint(ctx& c, cvec& z, const solve_options& o, path_result& p) {
  // src/solve.f90:217-252
  path_info info;
  endgame_result eg;
  double t_end = 0.0;
  if (o.use_endgame) t_end = o.endgame.t_start;
  track_path(c, z, 1.0, t_end, o.tracker, info);
  p.status = info.status;
  p.t = info.t.re;
  p.naccepted = info.naccepted;
  p.nrejected = info.nrejected;
  if (info.status != path_success || !o.use_endgame) return;
  cauchy_endgame(c, z, o.endgame, o.tracker, eg);
  p.naccepted += eg.naccepted;
  p.nrejected += eg.nrejected;
  if (eg.status == endgame_failed) {
    p.status = path_endgame_failed;
    return;
  }
  z = eg.z;
  p.t = 0.0;
  p.winding_number = eg.winding_number;
  p.endgame_status = eg.status;
  p.endgame_error = eg.error;
}

static void refine(ctx& c, cvec& z, int maxit) {  // src/solve.f90:254-286
  const int N = c.N;
  double dnorm_prev = kHuge;
  for (int it = 1; it <= maxit; ++it) {
    c.cnt.refine++;
    c.evaluate(z.data(), C(0.0));
    if (lu_factor(N, c.hz.data(), c.ipiv.data()) != status_ok) return;
    for (int i = 0; i < N; ++i) c.h[i] = -c.h[i];
    lu_solve(N, c.hz.data(), c.ipiv.data(), c.h.data());
    double dnorm = norm_inf(c.h.data(), N);
    if (dnorm > dnorm_prev) return;
    for (int i = 0; i < N; ++i) z[i] = z[i] + c.h[i];
    if (dnorm <= 4.0 * kEps * norm_inf(z)) return;
    dnorm_prev = dnorm;
  }
}

static void classify(ctx& c, cvec& z, const solve_options& o, path_result& p) {
  // src/solve.f90:288-328
  const int N = c.N, n = N - 1;
  c.cnt.eval++;
  c.evaluate(z.data(), C(0.0));
  c.cnt.cond++;
  p.cond = cond1(N, c.hz.data());
  p.singular = p.winding_number > 1 || p.cond > o.singular_cond;
  if (!p.singular) {
    refine(c, z, o.refine_maxit);
    c.cnt.eval++;
    c.evaluate(z.data(), C(0.0));
    c.cnt.cond++;
    p.cond = cond1(N, c.hz.data());
  }
  p.z = z;
  double znorm = norm_inf(z);
  double rmax = -kHuge;
  for (int i = 0; i < n; ++i)
    rmax = std::max(rmax, cabs_(c.h[i]) / rpowi(znorm, c.H->deg[i]));
  p.residual = rmax;
  p.at_infinity = cabs_(z[n]) <=
                  std::max(o.infinity_tol, 10.0 * std::min(p.endgame_error, 1.0e-4)) * znorm;
  if (!p.at_infinity) {
    p.x.resize(n);
    for (int i = 0; i < n; ++i) p.x[i] = z[i] / z[n];
    double imax = 0.0;
    for (int i = 0; i < n; ++i) imax = std::max(imax, std::fabs(p.x[i].im));
    p.is_real = imax <= o.real_tol * std::max(1.0, norm_inf(p.x));
  }
}

/* per-path body of the do-k loop in solve, src/solve.f90:190-198 */
static void solve_one_path(const total_degree_homotopy& hom,
                           const solve_options& o, int k, path_result& p) {
  ctx c(hom);
  cvec z(hom.n + 1);
  tdh_start_solution(hom, k, z.data());
  endpoint(c, z, o, p);
  if (p.status != path_success) {
    p.z = z;
  } else {
    classify(c, z, o, p);
  }
  p.cnt = c.cnt;
}

static int find(const cvec& x, const std::vector<cvec>& pts, double tol) {
  // src/solve.f90:379-400 (1-based result)
  double scale = std::max(1.0, norm_inf(x));
  cvec diff(x.size());
  for (size_t j = 0; j < pts.size(); ++j) {
    for (size_t i = 0; i < x.size(); ++i) diff[i] = x[i] - pts[j][i];
    if (norm_inf(diff) <= tol * scale) return (int)j + 1;
  }
  return 0;
}

struct solve_result {
  int n = 0;
  int npaths = 0;
  std::vector<path_result> paths;
  std::vector<cvec> solutions;
  std::vector<cvec> singular_solutions;
  std::vector<int> multiplicities;
  std::vector<std::vector<double>> real_solutions;
  int ninfinite = 0, nfailed = 0, nduplicates = 0;
};

static void bookkeeping(solve_result& res, const solve_options& o) {
  // the order-dependent part of the do-k loop, src/solve.f90:193-213,
  // add_solution :330-351, add_singular :353-377, collect_real :402-426
  for (auto& p : res.paths) {
    if (p.status != path_success) {
      res.nfailed++;
    } else if (p.at_infinity) {
      res.ninfinite++;
    } else if (p.singular) {
      int j = find(p.x, res.singular_solutions, o.singular_dedup_tol);
      if (j > 0) {
        res.multiplicities[j - 1]++;
      } else {
        res.singular_solutions.push_back(p.x);
        res.multiplicities.push_back(1);
        j = (int)res.singular_solutions.size();
      }
      p.singular_index = j;
    } else {
      int j = find(p.x, res.solutions, o.dedup_tol);
      if (j > 0) {
        res.nduplicates++;
      } else {
        res.solutions.push_back(p.x);
        j = (int)res.solutions.size();
      }
      p.solution_index = j;
    }
  }
  for (const auto& s : res.solutions) {
    double imax = 0.0;
    for (const auto& v : s) imax = std::max(imax, std::fabs(v.im));
    if (imax <= o.real_tol * std::max(1.0, norm_inf(s))) {
      std::vector<double> r(s.size());
      for (size_t i = 0; i < s.size(); ++i) r[i] = s[i].re;
      res.real_solutions.push_back(r);
    }
  }
}

static void run_paths_threaded(const total_degree_homotopy& hom,
                               const solve_options& o, int64_t k0, int64_t count,
                               int nthreads, std::vector<path_result>& out) {
  out.assign((size_t)count, path_result());
  if (nthreads < 1) nthreads = 1;
  if (nthreads > count) nthreads = (int)std::max<int64_t>(count, 1);
  std::atomic<int64_t> next(0);
  auto worker = [&]() {
    for (;;) {
      int64_t q = next.fetch_add(1);
      if (q >= count) break;
      solve_one_path(hom, o, (int)(k0 + q), out[(size_t)q]);
    }
  };
  if (nthreads == 1) {
    worker();
    return;
  }
  std::vector<std::thread> th;
  for (int i = 0; i < nthreads; ++i) th.emplace_back(worker);
  for (auto& t : th) t.join();
}

/* conversions from the C structs */
static tracker_options to_topts(const orc_tracker_options* c) {
  tracker_options t;
  t.step_init = c->step_init;
  t.step_max = c->step_max;
  t.step_min = c->step_min;
  t.corrector_tol = c->corrector_tol;
  t.corrector_maxit = c->corrector_maxit;
  t.contraction = c->contraction;
  t.grow_after = c->grow_after;
  t.max_steps = c->max_steps;
  return t;
}
static endgame_options to_eopts(const orc_endgame_options* c) {
  endgame_options e;
  e.t_start = c->t_start;
  e.nsamples = c->nsamples;
  e.radius_factor = c->radius_factor;
  e.radius_min = c->radius_min;
  e.max_winding = c->max_winding;
  e.loop_radius = c->loop_radius;
  e.winding_agreement = c->winding_agreement;
  e.tol = c->tol;
  e.residual_tol = c->residual_tol;
  e.closure_factor = c->closure_factor;
  return e;
}
static solve_options to_sopts(const orc_solve_options* c) {
  solve_options s;
  if (!c) return s;
  s.tracker = to_topts(&c->tracker);
  s.endgame = to_eopts(&c->endgame);
  s.use_endgame = c->use_endgame != 0;
  s.seed = c->seed;
  s.refine_maxit = c->refine_maxit;
  s.infinity_tol = c->infinity_tol;
  s.singular_cond = c->singular_cond;
  s.real_tol = c->real_tol;
  s.dedup_tol = c->dedup_tol;
  s.singular_dedup_tol = c->singular_dedup_tol;
  return s;
}

static void fill_path_out(const path_result& p, int n, orc_path_out* po,
                          double* z, double* x) {
  po->status = p.status;
  po->winding_number = p.winding_number;
  po->endgame_status = p.endgame_status;
  po->at_infinity = p.at_infinity;
  po->singular = p.singular;
  po->is_real = p.is_real;
  po->naccepted = p.naccepted;
  po->nrejected = p.nrejected;
  po->solution_index = p.solution_index;
  po->singular_index = p.singular_index;
  po->n_tangent = p.cnt.tangent;
  po->n_newton = p.cnt.newton;
  po->n_refine = p.cnt.refine;
  po->n_eval = p.cnt.eval;
  po->n_cond = p.cnt.cond;
  po->n_fp64_retry = 0;
  po->t = p.t;
  po->endgame_error = p.endgame_error;
  po->cond = p.cond;
  po->residual = p.residual;
  if (z)
    for (int i = 0; i <= n; ++i) {
      z[2 * i] = p.z[i].re;
      z[2 * i + 1] = p.z[i].im;
    }
  if (x)
    for (int i = 0; i < n; ++i) {
      x[2 * i] = p.x.empty() ? 0.0 : p.x[i].re;
      x[2 * i + 1] = p.x.empty() ? 0.0 : p.x[i].im;
    }
}

}  // namespace orc

using namespace orc;

static inline const cx* ccx(const double* p) { return reinterpret_cast<const cx*>(p); }
static inline cx* mcx(double* p) { return reinterpret_cast<cx*>(p); }

extern "C" {

void orc_default_solve_options(orc_solve_options* c) {
  solve_options s;
  std::memset(c, 0, sizeof(*c));
  c->tracker.step_init = s.tracker.step_init;
  c->tracker.step_max = s.tracker.step_max;
  c->tracker.step_min = s.tracker.step_min;
  c->tracker.corrector_tol = s.tracker.corrector_tol;
  c->tracker.corrector_maxit = s.tracker.corrector_maxit;
  c->tracker.grow_after = s.tracker.grow_after;
  c->tracker.contraction = s.tracker.contraction;
  c->tracker.max_steps = s.tracker.max_steps;
  c->endgame.t_start = s.endgame.t_start;
  c->endgame.radius_factor = s.endgame.radius_factor;
  c->endgame.radius_min = s.endgame.radius_min;
  c->endgame.loop_radius = s.endgame.loop_radius;
  c->endgame.winding_agreement = s.endgame.winding_agreement;
  c->endgame.tol = s.endgame.tol;
  c->endgame.residual_tol = s.endgame.residual_tol;
  c->endgame.closure_factor = s.endgame.closure_factor;
  c->endgame.nsamples = s.endgame.nsamples;
  c->endgame.max_winding = s.endgame.max_winding;
  c->use_endgame = 1;
  c->seed = s.seed;
  c->refine_maxit = s.refine_maxit;
  c->infinity_tol = s.infinity_tol;
  c->singular_cond = s.singular_cond;
  c->real_tol = s.real_tol;
  c->dedup_tol = s.dedup_tol;
  c->singular_dedup_tol = s.singular_dedup_tol;
}

void* orc_rng_new(void) { return new rng(); }
void orc_rng_free(void* g) { delete static_cast<rng*>(g); }
void orc_rng_seed(void* g, int32_t seed) { rng_seed(*static_cast<rng*>(g), seed); }
double orc_rng_uniform(void* g) { return rng_uniform(*static_cast<rng*>(g)); }
void orc_rng_unit_complex(void* g, double* z) {
  cx v = rng_unit_complex(*static_cast<rng*>(g));
  z[0] = v.re;
  z[1] = v.im;
}
void orc_rng_normal_complex(void* g, double* z) {
  cx v = rng_normal_complex(*static_cast<rng*>(g));
  z[0] = v.re;
  z[1] = v.im;
}

int32_t orc_lu_factor(int32_t n, double* a, int32_t* ipiv) {
  std::vector<int> ip(n, 0);
  int st = lu_factor(n, mcx(a), ip.data());
  for (int k = 0; k < n; ++k) ipiv[k] = ip[k] + 1;
  return st;
}
void orc_lu_solve(int32_t n, const double* a, const int32_t* ipiv, double* b) {
  std::vector<int> ip(n);
  for (int k = 0; k < n; ++k) ip[k] = ipiv[k] - 1;
  lu_solve(n, ccx(a), ip.data(), mcx(b));
}
int32_t orc_solve_linear(int32_t n, const double* a, const double* b, double* x) {
  // src/linalg.f90:116-133
  cvec lu(ccx(a), ccx(a) + (size_t)n * n);
  std::vector<int> ip(n);
  int st = lu_factor(n, lu.data(), ip.data());
  if (st != status_ok) return st;
  for (int i = 0; i < n; ++i) mcx(x)[i] = ccx(b)[i];
  lu_solve(n, lu.data(), ip.data(), mcx(x));
  return st;
}
double orc_cond1(int32_t n, const double* a) { return cond1(n, ccx(a)); }
double orc_norm_inf(int32_t n, const double* z) { return norm_inf(ccx(z), n); }

void orc_sparse_set_user(void* s, int32_t n, const int32_t* degrees, orc_user_evaluator fn,
                         void* ctx) {
  sparse_system& p = *static_cast<sparse_system*>(s);
  sparse_init(p, n);
  p.neq = n;
  p.first.assign(n + 1, 0);
  p.deg.assign(degrees, degrees + n);
  p.user = fn;
  p.user_ctx = ctx;
}
void* orc_sparse_new(void) { return new sparse_system(); }
void orc_sparse_free(void* s) { delete static_cast<sparse_system*>(s); }
void orc_sparse_init(void* s, int32_t n) { sparse_init(*static_cast<sparse_system*>(s), n); }
int32_t orc_sparse_add_equation(void* s, int32_t ncoefs, const double* coefs,
                                int32_t rows, int32_t cols, const int32_t* exps) {
  return sparse_add_equation(*static_cast<sparse_system*>(s), ncoefs, ccx(coefs),
                             rows, cols, exps);
}
int32_t orc_sparse_nvars(void* s) { return static_cast<sparse_system*>(s)->n; }
int32_t orc_sparse_nequations(void* s) { return static_cast<sparse_system*>(s)->neq; }
int32_t orc_sparse_nterms(void* s, int32_t i) {
  auto* p = static_cast<sparse_system*>(s);
  return p->first[i] - p->first[i - 1];
}
int32_t orc_sparse_total_terms(void* s) { return static_cast<sparse_system*>(s)->nt(); }
int32_t orc_sparse_maxexp(void* s) { return static_cast<sparse_system*>(s)->maxexp; }
void orc_sparse_degrees(void* s, int32_t* d) {
  auto* p = static_cast<sparse_system*>(s);
  for (int i = 0; i < p->neq; ++i) d[i] = p->deg[i];
}
void orc_sparse_table(void* s, int32_t* first, int32_t* hexps, double* coefs) {
  auto* p = static_cast<sparse_system*>(s);
  for (int i = 0; i <= p->neq; ++i) first[i] = p->first[i];
  for (size_t q = 0; q < p->hexps.size(); ++q) hexps[q] = p->hexps[q];
  for (int k = 0; k < p->nt(); ++k) {
    coefs[2 * k] = p->coefs[k].re;
    coefs[2 * k + 1] = p->coefs[k].im;
  }
}
void orc_sparse_evaluate(void* s, const double* x, double* f, double* jac) {
  // src/sparse.f90:197-207
  auto* p = static_cast<sparse_system*>(s);
  eval_scratch sc;
  eval_terms(p->neq, p->first.data(), p->exps.data(), p->n, p->coefs.data(),
             p->maxexp, ccx(x), mcx(f), mcx(jac), sc);
}
void orc_sparse_evaluate_homogeneous(void* s, const double* z, double* f, double* jac) {
  auto* p = static_cast<sparse_system*>(s);
  eval_scratch sc;
  sparse_evaluate_homogeneous(*p, ccx(z), mcx(f), mcx(jac), sc);
}

void* orc_hom_new(void) { return new total_degree_homotopy(); }
void orc_hom_free(void* h) { delete static_cast<total_degree_homotopy*>(h); }
int32_t orc_hom_init(void* h, void* sys, void* gen) {
  return tdh_init(*static_cast<total_degree_homotopy*>(h),
                  *static_cast<sparse_system*>(sys), *static_cast<rng*>(gen));
}
int32_t orc_hom_nstart(void* h) { return static_cast<total_degree_homotopy*>(h)->nstart; }
void orc_hom_constants(void* h, double* gamma, double* b, double* patch) {
  auto* H = static_cast<total_degree_homotopy*>(h);
  gamma[0] = H->gamma.re;
  gamma[1] = H->gamma.im;
  for (int i = 0; i < H->n; ++i) {
    b[2 * i] = H->b[i].re;
    b[2 * i + 1] = H->b[i].im;
  }
  for (int i = 0; i <= H->n; ++i) {
    patch[2 * i] = H->patch[i].re;
    patch[2 * i + 1] = H->patch[i].im;
  }
}
void orc_hom_start_solution(void* h, int32_t k, double* z) {
  tdh_start_solution(*static_cast<total_degree_homotopy*>(h), k, mcx(z));
}
void orc_hom_evaluate(void* h, const double* z, const double* t, double* hv,
                      double* hz, double* ht) {
  auto* H = static_cast<total_degree_homotopy*>(h);
  work w;
  w.resize(H->n);
  tdh_evaluate(*H, ccx(z), C(t[0], t[1]), mcx(hv), mcx(hz), mcx(ht), w);
}

static void info_out(const path_info& i, orc_path_info* o) {
  o->status = i.status;
  o->naccepted = i.naccepted;
  o->nrejected = i.nrejected;
  o->pad_ = 0;
  o->s = i.s;
  o->t_re = i.t.re;
  o->t_im = i.t.im;
  o->step = i.step;
}

static void track_generic(void* h, double* z, const segment& seg,
                          const orc_tracker_options* o, orc_path_info* out) {
  auto* H = static_cast<total_degree_homotopy*>(h);
  ctx c(*H);
  cvec zz(ccx(z), ccx(z) + H->n + 1);
  path_info info;
  track_segment(c, zz, seg, to_topts(o), info);
  for (int i = 0; i <= H->n; ++i) mcx(z)[i] = zz[i];
  info_out(info, out);
}
void orc_track_path(void* h, double* z, double t_start, double t_end,
                    const orc_tracker_options* o, orc_path_info* info) {
  track_generic(h, z, line_segment(C(t_start), C(t_end)), o, info);
}
void orc_track_line(void* h, double* z, const double* t0, const double* t1,
                    const orc_tracker_options* o, orc_path_info* info) {
  track_generic(h, z, line_segment(C(t0[0], t0[1]), C(t1[0], t1[1])), o, info);
}
void orc_track_arc(void* h, double* z, double radius, double theta0, double dtheta,
                   const orc_tracker_options* o, orc_path_info* info) {
  track_generic(h, z, arc_segment(radius, theta0, dtheta), o, info);
}

void orc_cauchy_endgame(void* h, double* z, const orc_endgame_options* eo,
                        const orc_tracker_options* to, orc_endgame_result* r,
                        double* zres) {
  auto* H = static_cast<total_degree_homotopy*>(h);
  ctx c(*H);
  cvec zz(ccx(z), ccx(z) + H->n + 1);
  endgame_result res;
  cauchy_endgame(c, zz, to_eopts(eo), to_topts(to), res);
  for (int i = 0; i <= H->n; ++i) {
    mcx(z)[i] = zz[i];
    mcx(zres)[i] = res.z[i];
  }
  r->status = res.status;
  r->winding_number = res.winding_number;
  r->naccepted = res.naccepted;
  r->nrejected = res.nrejected;
  r->error = res.error;
  r->residual = res.residual;
  r->radius = res.radius;
}

int64_t orc_bezout(void* sys) {
  auto* s = static_cast<sparse_system*>(sys);
  int64_t b = 1;
  for (int d : s->deg) b *= d;
  return b;
}

int32_t orc_solve_paths(void* sys, const orc_solve_options* co, int64_t k0,
                        int64_t count, int32_t nthreads, orc_path_out* paths,
                        double* z_out, double* x_out) {
  auto* s = static_cast<sparse_system*>(sys);
  solve_options o = to_sopts(co);
  rng gen;
  rng_seed(gen, o.seed);
  total_degree_homotopy hom;
  int st = tdh_init(hom, *s, gen);
  if (st != status_ok) return st;
  std::vector<path_result> res;
  run_paths_threaded(hom, o, k0, count, nthreads, res);
  const int n = hom.n;
  for (int64_t q = 0; q < count; ++q)
    fill_path_out(res[(size_t)q], n, &paths[q],
                  z_out ? z_out + 2 * (size_t)q * (n + 1) : nullptr,
                  x_out ? x_out + 2 * (size_t)q * n : nullptr);
  return status_ok;
}

int32_t orc_solve(void* sys, const orc_solve_options* co, int32_t nthreads,
                  orc_path_out* paths, double* z_out, double* x_out,
                  orc_solve_counts* counts, double* sols, double* realsols,
                  double* ssols, int32_t* mult) {
  // src/solve.f90:154-215
  auto* s = static_cast<sparse_system*>(sys);
  solve_options o = to_sopts(co);
  rng gen;
  rng_seed(gen, o.seed);
  total_degree_homotopy hom;
  std::memset(counts, 0, sizeof(*counts));
  int st = tdh_init(hom, *s, gen);
  if (st != status_ok) return st;
  solve_result res;
  res.n = hom.n;
  res.npaths = hom.nstart;
  run_paths_threaded(hom, o, 1, hom.nstart, nthreads, res.paths);
  bookkeeping(res, o);
  const int n = hom.n;
  for (int q = 0; q < res.npaths; ++q)
    fill_path_out(res.paths[q], n, &paths[q], z_out + 2 * (size_t)q * (n + 1),
                  x_out + 2 * (size_t)q * n);
  counts->n = n;
  counts->npaths = res.npaths;
  counts->nsolutions = (int)res.solutions.size();
  counts->nreal = (int)res.real_solutions.size();
  counts->nsingular = (int)res.singular_solutions.size();
  counts->ninfinite = res.ninfinite;
  counts->nfailed = res.nfailed;
  counts->nduplicates = res.nduplicates;
  for (size_t j = 0; j < res.solutions.size(); ++j)
    for (int i = 0; i < n; ++i) {
      sols[2 * (j * n + i)] = res.solutions[j][i].re;
      sols[2 * (j * n + i) + 1] = res.solutions[j][i].im;
    }
  for (size_t j = 0; j < res.real_solutions.size(); ++j)
    for (int i = 0; i < n; ++i) realsols[j * n + i] = res.real_solutions[j][i];
  for (size_t j = 0; j < res.singular_solutions.size(); ++j) {
    for (int i = 0; i < n; ++i) {
      ssols[2 * (j * n + i)] = res.singular_solutions[j][i].re;
      ssols[2 * (j * n + i) + 1] = res.singular_solutions[j][i].im;
    }
    mult[j] = res.multiplicities[j];
  }
  return status_ok;
}

}  // extern "C"

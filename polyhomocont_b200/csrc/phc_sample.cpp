// phc_sample.cpp -- user-evaluator systems as sparse tables.
//
// The reference accepts any extension of poly_system that provides nvars,
// degrees and evaluate (F(x) together with dF/dx, src/system.f90:27-67) and
// tracks it through the default homogenization F^h_i = w^{d_i} F_i(z/w)
// (src/system.f90:71-119). A Fortran procedure cannot run on the GPU, so
// such a system is turned into a sparse table once, on the host, and then
// tracked by the same kernels as a sparse_system.
//
// The degrees "must be exact" (src/system.f90:45-50), so F_i is a
// polynomial of total degree d_i in n variables and is fixed by its values
// at enough generic points. For each distinct degree d the sampler
//   1. lists the m = C(n+d, d) exponent vectors with |a| <= d (highest
//      total degree first, lexicographically descending within a degree);
//   2. evaluates the user's F at P = 2m points on the unit torus
//      (x_j = e^{i theta}, theta uniform; the design matrix [x_p^a] is then
//      a random Fourier matrix, well conditioned at 2x oversampling);
//   3. solves the least-squares problem [x_p^a] c = F_i(x_p) for every
//      equation of that degree by complex Householder QR;
//   4. sets to zero each real or imaginary coefficient part at or below
//      1e-12 * sum_a |c_a| (sum_a |c_a| bounds |F_i| on the torus, the
//      least-squares error is a few eps times it), and keeps the terms
//      that remain, in the order of step 1;
//   5. checks the table against the user's F AND Jacobian at 16 fresh
//      points (half on the torus, half at radii in [0.5, 1.5]) and rejects
//      it (err_invalid_input) when the relative error exceeds 1e-9: the
//      evaluator is then not a polynomial of the stated degrees, or its
//      Jacobian is not the derivative of F.
// An equation whose sampled top-degree part vanishes is rejected too: its
// stated degree would not be exact. The result is an ordinary sparse
// builder (phc_sparse_init + phc_sparse_add_equation), so the homotopy,
// the table compiler and the kernels see no difference. Tracking F^h
// directly is the accuracy the reference recommends for extensions that
// can do it (src/system.f90:15-19); its default homogenization divides by
// w and loses accuracy near infinity.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

#include "phc_host.h"
#include "polyhomocont_b200.h"

namespace {

using cd = std::complex<double>;

constexpr int kMaxMonomials = 1500;  // per equation: the QR is O(P m^2), P = 2m
constexpr double kSnap = 1e-12;
constexpr double kCheckTol = 1e-9;
constexpr int kCheckPoints = 16;

// splitmix64: the sample points only need to be generic and reproducible
struct Rng {
  uint64_t s;
  explicit Rng(int32_t seed) : s(0x9E3779B97F4A7C15ull * (uint64_t)(uint32_t)seed + 0x1234567ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// C(n+d, d), or kMaxMonomials + 1 once it is exceeded
int64_t monomial_count(int n, int d) {
  int64_t c = 1;
  for (int k = 1; k <= d; ++k) {
    c = c * (n + k) / k;  // exact: c is C(n+k, k) after this step
    if (c > kMaxMonomials) return kMaxMonomials + 1;
  }
  return c;
}

void list_degree(int n, int j, int rest, std::vector<int>& cur, std::vector<int>& out) {
  if (j == n - 1) {
    cur[j] = rest;
    out.insert(out.end(), cur.begin(), cur.end());
    return;
  }
  for (int e = rest; e >= 0; --e) {
    cur[j] = e;
    list_degree(n, j + 1, rest - e, cur, out);
  }
}

// exponent vectors with |a| <= d, n per vector, highest total degree first
std::vector<int> monomials(int n, int d) {
  std::vector<int> out, cur(n, 0);
  for (int t = d; t >= 0; --t) list_degree(n, 0, t, cur, out);
  return out;
}

// value of x^a from a power table pw[j * (d+1) + e] = x_j^e
inline cd mono(const cd* pw, int n, int d, const int* a) {
  cd v = 1.0;
  for (int j = 0; j < n; ++j)
    if (a[j]) v *= pw[j * (d + 1) + a[j]];
  return v;
}

void power_table(const cd* x, int n, int d, std::vector<cd>& pw) {
  pw.assign((size_t)n * (d + 1), cd(1.0));
  for (int j = 0; j < n; ++j)
    for (int e = 1; e <= d; ++e) pw[j * (d + 1) + e] = pw[j * (d + 1) + e - 1] * x[j];
}

// A reusable barrier for a fixed set of threads.
class Barrier {
 public:
  explicit Barrier(int n) : n_(n) {}
  void wait() {
    std::unique_lock<std::mutex> lk(mu_);
    const long gen = gen_;
    if (++count_ == n_) {
      count_ = 0;
      ++gen_;
      cv_.notify_all();
      return;
    }
    cv_.wait(lk, [&] { return gen_ != gen; });
  }

 private:
  std::mutex mu_;
  std::condition_variable cv_;
  int n_, count_ = 0;
  long gen_ = 0;
};

// Least squares min ||A X - B|| for A rows x cols (rows >= cols) and B
// rows x nrhs, both column-major, by Householder QR applied to B as the
// reflections are formed; X overwrites the first cols rows of B. Returns
// false when R has a negligible diagonal entry (rank-deficient design).
// For large designs each reflection is applied to the remaining columns
// by up to 16 threads, each column by one thread in the serial order of
// operations, so the result does not depend on the thread count.
bool least_squares(std::vector<cd>& A, int rows, int cols, std::vector<cd>& B, int nrhs) {
  std::vector<cd> diag(cols);
  double dmax = 0.0, vv = 0.0;
  bool failed = false;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  int T = cols >= 192 ? (int)std::min(hw, 16u) : 1;
  std::unique_ptr<Barrier> bar;
  auto work = [&](int t) {
    for (int k = 0; k < cols; ++k) {
      cd* a = &A[(size_t)k * rows];
      if (t == 0) {  // the reflection of column k: v = x - alpha e_k in place
        double ss = 0.0;
        for (int i = k; i < rows; ++i) ss += std::norm(a[i]);
        const double s = std::sqrt(ss);
        if (s == 0.0) {
          failed = true;
        } else {
          const double ak = std::abs(a[k]);
          const cd alpha = ak == 0.0 ? cd(-s) : -(a[k] / ak) * s;
          a[k] -= alpha;
          vv = 0.0;
          for (int i = k; i < rows; ++i) vv += std::norm(a[i]);
          diag[k] = alpha;
          dmax = std::max(dmax, s);
        }
      }
      if (T > 1) bar->wait();
      if (failed) return;
      // columns k+1 .. cols-1, then the right-hand sides, in T contiguous ranges
      const int rest = cols - k - 1, m = rest + nrhs;
      const int lo = (int)((long)m * t / T), hi = (int)((long)m * (t + 1) / T);
      for (int q = lo; q < hi; ++q) {
        cd* y = q < rest ? &A[(size_t)(k + 1 + q) * rows] : &B[(size_t)(q - rest) * rows];
        cd dot = 0.0;
        for (int i = k; i < rows; ++i) dot += std::conj(a[i]) * y[i];
        const cd f = 2.0 * dot / vv;
        for (int i = k; i < rows; ++i) y[i] -= f * a[i];
      }
      if (T > 1) bar->wait();
    }
  };
  // Helper threads wait at a gate until the whole pool exists. If a thread
  // cannot be created (std::system_error), the gate tells the ones already
  // started to return, and the factorization runs on this thread alone.
  std::vector<std::thread> pool;
  std::mutex gate_mu;
  std::condition_variable gate_cv;
  int gate = T > 1 ? 0 : 1;  // 0 closed, 1 run, 2 abandon
  bool pool_ok = true;
  try {
    for (int t = 1; t < T; ++t)
      pool.emplace_back([&, t] {
        {
          std::unique_lock<std::mutex> lk(gate_mu);
          gate_cv.wait(lk, [&] { return gate != 0; });
          if (gate == 2) return;
        }
        work(t);
      });
  } catch (const std::system_error&) {
    pool_ok = false;
  }
  if (!pool_ok) {
    {
      std::lock_guard<std::mutex> lk(gate_mu);
      gate = 2;
    }
    gate_cv.notify_all();
    for (auto& th : pool) th.join();
    pool.clear();
    T = 1;
  }
  bar.reset(new Barrier(T));
  if (T > 1) {
    {
      std::lock_guard<std::mutex> lk(gate_mu);
      gate = 1;
    }
    gate_cv.notify_all();
  }
  work(0);
  for (auto& th : pool) th.join();
  if (failed) return false;
  for (int k = 0; k < cols; ++k)
    if (std::abs(diag[k]) <= 1e-10 * dmax) return false;
  for (int r = 0; r < nrhs; ++r) {
    cd* b = &B[(size_t)r * rows];
    for (int k = cols - 1; k >= 0; --k) {
      cd acc = b[k];
      for (int c = k + 1; c < cols; ++c) acc -= A[(size_t)c * rows + k] * b[c];
      b[k] = acc / diag[k];
    }
  }
  return true;
}

struct Evaluator {
  phc_evaluator fn;
  void* ctx;
  int n;
  std::vector<double> xb, fb, jb;
  explicit Evaluator(phc_evaluator f, void* c, int n_)
      : fn(f), ctx(c), n(n_), xb(2 * n_), fb(2 * n_), jb(2 * (size_t)n_ * n_) {}
  // F(x) into f[n], dF/dx into jac (jac(i, j) at i + j n); status of the callback
  int32_t operator()(const cd* x, cd* f, cd* jac) {
    for (int j = 0; j < n; ++j) {
      xb[2 * j] = x[j].real();
      xb[2 * j + 1] = x[j].imag();
    }
    std::fill(fb.begin(), fb.end(), 0.0);
    std::fill(jb.begin(), jb.end(), 0.0);
    const int32_t st = fn(ctx, n, xb.data(), fb.data(), jb.data());
    if (st != 0) return st;
    for (int i = 0; i < n; ++i) f[i] = cd(fb[2 * i], fb[2 * i + 1]);
    if (jac)
      for (size_t q = 0; q < (size_t)n * n; ++q) jac[q] = cd(jb[2 * q], jb[2 * q + 1]);
    for (double v : fb)
      if (!std::isfinite(v)) return PHC_ERR_INVALID_INPUT;
    for (double v : jb)
      if (!std::isfinite(v)) return PHC_ERR_INVALID_INPUT;
    return 0;
  }
};

struct Equation {
  std::vector<int> exps;  // n per kept term
  std::vector<cd> coefs;
};

}  // namespace

extern "C" int32_t phc_sparse_sample(phc_sparse* s, int32_t n, const int32_t* degrees,
                                     phc_evaluator eval, void* ctx, int32_t seed,
                                     double* max_error) {
  phc::NvtxRange range("phc sample user system");
  if (max_error) *max_error = 0.0;
  if (!s) return PHC_ERR_BAD_HANDLE;
  if (n < 1 || n >= 32 || !degrees || !eval) return PHC_ERR_INVALID_INPUT;
  for (int i = 0; i < n; ++i)
    if (degrees[i] < 1) return PHC_ERR_INVALID_INPUT;
  std::map<int, std::vector<int>> by_degree;  // degree -> equations
  for (int i = 0; i < n; ++i) by_degree[degrees[i]].push_back(i);
  for (auto& kv : by_degree)
    if (monomial_count(n, kv.first) > kMaxMonomials) return PHC_ERR_UNSUPPORTED;

  Evaluator F(eval, ctx, n);
  Rng rng(seed);
  std::vector<Equation> eqs(n);
  std::vector<cd> x(n), f(n), pw;
  for (auto& kv : by_degree) {
    const int d = kv.first;
    const std::vector<int>& rows_of = kv.second;
    const std::vector<int> mon = monomials(n, d);
    const int m = (int)(mon.size() / n);
    const int P = 2 * m;
    std::vector<cd> A((size_t)P * m), B((size_t)P * rows_of.size());
    for (int p = 0; p < P; ++p) {
      for (int j = 0; j < n; ++j) x[j] = std::polar(1.0, 2.0 * M_PI * rng.uniform());
      const int32_t st = F(x.data(), f.data(), nullptr);
      if (st != 0) return st == PHC_ERR_INVALID_INPUT ? st : PHC_ERR_ABORTED;
      power_table(x.data(), n, d, pw);
      for (int k = 0; k < m; ++k) A[(size_t)k * P + p] = mono(pw.data(), n, d, &mon[(size_t)k * n]);
      for (size_t r = 0; r < rows_of.size(); ++r) B[r * P + p] = f[rows_of[r]];
    }
    if (!least_squares(A, P, m, B, (int)rows_of.size())) return PHC_ERR_NUMERICAL;
    for (size_t r = 0; r < rows_of.size(); ++r) {
      const cd* c = &B[r * P];
      double l1 = 0.0;
      for (int k = 0; k < m; ++k) l1 += std::abs(c[k]);
      const double tau = kSnap * l1;
      Equation& e = eqs[rows_of[r]];
      int top = 0;
      for (int k = 0; k < m; ++k) {
        const double re = std::abs(c[k].real()) <= tau ? 0.0 : c[k].real();
        const double im = std::abs(c[k].imag()) <= tau ? 0.0 : c[k].imag();
        if (re == 0.0 && im == 0.0) continue;
        const int* a = &mon[(size_t)k * n];
        int deg = 0;
        for (int j = 0; j < n; ++j) deg += a[j];
        top = std::max(top, deg);
        e.exps.insert(e.exps.end(), a, a + n);
        e.coefs.emplace_back(re, im);
      }
      if (top != d) return PHC_ERR_INVALID_INPUT;  // stated degree not exact
    }
  }

  // the table against the user's F and Jacobian at fresh points
  double worst = 0.0;
  std::vector<cd> jac((size_t)n * n);
  for (int p = 0; p < kCheckPoints; ++p) {
    const bool torus = p < kCheckPoints / 2;
    for (int j = 0; j < n; ++j)
      x[j] = std::polar(torus ? 1.0 : 0.5 + rng.uniform(), 2.0 * M_PI * rng.uniform());
    const int32_t st = F(x.data(), f.data(), jac.data());
    if (st != 0) return st == PHC_ERR_INVALID_INPUT ? st : PHC_ERR_ABORTED;
    for (int i = 0; i < n; ++i) {
      const int d = degrees[i];
      power_table(x.data(), n, d, pw);
      const Equation& e = eqs[i];
      const int T = (int)e.coefs.size();
      cd val = 0.0;
      double scale = 0.0;
      std::vector<cd> g(n, cd(0.0));
      std::vector<double> gscale(n, 0.0);
      for (int t = 0; t < T; ++t) {
        const int* a = &e.exps[(size_t)t * n];
        const cd term = e.coefs[t] * mono(pw.data(), n, d, a);
        val += term;
        scale += std::abs(term);
        for (int j = 0; j < n; ++j) {
          if (!a[j]) continue;
          // a_j c x^(a - e_j), from the power table without dividing by x_j
          cd v = e.coefs[t] * (double)a[j];
          for (int l = 0; l < n; ++l) {
            const int el = l == j ? a[l] - 1 : a[l];
            if (el) v *= pw[l * (d + 1) + el];
          }
          g[j] += v;
          gscale[j] += std::abs(v);
        }
      }
      worst = std::max(worst, std::abs(val - f[i]) / std::max(scale, 1e-300));
      for (int j = 0; j < n; ++j) {
        const double sc = std::max(gscale[j], scale);
        worst = std::max(worst, std::abs(g[j] - jac[i + (size_t)j * n]) / std::max(sc, 1e-300));
      }
    }
  }
  if (max_error) *max_error = worst;
  if (!(worst <= kCheckTol)) return PHC_ERR_INVALID_INPUT;

  int32_t st = phc_sparse_init(s, n);
  if (st != PHC_OK) return st;
  std::vector<double> cbuf;
  for (int i = 0; i < n; ++i) {
    const Equation& e = eqs[i];
    const int T = (int)e.coefs.size();
    cbuf.resize(2 * (size_t)T);
    for (int t = 0; t < T; ++t) {
      cbuf[2 * t] = e.coefs[t].real();
      cbuf[2 * t + 1] = e.coefs[t].imag();
    }
    st = phc_sparse_add_equation(s, T, cbuf.data(), n, T, e.exps.data());
    if (st != PHC_OK) return st;
  }
  return PHC_OK;
}

// host_fuzz.cpp -- randomized driver for the library's host C++ under
// AddressSanitizer and UndefinedBehaviorSanitizer (test infrastructure; it
// is built and run by tests/test_host_sanitizers.py, never shipped).
//
// It needs no GPU: it drives the host-only parts of the C ABI and the table
// compiler directly.
//   - sparse builder, homotopy set-up and the table compiler (with its
//     verifier) on random systems, and the verifier on corrupted tables;
//   - the compact request codec: round trips, truncated and bit-flipped
//     requests;
//   - the bookkeeping (phc_finish_solve) on random path records with
//     near-duplicate endpoints at the tolerance boundaries and extreme
//     magnitudes;
//   - the user-system sampler on random polynomial evaluators.
// Usage: host_fuzz <iterations> <seed>. Exit status 0 when every invariant
// held; the sanitizers abort the process on the first memory or UB error.
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "phc_host.h"
#include "polyhomocont_b200.h"

namespace {

std::mt19937_64 rng;
long n_plans = 0, n_rejected = 0, n_wire = 0, n_books = 0, n_samples = 0;

int uni(int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); }
double unif() { return std::uniform_real_distribution<double>(0.0, 1.0)(rng); }
double normal() { return std::normal_distribution<double>(0.0, 1.0)(rng); }

#define CHECK(c)                                                              \
  do {                                                                        \
    if (!(c)) {                                                               \
      std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c);    \
      std::exit(2);                                                           \
    }                                                                         \
  } while (0)

struct Sys {
  int n = 0;
  std::vector<int> deg;
  // per equation: coefs (interleaved) and the n x T exponent matrix
  std::vector<std::vector<double>> coefs;
  std::vector<std::vector<int32_t>> exps;
};

Sys random_system(int nmax, int dmax, int tmax) {
  Sys s;
  s.n = uni(1, nmax);
  for (int i = 0; i < s.n; ++i) {
    const int d = uni(1, dmax);
    const int T = uni(1, tmax);
    std::vector<double> c;
    std::vector<int32_t> e;
    for (int k = 0; k < T; ++k) {
      // one term of exact degree d, the rest of degree <= d
      int left = (k == 0) ? d : uni(0, d);
      std::vector<int32_t> a(s.n, 0);
      while (left > 0) {
        a[uni(0, s.n - 1)] += 1;
        --left;
      }
      e.insert(e.end(), a.begin(), a.end());
      c.push_back(normal());
      c.push_back(normal());
    }
    // the exponent matrix is n x T column-major: term k is column k
    s.deg.push_back(d);
    s.coefs.push_back(c);
    s.exps.push_back(e);
  }
  return s;
}

// n equations of exact degree d with T terms each
Sys fixed_system(int n, int d, int T) {
  Sys s;
  s.n = n;
  for (int i = 0; i < n; ++i) {
    std::vector<double> c;
    std::vector<int32_t> e;
    for (int k = 0; k < T; ++k) {
      int left = (k == 0) ? d : uni(0, d);
      std::vector<int32_t> a(n, 0);
      while (left-- > 0) a[uni(0, n - 1)] += 1;
      e.insert(e.end(), a.begin(), a.end());
      c.push_back(normal());
      c.push_back(normal());
    }
    s.deg.push_back(d);
    s.coefs.push_back(c);
    s.exps.push_back(e);
  }
  return s;
}

phc_sparse* build(const Sys& s) {
  phc_sparse* b = phc_sparse_create();
  CHECK(b != nullptr);
  CHECK(phc_sparse_init(b, s.n) == PHC_OK);
  for (int i = 0; i < s.n; ++i) {
    const int T = (int)s.coefs[i].size() / 2;
    CHECK(phc_sparse_add_equation(b, T, s.coefs[i].data(), s.n, T, s.exps[i].data()) == PHC_OK);
  }
  return b;
}

void fuzz_plan(const Sys& s) {
  phc_sparse* b = build(s);
  phc_system t;
  CHECK(phc_sparse_table(b, &t) == PHC_OK);
  std::vector<double> gamma(2), bb(2 * s.n), patch(2 * (s.n + 1));
  int64_t nstart = 0;
  const int32_t hs = phc_homotopy_init(&t, uni(1, 1000), gamma.data(), bb.data(), patch.data(),
                                       &nstart);
  if (hs != PHC_OK) {  // Bezout number out of range: rejected, nothing to compile
    ++n_rejected;
    phc_sparse_destroy(b);
    return;
  }
  phc_homotopy h{{gamma[0], gamma[1]}, bb.data(), patch.data()};
  // host evaluation of the table: F, F^h and their Jacobians at a random point
  {
    std::vector<double> z(2 * (s.n + 1)), f(2 * s.n), jac(2 * (size_t)s.n * (s.n + 1));
    for (auto& v : z) v = normal();
    CHECK(phc_sparse_evaluate(b, z.data(), f.data(), jac.data()) == PHC_OK);
    CHECK(phc_sparse_evaluate_homogeneous(b, z.data(), f.data(), jac.data()) == PHC_OK);
    for (double v : f) CHECK(std::isfinite(v));
  }
  phc::HostPlan hp;
  const int st = phc::build_plan(&t, &h, &hp);
  CHECK(st == PHC_OK || st == PHC_ERR_UNSUPPORTED || st == PHC_ERR_INVALID_INPUT);
  if (st == PHC_OK) {
    ++n_plans;
    CHECK(phc::verify_plan(hp.bytes.data(), hp.bytes.size()) == PHC_OK);
    // corrupted copies: the verifier must answer without reading out of bounds
    for (int r = 0; r < 8; ++r) {
      std::vector<unsigned char> bad(hp.bytes);
      const size_t at = (size_t)uni(0, (int)bad.size() - 1);
      bad[at] ^= (unsigned char)(1u << uni(0, 7));
      (void)phc::verify_plan(bad.data(), bad.size());
    }
    // header words overwritten with arbitrary values (sizes, offsets, counts)
    for (int r = 0; r < 8; ++r) {
      std::vector<unsigned char> bad(hp.bytes);
      const size_t word = (size_t)uni(0, (int)(sizeof(phc::PlanHeader) / 4) - 1);
      const uint32_t v = (uint32_t)rng();
      std::memcpy(bad.data() + 4 * word, &v, 4);
      (void)phc::verify_plan(bad.data(), bad.size());
    }
    std::vector<unsigned char> shortened(hp.bytes.begin(), hp.bytes.begin() + hp.bytes.size() / 2);
    CHECK(phc::verify_plan(shortened.data(), shortened.size()) != PHC_OK);
  }
  phc_sparse_destroy(b);
}

void fuzz_wire(const Sys& s) {
  phc_sparse* b = build(s);
  phc_system t;
  CHECK(phc_sparse_table(b, &t) == PHC_OK);
  phc_solve_options o;
  phc_default_solve_options(&o);
  o.seed = uni(1, 100);
  const int64_t size = phc_request_size(&t, 1);
  CHECK(size > 0);
  std::vector<unsigned char> buf((size_t)size);
  int64_t len = 0;
  CHECK(phc_request_encode(&t, &o, buf.data(), size, &len) == PHC_OK && len == size);
  // round trip: same table, same options
  phc_sparse* d = phc_sparse_create();
  phc_solve_options o2;
  CHECK(phc_request_decode(buf.data(), len, d, &o2) == PHC_OK);
  phc_system t2;
  CHECK(phc_sparse_table(d, &t2) == PHC_OK);
  CHECK(t2.n == t.n && t2.nterms == t.nterms);
  CHECK(std::memcmp(t2.first, t.first, sizeof(int32_t) * (t.n + 1)) == 0);
  CHECK(std::memcmp(t2.hexps, t.hexps, sizeof(int32_t) * (size_t)t.nterms * (t.n + 1)) == 0);
  CHECK(std::memcmp(t2.coefs, t.coefs, sizeof(double) * 2 * (size_t)t.nterms) == 0);
  CHECK(o2.seed == o.seed);
  ++n_wire;
  phc_sparse_destroy(d);
  // requests with a 16- or 32-bit field overwritten by an arbitrary value
  // (counts, sizes, exponents, variable indices): any status, no memory error
  for (int r = 0; r < 16 && len >= 4; ++r) {
    std::vector<unsigned char> bad(buf.begin(), buf.begin() + len);
    const size_t at = (size_t)uni(0, (int)len - 4);
    const uint32_t v = (uint32_t)rng();
    std::memcpy(bad.data() + at, &v, uni(0, 1) ? 4 : 2);
    phc_sparse* e = phc_sparse_create();
    phc_solve_options o3;
    (void)phc_request_decode(bad.data(), (int64_t)bad.size(), e, &o3);
    phc_sparse_destroy(e);
  }
  // damaged requests: any status, no memory error
  for (int r = 0; r < 16; ++r) {
    std::vector<unsigned char> bad(buf.begin(), buf.begin() + uni(0, (int)len));
    if (!bad.empty() && uni(0, 1)) bad[(size_t)uni(0, (int)bad.size() - 1)] ^= (unsigned char)uni(1, 255);
    phc_sparse* e = phc_sparse_create();
    phc_solve_options o3;
    (void)phc_request_decode(bad.empty() ? nullptr : bad.data(), (int64_t)bad.size(), e, &o3);
    phc_sparse_destroy(e);
  }
  phc_sparse_destroy(b);
}

void fuzz_bookkeeping() {
  const int n = uni(1, 12);
  const int64_t np = uni(1, 400);
  phc_solve_options o;
  phc_default_solve_options(&o);
  // a few base points; paths land on them with offsets around the tolerances
  std::vector<std::vector<std::complex<double>>> base(uni(1, 6));
  const double scale = std::pow(10.0, uni(-150, 150) * (uni(0, 3) == 0 ? 1.0 : 0.0));
  for (auto& p : base) {
    p.resize(n);
    for (auto& v : p) v = scale * std::complex<double>(normal(), uni(0, 2) ? normal() : 0.0);
  }
  std::vector<phc_path_out> paths((size_t)np);
  std::vector<double> x((size_t)np * n * 2);
  for (int64_t k = 0; k < np; ++k) {
    phc_path_out& p = paths[(size_t)k];
    std::memset(&p, 0, sizeof(p));
    p.status = uni(0, 9) == 0 ? uni(1, 3) : 0;
    p.at_infinity = uni(0, 7) == 0;
    p.singular = uni(0, 5) == 0;
    p.winding_number = 1 + p.singular * uni(1, 4);
    const auto& b = base[(size_t)uni(0, (int)base.size() - 1)];
    const double tol = p.singular ? o.singular_dedup_tol : o.dedup_tol;
    const double off = tol * std::max(1.0, scale) * (0.5 + unif()) * (uni(0, 1) ? 1.0 : 0.999999999);
    for (int j = 0; j < n; ++j) {
      const std::complex<double> v = b[j] + (j == 0 ? off * std::polar(1.0, 6.283 * unif()) : 0.0);
      x[((size_t)k * n + j) * 2] = v.real();
      x[((size_t)k * n + j) * 2 + 1] = v.imag();
    }
  }
  std::vector<double> sols((size_t)np * n * 2), rsols((size_t)np * n), ssols((size_t)np * n * 2);
  std::vector<int32_t> mult((size_t)np);
  phc_solve_result res;
  std::memset(&res, 0, sizeof(res));
  res.solutions = sols.data();
  res.real_solutions = rsols.data();
  res.singular_solutions = ssols.data();
  res.multiplicities = mult.data();
  CHECK(phc_finish_solve(n, np, &o, paths.data(), x.data(), &res) == PHC_OK);
  int64_t regular = 0, singular = 0, infinite = 0, failed = 0, msum = 0;
  for (int64_t k = 0; k < np; ++k) {
    const phc_path_out& p = paths[(size_t)k];
    if (p.status != 0) {
      ++failed;
    } else if (p.at_infinity) {
      ++infinite;
    } else if (p.singular) {
      ++singular;
      CHECK(p.singular_index >= 1 && p.singular_index <= res.counts.nsingular);
    } else {
      ++regular;
      CHECK(p.solution_index >= 1 && p.solution_index <= res.counts.nsolutions);
    }
  }
  for (int i = 0; i < res.counts.nsingular; ++i) msum += mult[(size_t)i];
  CHECK(res.counts.nfailed == failed && res.counts.ninfinite == infinite);
  CHECK(res.counts.nsolutions + res.counts.nduplicates == regular);
  CHECK(msum == singular);
  CHECK(res.counts.nreal <= res.counts.nsolutions);
  ++n_books;
}

// evaluator of a random sparse system for the sampler: F(x) and dF/dx
struct EvalCtx {
  const Sys* s;
};

int32_t evaluate(void* ctx, int32_t n, const double* xr, double* f, double* jac) {
  const Sys& s = *static_cast<EvalCtx*>(ctx)->s;
  std::vector<std::complex<double>> x(n);
  for (int j = 0; j < n; ++j) x[j] = {xr[2 * j], xr[2 * j + 1]};
  for (int i = 0; i < n; ++i) {
    std::complex<double> fi = 0.0;
    std::vector<std::complex<double>> g(n, 0.0);
    const int T = (int)s.coefs[i].size() / 2;
    for (int k = 0; k < T; ++k) {
      const std::complex<double> c(s.coefs[i][2 * k], s.coefs[i][2 * k + 1]);
      const int32_t* a = &s.exps[i][(size_t)k * n];
      std::complex<double> m = c;
      for (int j = 0; j < n; ++j)
        for (int e = 0; e < a[j]; ++e) m *= x[j];
      fi += m;
      for (int j = 0; j < n; ++j) {
        if (!a[j]) continue;
        std::complex<double> dm = c * (double)a[j];
        for (int l = 0; l < n; ++l)
          for (int e = 0; e < (l == j ? a[l] - 1 : a[l]); ++e) dm *= x[l];
        g[j] += dm;
      }
    }
    f[2 * i] = fi.real();
    f[2 * i + 1] = fi.imag();
    for (int j = 0; j < n; ++j) {
      jac[2 * ((size_t)i + (size_t)j * n)] = g[j].real();
      jac[2 * ((size_t)i + (size_t)j * n) + 1] = g[j].imag();
    }
  }
  return 0;
}

void fuzz_sampler(const Sys& s) {
  EvalCtx ctx{&s};
  phc_sparse* b = phc_sparse_create();
  double err = -1.0;
  const int32_t st = phc_sparse_sample(b, s.n, s.deg.data(), evaluate, &ctx, uni(1, 50), &err);
  CHECK(st == PHC_OK);
  CHECK(err >= 0.0 && err <= 1e-9);
  int32_t d[32];
  phc_sparse_degrees(b, d);
  for (int i = 0; i < s.n; ++i) CHECK(d[i] == s.deg[i]);
  // a stated degree one too high is not exact: rejected
  std::vector<int32_t> wrong(s.deg.begin(), s.deg.end());
  wrong[0] += 1;
  phc_sparse* c = phc_sparse_create();
  CHECK(phc_sparse_sample(c, s.n, wrong.data(), evaluate, &ctx, 1, &err) == PHC_ERR_INVALID_INPUT);
  ++n_samples;
  phc_sparse_destroy(c);
  phc_sparse_destroy(b);
}

}  // namespace

int main(int argc, char** argv) {
  const int iters = argc > 1 ? std::atoi(argv[1]) : 200;
  rng.seed(argc > 2 ? (uint64_t)std::atoll(argv[2]) : 1);
  for (int it = 0; it < iters; ++it) {
    const Sys a = random_system(it % 10 == 0 ? 31 : 12, 5, 30);
    fuzz_plan(a);
    fuzz_wire(a);
    fuzz_bookkeeping();
    if (it % 4 == 0) fuzz_sampler(random_system(5, 3, 8));
    // 210 monomials of degree <= 4 in 6 unknowns: the threaded least squares
    if (it % 150 == 0) fuzz_sampler(fixed_system(6, 4, 12));
  }
  std::printf("host_fuzz: %d iterations ok: %ld tables compiled and verified (%ld systems with "
              "too many paths), %ld request round trips, %ld bookkeeping runs, %ld sampled "
              "systems\n",
              iters, n_plans, n_rejected, n_wire, n_books, n_samples);
  // every part ran
  CHECK(n_plans > 0 && n_wire > 0 && n_books > 0 && n_samples > 0);
  return 0;
}

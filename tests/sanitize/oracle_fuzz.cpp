// oracle_fuzz.cpp -- the CPU restatement of solve() (oracle/phc_oracle.cpp)
// on random small systems under AddressSanitizer and
// UndefinedBehaviorSanitizer (test infrastructure; built and run by
// tests/test_host_sanitizers.py).
//
// Each iteration builds a random system (n <= 4, degrees <= 3, a few terms,
// sometimes with zero coefficients, repeated monomials or random seeds and
// options), solves it with two host threads, and checks the invariants of
// the result: every path is regular, singular, infinite or failed;
// solutions plus duplicates are the regular paths; multiplicities sum to
// the singular paths. Usage: oracle_fuzz <iterations> <seed>.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "phc_oracle.h"

namespace {

std::mt19937_64 rng;
int uni(int lo, int hi) { return std::uniform_int_distribution<int>(lo, hi)(rng); }
double normal() { return std::normal_distribution<double>(0.0, 1.0)(rng); }

#define CHECK(c)                                                            \
  do {                                                                      \
    if (!(c)) {                                                             \
      std::fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c);  \
      std::exit(2);                                                         \
    }                                                                       \
  } while (0)

}  // namespace

int main(int argc, char** argv) {
  const int iters = argc > 1 ? std::atoi(argv[1]) : 50;
  rng.seed(argc > 2 ? (uint64_t)std::atoll(argv[2]) : 1);
  long solved = 0, rejected = 0, paths_total = 0;
  for (int it = 0; it < iters; ++it) {
    const int n = uni(1, 4);
    void* sys = orc_sparse_new();
    orc_sparse_init(sys, n);
    int st = 0;
    for (int i = 0; i < n && st == 0; ++i) {
      const int d = uni(1, 3), T = uni(1, 6);
      std::vector<double> c;
      std::vector<int32_t> e((size_t)n * T, 0);
      for (int k = 0; k < T; ++k) {
        int left = (k == 0) ? d : uni(0, d);
        while (left-- > 0) e[(size_t)k * n + uni(0, n - 1)] += 1;
        const bool zero = uni(0, 9) == 0;
        c.push_back(zero ? 0.0 : normal());
        c.push_back(zero ? 0.0 : normal());
      }
      st = orc_sparse_add_equation(sys, T, c.data(), n, T, e.data());
    }
    orc_solve_options o;
    orc_default_solve_options(&o);
    o.seed = uni(1, 1000);
    o.use_endgame = uni(0, 4) != 0;
    o.tracker.max_steps = uni(0, 3) == 0 ? uni(1, 50) : o.tracker.max_steps;
    const int64_t np = (st == 0) ? orc_bezout(sys) : 0;
    const int64_t m = np > 0 ? np : 1;
    std::vector<orc_path_out> paths((size_t)m);
    std::vector<double> z((size_t)m * (n + 1) * 2), x((size_t)m * n * 2);
    std::vector<double> sols((size_t)m * n * 2), rsols((size_t)m * n), ssols((size_t)m * n * 2);
    std::vector<int32_t> mult((size_t)m);
    orc_solve_counts cnt{};
    const int32_t ss = orc_solve(sys, &o, 2, paths.data(), z.data(), x.data(), &cnt, sols.data(),
                                 rsols.data(), ssols.data(), mult.data());
    if (ss != 0) {
      ++rejected;
    } else {
      ++solved;
      paths_total += cnt.npaths;
      CHECK(cnt.npaths == np && cnt.n == n);
      long regular = 0, singular = 0, infinite = 0, failed = 0, msum = 0;
      for (int64_t k = 0; k < np; ++k) {
        const orc_path_out& p = paths[(size_t)k];
        if (p.status != 0)
          ++failed;
        else if (p.at_infinity)
          ++infinite;
        else if (p.singular)
          ++singular;
        else
          ++regular;
      }
      for (int i = 0; i < cnt.nsingular; ++i) msum += mult[(size_t)i];
      CHECK(cnt.nfailed == failed && cnt.ninfinite == infinite);
      CHECK(cnt.nsolutions + cnt.nduplicates == regular);
      CHECK(msum == singular);
    }
    orc_sparse_free(sys);
  }
  std::printf("oracle_fuzz: %d iterations ok: %ld systems solved (%ld paths), %ld rejected\n",
              iters, solved, paths_total, rejected);
  CHECK(solved > 0);
  return 0;
}

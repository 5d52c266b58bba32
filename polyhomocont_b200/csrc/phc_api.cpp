// phc_api.cpp -- C ABI of the B200 path tracker (include/polyhomocont_b200.h).
//
// Host side of the drop-in for solve() (src/solve.f90:154-215): the
// sparse_system builder, the homotopy set-up with the reference generator,
// device buffers and launches, and the order-dependent bookkeeping of the
// solve driver. There is no CPU fallback: without a usable CUDA device
// every entry point that needs one returns PHC_ERR_NO_DEVICE.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <complex>
#include <limits>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <chrono>
#include <mutex>
#include <thread>
#include <new>
#include <string>
#include <vector>

#include "phc_host.h"

namespace phc {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

void set_last_error(const std::string& s) { g_last_error = s; }
std::string last_error_text() { return g_last_error; }

int cuda_fail(cudaError_t e, const char* what) {
  set_last_error(std::string(what) + ": " + cudaGetErrorString(e));
  if (e == cudaErrorMemoryAllocation) return PHC_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice)
    return PHC_ERR_NO_DEVICE;
  return PHC_ERR_CUDA;
}

#define PHC_CUDA(call)                                   \
  do {                                                   \
    cudaError_t e_ = (call);                             \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);  \
  } while (0)

// ---------------------------------------------------------------------------
// options
// ---------------------------------------------------------------------------
phc_solve_options solve_defaults() {
  phc_solve_options o;
  std::memset(&o, 0, sizeof(o));
  o.tracker.step_init = 0.05;       // src/tracker.f90:60-76
  o.tracker.step_max = 0.1;
  o.tracker.step_min = 1.0e-14;
  o.tracker.corrector_tol = 1.0e-10;
  o.tracker.corrector_maxit = 3;
  o.tracker.contraction = 0.5;
  o.tracker.grow_after = 5;
  o.tracker.max_steps = 20000;
  o.endgame.t_start = 0.1;          // src/endgame.f90:75-100
  o.endgame.nsamples = 8;
  o.endgame.radius_factor = 0.25;
  o.endgame.radius_min = 1.0e-13;
  o.endgame.max_winding = 16;
  o.endgame.loop_radius = 1.0e-5;
  o.endgame.winding_agreement = 0.2;
  o.endgame.tol = 1.0e-11;
  o.endgame.residual_tol = 1.0e-8;
  o.endgame.closure_factor = 0.1;
  o.use_endgame = 1;                // src/solve.f90:63-83
  o.seed = 1;
  o.refine_maxit = 5;
  o.infinity_tol = 1.0e-8;
  o.singular_cond = 1.0e10;
  o.real_tol = 1.0e-8;
  o.dedup_tol = 1.0e-8;
  o.singular_dedup_tol = 1.0e-6;
  return o;
}

phc_gpu_options gpu_defaults() {
  phc_gpu_options g;
  std::memset(&g, 0, sizeof(g));
  g.precision = PHC_PREC_MIXED;
  g.schedule = PHC_SCHED_PERSISTENT;
  g.device = 0;
  g.warps_per_block = 0;
  g.blocks_per_sm = 0;
  g.chunk = 1;
  g.fp64_sticky = -1;
  return g;
}

// The reference runs with any option values; on the GPU, values that would
// make a loop run forever (radius_factor >= 1, no samples per loop, ...)
// are rejected up front.
int validate_options(const phc_solve_options* o) {
  const phc_tracker_options& t = o->tracker;
  const phc_endgame_options& e = o->endgame;
  if (!(t.step_min > 0.0) || !(t.step_init > 0.0) || !(t.step_max > 0.0)) return PHC_ERR_INVALID_INPUT;
  if (t.corrector_maxit < 1 || t.grow_after < 1 || t.max_steps < 0) return PHC_ERR_INVALID_INPUT;
  if (!(t.corrector_tol >= 0.0)) return PHC_ERR_INVALID_INPUT;
  if (o->use_endgame) {
    if (e.nsamples < 1 || e.max_winding < 1) return PHC_ERR_INVALID_INPUT;
    if (!(e.radius_factor > 0.0 && e.radius_factor < 1.0)) return PHC_ERR_INVALID_INPUT;
    if (!(e.radius_min > 0.0) || !(e.t_start > 0.0 && e.t_start < 1.0)) return PHC_ERR_INVALID_INPUT;
  }
  if (o->refine_maxit < 0) return PHC_ERR_INVALID_INPUT;
  return PHC_OK;
}

KOpts make_kopts(const phc_solve_options& so, const phc_gpu_options& g) {
  KOpts k;
  std::memset(&k, 0, sizeof(k));
  k.so = so;
  k.precision = g.precision;
  k.fp64_sticky = g.fp64_sticky < 0 ? 4 : g.fp64_sticky;
  // safety budget of evaluate+LU units per path; by default far above any
  // path the reference tracks in practice, it bounds every kernel's run time
  const int lg = g.unit_budget_log2 > 0 ? std::min(g.unit_budget_log2, 40) : 24;
  k.max_units = (int64_t)1 << lg;
  return k;
}

// ---------------------------------------------------------------------------
// reference generator (src/random.f90) and hom%init (src/homotopy.f90:104-149)
// ---------------------------------------------------------------------------
namespace {
struct Rng {
  int64_t s1 = 1234567, s2 = 7654321;
  void seed(int seed) {
    int64_t s = std::llabs((int64_t)seed);
    s1 = s % (2147483563LL - 1) + 1;
    s2 = (s * 7919LL + 104729LL) % (2147483399LL - 1) + 1;
    for (int i = 0; i < 16; ++i) uniform();
  }
  double uniform() {
    s1 = (40014LL * s1) % 2147483563LL;
    s2 = (40692LL * s2) % 2147483399LL;
    int64_t z = s1 - s2;
    if (z < 1) z += 2147483563LL - 1;
    return (double)z / 2147483563.0;
  }
  void unit_complex(double* z) {
    const double phi = 2.0 * 3.14159265358979323846 * uniform();
    z[0] = std::cos(phi);
    z[1] = std::sin(phi);
  }
  void normal_complex(double* z) {
    const double r = std::sqrt(-std::log(uniform()));
    const double phi = 2.0 * 3.14159265358979323846 * uniform();
    z[0] = r * std::cos(phi);
    z[1] = r * std::sin(phi);
  }
};
}  // namespace

int homotopy_init(const phc_system* sys, int seed, HostHomotopy* h) {
  if (sys == nullptr || sys->n < 1 || sys->deg == nullptr) return PHC_ERR_INVALID_INPUT;
  const int n = sys->n;
  int64_t nstart = 1;
  for (int i = 0; i < n; ++i) {
    if (sys->deg[i] < 1) return PHC_ERR_INVALID_INPUT;
    nstart *= sys->deg[i];
    if (nstart > (int64_t)INT32_MAX) return PHC_ERR_INVALID_INPUT;
  }
  Rng g;
  g.seed(seed);
  h->nstart = nstart;
  g.unit_complex(h->gamma);
  h->b.assign(2 * n, 0.0);
  for (int i = 0; i < n; ++i) g.unit_complex(&h->b[2 * i]);
  h->patch.assign(2 * (n + 1), 0.0);
  for (int i = 0; i <= n; ++i) g.normal_complex(&h->patch[2 * i]);
  double ss = 0.0;
  for (int i = 0; i <= n; ++i) {
    const double a = std::hypot(h->patch[2 * i], h->patch[2 * i + 1]);
    ss += a * a;
  }
  const double nrm = std::sqrt(ss);
  for (int i = 0; i < 2 * (n + 1); ++i) h->patch[i] = h->patch[i] / nrm;
  return PHC_OK;
}

// ---------------------------------------------------------------------------
// launch configuration
// ---------------------------------------------------------------------------
int device_smem_optin(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess)
    return 48 * 1024;
  return v;
}
int device_sms(int device) {
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 1;
  return v;
}

bool use_lean(int64_t paths, int device) {
  return paths > (int64_t)2 * kLeanPathsPerSm * device_sms(device);
}

int resolve_launch(const HostPlan& hp, const phc_gpu_options& g, int device, int64_t paths,
                   LaunchCfg* cfg) {
  cfg->nm = kernel_nm(hp.n);
  cfg->lean = use_lean(paths, device) ? 1 : 0;
  if (cfg->nm == 0) {
    set_last_error("more than 32 unknowns");
    return PHC_ERR_UNSUPPORTED;
  }
  cfg->precision = (g.precision == PHC_PREC_MIXED) ? PHC_PREC_MIXED : PHC_PREC_FP64;
  cfg->fac = hp.max_fac <= 1 ? 1 : (hp.max_fac == 2 ? 2 : 3);
  cfg->persistent = (g.schedule == PHC_SCHED_PERSISTENT) ? 1 : 0;
  int tw = 4, tc = 1;
  tuned_launch(device, cfg->precision, cfg->persistent, cfg->nm, cfg->lean, &tw, &tc);
  cfg->chunk = g.chunk > 0 ? g.chunk : tc;
  cfg->eval32 = kernel_eval32(cfg->nm, cfg->precision) ? 1 : 0;
  cfg->ws_bytes = ws_layout(hp.n, hp.S, hp.pw_size, cfg->eval32 != 0).bytes;
  // kernels without the FP32 evaluation stage the table without its FP32
  // coefficients
  const int plan_bytes = cfg->eval32 ? align16((int)hp.bytes.size()) : hp.bytes_fp64;
  cfg->plan_bytes = plan_bytes;
  const int smax = device_smem_optin(device);
  int warps = g.warps_per_block > 0 ? g.warps_per_block : tw;
  warps = std::min(std::max(warps, 1), max_warps_per_block(cfg->nm, cfg->lean != 0));
  while (warps > 1 && plan_bytes + warps * cfg->ws_bytes > smax) --warps;
  if (plan_bytes + warps * cfg->ws_bytes > smax) {
    set_last_error("system table does not fit in shared memory");
    return PHC_ERR_UNSUPPORTED;
  }
  cfg->warps = warps;
  cfg->smem = plan_bytes + warps * cfg->ws_bytes;
  int bps = track_blocks_per_sm(*cfg);
  if (bps < 1) bps = 1;
  if (g.blocks_per_sm > 0) bps = std::min(bps, g.blocks_per_sm);
  cfg->grid = device_sms(device) * bps;
  return PHC_OK;
}

// ---------------------------------------------------------------------------
// per-device workspace for the synchronous entry points
// ---------------------------------------------------------------------------
namespace {
struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t need) {
    if (need <= cap) return PHC_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(need, (size_t)4096);
    want += want / 2;
    cudaError_t e = cudaMalloc(&p, want);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc");
    cap = want;
    return PHC_OK;
  }
};
// Page-locked host memory mapped into the device's address space: the
// kernel writes results into it directly (phc_solve_sparse).
struct MappedBuf {
  void* p = nullptr;
  size_t cap = 0;
  int ensure(size_t need) {
    if (need <= cap) return PHC_OK;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(need, (size_t)4096);
    want += want / 2;
    cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocMapped);
    if (e != cudaSuccess) return cuda_fail(e, "cudaHostAlloc(mapped results)");
    cap = want;
    return PHC_OK;
  }
  template <class T>
  int device_ptr(T** d) const {
    cudaError_t e = cudaHostGetDevicePointer(reinterpret_cast<void**>(d), p, 0);
    return e == cudaSuccess ? PHC_OK : cuda_fail(e, "cudaHostGetDevicePointer");
  }
};
struct DeviceWS {
  std::mutex mu;
  bool ready = false;
  cudaStream_t stream = nullptr;
  DevBuf plan, out, z, x, counter;
  MappedBuf hout, hz, hx, hdone;
  unsigned char* stage = nullptr;  // pinned staging of the table upload
  size_t stage_cap = 0;
};
DeviceWS g_ws[64];

int check_device(int device) {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count < 1) {
    set_last_error(e != cudaSuccess ? cudaGetErrorString(e) : "no CUDA device");
    return PHC_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= count || device >= 64) {
    set_last_error("invalid device ordinal");
    return PHC_ERR_NO_DEVICE;
  }
  return PHC_OK;
}
}  // namespace

// Runs paths [k0, k0+count) of a compiled plan on the device workspace and
// copies the results to host buffers.
static int run_paths_sync(const HostPlan& hp, const phc_solve_options& so,
                          const phc_gpu_options& g, int64_t k0, int64_t count,
                          phc_path_out* out, double* z_out, double* x_out) {
  int st = check_device(g.device);
  if (st != PHC_OK) return st;
  if (count <= 0) return PHC_OK;
  DeviceWS& W = g_ws[g.device];
  std::lock_guard<std::mutex> lock(W.mu);
  PHC_CUDA(cudaSetDevice(g.device));
  if (!W.ready) {
    PHC_CUDA(cudaStreamCreateWithFlags(&W.stream, cudaStreamNonBlocking));
    W.ready = true;
  }
  LaunchCfg cfg;
  st = resolve_launch(hp, g, g.device, count, &cfg);
  if (st != PHC_OK) return st;
  const size_t nout = (size_t)count * sizeof(phc_path_out);
  const size_t nz = (size_t)count * hp.N * 2 * sizeof(double);
  const size_t nx = (size_t)count * hp.n * 2 * sizeof(double);
  if ((st = W.plan.ensure(hp.bytes.size() + 16)) != PHC_OK) return st;
  if ((st = W.out.ensure(nout)) != PHC_OK) return st;
  if ((st = W.z.ensure(nz)) != PHC_OK) return st;
  if ((st = W.x.ensure(nx)) != PHC_OK) return st;
  if ((st = W.counter.ensure(16)) != PHC_OK) return st;
  if (hp.bytes.size() > W.stage_cap) {
    if (W.stage) cudaFreeHost(W.stage);
    W.stage = nullptr;
    W.stage_cap = 0;
    PHC_CUDA(cudaMallocHost((void**)&W.stage, hp.bytes.size() * 2));
    W.stage_cap = hp.bytes.size() * 2;
  }
  std::memcpy(W.stage, hp.bytes.data(), hp.bytes.size());
  PHC_CUDA(cudaMemcpyAsync(W.plan.p, W.stage, hp.bytes.size(), cudaMemcpyHostToDevice, W.stream));
  KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.plan = static_cast<const unsigned char*>(W.plan.p);
  kp.plan_bytes = cfg.plan_bytes;
  kp.ws_bytes = cfg.ws_bytes;
  kp.warps = cfg.warps;
  kp.persistent = cfg.persistent;
  kp.chunk = cfg.chunk;
  kp.k0 = k0;
  kp.count = count;
  kp.counter = static_cast<unsigned long long*>(W.counter.p);
  kp.out = static_cast<phc_path_out*>(W.out.p);
  kp.z = static_cast<double*>(W.z.p);
  kp.x = static_cast<double*>(W.x.p);
  kp.opts = make_kopts(so, g);
  int grid;
  if (cfg.persistent) {
    PHC_CUDA(cudaMemsetAsync(W.counter.p, 0, sizeof(unsigned long long), W.stream));
    const int64_t need = (count + (int64_t)cfg.warps * cfg.chunk - 1) / ((int64_t)cfg.warps * cfg.chunk);
    grid = (int)std::min<int64_t>(cfg.grid, need);
  } else {
    grid = (int)((count + cfg.warps - 1) / cfg.warps);
  }
  cudaError_t e = launch_track(cfg, kp, grid, W.stream);
  if (e != cudaSuccess) return cuda_fail(e, "track kernel launch");
  PHC_CUDA(cudaMemcpyAsync(out, W.out.p, nout, cudaMemcpyDeviceToHost, W.stream));
  PHC_CUDA(cudaMemcpyAsync(z_out, W.z.p, nz, cudaMemcpyDeviceToHost, W.stream));
  if (x_out) PHC_CUDA(cudaMemcpyAsync(x_out, W.x.p, nx, cudaMemcpyDeviceToHost, W.stream));
  PHC_CUDA(cudaStreamSynchronize(W.stream));
  return PHC_OK;
}

// ---------------------------------------------------------------------------
// bookkeeping (src/solve.f90:193-213, :330-426)
// ---------------------------------------------------------------------------
static double norm_inf_exact(const double* v, int n) {
  double r = 0.0;
  for (int i = 0; i < n; ++i) r = std::max(r, std::hypot(v[2 * i], v[2 * i + 1]));
  return r;
}

// Squared moduli decide a comparison with |.| (hypot) unless they are
// within a relative kSqMargin of the threshold; only then is hypot itself
// compared, so every decision is the one the hypot test makes. Squares of
// magnitudes outside [kSqLo, kSqHi] could over- or underflow: those take
// the exact path.
constexpr double kSqMargin = 1e-12;
constexpr double kSqLo = 1e-140, kSqHi = 1e140;

// ||v||_inf (norm_inf, src/linalg.f90:176-189) with one hypot: the exact
// maximum is among the components whose square is within the margin of
// the largest square.
static double norm_inf_c(const double* v, int n) {
  double m2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double s = v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1];
    if (!(s <= kSqHi)) return norm_inf_exact(v, n);  // huge or NaN
    m2 = std::max(m2, s);
  }
  if (m2 < kSqLo) return norm_inf_exact(v, n);
  double r = 0.0;
  for (int i = 0; i < n; ++i) {
    const double s = v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1];
    if (s >= m2 * (1.0 - kSqMargin)) r = std::max(r, std::hypot(v[2 * i], v[2 * i + 1]));
  }
  return r;
}

// The square root of the largest squared modulus: within a few ulps of
// norm_inf, without a hypot. NaN when a square could over- or underflow
// or a value is not finite; the caller then takes the exact norm.
static double norm_inf_estimate(const double* v, int n) {
  double m2 = 0.0;
  for (int i = 0; i < n; ++i) {
    const double s = v[2 * i] * v[2 * i] + v[2 * i + 1] * v[2 * i + 1];
    if (!(s <= kSqHi)) return std::numeric_limits<double>::quiet_NaN();
    m2 = std::max(m2, s);
  }
  if (m2 < kSqLo) return std::numeric_limits<double>::quiet_NaN();
  return std::sqrt(m2);
}

// The reference's find (src/solve.f90:379-400) scans all stored points and
// returns the first (lowest index) within tol * max(1, ||x||). PointSet
// returns the same index without the O(P) scan: any match lies within the
// window |Re x_1 - Re s_1| <= tol * max(1, ||x||), so the points are
// hashed by Re x_1 into buckets of width 64*tol, a query visits the
// buckets its window covers, and the lowest index among the matches there
// is the first match of the scan. Points or queries with non-finite values,
// and windows wider than 64 buckets, take the linear scan, exactly as the
// reference.
class PointSet {
 public:
  // Points are rows of the caller's array x ([npaths][n] complex); the set
  // stores row indices, not copies.
  PointSet(int n, double tol, const double* x, int64_t expect)
      : n_(n), tol_(tol), width_(64.0 * tol), x_(x) {
    size_t cap = 64;
    while (cap < 2 * (size_t)std::max<int64_t>(expect, 1)) cap <<= 1;
    keys_.assign(cap, 0);
    heads_.assign(cap, -1);
  }
  int size() const { return (int)rows_.size(); }
  const double* point(int j) const { return x_ + (size_t)rows_[j] * 2 * n_; }

  // rho = tol * max(1, ||x||) comes from the norm estimate; the decisions
  // it makes keep a relative margin of 1e-12, far above the estimate's
  // error, and the few comparisons inside the margin use the exact norm.
  // est: norm_inf_estimate(x, n) (the caller has it already).
  int find(const double* x, double est) const {
    const bool approx = std::isfinite(est);
    const double rho = tol_ * std::max(1.0, approx ? est : norm_inf_c(x, n_));
    double rho_exact = approx ? -1.0 : rho;  // computed on first need
    auto exact_rho = [&]() {
      if (rho_exact < 0.0) rho_exact = tol_ * std::max(1.0, norm_inf_c(x, n_));
      return rho_exact;
    };
    const double x0 = x[0];
    int best = -1;
    auto test = [&](int j) {
      if (best >= 0 && j >= best) return;
      if (within(x, j, rho, exact_rho)) best = j;
    };
    const double margin = 1e-12 * (std::fabs(x0) + rho) + 1e-300;
    const double lo = x0 - rho - margin, hi = x0 + rho + margin;
    if (!std::isfinite(rho) || !std::isfinite(x0) || !(width_ > 0.0) ||
        (hi - lo) > 64.0 * width_ || std::fabs(x0) > 1e15 * width_) {
      for (int j = 0; j < size(); ++j) test(j);
      return best < 0 ? 0 : best + 1;
    }
    const long long b0 = bucket(lo), b1 = bucket(hi);
    for (long long b = b0; b <= b1; ++b)
      for (int j = head(b); j >= 0; j = next_[j]) test(j);
    for (int j : special_) test(j);
    return best < 0 ? 0 : best + 1;
  }

  // adds row k of x (the point x + k*2n)
  void add(int64_t k) {
    const int j = size();
    rows_.push_back(k);
    const double x0 = point(j)[0];
    if (std::isfinite(x0) && width_ > 0.0 && std::fabs(x0) <= 1e15 * width_) {
      const long long b = bucket(x0);
      size_t slot = probe(b);
      if (heads_[slot] < 0) {
        keys_[slot] = b;
        ++used_;
      }
      next_.push_back(heads_[slot]);
      heads_[slot] = j;
      if (2 * used_ > keys_.size()) rehash();
    } else {
      next_.push_back(-1);
      special_.push_back(j);
    }
  }

 private:
  long long bucket(double v) const { return (long long)std::floor(v / width_); }
  size_t hash(long long b) const {
    return (size_t)(((unsigned long long)b * 0x9E3779B97F4A7C15ull) >> 17);
  }
  // slot of bucket b: its own, or the empty one where it would go
  size_t probe(long long b) const {
    const size_t mask = keys_.size() - 1;
    size_t s = hash(b) & mask;
    while (heads_[s] >= 0 && keys_[s] != b) s = (s + 1) & mask;
    return s;
  }
  int head(long long b) const {
    const size_t s = probe(b);
    return heads_[s] >= 0 ? heads_[s] : -1;
  }
  void rehash() {
    std::vector<long long> k2;
    std::vector<int> h2;
    k2.swap(keys_);
    h2.swap(heads_);
    keys_.assign(2 * k2.size(), 0);
    heads_.assign(2 * k2.size(), -1);
    for (size_t s = 0; s < k2.size(); ++s) {
      if (h2[s] < 0) continue;
      const size_t t = probe(k2[s]);
      keys_[t] = k2[s];
      heads_[t] = h2[s];
    }
  }
  // max_i |x_i - p_i| <= rho, decided on squares away from the threshold;
  // at the threshold, hypot distances against the exact rho
  template <class ExactRho>
  bool within(const double* x, int j, double rho, ExactRho&& exact_rho) const {
    const double* p = point(j);
    const double r2 = rho * rho;
    bool exact = !(r2 >= kSqLo && r2 <= kSqHi);
    double m2 = 0.0;
    for (int i = 0; i < n_ && !exact; ++i) {
      const double dr = x[2 * i] - p[2 * i], di = x[2 * i + 1] - p[2 * i + 1];
      const double s = dr * dr + di * di;
      if (!(s <= kSqHi)) exact = true;  // huge or NaN
      m2 = std::max(m2, s);
    }
    if (!exact) {
      if (m2 <= r2 * (1.0 - kSqMargin)) return true;
      if (m2 >= r2 * (1.0 + kSqMargin)) return false;
    }
    double d = 0.0;
    for (int i = 0; i < n_; ++i)
      d = std::max(d, std::hypot(x[2 * i] - p[2 * i], x[2 * i + 1] - p[2 * i + 1]));
    return d <= exact_rho();
  }
  int n_;
  double tol_, width_;
  const double* x_;
  std::vector<int64_t> rows_;     // row of x of each stored point
  std::vector<int> next_;         // previous point in the same bucket, or -1
  std::vector<long long> keys_;   // open-addressing table: bucket -> newest point
  std::vector<int> heads_;
  size_t used_ = 0;
  std::vector<int> special_;
};

// collect_real's test for one solution (src/solve.f90:402-426):
// max_i |Im s_i| <= real_tol * max(1, ||s||), with the norm estimate
// deciding away from the threshold.
static bool is_real_solution(const double* s, int n, double est, double real_tol) {
  double imax = 0.0;
  for (int i = 0; i < n; ++i) imax = std::max(imax, std::fabs(s[2 * i + 1]));
  const double thr = real_tol * std::max(1.0, est);
  if (std::isfinite(est) && imax <= thr * (1.0 - kSqMargin)) return true;
  if (std::isfinite(est) && imax >= thr * (1.0 + kSqMargin)) return false;
  return imax <= real_tol * std::max(1.0, norm_inf_c(s, n));
}

// One pass in path order: each endpoint's norm estimate serves its dedup
// query and, for a new regular solution, collect_real's test; new
// solutions are copied out as they are found. collect_real runs over the
// solutions in index order, which is the order they are found in, so the
// real list is the same. Paths are added one at a time (add), so the pass
// can run while later paths are still being tracked; x is the caller's
// endpoint array, whose row k must hold path k's endpoint when it is added.
class Bookkeeper {
 public:
  Bookkeeper(int n, int64_t npaths, const phc_solve_options& o, const double* x,
             phc_solve_result* res)
      : n_(n), o_(o), x_(x), res_(res), sols_(n, o.dedup_tol, x, npaths),
        ssols_(n, o.singular_dedup_tol, x, 64) {}

  void add(int64_t k, phc_path_out& p) {
    phc_solve_counts& c = res_->counts;
    const int n = n_;
    const double* xk = x_ + (size_t)k * 2 * n;
    const size_t row = (size_t)2 * n * sizeof(double);
    p.solution_index = 0;
    p.singular_index = 0;
    if (p.status != PHC_PATH_SUCCESS) {
      c.nfailed++;
    } else if (p.at_infinity) {
      c.ninfinite++;
    } else if (p.singular) {  // add_singular, src/solve.f90:353-377
      int j = ssols_.find(xk, norm_inf_estimate(xk, n));
      if (j > 0) {
        mult_[j - 1]++;
      } else {
        ssols_.add(k);
        mult_.push_back(1);
        j = ssols_.size();
        if (res_->singular_solutions)
          std::memcpy(res_->singular_solutions + (size_t)(j - 1) * 2 * n, xk, row);
      }
      p.singular_index = j;
    } else {  // add_solution, src/solve.f90:330-351
      const double est = norm_inf_estimate(xk, n);
      int j = sols_.find(xk, est);
      if (j > 0) {
        c.nduplicates++;
      } else {
        sols_.add(k);
        j = sols_.size();
        if (res_->solutions) std::memcpy(res_->solutions + (size_t)(j - 1) * 2 * n, xk, row);
        if (is_real_solution(xk, n, est, o_.real_tol)) {
          if (res_->real_solutions)
            for (int i = 0; i < n; ++i) res_->real_solutions[(size_t)nreal_ * n + i] = xk[2 * i];
          ++nreal_;
        }
      }
      p.solution_index = j;
    }
  }

  void finish() {
    phc_solve_counts& c = res_->counts;
    c.nsolutions = sols_.size();
    c.nsingular = ssols_.size();
    if (res_->multiplicities)
      for (int j = 0; j < c.nsingular; ++j) res_->multiplicities[j] = mult_[j];
    c.nreal = nreal_;
  }

 private:
  int n_;
  phc_solve_options o_;
  const double* x_;
  phc_solve_result* res_;
  PointSet sols_, ssols_;
  std::vector<int> mult_;
  int nreal_ = 0;
};

void bookkeeping(int n, int64_t npaths, const phc_solve_options& o, phc_path_out* paths,
                 const double* x, phc_solve_result* res) {
  Bookkeeper b(n, npaths, o, x, res);
  for (int64_t k = 0; k < npaths; ++k) b.add(k, paths[k]);
  b.finish();
}

// solve()'s tracking and bookkeeping overlapped (src/solve.f90:190-213):
// the kernel writes every path's record, z and x into mapped host memory
// and then flags the path (KParams::done); this thread takes the paths in
// order as their flags appear, copies them into the caller's arrays and
// runs the bookkeeping on each, so that when the last path finishes only
// its own bookkeeping is left. The results are identical to tracking all
// paths first and running the bookkeeping afterwards.
static int solve_streamed(const HostPlan& hp, const phc_solve_options& so, const phc_gpu_options& g,
                          int64_t count, phc_solve_result* res) {
  int st = check_device(g.device);
  if (st != PHC_OK) return st;
  Bookkeeper book(hp.n, count, so, res->x, res);
  if (count <= 0) {
    book.finish();
    return PHC_OK;
  }
  DeviceWS& W = g_ws[g.device];
  std::lock_guard<std::mutex> lock(W.mu);
  PHC_CUDA(cudaSetDevice(g.device));
  if (!W.ready) {
    PHC_CUDA(cudaStreamCreateWithFlags(&W.stream, cudaStreamNonBlocking));
    W.ready = true;
  }
  LaunchCfg cfg;
  st = resolve_launch(hp, g, g.device, count, &cfg);
  if (st != PHC_OK) return st;
  const size_t zrow = (size_t)hp.N * 2, xrow = (size_t)hp.n * 2;
  if ((st = W.plan.ensure(hp.bytes.size() + 16)) != PHC_OK) return st;
  if ((st = W.counter.ensure(16)) != PHC_OK) return st;
  if ((st = W.hout.ensure((size_t)count * sizeof(phc_path_out))) != PHC_OK) return st;
  if ((st = W.hz.ensure((size_t)count * zrow * sizeof(double))) != PHC_OK) return st;
  if ((st = W.hx.ensure((size_t)count * xrow * sizeof(double))) != PHC_OK) return st;
  if ((st = W.hdone.ensure((size_t)count * sizeof(unsigned int))) != PHC_OK) return st;
  if (hp.bytes.size() > W.stage_cap) {
    if (W.stage) cudaFreeHost(W.stage);
    W.stage = nullptr;
    W.stage_cap = 0;
    PHC_CUDA(cudaMallocHost((void**)&W.stage, hp.bytes.size() * 2));
    W.stage_cap = hp.bytes.size() * 2;
  }
  // the previous launch on these buffers has finished (this function
  // returns only after its kernel), so the flags can be cleared here
  volatile unsigned int* done = static_cast<volatile unsigned int*>(W.hdone.p);
  std::memset(W.hdone.p, 0, (size_t)count * sizeof(unsigned int));
  std::memcpy(W.stage, hp.bytes.data(), hp.bytes.size());
  PHC_CUDA(cudaMemcpyAsync(W.plan.p, W.stage, hp.bytes.size(), cudaMemcpyHostToDevice, W.stream));
  KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.plan = static_cast<const unsigned char*>(W.plan.p);
  kp.plan_bytes = cfg.plan_bytes;
  kp.ws_bytes = cfg.ws_bytes;
  kp.warps = cfg.warps;
  kp.persistent = cfg.persistent;
  kp.chunk = cfg.chunk;
  kp.k0 = 1;
  kp.count = count;
  kp.counter = static_cast<unsigned long long*>(W.counter.p);
  if ((st = W.hout.device_ptr(&kp.out)) != PHC_OK) return st;
  if ((st = W.hz.device_ptr(&kp.z)) != PHC_OK) return st;
  if ((st = W.hx.device_ptr(&kp.x)) != PHC_OK) return st;
  if ((st = W.hdone.device_ptr(&kp.done)) != PHC_OK) return st;
  kp.opts = make_kopts(so, g);
  int grid;
  if (cfg.persistent) {
    PHC_CUDA(cudaMemsetAsync(W.counter.p, 0, sizeof(unsigned long long), W.stream));
    const int64_t need = (count + (int64_t)cfg.warps * cfg.chunk - 1) / ((int64_t)cfg.warps * cfg.chunk);
    grid = (int)std::min<int64_t>(cfg.grid, need);
  } else {
    grid = (int)((count + cfg.warps - 1) / cfg.warps);
  }
  cudaError_t e = launch_track(cfg, kp, grid, W.stream);
  if (e != cudaSuccess) return cuda_fail(e, "track kernel launch");
  const phc_path_out* hout = static_cast<const phc_path_out*>(W.hout.p);
  const double* hz = static_cast<const double*>(W.hz.p);
  const double* hx = static_cast<const double*>(W.hx.p);
  bool finished = false;  // the kernel has completed: every flag is set
  for (int64_t k = 0; k < count; ++k) {
    // wait for path k: spin briefly, then sleep; ask the stream now and
    // then, so that a failed launch ends the wait with its error
    for (int spin = 0; !finished && done[k] == 0u; ++spin) {
      if (spin < 256) continue;
      e = cudaStreamQuery(W.stream);
      if (e == cudaSuccess) {
        finished = true;
      } else if (e != cudaErrorNotReady) {
        return cuda_fail(e, "track kernel");
      } else {
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      }
    }
    if (done[k] == 0u) {
      set_last_error("track kernel finished without flagging a path");
      return PHC_ERR_CUDA;
    }
    // the path's results were made visible before its flag
    std::atomic_thread_fence(std::memory_order_acquire);
    res->paths[k] = hout[k];
    std::memcpy(res->z + (size_t)k * zrow, hz + (size_t)k * zrow, zrow * sizeof(double));
    std::memcpy(res->x + (size_t)k * xrow, hx + (size_t)k * xrow, xrow * sizeof(double));
    book.add(k, res->paths[k]);
  }
  PHC_CUDA(cudaStreamSynchronize(W.stream));
  book.finish();
  return PHC_OK;
}

}  // namespace phc

// ---------------------------------------------------------------------------
// type(sparse_system) builder
// ---------------------------------------------------------------------------
struct phc_sparse {
  int n = 0;
  int neq = 0;
  bool initialized = false;
  std::vector<int32_t> first;  // 0-based, neq + 1
  std::vector<int32_t> deg;
  std::vector<int32_t> hexps;  // term-major [nt][n+1]
  std::vector<double> coefs;   // [nt][2]
};

using namespace phc;

extern "C" {

const char* phc_version(void) { return "polyhomocont_b200 0.1.0 (sm_100a)"; }
const char* phc_last_error(void) { return g_last_error.c_str(); }

void phc_default_solve_options(phc_solve_options* o) {
  if (o) *o = solve_defaults();
}
void phc_default_gpu_options(phc_gpu_options* g) {
  if (g) *g = gpu_defaults();
}

phc_sparse* phc_sparse_create(void) { return new (std::nothrow) phc_sparse(); }
void phc_sparse_destroy(phc_sparse* s) { delete s; }

int32_t phc_sparse_init(phc_sparse* s, int32_t n) {  // src/sparse.f90:65-81
  if (!s) return PHC_ERR_BAD_HANDLE;
  s->n = n;
  s->neq = 0;
  s->initialized = true;
  s->first.assign(1, 0);
  s->deg.clear();
  s->hexps.clear();
  s->coefs.clear();
  return PHC_OK;
}

int32_t phc_sparse_add_equation(phc_sparse* s, int32_t ncoefs, const double* coefs,
                                int32_t rows, int32_t cols, const int32_t* exps) {
  // src/sparse.f90:83-141: validation, zero terms dropped, degree from the
  // kept terms, homogenized exponent of w = d - |a|
  if (!s || !s->initialized) return PHC_ERR_INVALID_INPUT;
  if (s->neq >= s->n) return PHC_ERR_INVALID_INPUT;
  if (rows != s->n) return PHC_ERR_INVALID_INPUT;
  if (cols != ncoefs || ncoefs < 0) return PHC_ERR_INVALID_INPUT;
  if (ncoefs > 0 && (coefs == nullptr || exps == nullptr)) return PHC_ERR_INVALID_INPUT;
  for (int64_t q = 0; q < (int64_t)rows * cols; ++q)
    if (exps[q] < 0) return PHC_ERR_INVALID_INPUT;
  int d = 0;
  for (int k = 0; k < ncoefs; ++k) {
    if (coefs[2 * k] == 0.0 && coefs[2 * k + 1] == 0.0) continue;
    int sum = 0;
    for (int j = 0; j < rows; ++j) sum += exps[(size_t)k * rows + j];
    d = std::max(d, sum);
  }
  if (d < 1) return PHC_ERR_INVALID_INPUT;
  int kept = 0;
  for (int k = 0; k < ncoefs; ++k) {
    if (coefs[2 * k] == 0.0 && coefs[2 * k + 1] == 0.0) continue;
    int sum = 0;
    for (int j = 0; j < rows; ++j) {
      const int e = exps[(size_t)k * rows + j];
      s->hexps.push_back(e);
      sum += e;
    }
    s->hexps.push_back(d - sum);
    s->coefs.push_back(coefs[2 * k]);
    s->coefs.push_back(coefs[2 * k + 1]);
    ++kept;
  }
  s->neq += 1;
  s->first.push_back(s->first.back() + kept);
  s->deg.push_back(d);
  return PHC_OK;
}

int32_t phc_sparse_nvars(const phc_sparse* s) { return s ? s->n : 0; }
int32_t phc_sparse_nequations(const phc_sparse* s) { return s ? s->neq : 0; }
int32_t phc_sparse_nterms(const phc_sparse* s, int32_t i) {
  if (!s || i < 1 || i > s->neq) return 0;
  return s->first[i] - s->first[i - 1];
}
int32_t phc_sparse_total_terms(const phc_sparse* s) { return s ? (int32_t)(s->coefs.size() / 2) : 0; }
void phc_sparse_degrees(const phc_sparse* s, int32_t* d) {
  if (!s || !d) return;
  for (int i = 0; i < s->neq; ++i) d[i] = s->deg[i];
}
// sys%evaluate and sys%evaluate_homogeneous (src/sparse.f90:197-221) on the
// host: f[neq] and jac (neq x m, column-major) of the table's terms at
// v[m], m = n (affine: the exponents without the w column) or n + 1. A
// term contributes c prod_l v_l^e_l to f_i and
// c e_j v_j^(e_j - 1) prod_{l != j} v_l^e_l to jac(i, j), the products
// taken over the nonzero exponents only, so zero coordinates need no
// division and w = 0 is exact.
namespace {
using cdh = std::complex<double>;
cdh powi(cdh x, int k) {  // x^k, k >= 0, square and multiply
  cdh r = 1.0;
  while (k > 0) {
    if (k & 1) r *= x;
    k >>= 1;
    if (k) x *= x;
  }
  return r;
}
void eval_table(const phc_sparse* s, int m, const double* v, double* f, double* jac) {
  const int n = s->n, neq = s->neq;
  std::vector<cdh> z(m), F(neq, cdh(0.0)), J((size_t)neq * m, cdh(0.0));
  for (int j = 0; j < m; ++j) z[j] = cdh(v[2 * j], v[2 * j + 1]);
  for (int i = 0; i < neq; ++i)
    for (int k = s->first[i]; k < s->first[i + 1]; ++k) {
      const int32_t* e = &s->hexps[(size_t)k * (n + 1)];
      const cdh c(s->coefs[2 * k], s->coefs[2 * k + 1]);
      cdh val = c;
      for (int l = 0; l < m; ++l)
        if (e[l] > 0) val *= powi(z[l], e[l]);
      F[i] += val;
      for (int j = 0; j < m; ++j) {
        if (e[j] <= 0) continue;
        cdh d = c * (double)e[j] * powi(z[j], e[j] - 1);
        for (int l = 0; l < m; ++l)
          if (l != j && e[l] > 0) d *= powi(z[l], e[l]);
        J[i + (size_t)j * neq] += d;
      }
    }
  for (int i = 0; i < neq; ++i) {
    f[2 * i] = F[i].real();
    f[2 * i + 1] = F[i].imag();
  }
  for (size_t q = 0; q < J.size(); ++q) {
    jac[2 * q] = J[q].real();
    jac[2 * q + 1] = J[q].imag();
  }
}
}  // namespace

int32_t phc_sparse_evaluate(const phc_sparse* s, const double* x, double* f, double* jac) {
  if (!s) return PHC_ERR_BAD_HANDLE;
  if (!s->initialized || s->neq != s->n || !x || !f || !jac) return PHC_ERR_INVALID_INPUT;
  eval_table(s, s->n, x, f, jac);
  return PHC_OK;
}

int32_t phc_sparse_evaluate_homogeneous(const phc_sparse* s, const double* z, double* f,
                                        double* jac) {
  if (!s) return PHC_ERR_BAD_HANDLE;
  if (!s->initialized || s->neq != s->n || !z || !f || !jac) return PHC_ERR_INVALID_INPUT;
  eval_table(s, s->n + 1, z, f, jac);
  return PHC_OK;
}

int32_t phc_sparse_table(const phc_sparse* s, phc_system* out) {
  if (!s || !out) return PHC_ERR_BAD_HANDLE;
  out->n = s->n;
  out->nterms = (int32_t)(s->coefs.size() / 2);
  out->first = s->first.data();
  out->deg = s->deg.data();
  out->hexps = s->hexps.data();
  out->coefs = s->coefs.data();
  // hom%init rejects systems whose equation count differs from n
  // (src/homotopy.f90:106-108)
  return (s->neq == s->n && s->n >= 1) ? PHC_OK : PHC_ERR_INVALID_INPUT;
}

int32_t phc_homotopy_init(const phc_system* sys, int32_t seed, double* gamma, double* b,
                          double* patch, int64_t* nstart) {
  HostHomotopy h;
  int st = homotopy_init(sys, seed, &h);
  if (st != PHC_OK) return st;
  if (gamma) {
    gamma[0] = h.gamma[0];
    gamma[1] = h.gamma[1];
  }
  if (b) std::memcpy(b, h.b.data(), h.b.size() * sizeof(double));
  if (patch) std::memcpy(patch, h.patch.data(), h.patch.size() * sizeof(double));
  if (nstart) *nstart = h.nstart;
  return PHC_OK;
}

int64_t phc_bezout(const phc_system* sys) {
  if (!sys || sys->n < 1 || !sys->deg) return 0;
  int64_t b = 1;
  for (int i = 0; i < sys->n; ++i) {
    if (sys->deg[i] < 1) return 0;
    b *= sys->deg[i];
    if (b > (int64_t)INT32_MAX) return 0;
  }
  return b;
}

int32_t phc_solve_paths(const phc_system* sys, const phc_homotopy* hom,
                        const phc_solve_options* opts, const phc_gpu_options* gpu,
                        int64_t k0, int64_t count, phc_path_out* out, double* z_out,
                        double* x_out) {
  const phc_solve_options so = opts ? *opts : solve_defaults();
  const phc_gpu_options g = gpu ? *gpu : gpu_defaults();
  int st = validate_options(&so);
  if (st != PHC_OK) return st;
  if (!out || !z_out || count < 0 || k0 < 1) return PHC_ERR_INVALID_INPUT;
  HostPlan hp;
  st = build_plan(sys, hom, &hp);
  if (st != PHC_OK) return st;
  if (k0 - 1 > hp.nstart - count) return PHC_ERR_INVALID_INPUT;  // k0 + count - 1 <= nstart
  return run_paths_sync(hp, so, g, k0, count, out, z_out, x_out);
}

int32_t phc_finish_solve(int32_t n, int64_t npaths, const phc_solve_options* opts,
                         phc_path_out* paths, const double* x, phc_solve_result* res) {
  if (n < 1 || npaths < 0 || !res || (npaths > 0 && (!paths || !x))) return PHC_ERR_INVALID_INPUT;
  const phc_solve_options so = opts ? *opts : solve_defaults();
  std::memset(&res->counts, 0, sizeof(res->counts));
  res->counts.n = n;
  res->counts.npaths = (int32_t)npaths;
  bookkeeping(n, npaths, so, paths, x, res);
  return PHC_OK;
}

int32_t phc_solve_sparse(const phc_system* sys, const phc_solve_options* opts,
                         const phc_gpu_options* gpu, phc_solve_result* res) {
  // solve(sys, res, status, options), src/solve.f90:154-215
  const phc_solve_options so = opts ? *opts : solve_defaults();
  const phc_gpu_options g = gpu ? *gpu : gpu_defaults();
  if (!res) return PHC_ERR_INVALID_INPUT;
  std::memset(&res->counts, 0, sizeof(res->counts));
  int st = validate_options(&so);
  if (st != PHC_OK) return st;
  st = validate_system(sys);
  if (st != PHC_OK) return st;
  HostHomotopy h;
  HostPlan hp;
  {
    NvtxRange r("phc setup: homotopy and table compile");
    st = homotopy_init(sys, so.seed, &h);  // gen%seed + hom%init
    if (st != PHC_OK) return st;
    if (!res->paths || !res->z || !res->x) return PHC_ERR_INVALID_INPUT;
    const phc_homotopy hv = h.view();
    st = build_plan(sys, &hv, &hp);
    if (st != PHC_OK) return st;
  }
  res->counts.n = sys->n;
  res->counts.npaths = (int32_t)h.nstart;
  NvtxRange r("phc track and bookkeeping");
  return solve_streamed(hp, so, g, h.nstart, res);
}

// ---------------------------------------------------------------------------
// device-resident plans
// ---------------------------------------------------------------------------
}  // extern "C"

struct phc_plan {
  int device = 0;
  HostPlan hp;
  LaunchCfg cfg;
  KOpts kopts;
  void* d_plan = nullptr;
  unsigned long long* d_counter = nullptr;
};

extern "C" {

int32_t phc_plan_create(const phc_system* sys, const phc_homotopy* hom,
                        const phc_solve_options* opts, const phc_gpu_options* gpu,
                        phc_plan** plan) {
  if (!plan) return PHC_ERR_INVALID_INPUT;
  *plan = nullptr;
  const phc_solve_options so = opts ? *opts : solve_defaults();
  const phc_gpu_options g = gpu ? *gpu : gpu_defaults();
  int st = validate_options(&so);
  if (st != PHC_OK) return st;
  st = check_device(g.device);
  if (st != PHC_OK) return st;
  std::unique_ptr<phc_plan> p(new (std::nothrow) phc_plan());
  if (!p) return PHC_ERR_OOM;
  st = build_plan(sys, hom, &p->hp);
  if (st != PHC_OK) return st;
  p->device = g.device;
  PHC_CUDA(cudaSetDevice(g.device));
  st = resolve_launch(p->hp, g, g.device, p->hp.nstart, &p->cfg);
  if (st != PHC_OK) return st;
  p->kopts = make_kopts(so, g);
  PHC_CUDA(cudaMalloc(&p->d_plan, p->hp.bytes.size() + 16));
  PHC_CUDA(cudaMalloc((void**)&p->d_counter, 16));
  PHC_CUDA(cudaMemcpy(p->d_plan, p->hp.bytes.data(), p->hp.bytes.size(), cudaMemcpyHostToDevice));
  *plan = p.release();
  return PHC_OK;
}

int32_t phc_plan_launch(phc_plan* p, int64_t k0, int64_t count, phc_path_out* d_out,
                        double* d_z, void* stream) {
  if (!p) return PHC_ERR_BAD_HANDLE;
  if (count <= 0) return PHC_OK;
  if (k0 < 1 || k0 - 1 > p->hp.nstart - count || !d_out || !d_z)
    return PHC_ERR_INVALID_INPUT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PHC_CUDA(cudaSetDevice(p->device));
  KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.plan = static_cast<const unsigned char*>(p->d_plan);
  kp.plan_bytes = p->cfg.plan_bytes;
  kp.ws_bytes = p->cfg.ws_bytes;
  kp.warps = p->cfg.warps;
  kp.persistent = p->cfg.persistent;
  kp.chunk = p->cfg.chunk;
  kp.k0 = k0;
  kp.count = count;
  kp.counter = p->d_counter;
  kp.out = d_out;
  kp.z = d_z;
  kp.x = nullptr;
  kp.opts = p->kopts;
  int grid;
  if (p->cfg.persistent) {
    PHC_CUDA(cudaMemsetAsync(p->d_counter, 0, sizeof(unsigned long long), s));
    const int64_t per = (int64_t)p->cfg.warps * p->cfg.chunk;
    grid = (int)std::min<int64_t>(p->cfg.grid, (count + per - 1) / per);
  } else {
    grid = (int)((count + p->cfg.warps - 1) / p->cfg.warps);
  }
  cudaError_t e = launch_track(p->cfg, kp, grid, s);
  if (e != cudaSuccess) return cuda_fail(e, "track kernel launch");
  return PHC_OK;
}

int32_t phc_plan_launch_count(const phc_plan* p) { return p ? 1 : 0; }

}  // extern "C"

struct phc_graph {
  int device = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

extern "C" {

int32_t phc_graph_create(phc_plan* p, int64_t k0, int64_t count, phc_path_out* d_out,
                         double* d_z, phc_graph** out) {
  if (!p || !out) return PHC_ERR_BAD_HANDLE;
  *out = nullptr;
  if (count <= 0 || k0 < 1 || k0 - 1 > p->hp.nstart - count || !d_out ||
      !d_z)
    return PHC_ERR_INVALID_INPUT;
  PHC_CUDA(cudaSetDevice(p->device));
  std::unique_ptr<phc_graph> g(new (std::nothrow) phc_graph());
  if (!g) return PHC_ERR_OOM;
  g->device = p->device;
  cudaStream_t s = nullptr;
  PHC_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  int st = PHC_OK;
  if (e == cudaSuccess) {
    st = phc_plan_launch(p, k0, count, d_out, d_z, s);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(s, &graph);
    if (st == PHC_OK && e2 != cudaSuccess) e = e2;
    g->graph = graph;
  }
  if (e == cudaSuccess && st == PHC_OK)
    e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  cudaStreamDestroy(s);
  if (st != PHC_OK || e != cudaSuccess) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    return st != PHC_OK ? st : cuda_fail(e, "graph capture");
  }
  *out = g.release();
  return PHC_OK;
}

int32_t phc_graph_launch(phc_graph* g, void* stream) {
  if (!g) return PHC_ERR_BAD_HANDLE;
  PHC_CUDA(cudaSetDevice(g->device));
  PHC_CUDA(cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream)));
  return PHC_OK;
}

int32_t phc_graph_destroy(phc_graph* g) {
  if (!g) return PHC_ERR_BAD_HANDLE;
  cudaSetDevice(g->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return PHC_OK;
}

int32_t phc_plan_config(const phc_plan* p, int32_t* warps, int32_t* grid, int32_t* smem,
                        int32_t* nm, int32_t* table_bytes) {
  if (!p) return PHC_ERR_BAD_HANDLE;
  if (table_bytes) *table_bytes = (int32_t)p->hp.bytes.size();
  if (warps) *warps = p->cfg.warps;
  if (grid) *grid = p->cfg.grid;
  if (smem) *smem = p->cfg.smem;
  if (nm) *nm = p->cfg.nm;
  return PHC_OK;
}

int32_t phc_plan_destroy(phc_plan* p) {
  if (!p) return PHC_ERR_BAD_HANDLE;
  cudaSetDevice(p->device);
  if (p->d_plan) cudaFree(p->d_plan);
  if (p->d_counter) cudaFree(p->d_counter);
  delete p;
  return PHC_OK;
}

}  // extern "C"

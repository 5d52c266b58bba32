// phc_server.cpp -- serving loop with continuous batching.
//
// Requests are whole solve() calls (a sparse system plus solve_options).
// An engine thread admits pending requests into batches as soon as a slot
// (a CUDA stream with its device and pinned buffers) and enough of the
// device-memory budget are free, launches the batch while other batches
// are still running, and finishes each request on the host (bookkeeping,
// src/solve.f90:193-213) when its batch's event has fired. Requests that
// arrive while the GPU is busy therefore start as soon as any slot frees
// up, and the work of different batches overlaps on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "phc_host.h"

namespace phc {
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t ticket = 0;
  // owned copy of the system table and options
  int n = 0;
  std::vector<int32_t> first, deg, hexps;
  std::vector<double> coefs;
  phc_solve_options opts;
  HostHomotopy hom;
  HostPlan plan;
  int64_t npaths = 0;
  size_t dev_bytes = 0;
  int status = PHC_OK;
  // why the request failed: error texts are per thread, so the engine's
  // text travels with the request to the thread that asks for the result
  std::string error;
  // results
  std::vector<phc_path_out> paths;
  std::vector<double> z, x, sols, realsols, ssols;
  std::vector<int32_t> mult;
  phc_solve_counts counts;
  Clock::time_point t_submit, t_done;
  bool done = false;
  // placement inside a batch
  size_t off_plan = 0, off_out = 0, off_z = 0, off_x = 0, end = 0;
  int stage = 0;  // 0: paths running, 1: results being copied, 2: finished
  LaunchCfg cfg;

  phc_system view() const {
    phc_system s;
    s.n = n;
    s.nterms = (int32_t)(coefs.size() / 2);
    s.first = first.data();
    s.deg = deg.data();
    s.hexps = hexps.data();
    s.coefs = coefs.data();
    return s;
  }
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaStream_t copy = nullptr;  // per-request result copies
  cudaEvent_t done = nullptr;   // the batch kernel has finished
  unsigned int* done_h = nullptr;  // finished paths per request (mapped host memory)
  unsigned int* done_d = nullptr;  // the same array as the device sees it
  std::vector<cudaEvent_t> copied;  // per request of the batch
  int nfinished = 0;
  void* dbuf = nullptr;
  size_t dcap = 0;
  unsigned char* hbuf = nullptr;  // pinned: plans in, results out
  size_t hcap = 0;
  unsigned long long* counters = nullptr;  // queue head of the batch kernel
  std::vector<std::shared_ptr<Request>> batch;
  size_t bytes = 0;
  bool busy = false;
};

inline size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace phc

using namespace phc;

struct phc_server {
  phc_server_config cfg;
  std::mutex mu;
  std::condition_variable cv;
  std::deque<std::shared_ptr<Request>> pending;
  std::map<uint64_t, std::shared_ptr<Request>> all;
  std::vector<Slot> slots;
  std::thread engine;
  bool stop = false;
  uint64_t next_ticket = 1;
  int64_t submitted = 0, completed = 0, batches = 0;
  size_t mem_in_use = 0;
  int init_status = PHC_OK;
  std::vector<void*> retired_host;  // outgrown pinned buffers
};

namespace phc {
namespace {

// Lays out a batch in one device buffer and one pinned buffer:
// [descriptors | tables | outputs(paths) | z | x], regions 256-aligned.
size_t layout_batch(std::vector<std::shared_ptr<Request>>& b) {
  size_t off = up256(b.size() * sizeof(BatchSys));
  for (auto& r : b) {
    r->off_plan = off;
    off += up256(r->plan.bytes.size());
  }
  for (auto& r : b) {
    r->off_out = off;
    off += up256((size_t)r->npaths * sizeof(phc_path_out));
    r->off_z = off;
    off += up256((size_t)r->npaths * (r->n + 1) * 16);
    r->off_x = off;
    off += up256((size_t)r->npaths * r->n * 16);
    r->end = off;
    r->stage = 0;
  }
  return off;
}

// Grows a slot's buffers geometrically without a device-wide
// synchronisation: device memory is stream-ordered (cudaMallocAsync /
// cudaFreeAsync on the slot's stream), and pinned buffers that are
// outgrown are kept until the server is destroyed, since cudaFreeHost
// would wait for the whole device.
int grow(Slot& s, size_t bytes, std::vector<void*>& retired_host) {
  if (bytes > s.dcap) {
    const size_t want = std::max(bytes, s.dcap + s.dcap / 2);
    if (s.dbuf) cudaFreeAsync(s.dbuf, s.stream);
    s.dbuf = nullptr;
    s.dcap = 0;
    cudaError_t e = cudaMallocAsync(&s.dbuf, want, s.stream);
    if (e != cudaSuccess) return cuda_fail(e, "server cudaMallocAsync");
    s.dcap = want;
  }
  if (bytes > s.hcap) {
    const size_t want = std::max(bytes, s.hcap + s.hcap / 2);
    if (s.hbuf) retired_host.push_back(s.hbuf);
    s.hbuf = nullptr;
    s.hcap = 0;
    cudaError_t e = cudaHostAlloc((void**)&s.hbuf, want, cudaHostAllocDefault);
    if (e != cudaSuccess) return cuda_fail(e, "server cudaHostAlloc");
    s.hcap = want;
  }
  return PHC_OK;
}

// One kernel per batch: every request's paths go into one queue, so small
// systems share the GPU instead of running one after another. The register
// capacity is the largest of the batch; each warp holds one table, one
// workspace and one option block in its shared-memory slice.
int launch_batch(phc_server* S, Slot& s) {
  const phc_gpu_options& g = S->cfg.gpu;
  size_t bytes = layout_batch(s.batch);
  int st = grow(s, bytes, S->retired_host);
  if (st != PHC_OK) return st;
  s.bytes = bytes;
  unsigned char* dev = static_cast<unsigned char*>(s.dbuf);
  const int prec = (g.precision == PHC_PREC_MIXED) ? PHC_PREC_MIXED : PHC_PREC_FP64;
  int nm = 0, table_cap = 0, ws_cap = 0, fac = 1;
  int64_t total = 0;
  BatchSys* d = reinterpret_cast<BatchSys*>(s.hbuf);
  size_t plan_end = up256(s.batch.size() * sizeof(BatchSys));
  for (size_t i = 0; i < s.batch.size(); ++i) {
    Request& r = *s.batch[i];
    // the batch kernels evaluate in FP64 only: their warps stage the table
    // without its FP32 coefficients
    const int tb = r.plan.bytes_fp64;
    std::memcpy(s.hbuf + r.off_plan, r.plan.bytes.data(), r.plan.bytes.size());
    plan_end = std::max(plan_end, r.off_plan + up256(r.plan.bytes.size()));
    std::memset(&d[i], 0, sizeof(BatchSys));
    d[i].table_off = (int64_t)r.off_plan;
    d[i].table_bytes = tb;
    d[i].path_begin = total;
    d[i].npaths = r.npaths;
    d[i].out_off = (int64_t)r.off_out;
    d[i].z_off = (int64_t)r.off_z;
    d[i].x_off = (int64_t)r.off_x;
    d[i].opts = make_kopts(r.opts, g);
    total += r.npaths;
    nm = std::max(nm, r.cfg.nm);
    fac = std::max(fac, r.cfg.fac);
    table_cap = std::max(table_cap, tb);
    ws_cap = std::max(ws_cap, ws_layout(r.plan.n, r.plan.S, r.plan.pw_size, false).bytes);
  }
  const int slice = table_cap + ws_cap + align16((int)sizeof(KOpts));
  // the lean kernel form for batches with many more paths than resident
  // warps, of systems with rows of at least 16 columns: for smaller rows
  // the form's register savings buy less than its extra work per unit
  // costs (the serving stream of n <= 8: 1,577 systems/s lean against
  // 2,075 not)
  const int lean = (nm >= 16 && use_lean(total, S->cfg.device)) ? 1 : 0;
  const int smax = device_smem_optin(S->cfg.device);
  int warps = g.warps_per_block > 0
                  ? std::min(std::max(g.warps_per_block, 1), max_warps_per_block(nm, lean != 0))
                  : 4;
  while (warps > 1 && warps * slice > smax) --warps;
  if (warps * slice > smax) {
    set_last_error("batch tables do not fit in shared memory");
    return PHC_ERR_UNSUPPORTED;
  }
  const int smem = warps * slice;
  int bps = track_batch_blocks_per_sm(nm, prec, fac, lean, warps, smem);
  if (bps < 1) bps = 1;
  if (g.blocks_per_sm > 0) bps = std::min(bps, g.blocks_per_sm);
  KParamsBatch kb;
  std::memset(&kb, 0, sizeof(kb));
  kb.base = dev;
  kb.sys = reinterpret_cast<const BatchSys*>(dev);
  kb.nsys = (int32_t)s.batch.size();
  kb.chunk = g.chunk > 0 ? g.chunk : 1;
  kb.table_cap = table_cap;
  kb.ws_cap = ws_cap;
  kb.slice_bytes = slice;
  kb.total_paths = total;
  kb.counter = s.counters;
  // the slot is free, so the previous batch's kernel has finished with it
  std::memset(s.done_h, 0, s.batch.size() * sizeof(unsigned int));
  kb.done = s.done_d;
  s.nfinished = 0;
  const int64_t per = (int64_t)warps * kb.chunk;
  const int grid =
      (int)std::min<int64_t>((int64_t)device_sms(S->cfg.device) * bps, (total + per - 1) / per);
  cudaError_t e = cudaMemcpyAsync(dev, s.hbuf, plan_end, cudaMemcpyHostToDevice, s.stream);
  if (e != cudaSuccess) return cuda_fail(e, "server H2D");
  e = cudaMemsetAsync(s.counters, 0, sizeof(unsigned long long), s.stream);
  if (e != cudaSuccess) return cuda_fail(e, "server counter reset");
  e = launch_track_batch(nm, prec, fac, lean, warps, smem, kb, grid, s.stream);
  if (e != cudaSuccess) return cuda_fail(e, "server kernel launch");
  // each request's results are copied back as soon as its paths are done
  // (see engine_main); the event marks the end of the whole batch
  e = cudaEventRecord(s.done, s.stream);
  if (e != cudaSuccess) return cuda_fail(e, "server event");
  return PHC_OK;
}

void finish_request(Request& r, const unsigned char* h) {
  const int n = r.n;
  r.paths.resize(r.npaths);
  std::memcpy(r.paths.data(), h + r.off_out, (size_t)r.npaths * sizeof(phc_path_out));
  r.z.resize((size_t)r.npaths * (n + 1) * 2);
  std::memcpy(r.z.data(), h + r.off_z, r.z.size() * sizeof(double));
  r.x.resize((size_t)r.npaths * n * 2);
  std::memcpy(r.x.data(), h + r.off_x, r.x.size() * sizeof(double));
  r.sols.assign((size_t)r.npaths * n * 2, 0.0);
  r.realsols.assign((size_t)r.npaths * n, 0.0);
  r.ssols.assign((size_t)r.npaths * n * 2, 0.0);
  r.mult.assign(r.npaths, 0);
  phc_solve_result res;
  std::memset(&res, 0, sizeof(res));
  res.solutions = r.sols.data();
  res.real_solutions = r.realsols.data();
  res.singular_solutions = r.ssols.data();
  res.multiplicities = r.mult.data();
  bookkeeping(n, r.npaths, r.opts, r.paths.data(), r.x.data(), &res);
  r.counts = res.counts;
  r.counts.n = n;
  r.counts.npaths = (int32_t)r.npaths;
}

void engine_main(phc_server* S) {
  cudaSetDevice(S->cfg.device);
  const int64_t max_paths = S->cfg.max_batch_paths > 0 ? S->cfg.max_batch_paths : (1 << 20);
  const int max_sys = S->cfg.max_batch_systems > 0 ? S->cfg.max_batch_systems : 256;
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    bool progressed = false;
    // 1. completions, request by request: a request whose paths are all
    // counted (or whose batch kernel has ended) gets its results copied back
    // on the slot's copy stream while the rest of the batch keeps running;
    // once the copy has landed it is finished on the host
    for (auto& s : S->slots) {
      if (!s.busy) continue;
      const cudaError_t kq = cudaEventQuery(s.done);
      const bool kfin = (kq == cudaSuccess);
      if (kq != cudaSuccess && kq != cudaErrorNotReady) {
        // the batch kernel failed: its unfinished requests fail with it
        set_last_error(std::string("batch kernel: ") + cudaGetErrorString(kq));
        for (auto& r : s.batch) {
          if (r->stage == 2) continue;
          r->status = PHC_ERR_CUDA;
          r->error = last_error_text();
          r->t_done = Clock::now();
          r->done = true;
          r->stage = 2;
          S->completed++;
          s.nfinished++;
        }
      }
      unsigned char* dev = static_cast<unsigned char*>(s.dbuf);
      for (size_t i = 0; i < s.batch.size(); ++i) {
        Request& r = *s.batch[i];
        if (r.stage == 0) {
          const unsigned int cnt = reinterpret_cast<volatile unsigned int*>(s.done_h)[i];
          if (kfin || cnt >= (unsigned int)r.npaths) {
            cudaError_t e = cudaMemcpyAsync(s.hbuf + r.off_out, dev + r.off_out,
                                            r.end - r.off_out, cudaMemcpyDeviceToHost, s.copy);
            if (e == cudaSuccess) e = cudaEventRecord(s.copied[i], s.copy);
            if (e != cudaSuccess) {
              cuda_fail(e, "server D2H");
              r.status = PHC_ERR_CUDA;
              r.error = last_error_text();
              r.t_done = Clock::now();
              r.done = true;
              r.stage = 2;
              S->completed++;
              s.nfinished++;
              progressed = true;
              continue;
            }
            r.stage = 1;
            progressed = true;
          }
        }
        if (r.stage == 1 && cudaEventQuery(s.copied[i]) == cudaSuccess) {
          {
            NvtxRange range("phc serve: finish request");
            finish_request(r, s.hbuf);
          }
          r.t_done = Clock::now();
          r.done = true;
          r.stage = 2;
          S->completed++;
          s.nfinished++;
          progressed = true;
          S->cv.notify_all();
        }
      }
      if ((kfin || (kq != cudaErrorNotReady)) && s.nfinished == (int)s.batch.size()) {
        S->mem_in_use -= s.bytes;
        s.batch.clear();
        s.busy = false;
        progressed = true;
        S->cv.notify_all();
      }
    }
    // 2. admissions: fill every free slot with pending requests (FIFO)
    for (auto& s : S->slots) {
      if (s.busy || S->pending.empty()) continue;
      const size_t budget = (size_t)S->cfg.mem_budget_bytes;
      std::vector<std::shared_ptr<Request>> b;
      int64_t paths = 0;
      size_t bytes = 0;
      while (!S->pending.empty() && (int)b.size() < max_sys) {
        auto& r = S->pending.front();
        const size_t need = r->dev_bytes;
        if (!b.empty() && (paths + r->npaths > max_paths)) break;
        if (S->mem_in_use + bytes + need > budget) break;
        bytes += need;
        paths += r->npaths;
        b.push_back(r);
        S->pending.pop_front();
      }
      if (b.empty()) break;  // memory budget exhausted: wait for completions
      s.batch = b;
      int st;
      {
        NvtxRange range("phc serve: launch batch");
        st = launch_batch(S, s);
      }
      if (st != PHC_OK) {
        for (auto& r : s.batch) {
          r->status = st;
          r->error = last_error_text();
          r->t_done = Clock::now();
          r->done = true;
          S->completed++;
        }
        s.batch.clear();
        S->cv.notify_all();
        continue;
      }
      s.busy = true;
      S->mem_in_use += s.bytes;
      S->batches++;
      progressed = true;
    }
    bool any_busy = false;
    for (auto& s : S->slots) any_busy |= s.busy;
    if (S->stop && !any_busy) break;
    if (!progressed) {
      if (any_busy)
        S->cv.wait_for(lk, std::chrono::microseconds(50));
      else
        S->cv.wait_for(lk, std::chrono::milliseconds(20));
    }
  }
  // abort what never started
  for (auto& r : S->pending) {
    r->status = PHC_ERR_ABORTED;
    r->error = "the server stopped before the request started";
    r->done = true;
  }
  S->pending.clear();
  S->cv.notify_all();
}

}  // namespace
}  // namespace phc

namespace phc {
namespace {
// Frees every CUDA resource of the server's slots (after its engine has
// stopped, or when creation failed part way) and the server itself.
void release_server(phc_server* S) {
  cudaSetDevice(S->cfg.device);
  for (auto& s : S->slots) {
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.copy) cudaStreamSynchronize(s.copy);
    if (s.dbuf && s.stream) cudaFreeAsync(s.dbuf, s.stream);
    if (s.stream) cudaStreamSynchronize(s.stream);
    if (s.hbuf) cudaFreeHost(s.hbuf);
    if (s.counters) cudaFree(s.counters);
    if (s.done) cudaEventDestroy(s.done);
    for (auto ev : s.copied)
      if (ev) cudaEventDestroy(ev);
    if (s.done_h) cudaFreeHost(s.done_h);
    if (s.copy) cudaStreamDestroy(s.copy);
    if (s.stream) cudaStreamDestroy(s.stream);
  }
  for (void* h : S->retired_host) cudaFreeHost(h);
  delete S;
}
}  // namespace
}  // namespace phc

extern "C" {

int32_t phc_server_create(const phc_server_config* cfg, phc_server** out) {
  if (!cfg || !out) return PHC_ERR_INVALID_INPUT;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count < 1 || cfg->device < 0 ||
      cfg->device >= count) {
    set_last_error("no CUDA device for the server");
    return PHC_ERR_NO_DEVICE;
  }
  phc_server* S = new (std::nothrow) phc_server();
  if (!S) return PHC_ERR_OOM;
  // on any failure below, everything created so far is released
  auto fail = [&](int st) {
    release_server(S);
    return st;
  };
  S->cfg = *cfg;
  if (S->cfg.nslots < 1) S->cfg.nslots = 4;
  if (S->cfg.mem_budget_bytes <= 0) S->cfg.mem_budget_bytes = (int64_t)1 << 30;
  S->cfg.gpu.device = cfg->device;
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice"));
  S->slots.resize(S->cfg.nslots);
  const int max_sys = S->cfg.max_batch_systems > 0 ? S->cfg.max_batch_systems : 256;
  for (auto& s : S->slots) {
    e = cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "server stream"));
    e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return fail(cuda_fail(e, "server event"));
    e = cudaMalloc((void**)&s.counters, sizeof(unsigned long long));
    if (e != cudaSuccess) return fail(cuda_fail(e, "server counter"));
    e = cudaStreamCreateWithFlags(&s.copy, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "server copy stream"));
    e = cudaHostAlloc((void**)&s.done_h, (size_t)max_sys * sizeof(unsigned int),
                      cudaHostAllocMapped);
    if (e != cudaSuccess) return fail(cuda_fail(e, "server path counters"));
    std::memset(s.done_h, 0, (size_t)max_sys * sizeof(unsigned int));
    e = cudaHostGetDevicePointer((void**)&s.done_d, s.done_h, 0);
    if (e != cudaSuccess) return fail(cuda_fail(e, "server path counters (device view)"));
    s.copied.assign(max_sys, nullptr);
    for (auto& ev : s.copied) {
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e != cudaSuccess) return fail(cuda_fail(e, "server copy event"));
    }
    // initial buffers sized for a typical batch, grown on demand
    const int st = grow(s, (size_t)1 << 22, S->retired_host);
    if (st != PHC_OK) return fail(st);
  }
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return fail(cuda_fail(e, "server setup"));
  S->engine = std::thread(engine_main, S);
  *out = S;
  return PHC_OK;
}

int32_t phc_server_submit(phc_server* S, const phc_system* sys, const phc_solve_options* opts,
                          uint64_t* ticket) {
  if (!S || !ticket) return PHC_ERR_BAD_HANDLE;
  const phc_solve_options so = opts ? *opts : solve_defaults();
  int st = validate_options(&so);
  if (st != PHC_OK) return st;
  st = validate_system(sys);
  if (st != PHC_OK) return st;
  auto r = std::make_shared<Request>();
  r->n = sys->n;
  r->first.assign(sys->first, sys->first + sys->n + 1);
  r->deg.assign(sys->deg, sys->deg + sys->n);
  r->hexps.assign(sys->hexps, sys->hexps + (size_t)sys->nterms * (sys->n + 1));
  r->coefs.assign(sys->coefs, sys->coefs + 2 * (size_t)sys->nterms);
  r->opts = so;
  st = homotopy_init(sys, so.seed, &r->hom);  // gen%seed + hom%init
  if (st != PHC_OK) return st;
  const phc_system v = r->view();
  const phc_homotopy hv = r->hom.view();
  st = build_plan(&v, &hv, &r->plan);
  if (st != PHC_OK) return st;
  r->npaths = r->hom.nstart;
  st = resolve_launch(r->plan, S->cfg.gpu, S->cfg.device, r->npaths, &r->cfg);
  if (st != PHC_OK) return st;
  r->dev_bytes = sizeof(BatchSys) + up256(r->plan.bytes.size()) + up256((size_t)r->npaths * sizeof(phc_path_out)) +
                 up256((size_t)r->npaths * (r->n + 1) * 16) + up256((size_t)r->npaths * r->n * 16);
  if (r->dev_bytes > (size_t)S->cfg.mem_budget_bytes) {
    set_last_error("request larger than the server's memory budget");
    return PHC_ERR_ADMISSION;
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return PHC_ERR_ABORTED;
    r->ticket = S->next_ticket++;
    S->all[r->ticket] = r;
    S->pending.push_back(r);
    S->submitted++;
  }
  S->cv.notify_all();
  *ticket = r->ticket;
  return PHC_OK;
}

int32_t phc_server_poll(phc_server* S, uint64_t ticket, int32_t* done) {
  if (!S || !done) return PHC_ERR_BAD_HANDLE;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return PHC_ERR_BAD_HANDLE;
  *done = it->second->done ? 1 : 0;
  return PHC_OK;
}

int32_t phc_server_wait(phc_server* S, uint64_t ticket, int64_t timeout_ms) {
  if (!S) return PHC_ERR_BAD_HANDLE;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return PHC_ERR_BAD_HANDLE;
  auto r = it->second;
  auto pred = [&] { return r->done; };
  if (timeout_ms < 0) {
    S->cv.wait(lk, pred);
  } else if (!S->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
    return PHC_ERR_NOT_READY;
  }
  return PHC_OK;
}

int64_t phc_server_npaths(phc_server* S, uint64_t ticket) {
  if (!S) return 0;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  return it == S->all.end() ? 0 : it->second->npaths;
}

int32_t phc_server_result(phc_server* S, uint64_t ticket, phc_solve_result* res,
                          double* latency_s) {
  if (!S || !res) return PHC_ERR_BAD_HANDLE;
  std::shared_ptr<Request> r;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->all.find(ticket);
    if (it == S->all.end()) return PHC_ERR_BAD_HANDLE;
    r = it->second;
    if (!r->done) return PHC_ERR_NOT_READY;
    S->all.erase(it);
  }
  if (latency_s)
    *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  if (r->status != PHC_OK) {
    set_last_error(r->error);
    return r->status;
  }
  const int n = r->n;
  res->counts = r->counts;
  if (res->paths) std::memcpy(res->paths, r->paths.data(), r->paths.size() * sizeof(phc_path_out));
  if (res->z) std::memcpy(res->z, r->z.data(), r->z.size() * sizeof(double));
  if (res->x) std::memcpy(res->x, r->x.data(), r->x.size() * sizeof(double));
  if (res->solutions)
    std::memcpy(res->solutions, r->sols.data(), (size_t)r->counts.nsolutions * n * 2 * sizeof(double));
  if (res->real_solutions)
    std::memcpy(res->real_solutions, r->realsols.data(), (size_t)r->counts.nreal * n * sizeof(double));
  if (res->singular_solutions)
    std::memcpy(res->singular_solutions, r->ssols.data(),
                (size_t)r->counts.nsingular * n * 2 * sizeof(double));
  if (res->multiplicities)
    std::memcpy(res->multiplicities, r->mult.data(), (size_t)r->counts.nsingular * sizeof(int32_t));
  return PHC_OK;
}

int32_t phc_server_stats(phc_server* S, int64_t* submitted, int64_t* completed, int64_t* batches,
                         int64_t* in_flight) {
  if (!S) return PHC_ERR_BAD_HANDLE;
  std::lock_guard<std::mutex> lk(S->mu);
  if (submitted) *submitted = S->submitted;
  if (completed) *completed = S->completed;
  if (batches) *batches = S->batches;
  if (in_flight) {
    int64_t k = 0;
    for (auto& s : S->slots) k += s.busy ? (int64_t)s.batch.size() : 0;
    *in_flight = k;
  }
  return PHC_OK;
}

int32_t phc_server_destroy(phc_server* S) {
  if (!S) return PHC_ERR_BAD_HANDLE;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv.notify_all();
  if (S->engine.joinable()) S->engine.join();
  release_server(S);
  return PHC_OK;
}

}  // extern "C"

// phc_tune.cpp -- the launch-configuration autotuner (phc_autotune) and
// the per-process table of tuned values that resolve_launch consults.
//
// Candidates are every schedule (persistent refill, one path per warp),
// warps per block in {1, 2, 4, 6, 8, 12, 16} that fit in shared memory, and refill
// chunks {1, 2, 4} for the persistent schedule. Each is timed with CUDA
// events on the same sample of paths (one untimed launch, then the best of
// two timed ones), and the fastest wins.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>

#include "phc_host.h"

namespace phc {
namespace {

struct TuneKey {
  int device, precision, schedule, nm, lean;
  bool operator<(const TuneKey& o) const {
    return std::tie(device, precision, schedule, nm, lean) <
           std::tie(o.device, o.precision, o.schedule, o.nm, o.lean);
  }
};
struct TuneVal {
  int warps, chunk;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tuned;

}  // namespace

bool tuned_launch(int device, int precision, int schedule, int nm, int lean, int* warps,
                  int* chunk) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tuned.find(TuneKey{device, precision, schedule, nm, lean});
  if (it == g_tuned.end()) return false;
  *warps = it->second.warps;
  *chunk = it->second.chunk;
  return true;
}

}  // namespace phc

using namespace phc;

extern "C" int32_t phc_autotune(const phc_system* sys, const phc_solve_options* opts,
                                phc_gpu_options* gpu, int64_t sample_paths,
                                phc_tune_report* report) {
  NvtxRange range("phc autotune");
  if (!gpu) return PHC_ERR_INVALID_INPUT;
  phc_gpu_options g = *gpu;
  const phc_solve_options so = opts ? *opts : solve_defaults();
  int st = validate_options(&so);
  if (st != PHC_OK) return st;
  st = validate_system(sys);
  if (st != PHC_OK) return st;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || g.device < 0 || g.device >= count) {
    set_last_error("no CUDA device for the autotuner");
    return PHC_ERR_NO_DEVICE;
  }
  cudaError_t e = cudaSetDevice(g.device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  HostHomotopy hh;
  st = homotopy_init(sys, so.seed, &hh);
  if (st != PHC_OK) return st;
  const phc_homotopy hv = hh.view();
  HostPlan hp;
  st = build_plan(sys, &hv, &hp);
  if (st != PHC_OK) return st;
  const int prec = (g.precision == PHC_PREC_MIXED) ? PHC_PREC_MIXED : PHC_PREC_FP64;
  const int nm = kernel_nm(hp.n);
  int64_t sample = sample_paths;
  if (sample <= 0) sample = (int64_t)device_sms(g.device) * 8 * 4;
  sample = std::min<int64_t>(sample, hp.nstart);
  if (sample < 1) return PHC_ERR_INVALID_INPUT;

  phc_path_out* d_out = nullptr;
  double* d_z = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  auto cleanup = [&]() {
    if (stream) cudaStreamSynchronize(stream);
    if (d_out) cudaFree(d_out);
    if (d_z) cudaFree(d_z);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  };
  if ((e = cudaMalloc((void**)&d_out, (size_t)sample * sizeof(phc_path_out))) != cudaSuccess ||
      (e = cudaMalloc((void**)&d_z, (size_t)sample * hp.N * 2 * sizeof(double))) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&ev0)) != cudaSuccess || (e = cudaEventCreate(&ev1)) != cudaSuccess) {
    cleanup();
    return cuda_fail(e, "autotuner set-up");
  }

  phc_tune_report rep;
  std::memset(&rep, 0, sizeof(rep));
  rep.sample_paths = sample;
  rep.best = -1;
  const int scheds[2] = {PHC_SCHED_PERSISTENT, PHC_SCHED_GRID};
  const int warps_c[7] = {1, 2, 4, 6, 8, 12, 16};
  const int chunks[3] = {1, 2, 4};
  for (int sch : scheds) {
    for (int w : warps_c) {
      for (int ci = 0; ci < (sch == PHC_SCHED_PERSISTENT ? 3 : 1); ++ci) {
        if (rep.ncand >= PHC_TUNE_MAX) break;
        phc_gpu_options gc = g;
        gc.schedule = sch;
        gc.warps_per_block = w;
        gc.chunk = chunks[ci];
        gc.precision = prec;
        LaunchCfg cfg;
        // the form a plan of the whole system uses (phc_plan_create)
        if (resolve_launch(hp, gc, g.device, hp.nstart, &cfg) != PHC_OK || cfg.warps != w)
          continue;
        phc_plan* plan = nullptr;
        st = phc_plan_create(sys, &hv, &so, &gc, &plan);
        if (st != PHC_OK) {
          cleanup();
          return st;
        }
        double best_ms = 0.0;
        for (int rpt = 0; rpt < 3 && st == PHC_OK; ++rpt) {
          if ((e = cudaEventRecord(ev0, stream)) != cudaSuccess) break;
          st = phc_plan_launch(plan, 1, sample, d_out, d_z, stream);
          if (st != PHC_OK) break;
          if ((e = cudaEventRecord(ev1, stream)) != cudaSuccess) break;
          if ((e = cudaEventSynchronize(ev1)) != cudaSuccess) break;
          float ms = 0.f;
          if ((e = cudaEventElapsedTime(&ms, ev0, ev1)) != cudaSuccess) break;
          if (rpt > 0 && (best_ms == 0.0 || ms < best_ms)) best_ms = ms;  // first launch warms up
        }
        phc_plan_destroy(plan);
        if (st != PHC_OK || e != cudaSuccess) {
          cleanup();
          return st != PHC_OK ? st : cuda_fail(e, "autotuner launch");
        }
        const int k = rep.ncand++;
        rep.schedule[k] = sch;
        rep.warps_per_block[k] = w;
        rep.chunk[k] = chunks[ci];
        rep.ms[k] = best_ms;
        if (rep.best < 0 || best_ms < rep.ms[rep.best]) rep.best = k;
      }
    }
  }
  cleanup();
  if (rep.best < 0) {
    set_last_error("no launch configuration fits this system");
    return PHC_ERR_UNSUPPORTED;
  }
  gpu->schedule = rep.schedule[rep.best];
  gpu->warps_per_block = rep.warps_per_block[rep.best];
  gpu->chunk = rep.chunk[rep.best];
  gpu->precision = prec;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[TuneKey{g.device, prec, gpu->schedule == PHC_SCHED_PERSISTENT ? 1 : 0, nm,
                    use_lean(hp.nstart, g.device) ? 1 : 0}] =
        TuneVal{gpu->warps_per_block, gpu->chunk};
  }
  if (report) *report = rep;
  return PHC_OK;
}

// phc_host.h -- host-side internals shared by the C ABI implementation,
// the plan builder, the kernel launcher and the serving loop.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <string>
#include <vector>

#include "phc_internal.h"
#include "polyhomocont_b200.h"

namespace phc {

struct HostPlan {
  std::vector<unsigned char> bytes;  // PlanHeader + records
  int n = 0, N = 0, S = 0, maxexp = 0, pw_size = 0, nrec = 0;
  int max_fac = 0;  // most power-table factors of a Jacobian record
  int bytes_fp64 = 0;  // leading bytes without the FP32 coefficients
  int64_t nstart = 0;
};

int validate_system(const phc_system* sys);
int validate_options(const phc_solve_options* o);
int build_plan(const phc_system* sys, const phc_homotopy* hom, HostPlan* out);
// Checks every index the kernels read from a compiled table (build_plan
// calls it on its result); PHC_ERR_UNSUPPORTED with the reason otherwise.
int verify_plan(const unsigned char* bytes, size_t size);

// Homotopy constants drawn on the host with the reference generator.
struct HostHomotopy {
  double gamma[2] = {1.0, 0.0};
  std::vector<double> b, patch;
  int64_t nstart = 0;
  phc_homotopy view() const {
    phc_homotopy h;
    h.gamma[0] = gamma[0];
    h.gamma[1] = gamma[1];
    h.b = b.data();
    h.patch = patch.data();
    return h;
  }
};
int homotopy_init(const phc_system* sys, int seed, HostHomotopy* h);

// Launch configuration resolved for a plan.
struct LaunchCfg {
  int nm = 0;          // register-row capacity
  int precision = 0;   // PHC_PREC_*
  int fac = 1;         // schedule form of the kernel: 1, 2 or 3 factors per record
  int warps = 4;       // warps per block
  int persistent = 0;
  int chunk = 1;
  int grid = 0;        // persistent grid (blocks)
  int lean = 0;        // the lean form of the kernel (track_one)
  int eval32 = 0;      // the kernel carries the FP32 evaluation
  int plan_bytes = 0;  // table bytes the kernel stages into shared memory
  int ws_bytes = 0;
  int smem = 0;        // dynamic shared memory per block
};

// Opt-in shared memory per block and SM count of a device (cached).
int device_smem_optin(int device);
int device_sms(int device);
// Tuned launch parameters remembered by phc_autotune for a device,
// precision, schedule and register-row width; false if none.
bool tuned_launch(int device, int precision, int schedule, int nm, int lean, int* warps,
                  int* chunk);
// Whether a launch of `paths` paths on a device uses the lean kernel form.
bool use_lean(int64_t paths, int device);
// Resolves the launch configuration for launches of about `paths` paths
// of a plan on a device.
int resolve_launch(const HostPlan& hp, const phc_gpu_options& g, int device, int64_t paths,
                   LaunchCfg* cfg);
// Launches the tracking kernel (phc_launch.cu).
cudaError_t launch_track(const LaunchCfg& cfg, const KParams& kp, int grid, cudaStream_t s);
// Occupancy (blocks per SM) of the kernel for a configuration.
int track_blocks_per_sm(const LaunchCfg& cfg);
// Batched kernel (many systems per launch) and its occupancy.
cudaError_t launch_track_batch(int nm, int prec, int fac, int lean, int warps, int smem,
                               const KParamsBatch& kb, int grid, cudaStream_t s);
int track_batch_blocks_per_sm(int nm, int prec, int fac, int lean, int warps, int smem);
// Kernel variant: bit 0 the precision, (mode / 2) % 3 the schedule form (1,
// 2, 3 factors per record), mode / 6 the lean form.
inline int kernel_mode(int prec, int fac, int lean) {
  const int f = fac <= 1 ? 0 : (fac == 2 ? 1 : 2);
  return (prec == PHC_PREC_MIXED ? 1 : 0) + 2 * f + (lean ? 6 : 0);
}

KOpts make_kopts(const phc_solve_options& so, const phc_gpu_options& g);
phc_gpu_options gpu_defaults();
phc_solve_options solve_defaults();

// A named NVTX range over a host phase (table compile, tracking,
// bookkeeping, sampling, tuning, serving batches), visible to profilers
// that record NVTX (ncu --nvtx); without an attached tool it costs a
// branch.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

void set_last_error(const std::string& s);
// The calling thread's last error text (error texts are per thread).
std::string last_error_text();
int cuda_fail(cudaError_t e, const char* what);

// Host bookkeeping of solve() (add_solution, add_singular, find,
// collect_real; src/solve.f90:193-213, :330-426), in path order.
void bookkeeping(int n, int64_t npaths, const phc_solve_options& o, phc_path_out* paths,
                 const double* x, phc_solve_result* res);

}  // namespace phc

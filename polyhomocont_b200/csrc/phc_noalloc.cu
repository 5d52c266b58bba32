// phc_noalloc.cu -- a tracker entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc: services whose device memory is
// reserved and accounted for up front (a memory pool sized at start-up
// that must not grow), and hosts whose policy forbids device allocations
// after start-up because an allocation can block or fail at an
// unpredictable moment. phc_solve_paths_noalloc serves them. The caller
// passes its inputs (the system table and homotopy constants, in host
// memory) and its outputs (device buffers it owns); the only other device
// memory the tracker needs -- the compiled copy of the table and the
// path-queue counter -- lives in the fixed-size array below, which every
// GPU that loads the library holds until the process exits.
//
// The array's device address is looked up on the first call on each
// device and cached; a cudaDeviceReset (or anything else that destroys the
// device's primary context) invalidates the cached address, so the entry
// point must not be used on a device after such a reset.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "phc_host.h"

namespace phc {
namespace {

// Room for the persistent-queue counter (first 256 bytes) and the compiled
// table (all records of systems of up to about 7000 Jacobian terms).
constexpr size_t kNoAllocBytes = 256 * 1024;
constexpr size_t kTableOffset = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_scratch_mu;
void* g_scratch_ptr[64] = {nullptr};

// The array's name is a host-side stand-in in host code; its device
// address is looked up once per device, with that device current.
int scratch_address(int device, unsigned char** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (g_scratch_ptr[device] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_ptr[device] = p;
  }
  *out = static_cast<unsigned char*>(g_scratch_ptr[device]);
  return PHC_OK;
}

}  // namespace
}  // namespace phc

using namespace phc;

extern "C" int32_t phc_solve_paths_noalloc(const phc_system* sys, const phc_homotopy* hom,
                                           const phc_solve_options* opts,
                                           const phc_gpu_options* gpu, int64_t k0,
                                           int64_t count, phc_path_out* d_out, double* d_z,
                                           double* d_x, void* stream) {
  const phc_solve_options so = opts ? *opts : solve_defaults();
  const phc_gpu_options g = gpu ? *gpu : gpu_defaults();
  int st = validate_options(&so);
  if (st != PHC_OK) return st;
  if (count < 0 || k0 < 1 || (count > 0 && (d_out == nullptr || d_z == nullptr)))
    return PHC_ERR_INVALID_INPUT;
  if (g.device < 0 || g.device >= 64) return PHC_ERR_NO_DEVICE;
  HostPlan hp;
  st = build_plan(sys, hom, &hp);
  if (st != PHC_OK) return st;
  // k0 + count - 1 <= nstart, written so that no sum can overflow
  if (k0 - 1 > hp.nstart - count) return PHC_ERR_INVALID_INPUT;
  if (hp.bytes.size() > kNoAllocBytes - kTableOffset) {
    set_last_error("system table larger than the no-alloc scratch array (256 KiB); "
                   "use phc_solve_paths or phc_plan_create");
    return PHC_ERR_UNSUPPORTED;
  }
  if (count == 0) return PHC_OK;
  cudaError_t e = cudaSetDevice(g.device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  unsigned char* scratch = nullptr;
  st = scratch_address(g.device, &scratch);
  if (st != PHC_OK) return st;
  LaunchCfg cfg;
  st = resolve_launch(hp, g, g.device, count, &cfg);
  if (st != PHC_OK) return st;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the counter must start at zero; the table is rewritten by every call.
  // hp.bytes is pageable host memory: the copy has been staged by the time
  // cudaMemcpyAsync returns, so the buffer may be freed when this call ends.
  e = cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemsetAsync(no-alloc counter)");
  e = cudaMemcpyAsync(scratch + kTableOffset, hp.bytes.data(), hp.bytes.size(),
                      cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyAsync(no-alloc table)");
  KParams kp;
  std::memset(&kp, 0, sizeof(kp));
  kp.plan = scratch + kTableOffset;
  kp.plan_bytes = cfg.plan_bytes;
  kp.ws_bytes = cfg.ws_bytes;
  kp.warps = cfg.warps;
  kp.persistent = cfg.persistent;
  kp.chunk = cfg.chunk;
  kp.k0 = k0;
  kp.count = count;
  kp.counter = reinterpret_cast<unsigned long long*>(scratch);
  kp.out = d_out;
  kp.z = d_z;
  kp.x = d_x;
  kp.opts = make_kopts(so, g);
  int grid;
  if (cfg.persistent) {
    const int64_t per = (int64_t)cfg.warps * cfg.chunk;
    grid = (int)std::min<int64_t>(cfg.grid, (count + per - 1) / per);
  } else {
    grid = (int)((count + cfg.warps - 1) / cfg.warps);
  }
  e = launch_track(cfg, kp, grid, s);
  if (e != cudaSuccess) return cuda_fail(e, "track kernel launch (no-alloc)");
  return PHC_OK;
}

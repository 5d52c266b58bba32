// phc_launch.cu -- dispatch of the tracking kernel over the compiled
// register-row widths.
#include <cuda_runtime.h>

#include "phc_host.h"

namespace phc {

#define PHC_DECLARE_NM(NMV)                                                      \
  cudaError_t launch_nm_##NMV(int mode, const KParams& kp, int grid, int block, \
                              int smem, cudaStream_t s);                        \
  int occupancy_nm_##NMV(int mode, int block, int smem);                        \
  cudaError_t launch_batch_nm_##NMV(int mode, const KParamsBatch& kb, int grid, \
                                    int block, int smem, cudaStream_t s);       \
  int occupancy_batch_nm_##NMV(int mode, int block, int smem);
PHC_DECLARE_NM(6)
PHC_DECLARE_NM(8)
PHC_DECLARE_NM(12)
PHC_DECLARE_NM(16)
PHC_DECLARE_NM(17)
PHC_DECLARE_NM(18)
PHC_DECLARE_NM(24)
PHC_DECLARE_NM(32)

cudaError_t launch_track(const LaunchCfg& cfg, const KParams& kp, int grid, cudaStream_t s) {
  if (grid < 1) return cudaSuccess;
  const int block = cfg.warps * kWarp;
  const int mode = kernel_mode(cfg.precision, cfg.fac, cfg.lean);
  switch (cfg.nm) {
    case 6: return launch_nm_6(mode, kp, grid, block, cfg.smem, s);
    case 8: return launch_nm_8(mode, kp, grid, block, cfg.smem, s);
    case 12: return launch_nm_12(mode, kp, grid, block, cfg.smem, s);
    case 16: return launch_nm_16(mode, kp, grid, block, cfg.smem, s);
    case 17: return launch_nm_17(mode, kp, grid, block, cfg.smem, s);
    case 18: return launch_nm_18(mode, kp, grid, block, cfg.smem, s);
    case 24: return launch_nm_24(mode, kp, grid, block, cfg.smem, s);
    case 32: return launch_nm_32(mode, kp, grid, block, cfg.smem, s);
    default: return cudaErrorInvalidValue;
  }
}

int track_blocks_per_sm(const LaunchCfg& cfg) {
  const int block = cfg.warps * kWarp;
  const int mode = kernel_mode(cfg.precision, cfg.fac, cfg.lean);
  switch (cfg.nm) {
    case 6: return occupancy_nm_6(mode, block, cfg.smem);
    case 8: return occupancy_nm_8(mode, block, cfg.smem);
    case 12: return occupancy_nm_12(mode, block, cfg.smem);
    case 16: return occupancy_nm_16(mode, block, cfg.smem);
    case 17: return occupancy_nm_17(mode, block, cfg.smem);
    case 18: return occupancy_nm_18(mode, block, cfg.smem);
    case 24: return occupancy_nm_24(mode, block, cfg.smem);
    case 32: return occupancy_nm_32(mode, block, cfg.smem);
    default: return 0;
  }
}

cudaError_t launch_track_batch(int nm, int prec, int fac, int lean, int warps, int smem,
                               const KParamsBatch& kb, int grid, cudaStream_t s) {
  if (grid < 1) return cudaSuccess;
  const int block = warps * kWarp;
  const int mode = kernel_mode(prec, fac, lean);
  switch (nm) {
    case 6: return launch_batch_nm_6(mode, kb, grid, block, smem, s);
    case 8: return launch_batch_nm_8(mode, kb, grid, block, smem, s);
    case 12: return launch_batch_nm_12(mode, kb, grid, block, smem, s);
    case 16: return launch_batch_nm_16(mode, kb, grid, block, smem, s);
    case 17: return launch_batch_nm_17(mode, kb, grid, block, smem, s);
    case 18: return launch_batch_nm_18(mode, kb, grid, block, smem, s);
    case 24: return launch_batch_nm_24(mode, kb, grid, block, smem, s);
    case 32: return launch_batch_nm_32(mode, kb, grid, block, smem, s);
    default: return cudaErrorInvalidValue;
  }
}

int track_batch_blocks_per_sm(int nm, int prec, int fac, int lean, int warps, int smem) {
  const int block = warps * kWarp;
  const int mode = kernel_mode(prec, fac, lean);
  switch (nm) {
    case 6: return occupancy_batch_nm_6(mode, block, smem);
    case 8: return occupancy_batch_nm_8(mode, block, smem);
    case 12: return occupancy_batch_nm_12(mode, block, smem);
    case 16: return occupancy_batch_nm_16(mode, block, smem);
    case 17: return occupancy_batch_nm_17(mode, block, smem);
    case 18: return occupancy_batch_nm_18(mode, block, smem);
    case 24: return occupancy_batch_nm_24(mode, block, smem);
    case 32: return occupancy_batch_nm_32(mode, block, smem);
    default: return 0;
  }
}

}  // namespace phc

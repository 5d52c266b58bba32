// phc_launch.cu -- dispatch of the tracking kernel over the compiled
// register-row widths.
#include <cuda_runtime.h>

#include "phc_host.h"

namespace phc {

#define PHC_DECLARE_NM(NMV)                                                      \
  cudaError_t launch_nm_##NMV(int prec, const KParams& kp, int grid, int block, \
                              int smem, cudaStream_t s);                        \
  int occupancy_nm_##NMV(int prec, int block, int smem);                        \
  cudaError_t launch_batch_nm_##NMV(int prec, const KParamsBatch& kb, int grid, \
                                    int block, int smem, cudaStream_t s);       \
  int occupancy_batch_nm_##NMV(int prec, int block, int smem);
PHC_DECLARE_NM(6)
PHC_DECLARE_NM(8)
PHC_DECLARE_NM(12)
PHC_DECLARE_NM(16)
PHC_DECLARE_NM(18)
PHC_DECLARE_NM(24)
PHC_DECLARE_NM(32)

cudaError_t launch_track(const LaunchCfg& cfg, const KParams& kp, int grid, cudaStream_t s) {
  if (grid < 1) return cudaSuccess;
  const int block = cfg.warps * kWarp;
  switch (cfg.nm) {
    case 6: return launch_nm_6(cfg.precision, kp, grid, block, cfg.smem, s);
    case 8: return launch_nm_8(cfg.precision, kp, grid, block, cfg.smem, s);
    case 12: return launch_nm_12(cfg.precision, kp, grid, block, cfg.smem, s);
    case 16: return launch_nm_16(cfg.precision, kp, grid, block, cfg.smem, s);
    case 18: return launch_nm_18(cfg.precision, kp, grid, block, cfg.smem, s);
    case 24: return launch_nm_24(cfg.precision, kp, grid, block, cfg.smem, s);
    case 32: return launch_nm_32(cfg.precision, kp, grid, block, cfg.smem, s);
    default: return cudaErrorInvalidValue;
  }
}

int track_blocks_per_sm(const LaunchCfg& cfg) {
  const int block = cfg.warps * kWarp;
  switch (cfg.nm) {
    case 6: return occupancy_nm_6(cfg.precision, block, cfg.smem);
    case 8: return occupancy_nm_8(cfg.precision, block, cfg.smem);
    case 12: return occupancy_nm_12(cfg.precision, block, cfg.smem);
    case 16: return occupancy_nm_16(cfg.precision, block, cfg.smem);
    case 18: return occupancy_nm_18(cfg.precision, block, cfg.smem);
    case 24: return occupancy_nm_24(cfg.precision, block, cfg.smem);
    case 32: return occupancy_nm_32(cfg.precision, block, cfg.smem);
    default: return 0;
  }
}

cudaError_t launch_track_batch(int nm, int prec, int warps, int smem, const KParamsBatch& kb,
                               int grid, cudaStream_t s) {
  if (grid < 1) return cudaSuccess;
  const int block = warps * kWarp;
  switch (nm) {
    case 6: return launch_batch_nm_6(prec, kb, grid, block, smem, s);
    case 8: return launch_batch_nm_8(prec, kb, grid, block, smem, s);
    case 12: return launch_batch_nm_12(prec, kb, grid, block, smem, s);
    case 16: return launch_batch_nm_16(prec, kb, grid, block, smem, s);
    case 18: return launch_batch_nm_18(prec, kb, grid, block, smem, s);
    case 24: return launch_batch_nm_24(prec, kb, grid, block, smem, s);
    case 32: return launch_batch_nm_32(prec, kb, grid, block, smem, s);
    default: return cudaErrorInvalidValue;
  }
}

int track_batch_blocks_per_sm(int nm, int prec, int warps, int smem) {
  const int block = warps * kWarp;
  switch (nm) {
    case 6: return occupancy_batch_nm_6(prec, block, smem);
    case 8: return occupancy_batch_nm_8(prec, block, smem);
    case 12: return occupancy_batch_nm_12(prec, block, smem);
    case 16: return occupancy_batch_nm_16(prec, block, smem);
    case 18: return occupancy_batch_nm_18(prec, block, smem);
    case 24: return occupancy_batch_nm_24(prec, block, smem);
    case 32: return occupancy_batch_nm_32(prec, block, smem);
    default: return 0;
  }
}

}  // namespace phc

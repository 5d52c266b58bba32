// phc_peaks.cu -- FMA microbenchmark for the CUDA-core FP64 and FP32 peaks,
// the denominators of the tracker's roofline (the tracker runs on the FP64
// and FP32 pipes, not on tensor cores or HBM).
#include <cuda_runtime.h>

#include "phc_host.h"

namespace phc {
namespace {

constexpr int kChains = 8;

template <typename T>
__global__ void __launch_bounds__(256) fma_kernel(T* out, int iters, T a, T b) {
  T acc[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) acc[c] = (T)(threadIdx.x + c);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = fma(acc[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += acc[c];
  if (s == (T)-1.2345) out[threadIdx.x] = s;  // keeps the chains alive
}

template <typename T>
int time_fma(int device, double* tflops) {
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  T* out = nullptr;
  cudaError_t e = cudaMalloc(&out, 256 * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(e, "peaks cudaMalloc");
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  fma_kernel<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(t0);
    fma_kernel<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    if (ms < best) best = ms;
  }
  e = cudaGetLastError();
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(out);
  if (e != cudaSuccess) return cuda_fail(e, "peaks kernel");
  const double flops = 2.0 * kChains * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return PHC_OK;
}

}  // namespace
}  // namespace phc

extern "C" int32_t phc_measure_fma_peaks(int32_t device, double* fp64_tflops,
                                         double* fp32_tflops) {
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return phc::cuda_fail(e, "cudaSetDevice");
  int st = phc::time_fma<double>(device, fp64_tflops);
  if (st != PHC_OK) return st;
  return phc::time_fma<float>(device, fp32_tflops);
}

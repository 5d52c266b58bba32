// phc_probe.cu -- device probe of the tracker's reciprocal helpers (test
// infrastructure, not part of the library): rcp_nr (the hardware
// reciprocal approximation refined by Newton-Raphson) and crcp (complex
// reciprocal with Smith's division as the fallback) from phc_device.cuh,
// evaluated on caller-given inputs beside CUDA's own correctly rounded
// division 1/d and its complex division cuCdiv(1, a), so that a test can
// compare them.
#include <cuComplex.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "phc_device.cuh"

namespace {

__global__ void rcp64_kernel(const double* d, int n, double* nr, double* div) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  nr[i] = phc::rcp_nr(d[i]);
  div[i] = 1.0 / d[i];
}

__global__ void rcp32_kernel(const float* d, int n, float* nr, float* div) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  nr[i] = phc::rcp_nr(d[i]);
  div[i] = 1.0f / d[i];
}

// a, out, div: n interleaved complex values
__global__ void crcp64_kernel(const double* a, int n, double* out, double* div) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const phc::cd v = phc::mkc<double>(a[2 * i], a[2 * i + 1]);
  const phc::cd r = phc::crcp(v);
  out[2 * i] = r.re;
  out[2 * i + 1] = r.im;
  const cuDoubleComplex q =
      cuCdiv(make_cuDoubleComplex(1.0, 0.0), make_cuDoubleComplex(v.re, v.im));
  div[2 * i] = cuCreal(q);
  div[2 * i + 1] = cuCimag(q);
}

__global__ void crcp32_kernel(const float* a, int n, float* out, float* div) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const phc::cf v = phc::mkc<float>(a[2 * i], a[2 * i + 1]);
  const phc::cf r = phc::crcp(v);
  out[2 * i] = r.re;
  out[2 * i + 1] = r.im;
  const cuFloatComplex q =
      cuCdivf(make_cuFloatComplex(1.0f, 0.0f), make_cuFloatComplex(v.re, v.im));
  div[2 * i] = cuCrealf(q);
  div[2 * i + 1] = cuCimagf(q);
}

// Copies `in` (bytes_in) to the device, runs launch(d_in, d_out1, d_out2)
// and copies both outputs (bytes_out each) back. Returns a cudaError_t.
template <typename L>
int run(const void* in, size_t bytes_in, void* out1, void* out2, size_t bytes_out, L launch) {
  void *d_in = nullptr, *d_o1 = nullptr, *d_o2 = nullptr;
  cudaError_t e = cudaMalloc(&d_in, bytes_in);
  if (e == cudaSuccess) e = cudaMalloc(&d_o1, bytes_out);
  if (e == cudaSuccess) e = cudaMalloc(&d_o2, bytes_out);
  if (e == cudaSuccess) e = cudaMemcpy(d_in, in, bytes_in, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    launch(d_in, d_o1, d_o2);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out1, d_o1, bytes_out, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(out2, d_o2, bytes_out, cudaMemcpyDeviceToHost);
  cudaFree(d_in);
  cudaFree(d_o1);
  cudaFree(d_o2);
  return (int)e;
}

constexpr int kBlock = 256;
int blocks(int n) { return (n + kBlock - 1) / kBlock; }

}  // namespace

extern "C" {

int phc_probe_rcp64(const double* d, int32_t n, double* nr, double* div) {
  if (n <= 0) return 0;
  return run(d, n * sizeof(double), nr, div, n * sizeof(double), [&](void* i, void* a, void* b) {
    rcp64_kernel<<<blocks(n), kBlock>>>((const double*)i, n, (double*)a, (double*)b);
  });
}

int phc_probe_rcp32(const float* d, int32_t n, float* nr, float* div) {
  if (n <= 0) return 0;
  return run(d, n * sizeof(float), nr, div, n * sizeof(float), [&](void* i, void* a, void* b) {
    rcp32_kernel<<<blocks(n), kBlock>>>((const float*)i, n, (float*)a, (float*)b);
  });
}

int phc_probe_crcp64(const double* a, int32_t n, double* out, double* div) {
  if (n <= 0) return 0;
  return run(a, 2 * n * sizeof(double), out, div, 2 * n * sizeof(double),
             [&](void* i, void* o, void* q) {
               crcp64_kernel<<<blocks(n), kBlock>>>((const double*)i, n, (double*)o, (double*)q);
             });
}

int phc_probe_crcp32(const float* a, int32_t n, float* out, float* div) {
  if (n <= 0) return 0;
  return run(a, 2 * n * sizeof(float), out, div, 2 * n * sizeof(float),
             [&](void* i, void* o, void* q) {
               crcp32_kernel<<<blocks(n), kBlock>>>((const float*)i, n, (float*)o, (float*)q);
             });
}

}  // extern "C"

// peaks.cu -- self-tests of the device's FP64 / FP32 FMA throughput and of
// the HBM copy bandwidth, the denominators of the Newton and stencil
// rooflines.  The reference measures its own bandwidth at construction
// (timeStepper::bandwidthTest, timestepper.cpp:473-526); this extends that
// to the arithmetic pipes the Newton kernels run on.
#include <cuda_runtime.h>

#include "../../include/grim_b200.h"

namespace {

template <class T>
__global__ void k_fma_chain(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
    x7 = x0 + 7;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int u = 0; u < 16; u++) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-12345.) out[0] = s;  // keeps the chain alive
}

__global__ void k_copy(const double4* __restrict__ a, double4* __restrict__ b, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long st = (long long)gridDim.x * blockDim.x;
  for (; i < n; i += st) b[i] = a[i];
}

template <class T>
double fma_rate(int sms) {
  T* d = nullptr;
  cudaMalloc(&d, sizeof(T));
  const int iters = 256, threads = 256, blocks = sms * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma_chain<T><<<blocks, threads>>>(d, iters, (T)0.999999, (T)1e-7);
  cudaEventRecord(e0);
  const int reps = 5;
  for (int r = 0; r < reps; r++) k_fma_chain<T><<<blocks, threads>>>(d, iters, (T)0.999999, (T)1e-7);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks * reps;
  return flops / (ms * 1e-3) / 1e12;
}

}  // namespace

extern "C" int grim_measure_peaks(int device, double* fp64_tflops, double* fp32_tflops, double* hbm_gbs) {
  if (cudaSetDevice(device) != cudaSuccess) return GRIM_ECUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (fp64_tflops) *fp64_tflops = fma_rate<double>(sms);
  if (fp32_tflops) *fp32_tflops = fma_rate<float>(sms);
  if (hbm_gbs) {
    const long long n = (1LL << 30) / 32;  // 1 GiB per buffer
    double4 *a = nullptr, *b = nullptr;
    if (cudaMalloc(&a, n * 32) != cudaSuccess) return GRIM_ENOMEM;
    if (cudaMalloc(&b, n * 32) != cudaSuccess) { cudaFree(a); return GRIM_ENOMEM; }
    cudaMemset(a, 0, n * 32);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int r = 0; r < 6; r++) {
      cudaEventRecord(e0);
      k_copy<<<sms * 16, 256>>>(a, b, n);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      if (r > 0 && ms < best) best = ms;
    }
    *hbm_gbs = 2.0 * n * 32 / (best * 1e-3) / 1e9;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(a);
    cudaFree(b);
  }
  return cudaGetLastError() == cudaSuccess ? GRIM_OK : GRIM_ECUDA;
}

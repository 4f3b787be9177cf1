// FP64 / FP32 FMA throughput probe (measurement utility for the roofline
// denominator; not part of the hot path). Each thread runs 8 independent FMA
// chains so the pipe, not latency, bounds the rate; the result is written to
// global memory so the chains are not dead code.
#include <cuda_runtime.h>

namespace {

template <class T>
__global__ void k_fma(T* out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x * (T)1e-7, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
      x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
}

template <class T>
int run(int blocks, int threads, int iters, double* tflops) {
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * blocks * threads) != cudaSuccess) return 2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_fma<T><<<blocks, threads>>>(out, iters / 4, (T)0.999999, (T)1e-9);  // warm-up
  cudaEventRecord(e0);
  k_fma<T><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-9);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  const double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  return cudaGetLastError() == cudaSuccess ? 0 : 4;
}

}  // namespace

extern "C" int cco_peak_fma(int fp64, int blocks, int threads, int iters, double* tflops) {
  if (!tflops || blocks < 1 || threads < 32 || iters < 1) return 1;
  return fp64 ? run<double>(blocks, threads, iters, tflops) : run<float>(blocks, threads, iters, tflops);
}

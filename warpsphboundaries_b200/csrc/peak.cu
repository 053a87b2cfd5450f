// FMA-throughput probes of this GPU (the roofline denominators of the FP64-bound closed-form kernels):
// many independent fused multiply-add chains per thread, a grid of several CTAs per SM, timed with CUDA events.
#include <cuda_runtime.h>
#include <stdint.h>

template <typename T, int CHAINS>
__global__ void k_fma(T* out, int iters, T a, T b) {
  T x[CHAINS];
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) x[c] = (T)(threadIdx.x + c) * (T)1e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
  }
  T s = 0;
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) s += x[c];
  if (s == (T)12345.678) out[0] = s;     // keeps the chains alive
}

template <typename T>
static double run(int iters) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return -1.0;
  const int threads = 256, blocks = sms * 8;
  constexpr int CH = 8;
  k_fma<T, CH><<<blocks, threads>>>(out, iters / 8, (T)0.999999, (T)1e-7);   // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  k_fma<T, CH><<<blocks, threads>>>(out, iters, (T)0.999999, (T)1e-7);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
  const double flops = 2.0 * CH * (double)iters * threads * blocks;
  return flops / (ms * 1e-3) / 1e12;
}

// measured TFLOP/s of dependent-free FMA streams (2 flops per FMA); negative on error
extern "C" double wsbpeak_fp64_tflops(int iters) { return run<double>(iters); }
extern "C" double wsbpeak_fp32_tflops(int iters) { return run<float>(iters); }

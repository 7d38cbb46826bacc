// peak.cu -- FMA-pipe throughput of this GPU, the denominators of the FP32 / FP64 pipe
// fractions that bench.py reports beside the HBM roofline.  Not part of the energy path
// (libffxpeak.so is a separate library; include/ffxcuda.h does not declare it).
//
// Each thread runs kChains independent FMA chains for `iters` steps, so the FMA pipe sees
// kChains independent instructions per thread between dependent ones; the grid covers
// every SM several times.  The chains' sum is stored so the compiler keeps every FMA.
#include <cuda_runtime.h>
#include <stdint.h>

namespace {

constexpr int kChains = 16;
constexpr int kThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fma(int iters, T a, T b, T *out) {
  T c[kChains];
#pragma unroll
  for (int q = 0; q < kChains; q++) c[q] = (T)(threadIdx.x + q);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int q = 0; q < kChains; q++) c[q] = fma(c[q], a, b);
  }
  T s = 0;
#pragma unroll
  for (int q = 0; q < kChains; q++) s += c[q];
  out[blockIdx.x * kThreads + threadIdx.x] = s;
}

template <typename T>
int run(double *tflops, double *ms_out) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 2;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 2;
  const int blocks = sms * 8;
  const int iters = (sizeof(T) == 4) ? 8192 : 4096;
  T *out = nullptr;
  if (cudaMalloc(&out, (size_t)blocks * kThreads * sizeof(T)) != cudaSuccess) return 2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const T a = (T)0.999999, b = (T)1e-7;
  for (int w = 0; w < 3; w++) k_fma<T><<<blocks, kThreads>>>(iters, a, b, out);
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(e0);
    k_fma<T><<<blocks, kThreads>>>(iters, a, b, out);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  const cudaError_t err = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return 2;
  const double flops = 2.0 * (double)blocks * kThreads * kChains * (double)iters;
  *tflops = flops / (best * 1e-3) / 1e12;
  if (ms_out) *ms_out = best;
  return 0;
}

}  // namespace

// Best of five launches after three warm-ups: FMA throughput in TFLOP/s (2 FLOPs per FMA)
// of FP64 (fp64 != 0) or FP32 arithmetic on the current device.  Returns 0, or 2 on a CUDA
// error.
extern "C" int ffxpeak_fma_tflops(int fp64, double *tflops, double *ms) {
  if (!tflops) return 1;
  return fp64 ? run<double>(tflops, ms) : run<float>(tflops, ms);
}

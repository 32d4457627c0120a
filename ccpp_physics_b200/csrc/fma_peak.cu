// fma_peak.cu -- measured FMA throughput of the current GPU, the denominator of
// the FP-pipe roofline the benchmark reports beside the HBM one.  Built as a
// library of its own (libfma_peak.so) that only bench.py loads; it is not
// part of the RRTMG library.
//
// Each thread runs 8 independent FMA chains (so issue, not latency, limits
// it) over `iters` steps; the grid covers every SM several times.  The result
// is 2 * chains * iters * threads flops over the CUDA-event time of the
// launch.
#include <cstdint>
#include <cstdio>

#include <cuda_runtime.h>


namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T b, T c) {
  T a0 = T(threadIdx.x) * T(1e-3), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
  T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
      a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
    }
  }
  const T s = ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
  if (s == T(-1.2345)) out[blockIdx.x] = s;   // keeps the chains alive; never true
}

template <typename T>
int time_chains(int iters, double* tflops) {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
  const int blocks = sms * 8, threads = 256;
  T* out = nullptr;
  if (cudaMalloc(&out, sizeof(T) * blocks) != cudaSuccess) return 1;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chains<T><<<blocks, threads>>>(out, iters / 4, T(0.999), T(1e-4));   // warm-up
  cudaEventRecord(e0);
  fma_chains<T><<<blocks, threads>>>(out, iters, T(0.999), T(1e-4));
  cudaEventRecord(e1);
  cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess || ms <= 0.f) return 1;
  const double flops = 2.0 * 64.0 * (double)iters * (double)blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return 0;
}

}  // namespace

// FP64 and FP32 FMA throughput in TFLOP/s (either pointer may be NULL); 0 on success.
extern "C" int fma_peak_tflops(double* fp64_tflops, double* fp32_tflops) {
  if (fp64_tflops && time_chains<double>(4096, fp64_tflops)) return 1;
  if (fp32_tflops && time_chains<float>(8192, fp32_tflops)) return 1;
  return 0;
}

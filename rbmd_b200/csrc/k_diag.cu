// k_diag.cu -- FMA-chain microbenchmark for the non-tensor FP32 / FP64 pipe peaks (the roofline
// denominators of the pair and k-space kernels, which no tensor core can serve).
#include "kernels.h"

namespace rbmd {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chain(T* out, int iters, T a, T b) {
  // 8 independent dependent chains per thread hide the FMA latency
  T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6,
    x7 = x0 + 7;
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == T(-12345.678)) out[blockIdx.x] = s;  // keeps the chains alive
}

double fma_peak_tflops(int fp64, cudaStream_t st) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = fp64 ? 512 : 2048;
  void* out = nullptr;
  cudaMalloc(&out, sizeof(double) * blocks);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best = 0.0;
  for (int rep = 0; rep < 4; ++rep) {
    cudaEventRecord(a, st);
    if (fp64) k_fma_chain<double><<<blocks, threads, 0, st>>>((double*)out, iters, 0.999999, 1e-7);
    else k_fma_chain<float><<<blocks, threads, 0, st>>>((float*)out, iters, 0.999999f, 1e-7f);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    const double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
    if (rep > 0 && ms > 0) best = fmax(best, flops / (ms * 1e-3) / 1e12);
  }
  note_launch(4);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  return best;
}

}  // namespace rbmd

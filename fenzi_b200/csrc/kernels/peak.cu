// FP32 FMA throughput microbenchmark: independent FMA chains per thread, all
// operands in registers, grid sized to fill every SM several times.
#include "common.cuh"

namespace fzk {

__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float seed) {
  float a0 = seed + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
  float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
  const float m = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      a0 = fmaf(a0, m, c); a1 = fmaf(a1, m, c); a2 = fmaf(a2, m, c); a3 = fmaf(a3, m, c);
      a4 = fmaf(a4, m, c); a5 = fmaf(a5, m, c); a6 = fmaf(a6, m, c); a7 = fmaf(a7, m, c);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keep the chains live
}

double measure_fp32_peak(int device) {
  cudaSetDevice(device);
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  float* out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess) return 0.0;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  k_fma_peak<<<blocks, threads>>>(out, iters, 1.f);  // warm up / clocks up
  k_fma_peak<<<blocks, threads>>>(out, iters, 1.f);
  float best = 1e30f;
  for (int r = 0; r < 5; ++r) {
    cudaEventRecord(a);
    k_fma_peak<<<blocks, threads>>>(out, iters, 1.f);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    best = ms < best ? ms : best;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  const double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * threads;
  return flops / (best * 1e-3) / 1e12;
}

}  // namespace fzk

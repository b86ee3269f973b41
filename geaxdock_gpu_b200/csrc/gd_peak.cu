/*
 * gd_peak.cu -- measured FP32 FMA throughput of the device, the roofline denominator of the
 * pair-energy kernel (an FP32/MUFU-bound loop; neither an HBM copy nor a tensor-core GEMM
 * describes its ceiling). Eight independent FMA chains per thread, every SM busy, timed with
 * CUDA events; 2 FLOP per FMA.
 */
#include <cuda_runtime.h>

#include "../../include/geauxdock_b200.h"

namespace {

__global__ void fma_chains(float *out, int iters, float b, float c) {
  float a0 = threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5,
        a6 = a0 + 6, a7 = a0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = __fmaf_rn(a0, b, c); a1 = __fmaf_rn(a1, b, c); a2 = __fmaf_rn(a2, b, c);
      a3 = __fmaf_rn(a3, b, c); a4 = __fmaf_rn(a4, b, c); a5 = __fmaf_rn(a5, b, c);
      a6 = __fmaf_rn(a6, b, c); a7 = __fmaf_rn(a7, b, c);
    }
  }
  const float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678f) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int gd_probe_fp32_peak(int device, int repeats, double *tflops) {
  if (!tflops || repeats < 1) return GD_ERR_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return GD_ERR_NODEVICE;
  cudaDeviceProp p;
  if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return GD_ERR_CUDA;
  const int threads = 512, blocks = p.multiProcessorCount * 4, iters = 4096;
  float *out = nullptr;
  if (cudaMalloc(&out, sizeof(float) * threads * blocks) != cudaSuccess) return GD_ERR_NOMEM;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chains<<<blocks, threads>>>(out, iters / 8, 0.999f, 1e-3f); /* warm-up */
  double best = 0.0;
  for (int r = 0; r < repeats; ++r) {
    cudaEventRecord(e0);
    fma_chains<<<blocks, threads>>>(out, iters, 0.999f, 1e-3f);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    const double flops = 2.0 * 8.0 * 16.0 * iters * (double)threads * blocks;
    if (ms > 0) best = flops / (ms * 1e-3) / 1e12 > best ? flops / (ms * 1e-3) / 1e12 : best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return GD_ERR_CUDA;
  *tflops = best;
  return GD_OK;
}

// kmhd_probe.cu -- FP64 tensor-pipe peak probe for roofline denominators.
#include <cuda_runtime.h>

#include "../../include/kmhd_probe.h"
#include "kmhd_internal.cuh"

namespace {
__global__ void k_dmma_chain(double* out, int iters) {
  double c[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) c[i][0] = c[i][1] = 0.0;
  const double a = 1.0 + 1e-3 * threadIdx.x, b = 1.0 - 1e-3 * threadIdx.x;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int i = 0; i < 8; ++i) kmhd::dmma(c[i][0], c[i][1], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < 8; ++i) s += c[i][0] + c[i][1];
  if (s == 12345.678) out[0] = s;  // keeps the chain live
}
}  // namespace

extern "C" int kmhd_probe_fp64_tflops(int device, double* tflops) {
  if (!tflops) return KMHD_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return KMHD_ERR_DEVICE;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return KMHD_ERR_NOMEM;
  const int iters = 4096, threads = 256, blocks = nsm * 4;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  k_dmma_chain<<<blocks, threads>>>(out, 64);  // warm-up
  cudaEventRecord(e0);
  k_dmma_chain<<<blocks, threads>>>(out, iters);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return KMHD_ERR_CUDA;
  // one m8n8k4 = 8*8*4 FMA = 512 flop per warp instruction
  const double flops = (double)blocks * (threads / 32) * iters * 8 * 512.0;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return KMHD_OK;
}

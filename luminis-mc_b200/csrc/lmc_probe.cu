// lmc_probe.cu -- measured FP32 FMA issue peak of the current GPU.
//
// The transport kernel is bound by FP32/SFU issue, not by HBM or the tensor
// cores, so its roofline denominator is the rate at which this GPU retires
// dependent-free FFMA instructions: 16 independent FMA chains per thread,
// enough resident warps to cover the FMA latency on every SM sub-partition.
#include <cuda_runtime.h>

#include <string>

#include "lmc_internal.h"
#include "luminis_b200.h"

namespace {

__global__ void __launch_bounds__(256) ffma_chains(float *out, int iters, float b, float c)
{
  float a[16];
#pragma unroll
  for (int k = 0; k < 16; ++k)
    a[k] = (float)(threadIdx.x + k) * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k)
      a[k] = fmaf(a[k], b, c);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k)
    s += a[k];
  if (s == 1234.5f)                         // never true; keeps the chains live
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" LMC_API lmc_status lmc_probe_fp32_peak(int iters, double *tflops, double *ms)
{
  using lmc::fail;
  if (iters <= 0 || !tflops)
    return fail(LMC_ERR_INVALID, "lmc_probe_fp32_peak: iters > 0 and tflops required");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256;
  float *out = nullptr;
  cudaEvent_t e0, e1;
  if (cudaMalloc(&out, sizeof(float) * blocks * threads) != cudaSuccess)
    return fail(LMC_ERR_CUDA, "lmc_probe_fp32_peak: cudaMalloc failed");
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  ffma_chains<<<blocks, threads>>>(out, 64, 1.0000001f, 1e-7f);   // warm-up
  cudaEventRecord(e0);
  ffma_chains<<<blocks, threads>>>(out, iters, 1.0000001f, 1e-7f);
  cudaEventRecord(e1);
  const cudaError_t err = cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess)
    return fail(LMC_ERR_CUDA, std::string("lmc_probe_fp32_peak: ") + cudaGetErrorString(err));
  const double flops = 2.0 * 16.0 * (double)iters * blocks * threads;
  *tflops = flops / (t * 1e-3) / 1e12;
  if (ms)
    *ms = t;
  return LMC_OK;
}

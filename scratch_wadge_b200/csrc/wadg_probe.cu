// FP64 FMA throughput probe: the denominator of the volume kernel's roofline.
// Independent FMA chains per thread (enough ILP to saturate the FP64 pipe),
// a grid of several CTAs per SM; timed with CUDA events on the given stream.
#include <cuda_runtime.h>

#include <string>

#include "../../include/wadg.h"

namespace wadg_internal {
void set_error(const std::string &msg);
}

namespace {
constexpr int CHAINS = 8;

__global__ void __launch_bounds__(256) fp64_fma_probe(int iters, double a, double b,
                                                       double *sink) {
  double x[CHAINS];
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) x[c] = threadIdx.x * 1e-3 + c;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int c = 0; c < CHAINS; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < CHAINS; ++c) s += x[c];
  if (s == 12345.678) sink[0] = s;  // keeps the chains alive
}
}  // namespace

extern "C" int wadg_probe_fp64_fma(void *stream, int iters, double *tflops, float *ms_out) {
  if (!tflops || iters <= 0) return WADG_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double *sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return WADG_ERR_CUDA;
  const int blocks = sms * 8, threads = 256;
  // warm-up
  fp64_fma_probe<<<blocks, threads, 0, s>>>(iters / 4 + 1, 0.999999, 1e-7, sink);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, s);
  fp64_fma_probe<<<blocks, threads, 0, s>>>(iters, 0.999999, 1e-7, sink);
  cudaEventRecord(e1, s);
  cudaError_t err = cudaEventSynchronize(e1);
  float ms = 0.f;
  if (err == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  if (err != cudaSuccess) {
    wadg_internal::set_error(cudaGetErrorString(err));
    return WADG_ERR_CUDA;
  }
  const double flops = 2.0 * CHAINS * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  if (ms_out) *ms_out = ms;
  return WADG_OK;
}

// FMA-pipe throughput probe: the denominator for the sweep kernels' roofline
// (they are bound by FP32 / FP64 fused multiply-adds, not by HBM or tensor
// cores).  Every thread runs 8 independent FMA chains so the pipe, not the
// FMA latency, limits the rate; the result is stored so nothing is removed.
#include <cuda_runtime.h>

#include "../../include/chaos_lyap.h"

namespace {

template <class T>
__global__ void __launch_bounds__(256) fma_chains(T *out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int i = 0; i < 8; i++) x[i] = (T)(threadIdx.x + i);
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 16; r++)
#pragma unroll
      for (int i = 0; i < 8; i++) x[i] = x[i] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += x[i];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" int chaos_lyap_fma_peak(int device, int precision, double seconds, double *tflops) {
  if (!tflops || (precision != CHAOS_PREC_FP32 && precision != CHAOS_PREC_FP64)) return CHAOS_LYAP_EINVAL;
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return CHAOS_LYAP_ECUDA;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int block = 256, grid = sms * 8;
  void *buf = nullptr;
  if (cudaMalloc(&buf, sizeof(double) * grid * block) != cudaSuccess) {
    cudaSetDevice(prev);
    return CHAOS_LYAP_ENOMEM;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto launch = [&](int iters) {
    if (precision == CHAOS_PREC_FP32)
      fma_chains<float><<<grid, block>>>((float *)buf, iters, 0.999999f, 1e-7f);
    else
      fma_chains<double><<<grid, block>>>((double *)buf, iters, 0.999999999, 1e-12);
  };
  int iters = 64;
  float ms = 0;
  launch(iters);  // warm-up
  for (;;) {      // grow the launch until it runs for the requested time
    cudaEventRecord(e0);
    launch(iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms >= 1000.0 * seconds || iters >= (1 << 28)) break;
    iters *= ms > 1.0f ? (int)(1000.0 * seconds / ms) + 1 : 8;
  }
  const double flops = 2.0 * 8 * 16 * (double)iters * grid * block;
  *tflops = flops / (ms * 1e-3) / 1e12;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  cudaError_t e = cudaGetLastError();
  cudaSetDevice(prev);
  return e == cudaSuccess ? CHAOS_LYAP_OK : CHAOS_LYAP_ECUDA;
}

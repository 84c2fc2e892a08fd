// FMA-pipe throughput probe: the denominator for the sweep kernels' roofline
// (they are bound by FP32 / FP64 fused multiply-adds, not by HBM or tensor
// cores).  Every thread runs 8 independent FMA chains so the pipe, not the
// FMA latency, limits the rate; the result is stored so nothing is removed.
// FP32 is measured both as scalar FFMA and as packed FFMA2 chains, and the
// faster rate is the peak.
#include <cuda_runtime.h>

#include <algorithm>

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

// The same chains with FP32 pairs advanced by the packed multiply-add of
// sm_100 (one FFMA2 instruction for two FMAs), which the FP32 sweep kernels
// issue for their paired rows.
__global__ void __launch_bounds__(256) ffma2_chains(float *out, int iters, float a, float b) {
  float2 x[8];
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
  for (int i = 0; i < 8; i++) x[i] = make_float2((float)(threadIdx.x + i), (float)(threadIdx.x - i));
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int r = 0; r < 16; r++)
#pragma unroll
      for (int i = 0; i < 8; i++) x[i] = __ffma2_rn(x[i], a2, b2);
  }
  float s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += x[i].x + x[i].y;
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
  // form 0: scalar FMA chains; form 1 (FP32 only): packed FFMA2 chains, two
  // FMAs per instruction.  The peak is the faster of the two.
  auto launch = [&](int form, int iters) {
    if (precision == CHAOS_PREC_FP64)
      fma_chains<double><<<grid, block>>>((double *)buf, iters, 0.999999999, 1e-12);
    else if (form == 0)
      fma_chains<float><<<grid, block>>>((float *)buf, iters, 0.999999f, 1e-7f);
    else
      ffma2_chains<<<grid, block>>>((float *)buf, iters, 0.999999f, 1e-7f);
  };
  double best = 0.0;
  const int forms = precision == CHAOS_PREC_FP32 ? 2 : 1;
  for (int form = 0; form < forms; form++) {
    int iters = 64;
    float ms = 0;
    launch(form, iters);  // warm-up
    for (;;) {            // grow the launch until it runs for the requested time
      cudaEventRecord(e0);
      launch(form, iters);
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms >= 1000.0 * seconds || iters >= (1 << 24)) break;
      const long long grow = ms > 1.0f ? (long long)(1000.0 * seconds / ms) + 1 : 8;
      iters = (int)std::min<long long>((long long)iters * grow, 1 << 24);
    }
    const double fma_per_iter = 8.0 * 16 * (form == 1 ? 2 : 1);
    const double flops = 2.0 * fma_per_iter * (double)iters * grid * block;
    const double tf = flops / (ms * 1e-3) / 1e12;
    if (tf > best) best = tf;
  }
  *tflops = best;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(buf);
  cudaError_t e = cudaGetLastError();
  cudaSetDevice(prev);
  return e == cudaSuccess ? CHAOS_LYAP_OK : CHAOS_LYAP_ECUDA;
}

// Longest-first hand-out order for the persistent work queues.
//
// When points carry their own averaging time, the run's length is bounded by
// its longest point: a point started late that needs many steps finishes
// long after the rest.  Handing out points in decreasing averaging time
// starts the long ones first, so they overlap with everything else.
//
// A counting sort on the device (capturable in a CUDA graph, no host copy of
// the times): min / max of the times, a histogram over kOrderBuckets buckets
// spanning [min, max] (bucket 0 = longest), an exclusive scan of the counts,
// and a scatter of the point indices.  Points within a bucket come in no
// particular order; the result is a permutation of [0, P).
#include <cstdint>

#include "kernels.h"

namespace chaos {
namespace {

constexpr int kScanThreads = kOrderBuckets;  // one thread per bucket in the scan

// Non-negative doubles order like their bit patterns read as unsigned
// integers, so min / max reduce with integer atomics.  Negative or NaN times
// (rejected by the API) would only misplace points, never break the
// permutation: bucket indices are clamped.
__device__ __forceinline__ unsigned long long key(double t) {
  return (unsigned long long)__double_as_longlong(t > 0.0 ? t : 0.0);
}

__global__ void minmax_kernel(const double *__restrict__ t, int64_t P,
                              unsigned long long *__restrict__ mm) {
  unsigned long long lo = ~0ULL, hi = 0ULL;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long k = key(t[i]);
    lo = k < lo ? k : lo;
    hi = k > hi ? k : hi;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long l2 = __shfl_xor_sync(0xffffffffu, lo, o);
    const unsigned long long h2 = __shfl_xor_sync(0xffffffffu, hi, o);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
  }
}

__device__ __forceinline__ int bucket_of(double t, const unsigned long long *mm) {
  const double lo = __longlong_as_double((long long)mm[0]);
  const double hi = __longlong_as_double((long long)mm[1]);
  const double span = hi - lo;
  if (!(span > 0.0)) return 0;
  const double f = (hi - (t > 0.0 ? t : 0.0)) / span * (double)(kOrderBuckets - 1);
  return (int)fmin(fmax(f, 0.0), (double)(kOrderBuckets - 1));  // NaN -> 0
}

__global__ void histogram_kernel(const double *__restrict__ t, int64_t P,
                                 const unsigned long long *__restrict__ mm,
                                 unsigned int *__restrict__ count) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P;
       i += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&count[bucket_of(t[i], mm)], 1u);
}

// One block of kOrderBuckets threads: count[] -> exclusive prefix sums in
// place (Hillis-Steele in shared memory).
__global__ void __launch_bounds__(kScanThreads) scan_kernel(unsigned int *__restrict__ count) {
  __shared__ unsigned int buf[2][kScanThreads];
  const int i = threadIdx.x;
  buf[0][i] = i > 0 ? count[i - 1] : 0u;
  __syncthreads();
  int cur = 0;
  for (int o = 1; o < kScanThreads; o <<= 1) {
    buf[cur ^ 1][i] = buf[cur][i] + (i >= o ? buf[cur][i - o] : 0u);
    cur ^= 1;
    __syncthreads();
  }
  count[i] = buf[cur][i];
}

__global__ void scatter_kernel(const double *__restrict__ t, int64_t P,
                               const unsigned long long *__restrict__ mm,
                               unsigned int *__restrict__ next, int32_t *__restrict__ order) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < P;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned int pos = atomicAdd(&next[bucket_of(t[i], mm)], 1u);
    order[pos] = (int32_t)i;  // pos < P: the buckets' counts add up to P
  }
}

}  // namespace

int launch_order_longest_first(const double *t_avg, int64_t P, int32_t *order, void *scratch,
                               cudaStream_t s) {
  if (P <= 0) return 0;
  if (P > INT32_MAX) return kErrUnsupported;
  auto *mm = static_cast<unsigned long long *>(scratch);
  auto *count = reinterpret_cast<unsigned int *>(mm + 2);
  cudaError_t e = cudaMemsetAsync(mm, 0xff, sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(mm + 1, 0, sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(count, 0, sizeof(unsigned int) * kOrderBuckets, s);
  if (e != cudaSuccess) return (int)e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int threads = 256;
  const int64_t want = (P + threads - 1) / threads;
  const unsigned grid = (unsigned)(want < 4LL * sms ? want : 4LL * sms);
  minmax_kernel<<<grid, threads, 0, s>>>(t_avg, P, mm);
  histogram_kernel<<<grid, threads, 0, s>>>(t_avg, P, mm, count);
  scan_kernel<<<1, kScanThreads, 0, s>>>(count);
  scatter_kernel<<<grid, threads, 0, s>>>(t_avg, P, mm, count, order);
  return (int)cudaGetLastError();
}

}  // namespace chaos

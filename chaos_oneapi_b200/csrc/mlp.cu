// Learned surrogate: an ensemble of small MLPs mapping a parameter point
// (p1, p2) to its Lyapunov spectrum, trained and evaluated on the GPU by the
// kernels below (no library GEMM).
//
//   features: 16 Fourier features of the point normalised to [0, 1]^2:
//             sin / cos (2 pi w_f . (u, v)) for 8 frequency vectors (default
//             sin / cos (pi j u), sin / cos (pi j v), j = 1..4)
//   network:  16 -> W -> W -> W -> 3 (W = 128), SiLU between layers
//   numerics: weights and activations in BF16 for the tensor-core products
//             (tcgen05.mma, FP32 accumulate in tensor memory); FP32 master weights, FP32
//             pre-activations for the backward pass, FP32 Adam moments
//
// All E networks advance together: every kernel takes the network index from
// blockIdx.z.  The loss is the mean squared error of standardised targets
// (each exponent shifted and scaled by the training data's mean and std).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/chaos_lyap.h"
#include "../../include/chaos_lyap_surrogate.h"

namespace {

using bf16 = __nv_bfloat16;

constexpr int kFeat = 16;   // input features
constexpr int kOutPad = 16; // output width padded for the tensor-core tiles

thread_local std::string g_err;
int fail(int code, const std::string &m) {
  g_err = m;
  return code;
}
int cuda_fail(cudaError_t e, const char *what) {
  return fail(CHAOS_LYAP_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ------------------------------------------------------------------- GEMM
// C[z](m, n) = sum_k A[z](m, k) B[z](k, n), A and B in BF16 at arbitrary
// strides, C in FP32 (row-major, ldc), on the 5th-generation tensor cores:
//
//  * one CTA (4 warps) per 128-row x BN-column tile of C (BN = N rounded up to
//    a multiple of 16, at most 128; blockIdx.z = the network);
//  * K in blocks of 64: all threads gather the A block (128 x 64) and the B
//    block (BN x 64, i.e. B^T, K-major) from global memory into shared memory
//    in the tensor core's no-swizzle K-major layout -- 8 x 8 "core matrices"
//    of 128 contiguous bytes, core matrices adjacent in K 128 bytes apart
//    (the descriptor's leading byte offset), adjacent in M / N 1024 bytes
//    apart (its stride byte offset); rows beyond M / N and k beyond K are
//    zero.  Two shared-memory stages: the next block is gathered while the
//    tensor core works on the current one;
//  * one thread issues tcgen05.mma.cta_group::1.kind::f16 (M = 128, N = BN,
//    K = 16, BF16 x BF16 -> FP32) per 16-wide slice of the block, with the
//    accumulator in tensor memory (TMEM, 128 columns allocated per CTA), and
//    tcgen05.commit onto the stage's mbarrier, which the threads wait on
//    before they overwrite that stage;
//  * epilogue: each warp reads its 32 accumulator rows from TMEM
//    (tcgen05.ld 32x32b, 16 columns at a time) and writes C (or adds to it).
// No TMA: operands are gathered with ordinary loads, so any strides work
// (the same kernel computes X W, A^T dZ and dZ W^T).  Every wait is bounded:
// a wait that gives up sets *err and the kernel still frees its TMEM.
struct GemmArgs {
  int M, N, K;
  const bf16 *A;
  int64_t sam, sak, saz;  // A(m, k) = A[z * saz + m * sam + k * sak]
  const bf16 *B;
  int64_t sbk, sbn, sbz;  // B(k, n) = B[z * sbz + k * sbk + n * sbn]
  float *C;
  int64_t ldc, scz;
  int accumulate;         // 1: C += A B
  int *err;               // set to 1 if a wait on the tensor core gave up
};

constexpr int kTcM = 128, kTcN = 128, kTcK = 64;
constexpr int kTcTileBytes = kTcM * kTcK * 2;                // one operand stage: 16 KB
constexpr int kTcSmemBytes = 4 * kTcTileBytes + 64;          // A, B x 2 stages + barriers
constexpr int kTcTmemCols = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor of tcgen05.mma: start address, leading
// byte offset (between core matrices adjacent in K), stride byte offset
// (between core matrices adjacent in M / N), all in 16-byte units; version
// 1 (bits 46-47); base offset 0; no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)((lbo & 0x3FFFFu) >> 4) << 16) |
         ((uint64_t)((sbo & 0x3FFFFu) >> 4) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: D in FP32 (bits 4-5 = 1), A and B in
// BF16 (bits 7-9 = 1, bits 10-12 = 1), both K-major (bits 15, 16 = 0),
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
__device__ __forceinline__ uint32_t umma_instr_desc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

// Bounded wait for the phase of `parity` of an mbarrier; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (int i = 0; i < (1 << 22); i++) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Offset (in elements) of element (r, k) of a rows x 64 stage in the
// no-swizzle K-major core-matrix layout: core matrix (r / 8, k / 8) at
// ((r / 8) * 8 + k / 8) * 64, element (r % 8, k % 8) inside it.
__device__ __forceinline__ int core_offset(int r, int k) {
  return (((r >> 3) << 3) + (k >> 3)) * 64 + ((r & 7) << 3) + (k & 7);
}

// Gathers rows [row0, row0 + nrows) x k [k0, k0 + 64) of an operand X(row, k)
// = X[row * srow + k * sk] into a stage (zero outside rows < rmax, k < kmax).
// nrows is a multiple of 16.  Three ways, by the operand's layout:
//  * k contiguous (sk = 1, rows 16-byte aligned): 16-byte loads of 8
//    consecutive k, stored whole as one row of a core matrix;
//  * rows contiguous (srow = 1, k 16-byte aligned): 16-byte loads of 8
//    consecutive rows at one k, scattered into the 8 rows of a core matrix
//    (threads of a warp take consecutive k, so a warp's stores spread over
//    four core matrices);
//  * otherwise element by element.
// Each thread issues its loads for several chunks before it stores any, so
// the loads of a stage overlap instead of waiting one after another.
__device__ __forceinline__ void gather_stage(bf16 *dst, const bf16 *src, int nrows, int row0,
                                             int rmax, int64_t srow, int k0, int kmax,
                                             int64_t sk) {
  const bf16 zero = __float2bfloat16(0.f);
  const bool aligned = ((reinterpret_cast<uintptr_t>(src) & 15) == 0);
  constexpr int U = 4;  // chunks in flight per thread
  if (sk == 1 && aligned && srow % 8 == 0) {
    const int chunks = nrows * (kTcK / 8);
    for (int c0 = threadIdx.x; c0 < chunks; c0 += U * blockDim.x) {
      uint4 v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int c = c0 + u * blockDim.x;
        const int r = c >> 3, kk = (c & 7) << 3, row = row0 + r, k = k0 + kk;
        v[u] = make_uint4(0, 0, 0, 0);
        if (c < chunks && row < rmax) {
          if (k + 8 <= kmax) {
            v[u] = *reinterpret_cast<const uint4 *>(src + (int64_t)row * srow + k);
          } else {
            __align__(16) bf16 t[8];
#pragma unroll
            for (int i = 0; i < 8; i++) t[i] = (k + i < kmax) ? src[(int64_t)row * srow + k + i] : zero;
            v[u] = *reinterpret_cast<const uint4 *>(t);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int c = c0 + u * blockDim.x;
        if (c < chunks)
          *reinterpret_cast<uint4 *>(dst + core_offset(c >> 3, (c & 7) << 3)) = v[u];
      }
    }
  } else if (srow == 1 && aligned && sk % 8 == 0 && row0 % 8 == 0) {
    const int chunks = (nrows / 8) * kTcK;  // (8-row group, k) pairs, k fastest
    for (int c0 = threadIdx.x; c0 < chunks; c0 += U * blockDim.x) {
      uint4 v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int c = c0 + u * blockDim.x;
        const int kk = c % kTcK, r = (c / kTcK) * 8, row = row0 + r, k = k0 + kk;
        v[u] = make_uint4(0, 0, 0, 0);
        if (c < chunks && k < kmax) {
          if (row + 8 <= rmax) {
            v[u] = *reinterpret_cast<const uint4 *>(src + row + (int64_t)k * sk);
          } else {
            __align__(16) bf16 t[8];
#pragma unroll
            for (int i = 0; i < 8; i++) t[i] = (row + i < rmax) ? src[row + i + (int64_t)k * sk] : zero;
            v[u] = *reinterpret_cast<const uint4 *>(t);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int c = c0 + u * blockDim.x;
        if (c < chunks) {
          const int kk = c % kTcK, r = (c / kTcK) * 8;
          const bf16 *t = reinterpret_cast<const bf16 *>(&v[u]);
#pragma unroll
          for (int i = 0; i < 8; i++) dst[core_offset(r + i, kk)] = t[i];
        }
      }
    }
  } else {
    const int total = nrows * kTcK;
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      const int r = e >> 6, kk = e & 63;
      const int row = row0 + r, k = k0 + kk;
      dst[core_offset(r, kk)] = (row < rmax && k < kmax) ? src[row * srow + k * sk] : zero;
    }
  }
}

__global__ void __launch_bounds__(128) gemm_bf16_tc_kernel(const GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  bf16 *As = reinterpret_cast<bf16 *>(smem);                       // 2 stages
  bf16 *Bs = reinterpret_cast<bf16 *>(smem + 2 * kTcTileBytes);    // 2 stages
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + 4 * kTcTileBytes);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + 4 * kTcTileBytes + 16);
  const int z = blockIdx.z;
  const int m0 = blockIdx.y * kTcM, n0 = blockIdx.x * kTcN;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int bn = min(kTcN, ((g.N - n0 + 15) / 16) * 16);  // tile width, multiple of 16
  const bf16 *A = g.A + z * g.saz;
  const bf16 *B = g.B + z * g.sbz;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; i++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[i])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {  // the whole warp allocates the accumulator's TMEM columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTcTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_instr_desc(kTcM, bn);

  bool ok = true;
  const int nkb = (g.K + kTcK - 1) / kTcK;
  for (int kb = 0; kb < nkb; kb++) {
    const int st = kb & 1, k0 = kb * kTcK;
    // the MMAs that read this stage two blocks ago must be done with it
    if (kb >= 2 && ok) ok = mbar_wait(smem_u32(&bars[st]), ((kb - 2) >> 1) & 1);
    bf16 *as = As + st * (kTcTileBytes / 2), *bs = Bs + st * (kTcTileBytes / 2);
    gather_stage(as, A, kTcM, m0, g.M, g.sam, k0, g.K, g.sak);
    gather_stage(bs, B, bn, n0, g.N, g.sbn, k0, g.K, g.sbk);
    // generic-proxy stores -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const int slices = (min(kTcK, g.K - k0) + 15) / 16;
      for (int j = 0; j < slices; j++) {
        const uint64_t ad = umma_smem_desc(smem_u32(as) + j * 256, 128, 1024);
        const uint64_t bd = umma_smem_desc(smem_u32(bs) + j * 256, 128, 1024);
        const uint32_t accum = (kb > 0 || j > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(accum)
            : "memory");
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(&bars[st]))
          : "memory");
    }
  }
  // the last commit covers every MMA of the tile
  if (ok) ok = mbar_wait(smem_u32(&bars[(nkb - 1) & 1]), ((nkb - 1) >> 1) & 1);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok) {
    if (lane == 0) atomicExch(g.err, 1);
  } else {
    float *C = g.C + z * g.scz;
    const int m = m0 + warp * 32 + lane;  // this thread's accumulator row (TMEM lane)
    for (int c0 = 0; c0 < bn; c0 += 16) {
      uint32_t v[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
          "%11, %12, %13, %14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
            "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
            "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(taddr)
          : "memory");
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < g.M) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int n = n0 + c0 + j;
          if (n < g.N) {
            float *p = &C[m * g.ldc + n];
            const float d = __uint_as_float(v[j]);
            *p = g.accumulate ? *p + d : d;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcTmemCols)
                 : "memory");
}

int gemm(GemmArgs g, int nz, cudaStream_t s, int *err) {
  static unsigned long long attr_set = 0;  // devices whose kernel attribute is set
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !(attr_set >> dev & 1ull)) {
    cudaError_t e = cudaFuncSetAttribute(gemm_bf16_tc_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         kTcSmemBytes);
    if (e != cudaSuccess) return (int)e;
    if (dev < 64) attr_set |= 1ull << dev;
  }
  g.err = err;
  dim3 grid((g.N + kTcN - 1) / kTcN, (g.M + kTcM - 1) / kTcM, nz);
  gemm_bf16_tc_kernel<<<grid, 128, kTcSmemBytes, s>>>(g);
  return (int)cudaGetLastError();
}

// ------------------------------------------------------- elementwise parts
__device__ __forceinline__ float silu(float z) { return z / (1.f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
  const float sg = 1.f / (1.f + __expf(-z));
  return sg * (1.f + z * (1.f - sg));
}

// 16 Fourier features of the normalised point (shared by all networks):
// sin and cos of 2 pi (w_f . (u, v)) for 8 frequency vectors w_f.
struct Freqs {
  float w[8][2];
};
__global__ void features_kernel(const double *xy, int64_t N, double u0, double us, double v0,
                                double vs, Freqs fr, bf16 *X) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float u = (float)((xy[2 * i] - u0) * us), v = (float)((xy[2 * i + 1] - v0) * vs);
#pragma unroll
  for (int f = 0; f < 8; f++) {
    float sn, cs;
    sincospif(2.f * (fr.w[f][0] * u + fr.w[f][1] * v), &sn, &cs);
    X[i * kFeat + 2 * f] = __float2bfloat16(sn);
    X[i * kFeat + 2 * f + 1] = __float2bfloat16(cs);
  }
}

// Z += b (per column); A = SiLU(Z) in BF16.  z = network.
__global__ void bias_silu_kernel(float *Z, const float *b, int64_t sbz, bf16 *A, int64_t rows,
                                 int cols, int64_t sz) {
  const int z = blockIdx.z;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int c = (int)(i % cols);
  const float v = Z[z * sz + i] + b[z * sbz + c];
  Z[z * sz + i] = v;
  A[z * sz + i] = __float2bfloat16(silu(v));
}

// Output layer: Y = Z + b on the first `outs` columns; for training, the
// loss gradient dY = 2 (Y - T) / (rows * outs) in BF16 (zero on the padding)
// and the squared error summed into loss[z].
__global__ void output_kernel(float *Y, const float *b, int64_t sbz, int64_t rows, int outs,
                              const float *T, const float *tmean, const float *tinv, bf16 *dY,
                              float *loss) {
  const int z = blockIdx.z;
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  float l = 0.f;
  for (int c = 0; c < kOutPad; c++) {
    float *y = &Y[(z * rows + r) * kOutPad + c];
    if (c < outs) {
      *y += b[z * sbz + c];
      if (T) {
        const float t = (T[r * outs + c] - tmean[c]) * tinv[c];
        const float d = *y - t;
        l += d * d;
        dY[(z * rows + r) * kOutPad + c] = __float2bfloat16(2.f * d / (float)(rows * outs));
      }
    } else if (T) {
      dY[(z * rows + r) * kOutPad + c] = __float2bfloat16(0.f);
    }
  }
  if (T) atomicAdd(&loss[z], l / (float)(rows * outs));
}

// dZ = dA * SiLU'(Z) in BF16 (dA in FP32, from the transposed product).
__global__ void silu_back_kernel(const float *dA, const float *Z, bf16 *dZ, int64_t n, int64_t sz) {
  const int z = blockIdx.z;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  dZ[z * sz + i] = __float2bfloat16(dA[z * sz + i] * dsilu(Z[z * sz + i]));
}

// db[c] = sum_r dZ[r, c] (one thread per column, per network).
__global__ void bias_grad_kernel(const bf16 *dZ, int64_t rows, int cols, int64_t sz, float *db,
                                 int64_t sdz) {
  const int z = blockIdx.z;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int64_t r = 0; r < rows; r++) s += __bfloat162float(dZ[z * sz + r * cols + c]);
  db[z * sdz + c] = s;
}

// Adam on the FP32 master parameters, then the BF16 copy of the weights.
__global__ void adam_kernel(float *p, const float *gr, float *m, float *v, bf16 *pb, int64_t n,
                            float lr, float b1, float b2, float eps, float c1, float c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = gr[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float upd = lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  p[i] -= upd;
  pb[i] = __float2bfloat16(p[i]);
}

// Minibatch rows idx[0..B) of the training set (device xy N x 2, T N x outs
// doubles) into the step's buffers, targets to FP32.
__global__ void gather_batch_kernel(const int *idx, int64_t B, const double *xy, const double *T,
                                    int outs, double *xyb, float *Tb) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= B) return;
  const int64_t j = idx[r];
  xyb[2 * r] = xy[2 * j];
  xyb[2 * r + 1] = xy[2 * j + 1];
  for (int c = 0; c < outs; c++) Tb[r * outs + c] = (float)T[j * outs + c];
}

__global__ void to_bf16_kernel(const float *p, bf16 *pb, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pb[i] = __float2bfloat16(p[i]);
}

// Ensemble mean and standard deviation (de-standardised) of the outputs.
__global__ void ensemble_kernel(const float *Y, int E, int64_t rows, int outs, const float *tmean,
                                const float *tstd, float *mean, float *std) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= rows) return;
  for (int c = 0; c < outs; c++) {
    float s = 0.f, s2 = 0.f;
    for (int z = 0; z < E; z++) {
      const float y = Y[(z * rows + r) * kOutPad + c] * tstd[c] + tmean[c];
      s += y;
      s2 += y * y;
    }
    const float mu = s / E;
    if (mean) mean[r * outs + c] = mu;
    if (std) std[r * outs + c] = sqrtf(fmaxf(s2 / E - mu * mu, 0.f));
  }
}

inline unsigned blocks(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// Parameter layout per network (FP32 master, BF16 copy, Adam moments):
//   W1 [16 x W] b1 [W] W2 [W x W] b2 [W] W3 [W x W] b3 [W] W4 [W x 16] b4 [16]
// (W4 and b4 padded to 16 outputs; the padding stays zero).
struct chaos_mlp {
  int E, W, outs, device;
  int64_t np;  // parameters per network
  int64_t off_w[4], off_b[4];
  float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;
  bf16 *pb = nullptr;
  float tmean[kOutPad], tstd[kOutPad];
  float *d_tmean = nullptr, *d_tstd = nullptr, *d_tinv = nullptr;
  double u0 = 0, us = 1, v0 = 0, vs = 1;
  Freqs freqs;    // feature frequencies (cycles over the unit box)
  int64_t t = 0;  // Adam step
  // workspace for `cap` rows
  int64_t cap = 0;
  bf16 *X = nullptr, *A1 = nullptr, *A2 = nullptr, *A3 = nullptr, *dZ = nullptr, *dY = nullptr;
  float *Z1 = nullptr, *Z2 = nullptr, *Z3 = nullptr, *Y = nullptr, *dA = nullptr, *loss = nullptr;
  float *Tb = nullptr;
  double *xyb = nullptr;
  int *idx = nullptr;      // minibatch row indices of kTrainChunk steps
  int64_t idx_cap = 0;
  int *d_err = nullptr;  // set by a GEMM whose wait on the tensor core gave up
};

namespace {

void free_ws(chaos_mlp *h) {
  void *ps[] = {h->X, h->A1, h->A2, h->A3, h->dZ, h->dY, h->Z1, h->Z2, h->Z3, h->Y, h->dA, h->Tb,
                h->xyb};
  for (void *p : ps) cudaFree(p);
  h->X = h->A1 = h->A2 = h->A3 = h->dZ = h->dY = nullptr;
  h->Z1 = h->Z2 = h->Z3 = h->Y = h->dA = h->Tb = nullptr;
  h->xyb = nullptr;
  h->cap = 0;
}

int ensure_ws(chaos_mlp *h, int64_t rows) {
  if (rows <= h->cap) return 0;
  free_ws(h);
  const int64_t E = h->E, W = h->W;
  cudaError_t e = cudaSuccess;
  auto al = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  al((void **)&h->X, sizeof(bf16) * rows * kFeat);
  al((void **)&h->A1, sizeof(bf16) * E * rows * W);
  al((void **)&h->A2, sizeof(bf16) * E * rows * W);
  al((void **)&h->A3, sizeof(bf16) * E * rows * W);
  al((void **)&h->dZ, sizeof(bf16) * E * rows * W);
  al((void **)&h->dY, sizeof(bf16) * E * rows * kOutPad);
  al((void **)&h->Z1, sizeof(float) * E * rows * W);
  al((void **)&h->Z2, sizeof(float) * E * rows * W);
  al((void **)&h->Z3, sizeof(float) * E * rows * W);
  al((void **)&h->Y, sizeof(float) * E * rows * kOutPad);
  al((void **)&h->dA, sizeof(float) * E * rows * W);
  al((void **)&h->Tb, sizeof(float) * rows * kOutPad);
  al((void **)&h->xyb, sizeof(double) * rows * 2);
  if (e != cudaSuccess) {
    free_ws(h);
    return fail(CHAOS_LYAP_ENOMEM, std::string("surrogate workspace: ") + cudaGetErrorString(e));
  }
  h->cap = rows;
  return 0;
}

GemmArgs mk(int M, int N, int K, const bf16 *A, int64_t sam, int64_t sak, int64_t saz, const bf16 *B,
            int64_t sbk, int64_t sbn, int64_t sbz, float *C, int64_t ldc, int64_t scz, int acc = 0) {
  return GemmArgs{M, N, K, A, sam, sak, saz, B, sbk, sbn, sbz, C, ldc, scz, acc, nullptr};
}

// Forward pass of all networks on `rows` points (features already in h->X).
int forward(chaos_mlp *h, int64_t rows, cudaStream_t s) {
  const int E = h->E, W = h->W;
  const int64_t np = h->np, sz = rows * W;
  const bf16 *Wb = h->pb;
  int rc = 0;
  // Z1 = X W1 ; A1 = silu(Z1 + b1)
  rc |= gemm(mk(rows, W, kFeat, h->X, kFeat, 1, 0, Wb + h->off_w[0], W, 1, np, h->Z1, W, sz), E, s, h->d_err);
  bias_silu_kernel<<<dim3(blocks(sz, 256), 1, E), 256, 0, s>>>(h->Z1, h->p + h->off_b[0], np, h->A1, rows, W, sz);
  rc |= gemm(mk(rows, W, W, h->A1, W, 1, sz, Wb + h->off_w[1], W, 1, np, h->Z2, W, sz), E, s, h->d_err);
  bias_silu_kernel<<<dim3(blocks(sz, 256), 1, E), 256, 0, s>>>(h->Z2, h->p + h->off_b[1], np, h->A2, rows, W, sz);
  rc |= gemm(mk(rows, W, W, h->A2, W, 1, sz, Wb + h->off_w[2], W, 1, np, h->Z3, W, sz), E, s, h->d_err);
  bias_silu_kernel<<<dim3(blocks(sz, 256), 1, E), 256, 0, s>>>(h->Z3, h->p + h->off_b[2], np, h->A3, rows, W, sz);
  rc |= gemm(mk(rows, kOutPad, W, h->A3, W, 1, sz, Wb + h->off_w[3], kOutPad, 1, np, h->Y, kOutPad,
                rows * kOutPad), E, s, h->d_err);
  if (rc) return rc;
  return (int)cudaGetLastError();
}

// Backward pass after forward + output_kernel (dY set); gradients into h->g.
int backward(chaos_mlp *h, int64_t rows, cudaStream_t s) {
  const int E = h->E, W = h->W;
  const int64_t np = h->np, sz = rows * W, syz = rows * kOutPad;
  const bf16 *Wb = h->pb;
  float *g = h->g;
  int rc = 0;
  // layer 4: dW4 = A3^T dY ; db4 = sum dY ; dA3 = dY W4^T
  rc |= gemm(mk(W, kOutPad, rows, h->A3, 1, W, sz, h->dY, kOutPad, 1, syz, g + h->off_w[3], kOutPad, np), E, s, h->d_err);
  bias_grad_kernel<<<dim3(1, 1, E), kOutPad, 0, s>>>(h->dY, rows, kOutPad, syz, g + h->off_b[3], np);
  rc |= gemm(mk(rows, W, kOutPad, h->dY, kOutPad, 1, syz, Wb + h->off_w[3], 1, kOutPad, np, h->dA, W, sz), E, s, h->d_err);
  // layer 3
  silu_back_kernel<<<dim3(blocks(sz, 256), 1, E), 256, 0, s>>>(h->dA, h->Z3, h->dZ, sz, sz);
  rc |= gemm(mk(W, W, rows, h->A2, 1, W, sz, h->dZ, W, 1, sz, g + h->off_w[2], W, np), E, s, h->d_err);
  bias_grad_kernel<<<dim3(blocks(W, 128), 1, E), 128, 0, s>>>(h->dZ, rows, W, sz, g + h->off_b[2], np);
  rc |= gemm(mk(rows, W, W, h->dZ, W, 1, sz, Wb + h->off_w[2], 1, W, np, h->dA, W, sz), E, s, h->d_err);
  // layer 2
  silu_back_kernel<<<dim3(blocks(sz, 256), 1, E), 256, 0, s>>>(h->dA, h->Z2, h->dZ, sz, sz);
  rc |= gemm(mk(W, W, rows, h->A1, 1, W, sz, h->dZ, W, 1, sz, g + h->off_w[1], W, np), E, s, h->d_err);
  bias_grad_kernel<<<dim3(blocks(W, 128), 1, E), 128, 0, s>>>(h->dZ, rows, W, sz, g + h->off_b[1], np);
  rc |= gemm(mk(rows, W, W, h->dZ, W, 1, sz, Wb + h->off_w[1], 1, W, np, h->dA, W, sz), E, s, h->d_err);
  // layer 1
  silu_back_kernel<<<dim3(blocks(sz, 256), 1, E), 256, 0, s>>>(h->dA, h->Z1, h->dZ, sz, sz);
  rc |= gemm(mk(kFeat, W, rows, h->X, 1, kFeat, 0, h->dZ, W, 1, sz, g + h->off_w[0], W, np), E, s, h->d_err);
  bias_grad_kernel<<<dim3(blocks(W, 128), 1, E), 128, 0, s>>>(h->dZ, rows, W, sz, g + h->off_b[0], np);
  if (rc) return rc;
  return (int)cudaGetLastError();
}

// One forward / backward on `rows` points starting at xy / T (device).
int grad_step(chaos_mlp *h, const double *xy, const float *T, int64_t rows, cudaStream_t s) {
  features_kernel<<<blocks(rows, 256), 256, 0, s>>>(xy, rows, h->u0, h->us, h->v0, h->vs, h->freqs,
                                                    h->X);
  int rc = forward(h, rows, s);
  if (rc) return rc;
  cudaMemsetAsync(h->loss, 0, sizeof(float) * h->E, s);
  output_kernel<<<dim3(blocks(rows, 128), 1, h->E), 128, 0, s>>>(
      h->Y, h->p + h->off_b[3], h->np, rows, h->outs, T, h->d_tmean, h->d_tinv, h->dY, h->loss);
  return backward(h, rows, s);
}

// Deterministic uniform(-1, 1) for the initial weights.
inline float uhash(uint64_t seed, uint64_t i) {
  uint64_t x = seed * 0x9E3779B97F4A7C15ULL + i * 0xBF58476D1CE4E5B9ULL + 0x94D049BB133111EBULL;
  x ^= x >> 30;
  x *= 0xBF58476D1CE4E5B9ULL;
  x ^= x >> 27;
  x *= 0x94D049BB133111EBULL;
  x ^= x >> 31;
  return (float)((x >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int d) {
    cudaGetDevice(&prev);
    if (prev != d) cudaSetDevice(d);
  }
  ~DevGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

const char *chaos_mlp_last_error(void) { return g_err.c_str(); }

int chaos_mlp_create(int ensemble, int width, int outputs, uint64_t seed, int device,
                     chaos_mlp **out) {
  if (!out) return fail(CHAOS_LYAP_EINVAL, "out is null");
  *out = nullptr;
  if (ensemble < 1 || ensemble > 16 || width < 16 || width > 1024 || width % 16 ||
      outputs < 1 || outputs > kOutPad)
    return fail(CHAOS_LYAP_EINVAL, "ensemble 1..16, width multiple of 16 in 16..1024, outputs 1..16");
  DevGuard g(device);
  auto *h = new chaos_mlp();
  h->E = ensemble;
  h->W = width;
  h->outs = outputs;
  h->device = device;
  const int64_t W = width;
  const int64_t sizes_w[4] = {kFeat * W, W * W, W * W, W * kOutPad};
  const int64_t sizes_b[4] = {W, W, W, kOutPad};
  int64_t off = 0;
  for (int l = 0; l < 4; l++) {
    h->off_w[l] = off;
    off += sizes_w[l];
    h->off_b[l] = off;
    off += sizes_b[l];
  }
  h->np = off;
  const int64_t n = h->np * ensemble;
  // He-style uniform init, scaled by fan-in; zero biases and output padding
  std::vector<float> init(n, 0.f);
  const int64_t fan_in[4] = {kFeat, W, W, W};
  const int64_t cols[4] = {W, W, W, kOutPad};
  for (int z = 0; z < ensemble; z++)
    for (int l = 0; l < 4; l++) {
      const float a = std::sqrt(6.f / (float)fan_in[l]) * (l == 3 ? 0.5f : 1.f);
      for (int64_t i = 0; i < sizes_w[l]; i++) {
        const int64_t col = i % cols[l];
        if (l == 3 && col >= outputs) continue;
        init[z * h->np + h->off_w[l] + i] = a * uhash(seed + 7919ULL * z, (uint64_t)(l * 1000003 + i));
      }
    }
  cudaError_t e = cudaSuccess;
  auto al = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
  };
  al((void **)&h->p, sizeof(float) * n);
  al((void **)&h->g, sizeof(float) * n);
  al((void **)&h->m, sizeof(float) * n);
  al((void **)&h->v, sizeof(float) * n);
  al((void **)&h->pb, sizeof(bf16) * n);
  al((void **)&h->d_tmean, sizeof(float) * kOutPad * 3);
  al((void **)&h->loss, sizeof(float) * ensemble);
  al((void **)&h->d_err, sizeof(int));
  if (e != cudaSuccess) {
    cudaFree(h->p);
    cudaFree(h->g);
    cudaFree(h->m);
    cudaFree(h->v);
    cudaFree(h->pb);
    cudaFree(h->d_tmean);
    cudaFree(h->loss);
    cudaFree(h->d_err);
    delete h;
    return fail(CHAOS_LYAP_ENOMEM, std::string("surrogate parameters: ") + cudaGetErrorString(e));
  }
  // default frequencies: half-integer multiples along each axis,
  // sin / cos (pi j u) and (pi j v), j = 1..4
  for (int j = 0; j < 4; j++) {
    h->freqs.w[2 * j][0] = 0.5f * (j + 1);
    h->freqs.w[2 * j][1] = 0.f;
    h->freqs.w[2 * j + 1][0] = 0.f;
    h->freqs.w[2 * j + 1][1] = 0.5f * (j + 1);
  }
  h->d_tstd = h->d_tmean + kOutPad;
  h->d_tinv = h->d_tmean + 2 * kOutPad;
  cudaMemcpy(h->p, init.data(), sizeof(float) * n, cudaMemcpyHostToDevice);
  cudaMemset(h->g, 0, sizeof(float) * n);
  cudaMemset(h->m, 0, sizeof(float) * n);
  cudaMemset(h->v, 0, sizeof(float) * n);
  cudaMemset(h->d_err, 0, sizeof(int));
  to_bf16_kernel<<<blocks(n, 256), 256>>>(h->p, h->pb, n);
  for (int c = 0; c < kOutPad; c++) h->tmean[c] = 0.f, h->tstd[c] = 1.f;
  float tb[3 * kOutPad];
  for (int c = 0; c < kOutPad; c++) tb[c] = 0.f, tb[kOutPad + c] = 1.f, tb[2 * kOutPad + c] = 1.f;
  cudaMemcpy(h->d_tmean, tb, sizeof tb, cudaMemcpyHostToDevice);
  if ((e = cudaDeviceSynchronize()) != cudaSuccess) {
    delete h;
    return cuda_fail(e, "surrogate init");
  }
  *out = h;
  return CHAOS_LYAP_OK;
}

int chaos_mlp_destroy(chaos_mlp *h) {
  if (!h) return CHAOS_LYAP_OK;
  DevGuard g(h->device);
  cudaDeviceSynchronize();
  free_ws(h);
  cudaFree(h->idx);
  cudaFree(h->p);
  cudaFree(h->g);
  cudaFree(h->m);
  cudaFree(h->v);
  cudaFree(h->pb);
  cudaFree(h->d_tmean);
  cudaFree(h->loss);
  cudaFree(h->d_err);
  delete h;
  return CHAOS_LYAP_OK;
}

namespace {
// A GEMM whose wait on the tensor core gave up leaves *d_err set; the calls
// that wait for their work report it (and clear it).
int check_tc(chaos_mlp *h) {
  int v = 0;
  cudaMemcpy(&v, h->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (!v) return CHAOS_LYAP_OK;
  cudaMemset(h->d_err, 0, sizeof(int));
  return fail(CHAOS_LYAP_ECUDA, "surrogate GEMM: a wait on the tensor core timed out");
}
}  // namespace

int chaos_mlp_set_domain(chaos_mlp *h, double u0, double u1, double v0, double v1) {
  if (!h || !(u1 != u0) || !(v1 != v0)) return fail(CHAOS_LYAP_EINVAL, "empty domain");
  h->u0 = u0;
  h->us = 1.0 / (u1 - u0);
  h->v0 = v0;
  h->vs = 1.0 / (v1 - v0);
  return CHAOS_LYAP_OK;
}

int chaos_mlp_set_features(chaos_mlp *h, const float *freqs) {
  if (!h || !freqs) return fail(CHAOS_LYAP_EINVAL, "null argument");
  for (int f = 0; f < 8; f++) {
    h->freqs.w[f][0] = freqs[2 * f];
    h->freqs.w[f][1] = freqs[2 * f + 1];
  }
  return CHAOS_LYAP_OK;
}

int chaos_mlp_set_target_scale(chaos_mlp *h, const float *mean, const float *stdev) {
  if (!h || !mean || !stdev) return fail(CHAOS_LYAP_EINVAL, "null argument");
  float tb[3 * kOutPad];
  for (int c = 0; c < kOutPad; c++) {
    const bool used = c < h->outs;
    h->tmean[c] = used ? mean[c] : 0.f;
    h->tstd[c] = used ? std::max(stdev[c], 1e-12f) : 1.f;
    tb[c] = h->tmean[c];
    tb[kOutPad + c] = h->tstd[c];
    tb[2 * kOutPad + c] = 1.f / h->tstd[c];
  }
  DevGuard g(h->device);
  cudaError_t e = cudaMemcpy(h->d_tmean, tb, sizeof tb, cudaMemcpyHostToDevice);
  return e == cudaSuccess ? CHAOS_LYAP_OK : cuda_fail(e, "set_target_scale");
}

int64_t chaos_mlp_num_params(chaos_mlp *h) { return h ? h->np * h->E : -1; }

// FP32 master parameters (E x np) to / from host memory.
int chaos_mlp_get_params(chaos_mlp *h, float *host) {
  if (!h || !host) return fail(CHAOS_LYAP_EINVAL, "null argument");
  DevGuard g(h->device);
  cudaError_t e = cudaMemcpy(host, h->p, sizeof(float) * h->np * h->E, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? CHAOS_LYAP_OK : cuda_fail(e, "get_params");
}
int chaos_mlp_set_params(chaos_mlp *h, const float *host) {
  if (!h || !host) return fail(CHAOS_LYAP_EINVAL, "null argument");
  DevGuard g(h->device);
  const int64_t n = h->np * h->E;
  cudaError_t e = cudaMemcpy(h->p, host, sizeof(float) * n, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "set_params");
  to_bf16_kernel<<<blocks(n, 256), 256>>>(h->p, h->pb, n);
  e = cudaDeviceSynchronize();
  return e == cudaSuccess ? CHAOS_LYAP_OK : cuda_fail(e, "set_params");
}

// Loss gradient of every network on `rows` points (device xy: rows x 2
// doubles, T: rows x outputs doubles), copied to host (E x np floats); the
// per-network losses into loss_out (E floats).  No parameter update.
int chaos_mlp_gradient(chaos_mlp *h, const double *xy, const double *T, int64_t rows,
                       float *grads_out, float *loss_out) {
  if (!h || !xy || !T || rows <= 0) return fail(CHAOS_LYAP_EINVAL, "bad arguments");
  DevGuard g(h->device);
  int rc = ensure_ws(h, rows);
  if (rc) return rc;
  std::vector<double> td(rows * h->outs);
  cudaMemcpy(td.data(), T, sizeof(double) * td.size(), cudaMemcpyDeviceToHost);
  std::vector<float> tf(td.begin(), td.end());
  cudaMemcpy(h->Tb, tf.data(), sizeof(float) * tf.size(), cudaMemcpyHostToDevice);
  rc = grad_step(h, xy, h->Tb, rows, 0);
  if (rc) return cuda_fail((cudaError_t)rc, "gradient");
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) return cuda_fail(e, "gradient");
  if ((rc = check_tc(h))) return rc;
  if (grads_out) cudaMemcpy(grads_out, h->g, sizeof(float) * h->np * h->E, cudaMemcpyDeviceToHost);
  if (loss_out) cudaMemcpy(loss_out, h->loss, sizeof(float) * h->E, cudaMemcpyDeviceToHost);
  return CHAOS_LYAP_OK;
}

// Adam training on N points (device xy: N x 2, T: N x outputs doubles):
// `steps` mini-batches of `batch` rows drawn without replacement per epoch
// from a seeded permutation (a different one per call seed); lr, betas
// (0.9, 0.999), eps 1e-8.  Every network sees the same batches.  The last
// step's per-network losses go to loss_out (E floats, may be NULL).
int chaos_mlp_train(chaos_mlp *h, const double *xy, const double *T, int64_t N, int steps,
                    int batch, float lr, uint64_t seed, void *stream, float *loss_out) {
  if (!h || !xy || !T || N <= 0 || steps < 0 || batch < 16)
    return fail(CHAOS_LYAP_EINVAL, "bad arguments");
  if (N > INT32_MAX) return fail(CHAOS_LYAP_EINVAL, "at most 2^31 - 1 training rows");
  DevGuard g(h->device);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t B = std::min<int64_t>(batch, N);
  int rc = ensure_ws(h, B);
  if (rc) return rc;
  // The minibatches are drawn on the host (a seeded Fisher-Yates shuffle per
  // epoch), kTrainChunk steps of row indices at a time, and gathered on the
  // device from the training set where it lies: a step is three kernels
  // and a copy of nothing, and the host never waits for the GPU until the
  // end (each index chunk is copied on the stream, after the steps that read
  // the previous one).
  constexpr int kTrainChunk = 256;
  if (h->idx_cap < kTrainChunk * B) {
    cudaFree(h->idx);
    h->idx = nullptr;
    h->idx_cap = 0;
    cudaError_t e = cudaMalloc((void **)&h->idx, sizeof(int) * kTrainChunk * B);
    if (e != cudaSuccess) return fail(CHAOS_LYAP_ENOMEM, std::string("batch indices: ") + cudaGetErrorString(e));
    h->idx_cap = kTrainChunk * B;
  }
  std::vector<int> perm(N);
  for (int64_t i = 0; i < N; i++) perm[i] = (int)i;
  uint64_t st = seed * 0x9E3779B97F4A7C15ULL + 1;
  auto rnd = [&]() {
    st ^= st << 13;
    st ^= st >> 7;
    st ^= st << 17;
    return st;
  };
  int64_t pos = N;
  std::vector<int> chunk(kTrainChunk * B);
  const int64_t n = h->np * h->E;
  for (int it0 = 0; it0 < steps; it0 += kTrainChunk) {
    const int cs = std::min(kTrainChunk, steps - it0);
    for (int64_t r = 0; r < cs * B; r++) {
      if (pos >= N) {  // new epoch
        for (int64_t i = N - 1; i > 0; i--) std::swap(perm[i], perm[rnd() % (uint64_t)(i + 1)]);
        pos = 0;
      }
      chunk[r] = perm[pos++];
    }
    // pageable source: staged before the call returns, so the vector can be
    // refilled while the copy and the steps before it are still queued
    cudaError_t e = cudaMemcpyAsync(h->idx, chunk.data(), sizeof(int) * cs * B,
                                    cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_fail(e, "batch indices");
    for (int k = 0; k < cs; k++) {
      gather_batch_kernel<<<blocks(B, 256), 256, 0, s>>>(h->idx + (int64_t)k * B, B, xy, T, h->outs,
                                                         h->xyb, h->Tb);
      rc = grad_step(h, h->xyb, h->Tb, B, s);
      if (rc) return cuda_fail((cudaError_t)rc, "train step");
      h->t++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f / (1.f - std::pow(b1, (float)h->t));
      const float c2 = 1.f / (1.f - std::pow(b2, (float)h->t));
      adam_kernel<<<blocks(n, 256), 256, 0, s>>>(h->p, h->g, h->m, h->v, h->pb, n, lr, b1, b2,
                                                 1e-8f, c1, c2);
    }
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "train");
  if ((rc = check_tc(h))) return rc;
  if (loss_out && steps > 0) cudaMemcpy(loss_out, h->loss, sizeof(float) * h->E, cudaMemcpyDeviceToHost);
  return CHAOS_LYAP_OK;
}

// Ensemble prediction on N points (device xy: N x 2 doubles): mean and
// standard deviation over the networks, de-standardised, N x outputs floats
// each (either may be NULL).  Processes `chunk` points at a time.
int chaos_mlp_predict(chaos_mlp *h, const double *xy, int64_t N, float *mean, float *stdev,
                      void *stream) {
  if (!h || !xy || N < 0) return fail(CHAOS_LYAP_EINVAL, "bad arguments");
  DevGuard g(h->device);
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t chunk = std::min<int64_t>(N, 1 << 16);
  int rc = ensure_ws(h, std::max<int64_t>(chunk, 1));
  if (rc) return rc;
  for (int64_t o = 0; o < N; o += chunk) {
    const int64_t rows = std::min(chunk, N - o);
    features_kernel<<<blocks(rows, 256), 256, 0, s>>>(xy + 2 * o, rows, h->u0, h->us, h->v0,
                                                      h->vs, h->freqs, h->X);
    rc = forward(h, rows, s);
    if (rc) return cuda_fail((cudaError_t)rc, "predict");
    output_kernel<<<dim3(blocks(rows, 128), 1, h->E), 128, 0, s>>>(
        h->Y, h->p + h->off_b[3], h->np, rows, h->outs, nullptr, nullptr, nullptr, nullptr, nullptr);
    ensemble_kernel<<<blocks(rows, 128), 128, 0, s>>>(
        h->Y, h->E, rows, h->outs, h->d_tmean, h->d_tstd, mean ? mean + o * h->outs : nullptr,
        stdev ? stdev + o * h->outs : nullptr);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "predict");
  return check_tc(h);
}

}  // extern "C"

// Warp-per-point sweep for the 40-dimensional Lorenz-96 model
//   x_i' = (x_{i+1} - x_{i-2}) x_{i-1} - gamma x_i + F   (cyclic)
// with its k <= 40 tangent vectors: Dormand-Prince 5(4) in FP32, modified
// Gram-Schmidt QR in FP64, log-norms in FP64.
//
// Layout.  One warp owns one point.  Its 32 lanes form 4 groups of 8; a group
// holds one 40-vector, 5 consecutive components per lane, so the stencil's
// neighbours i-2, i-1, i+1 are in the lane except at its edges, where 3
// shuffles per stage fetch them from the adjacent lanes (cyclically within
// the group).  A step runs the state first (every group computes it, so each
// lane has the stage points it needs for J without any exchange), then the k
// tangent vectors four at a time.  Per-step registers: the lane's 5
// components of the 7 stage points as Jacobian coefficients, plus one
// vector's Dopri5 stages.  Between steps the tangent vectors live in shared
// memory, double-buffered (accepted / candidate, swapped on acceptance):
// 2 x k x 40 floats per warp.  Their first-stage derivatives are not stored:
// J(x) v at the step's start costs one stencil pass with the stage-0
// Jacobian coefficients the state pass computes anyway (the same floats an
// FSAL copy would hold), and leaving them out halves the shared memory per
// point, so twice as many points fit on an SM.  The FP64 QR widens the
// vectors in place over both halves (k x 40 doubles).
//
// The phase and renormalisation logic follows adaptive.cuh (transient /
// alignment / averaging with clamped landings, the renormalisation interval
// of renorm.cuh from the Gram-Schmidt cancellation and the shrinking of the
// norms, norm products flushed into Kahan sums, escape radius, step budget);
// every decision is warp-uniform.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "renorm.cuh"

namespace chaos {
namespace l96 {

constexpr int N = 40;        // model dimension
constexpr int G = 4;         // vectors processed at once per warp (lane groups)
constexpr int C = 5;         // components per lane
constexpr int WARPS = 4;     // warps (points) per block
constexpr int PV = 4;        // Gram-Schmidt: later vectors per lane group per projection round
constexpr unsigned FULL = 0xffffffffu;

struct DPc {  // Dormand-Prince 5(4), cuda/tools/dopri.dp.cpp:14-44
  static constexpr float a21 = 0.2f;
  static constexpr float a31 = 3.f / 40.f, a32 = 9.f / 40.f;
  static constexpr float a41 = 44.f / 45.f, a42 = -56.f / 15.f, a43 = 32.f / 9.f;
  static constexpr float a51 = 19372.f / 6561.f, a52 = -25360.f / 2187.f, a53 = 64448.f / 6561.f,
                         a54 = -212.f / 729.f;
  static constexpr float a61 = 9017.f / 3168.f, a62 = -355.f / 33.f, a63 = 46732.f / 5247.f,
                         a64 = 49.f / 176.f, a65 = -5103.f / 18656.f;
  static constexpr float b1 = 35.f / 384.f, b3 = 500.f / 1113.f, b4 = 125.f / 192.f,
                         b5 = -2187.f / 6784.f, b6 = 11.f / 84.f;
  static constexpr float e1 = 71.f / 57600.f, e3 = -71.f / 16695.f, e4 = 71.f / 1920.f,
                         e5 = -17253.f / 339200.f, e6 = 22.f / 525.f, e7 = -1.f / 40.f;
};

// Neighbour fetch within the lane's group: left lane's components 3, 4 and
// the right lane's component 0.
struct Nb {
  float l3, l4, r0;
};
__device__ __forceinline__ Nb neighbours(const float (&v)[C], int left, int right) {
  Nb n;
  n.l3 = __shfl_sync(FULL, v[3], left);
  n.l4 = __shfl_sync(FULL, v[4], left);
  n.r0 = __shfl_sync(FULL, v[0], right);
  return n;
}
// Extended window w[-2..5] of the lane's components: at(j) = w[j] for j in -2..5.
struct Win {
  float w[C + 3];
  __device__ __forceinline__ float at(int j) const { return w[j + 2]; }
};
__device__ __forceinline__ Win window(const float (&v)[C], const Nb &n) {
  Win e;
  e.w[0] = n.l3;
  e.w[1] = n.l4;
#pragma unroll
  for (int j = 0; j < C; j++) e.w[j + 2] = v[j];
  e.w[C + 2] = n.r0;
  return e;
}

// Jacobian coefficients of one stage point for the lane's components:
// (J v)_i = (v_{i+1} - v_{i-2}) A_i + B_i v_{i-1} - gamma v_i,
// A_i = x_{i-1}, B_i = x_{i+1} - x_{i-2}.
struct Jc {
  float A[C], B[C];
};

__device__ __forceinline__ void rhs_state(const float (&x)[C], float (&dx)[C], Jc &jc, float F,
                                          float gam, int left, int right) {
  const Win e = window(x, neighbours(x, left, right));
#pragma unroll
  for (int j = 0; j < C; j++) {
    jc.A[j] = e.at(j - 1);
    jc.B[j] = e.at(j + 1) - e.at(j - 2);
    dx[j] = jc.B[j] * jc.A[j] - gam * e.at(j) + F;
  }
}

__device__ __forceinline__ void rhs_tangent(const float (&v)[C], float (&dv)[C], const Jc &jc,
                                            float gam, int left, int right) {
  const Win e = window(v, neighbours(v, left, right));
#pragma unroll
  for (int j = 0; j < C; j++)
    dv[j] = (e.at(j + 1) - e.at(j - 2)) * jc.A[j] + jc.B[j] * e.at(j - 1) - gam * e.at(j);
}

__device__ __forceinline__ float err_term(float y0, float y1, float e, float rtol, float atol) {
  const float m = fmaxf(fabsf(y0), fabsf(y1));
  const float r = __fdividef(e, fmaf(rtol, m, atol));
  return r * r;
}

// One Dopri5 pass over the lane's 5 components.  rhs(s, arg, out) evaluates
// stage s (1..6; stage 0 = k1 is given) at arg.
template <class RHS>
__device__ __forceinline__ void dopri_pass(const float (&y)[C], const float (&k1)[C], float h,
                                           const RHS &rhs, float (&y1)[C], float (&k7)[C],
                                           float &err2, float rtol, float atol) {
  using T = DPc;
  float k2[C], k3[C], k4[C], k5[C], arg[C], e[C];
#pragma unroll
  for (int j = 0; j < C; j++) arg[j] = y[j] + h * (T::a21 * k1[j]);
  rhs(1, arg, k2);
#pragma unroll
  for (int j = 0; j < C; j++) arg[j] = y[j] + h * (T::a31 * k1[j] + T::a32 * k2[j]);
  rhs(2, arg, k3);
#pragma unroll
  for (int j = 0; j < C; j++) arg[j] = y[j] + h * (T::a41 * k1[j] + T::a42 * k2[j] + T::a43 * k3[j]);
  rhs(3, arg, k4);
#pragma unroll
  for (int j = 0; j < C; j++)
    arg[j] = y[j] + h * (T::a51 * k1[j] + T::a52 * k2[j] + T::a53 * k3[j] + T::a54 * k4[j]);
  rhs(4, arg, k5);
#pragma unroll
  for (int j = 0; j < C; j++) {
    arg[j] = y[j] + h * (T::a61 * k1[j] + T::a62 * k2[j] + T::a63 * k3[j] + T::a64 * k4[j] +
                         T::a65 * k5[j]);
    e[j] = T::e1 * k1[j] + T::e3 * k3[j] + T::e4 * k4[j] + T::e5 * k5[j];
    y1[j] = T::b1 * k1[j] + T::b3 * k3[j] + T::b4 * k4[j] + T::b5 * k5[j];
  }
  {
    float k6[C];
    rhs(5, arg, k6);
#pragma unroll
    for (int j = 0; j < C; j++) {
      y1[j] = y[j] + h * (y1[j] + T::b6 * k6[j]);
      e[j] += T::e6 * k6[j];
    }
  }
  rhs(6, y1, k7);
#pragma unroll
  for (int j = 0; j < C; j++) {
    e[j] += T::e7 * k7[j];
    err2 += err_term(y[j], y1[j], h * e[j], rtol, atol);
  }
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ double group_sum(double v) {  // over the 8 lanes of a group
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}

enum Phase : int { kTransient = 0, kAlign = 1, kAverage = 2 };

struct Warp {
  // per lane
  float x[C], kx[C];
  double sum[2], comp[2], prod[2];  // exponents lane and lane + 32
  // warp-uniform
  float F, gam, h, fac_old;
  bool reject;
  int phase;
  double t_phase, phase_len, t_gs, L, rate_max, t_avg;
  long long steps;
  long long pt;
};

__device__ __forceinline__ void flush_logs(Warp &w) {
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const double y = log(w.prod[i]) - w.comp[i];
    const double s = w.sum[i] + y;
    w.comp[i] = (s - w.sum[i]) - y;
    w.sum[i] = s;
    w.prod[i] = 1.0;
  }
}

// In-place conversions between the k x 40 FP32 vectors and their FP64 copy
// W, which covers the warp's whole 2 x k x 40-float area (base).  The FP32
// vectors are in its lower half (src_upper false) or upper half.  Chunks of
// 32 elements, each read whole (__syncwarp) before it is written, in the
// order that never overwrites an element not yet read: widening from the
// lower half runs downwards (double i covers floats 2i, 2i + 1 >= i),
// widening from the upper half and narrowing into the lower half run upwards.
__device__ void widen(const float *src, double *W, int n, int lane, bool src_upper) {
  const int nch = (n + 31) / 32;
  for (int c = 0; c < nch; c++) {
    const int idx = 32 * (src_upper ? c : nch - 1 - c) + lane;
    const float f = idx < n ? src[idx] : 0.f;
    __syncwarp();
    if (idx < n) W[idx] = (double)f;
    __syncwarp();
  }
}
__device__ void narrow(const double *W, float *dst, int n, int lane) {
  const int nch = (n + 31) / 32;
  for (int c = 0; c < nch; c++) {
    const int idx = 32 * c + lane;
    const double d = idx < n ? W[idx] : 0.0;
    __syncwarp();
    if (idx < n) dst[idx] = (float)d;
    __syncwarp();
  }
}

// Modified Gram-Schmidt in FP64 on the k vectors of V (k x 40, FP32, in the
// lower or upper half of the warp's area `base`), through the FP64 work area
// W = base (k x 40 doubles); the orthonormal vectors end in the lower half.
// Returns max |v_q|^2 / r_q^2 (the cancellation factor), the smallest r_q in
// rmin, and multiplies r_q into the lane that owns exponent q.
__device__ double mgs_qr(Warp &w, const float *V, float *base, int k, int g, int li, int lane,
                         bool accumulate, bool &ok, double &rmin) {
  double *W = reinterpret_cast<double *>(base);
  widen(V, W, k * N, lane, V != base);
  // squared norms before orthogonalisation: vector q's in lane q % 32, slot q / 32
  double nb[2] = {0.0, 0.0};
  for (int r = 0; r < (k + G - 1) / G; r++) {
    const int vec = r * G + g;
    double b = 0;
    if (vec < k) {
#pragma unroll
      for (int j = 0; j < C; j++) {
        const double vb = W[vec * N + li * C + j];
        b = fma(vb, vb, b);
      }
    }
    b = group_sum(b);
#pragma unroll
    for (int gg = 0; gg < G; gg++) {
      const double bv = __shfl_sync(FULL, b, gg * 8);
      const int q = r * G + gg;
      if (q < k && (q & 31) == lane) nb[q >> 5] = bv;
    }
  }
  __syncwarp();
  double cancel = 1.0;
  ok = true;
  rmin = 1e300;
  for (int q = 0; q < k; q++) {
    double wq[C];
#pragma unroll
    for (int j = 0; j < C; j++) wq[j] = W[q * N + li * C + j];
    double s = 0;
#pragma unroll
    for (int j = 0; j < C; j++) s = fma(wq[j], wq[j], s);
    s = group_sum(s);
    const double inv = rsqrt(s);
    const double r = s * inv;
    ok = ok && (r > 0.0) && (r < 1e300);
    rmin = fmin(rmin, r);
#pragma unroll
    for (int j = 0; j < C; j++) wq[j] *= inv;
    __syncwarp();
    if (g == 0) {
#pragma unroll
      for (int j = 0; j < C; j++) W[q * N + li * C + j] = wq[j];
    }
    // projections of the later vectors, G x PV at a time: each group takes
    // PV vectors per round, whose dot products and group sums are
    // independent chains that overlap (a round is latency-bound: a 5-term
    // FP64 dot product and three shuffle levels)
    for (int j0 = q + 1; j0 < k; j0 += G * PV) {
      double wj[PV][C], c[PV];
#pragma unroll
      for (int u = 0; u < PV; u++) {
        const int vj = j0 + u * G + g;
        const bool valid = vj < k;
#pragma unroll
        for (int j = 0; j < C; j++) wj[u][j] = valid ? W[vj * N + li * C + j] : 0.0;
        c[u] = 0.0;
#pragma unroll
        for (int j = 0; j < C; j++) c[u] = fma(wq[j], wj[u][j], c[u]);
      }
#pragma unroll
      for (int u = 0; u < PV; u++) c[u] = group_sum(c[u]);
#pragma unroll
      for (int u = 0; u < PV; u++) {
        const int vj = j0 + u * G + g;
        if (vj < k)
#pragma unroll
          for (int j = 0; j < C; j++) W[vj * N + li * C + j] = fma(-c[u], wq[j], wj[u][j]);
      }
    }
    __syncwarp();
    if (ok) {
      // cancellation: norm before any projection vs r (the first vector has none)
      if (q > 0) {
        const double b = __shfl_sync(FULL, (q >> 5) ? nb[1] : nb[0], q & 31);
        cancel = fmax(cancel, b / s);
      }
      if (accumulate && (q & 31) == lane) {
        const int slot = q >> 5;
        w.prod[slot] *= r;
      }
    }
  }
  __syncwarp();
  narrow(W, base, k * N, lane);
  return cancel;
}

__device__ void finish(Warp &w, const AdaptiveArgs &a, int k, int lane, int status) {
  flush_logs(w);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const int q = lane + 32 * i;
    if (q < k) {
      const double lam = status ? __longlong_as_double(0x7ff8000000000000ULL) : w.sum[i] / w.t_avg;
      a.spectrum.base[w.pt * a.spectrum.ps + q * a.spectrum.cs] = lam;
    }
  }
  if (lane == 0) {
    if (a.status) a.status[w.pt] = status;
    if (a.steps) a.steps[w.pt] = w.steps;
  }
}

__device__ __forceinline__ long long fetch(const AdaptiveArgs &a, int lane, long long direct) {
  if (!a.queue) return direct;
  unsigned long long q = 0;
  if (lane == 0) q = atomicAdd(a.queue, 1ULL);
  q = __shfl_sync(FULL, q, 0);
  if (q >= (unsigned long long)a.P) return a.P;
  return (long long)((q * (unsigned long long)a.queue_stride) % (unsigned long long)a.P);
}

__global__ void __launch_bounds__(WARPS * 32, 4) l96_kernel(const AdaptiveArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int g = lane >> 3, li = lane & 7;
  const int left = g * 8 + ((li + 7) & 7), right = g * 8 + ((li + 1) & 7);
  const int k = a.k;
  const size_t per_warp = (size_t)2 * k * N;  // floats: accepted and candidate vectors
  float *base = reinterpret_cast<float *>(smem) + wid * per_warp;
  float *V = base, *V1 = base + k * N;

  const float rtol = (float)a.rtol, atol = (float)a.atol;
  const float tau = 0.3f * logf(1.0f / fmaxf(rtol, 5.96e-8f));
  const double hmax = a.hmax > 0 ? a.hmax : 1e300, hmin = fmax(a.hmin, 1e-12);
  const float esc = (float)(a.escape > 0 ? a.escape : 1e4);
  constexpr float safe = 0.9f, beta = 0.04f, facc1 = 5.0f, facc2 = 0.1f;
  constexpr float expo1 = 0.2f - beta * 0.75f;

  Warp w;
  long long direct = (long long)blockIdx.x * WARPS + wid;
  w.pt = fetch(a, lane, direct);

  auto start_tangent = [&]() {
    for (int idx = lane; idx < k * N; idx += 32) V[idx] = (idx / N == idx % N) ? 1.f : 0.f;
    __syncwarp();
    w.fac_old = 1e-4f;
    w.t_phase = 0.0;
    w.t_gs = 0.0;
    if (a.t_align > 0) {
      w.phase = kAlign;
      w.phase_len = a.t_align;
    } else {
      w.phase = kAverage;
      w.phase_len = w.t_avg;
    }
  };
  auto start_point = [&]() {
    w.F = (float)a.params.base[w.pt * a.params.ps + 0 * a.params.cs];
    w.gam = (float)a.params.base[w.pt * a.params.ps + 1 * a.params.cs];
#pragma unroll
    for (int j = 0; j < C; j++) w.x[j] = (float)a.inits.base[w.pt * a.inits.ps + (li * C + j) * a.inits.cs];
    w.h = (float)a.h0;
    w.fac_old = 1e-4f;
    w.reject = false;
    w.steps = 0;
    w.t_avg = a.t_avg_per_point ? a.t_avg_per_point[w.pt] : a.t_avg;
    w.L = a.dt_renorm / adaptive::kRenormSplitInit;
    w.rate_max = adaptive::initial_renorm_rate(tau, (float)a.dt_renorm);
#pragma unroll
    for (int i = 0; i < 2; i++) w.sum[i] = w.comp[i] = 0.0, w.prod[i] = 1.0;
    Jc jc;
    rhs_state(w.x, w.kx, jc, w.F, w.gam, left, right);
    if (a.t_transient > 0) {
      w.phase = kTransient;
      w.phase_len = a.t_transient;
      w.t_phase = 0.0;
      w.t_gs = 0.0;
    } else {
      start_tangent();
    }
  };
  // Gram-Schmidt of the warp's point; false on a degenerate basis.
  auto gram_schmidt = [&]() -> bool {
    bool ok;
    double rmin;
    const double cancel = mgs_qr(w, V, base, k, g, li, lane, w.phase == kAverage, ok, rmin);
    V = base;  // the orthonormal vectors are in the lower half now
    V1 = base + k * N;
    if (!ok) return false;
    if (w.phase == kAverage) {
      bool fl = false;
#pragma unroll
      for (int i = 0; i < 2; i++) fl = fl || !(w.prod[i] < 1e150 && w.prod[i] > 1e-150);
      if (__any_sync(FULL, fl)) flush_logs(w);
    }
    if (w.t_gs > 0.0)  // the policy of every adaptive form (renorm.cuh)
      adaptive::next_renorm_interval(w.L, w.rate_max, (float)cancel, rmin, w.t_gs, tau,
                                     a.dt_renorm);
    w.t_gs = 0.0;
    return true;
  };

  if (w.pt < a.P) start_point();
  while (w.pt < a.P) {
    int status = -1;  // -1: running
    if (w.steps == 0) {  // an initial state outside the escape radius (adaptive.cuh: state_inside)
      bool inside = true;
#pragma unroll
      for (int j = 0; j < C; j++) inside = inside && (fabsf(w.x[j]) <= esc);
      if (!__all_sync(FULL, inside)) status = 4;
    }
    if (status < 0 && w.steps >= a.max_steps) status = 3;
    if (status < 0 && !((double)w.h >= hmin)) status = 2;
    if (status < 0) {
      const double remaining = w.phase_len - w.t_phase;
      const bool clamped = (double)w.h >= remaining;
      const float h = clamped ? (float)remaining : w.h;
      const bool joint = w.phase != kTransient;
      w.steps++;
      // state pass: every group computes it; the stage points become J coefficients
      Jc jcs[7];
      float x1[C], kx1[C], err_state = 0.f;
      {
        auto rhs = [&](int s, const float (&arg)[C], float (&out)[C]) {
          rhs_state(arg, out, jcs[s], w.F, w.gam, left, right);
        };
        // stage 0 coefficients at the current state
        float dummy[C];
        rhs_state(w.x, dummy, jcs[0], w.F, w.gam, left, right);
        dopri_pass(w.x, w.kx, h, rhs, x1, kx1, err_state, rtol, atol);
      }
      float err2 = (g == 0) ? err_state : 0.f;
      if (joint) {
        for (int r = 0; r < (k + G - 1) / G; r++) {
          const int vec = r * G + g;
          const bool valid = vec < k;
          float v[C], kv[C], v1[C], kv1[C];
#pragma unroll
          for (int j = 0; j < C; j++) v[j] = valid ? V[vec * N + li * C + j] : 0.f;
          // first stage: J(x) v with the state pass's stage-0 coefficients
          rhs_tangent(v, kv, jcs[0], w.gam, left, right);
          float e2 = 0.f;
          auto rhs = [&](int s, const float (&arg)[C], float (&out)[C]) {
            rhs_tangent(arg, out, jcs[s], w.gam, left, right);
          };
          dopri_pass(v, kv, h, rhs, v1, kv1, e2, rtol, atol);
          if (valid) {
            err2 += e2;
#pragma unroll
            for (int j = 0; j < C; j++) V1[vec * N + li * C + j] = v1[j];
          }
        }
      }
      const float nc = joint ? (float)(N * (1 + k)) : (float)N;
      const float err = sqrtf(warp_sum(err2) / nc);
      if (!(err == err) || err > 3.0e38f) {  // the other forms' rule (adaptive.cuh: point_finite)
        bool fin = (w.F - w.F == 0.f) && (w.gam - w.gam == 0.f);
#pragma unroll
        for (int j = 0; j < C; j++) fin = fin && (w.x[j] - w.x[j] == 0.f);
        if (!__all_sync(FULL, fin)) {
          status = 1;
        } else {
          w.h = h / 5.0f;  // the controller's largest reduction
          w.reject = true;
        }
      } else {
        const float fac11 = exp2f(expo1 * __log2f(fmaxf(err, 1e-30f)));
        if (err <= 1.0f) {
          float fac = fac11 * exp2f(-beta * __log2f(w.fac_old));
          fac = fmaxf(facc2, fminf(facc1, fac * (1.0f / safe)));
          float hnew = h * __fdividef(1.0f, fac);
          w.fac_old = fmaxf(err, 1e-4f);
#pragma unroll
          for (int j = 0; j < C; j++) {
            w.x[j] = x1[j];
            w.kx[j] = kx1[j];
          }
          __syncwarp();
          if (joint) {  // accept the candidate: swap buffers
            float *t0 = V;
            V = V1;
            V1 = t0;
          }
          if ((double)hnew > hmax) hnew = (float)hmax;
          if (w.reject && hnew > h) hnew = h;
          w.reject = false;
          if (!clamped || hnew < h) w.h = hnew;
          w.t_phase = clamped ? w.phase_len : w.t_phase + (double)h;
          w.t_gs += (double)h;
          bool inside = true;
#pragma unroll
          for (int j = 0; j < C; j++) inside = inside && (fabsf(w.x[j]) <= esc);
          if (!__all_sync(FULL, inside)) {
            status = 4;
          } else if (clamped) {
            if (w.phase == kTransient) {
              start_tangent();
            } else if (w.phase == kAlign) {
              if (!gram_schmidt()) status = 1;
              w.phase = kAverage;
              w.phase_len = w.t_avg;
              w.t_phase = 0.0;
            } else {
              status = gram_schmidt() ? 0 : 1;
            }
          } else if (joint && w.t_gs >= w.L) {
            if (!gram_schmidt()) status = 1;
          }
        } else {
          w.h = h * __fdividef(1.0f, fminf(facc1, fac11 * (1.0f / safe)));
          w.reject = true;
        }
      }
    }
    if (status >= 0) {
      finish(w, a, k, lane, status);
      w.pt = fetch(a, lane, a.P);
      if (w.pt < a.P) start_point();
    }
  }
}

}  // namespace l96

int launch_l96_warp(int integrator, int precision, const AdaptiveArgs &a, int, cudaStream_t s) {
  using namespace l96;
  if (integrator != kDopri5 || precision != kFP32) return kErrUnsupported;
  if (a.k < 1 || a.k > N) return kErrUnsupported;
  const size_t smem = (size_t)WARPS * 2 * a.k * N * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(l96_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return (int)e;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned grid;
  if (a.queue) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, l96_kernel, WARPS * 32, smem);
    grid = (unsigned)std::min<int64_t>((int64_t)std::max(1, per_sm) * sms, (a.P + WARPS - 1) / WARPS);
  } else {
    grid = (unsigned)((a.P + WARPS - 1) / WARPS);
  }
  l96_kernel<<<grid, WARPS * 32, smem, s>>>(a);
  return (int)cudaGetLastError();
}

}  // namespace chaos

// Reference-exact FP64 sweep ("compat" precision).
//
// One thread per parameter point, the model inlined as a template parameter,
// state / tangent vectors / DVERK stages in registers (the reference keeps
// them in per-work-item global scratch, tasklyapunov.cpp:104-176).  The
// arithmetic follows the reference operation by operation so that, compiled
// with -fmad=false (no FMA contraction), trajectories agree bit for bit with
// the reference built for the host CPU:
//   * DVERK step: cuda/tools/dverk.dp.cpp:7-43 (state), :45-81 (tangent with
//     the base point frozen) -- same stage order and coefficient grouping;
//   * phase loops with double time counters (`for (t = 0; t < T; t += h)`),
//     renormalisation on `skipCount == addSkipSteps`:
//     cuda/lyapunov.dp.cpp:5-68 (FD), :133-180 (VAR), :229-259 (QR);
//   * classical Gram-Schmidt with an accumulated projection and rescaling to
//     length eps: cuda/tools/linalg.dp.cpp:20-51; QR by column CGS and
//     R = Q^T A: :54-127 (square case).
// This translation unit must be compiled with -fmad=false.
#include "kernels.h"
#include "models.cuh"

namespace chaos {
namespace {

template <class M> struct DState {
  const double *p;
  __device__ __forceinline__ void operator()(const double *y, double *dy) const { M::f(y, dy, p); }
};
template <class M> struct DVar {
  const double *p, *x;
  __device__ __forceinline__ void operator()(const double *y, double *dy) const { M::jv(y, dy, p, x); }
};
template <class M> struct DQcol {
  const double *p, *x;
  __device__ __forceinline__ void operator()(const double *y, double *dy) const { M::jq_col(y, dy, p, x); }
};

// One fixed DVERK step, cuda/tools/dverk.dp.cpp:7-43.
template <int D, class F>
__device__ __forceinline__ void dverk(double *val, const F &fn, double step) {
  double arg[D], k1[D], k2[D], k3[D], k4[D], k5[D], k6[D], k7[D], k8[D];
  fn(val, k1);
  for (int j = 0; j < D; j++) arg[j] = val[j] + step / 6. * k1[j];
  fn(arg, k2);
  for (int j = 0; j < D; j++) arg[j] = val[j] + step * (4. / 75. * k1[j] + 16. / 75. * k2[j]);
  fn(arg, k3);
  for (int j = 0; j < D; j++)
    arg[j] = val[j] + step * (5. / 6. * k1[j] - 8. / 3. * k2[j] + 5. / 2. * k3[j]);
  fn(arg, k4);
  for (int j = 0; j < D; j++)
    arg[j] = val[j] + step * (-165. / 64. * k1[j] + 55. / 6. * k2[j] - 425. / 64. * k3[j] +
                              85. / 96. * k4[j]);
  fn(arg, k5);
  for (int j = 0; j < D; j++)
    arg[j] = val[j] + step * (12. / 5. * k1[j] - 8. * k2[j] + 4015. / 612. * k3[j] -
                              11. / 36. * k4[j] + 88. / 255. * k5[j]);
  fn(arg, k6);
  for (int j = 0; j < D; j++)
    arg[j] = val[j] + step * (-8263. / 15000. * k1[j] + 124. / 75. * k2[j] - 643. / 680. * k3[j] -
                              81. / 250. * k4[j] + 2484. / 10625. * k5[j]);
  fn(arg, k7);
  for (int j = 0; j < D; j++)
    arg[j] = val[j] + step * (3501. / 1720. * k1[j] - 300. / 43. * k2[j] +
                              297275. / 52632. * k3[j] - 319. / 2322. * k4[j] +
                              24068. / 84065. * k5[j] + 3850. / 26703. * k7[j]);
  fn(arg, k8);
  for (int j = 0; j < D; j++)
    val[j] = val[j] + step * (3. / 40. * k1[j] + 875. / 2244. * k3[j] + 23. / 72. * k4[j] +
                              264. / 1955. * k5[j] + 125. / 11592. * k7[j] + 43. / 616. * k8[j]);
}

// One map iteration, cuda/tools/mapstep.dp.cpp:6-19: val <- fn(val) through
// a scratch copy (StepMAP for the state, StepMAPVAR for a tangent vector).
template <int D, class F> __device__ __forceinline__ void map_step(double *val, const F &fn) {
  double arg[D];
  fn(val, arg);
  for (int j = 0; j < D; j++) val[j] = arg[j];
}

template <int N> __device__ __forceinline__ double dot_seq(const double *a, const double *b) {
  double r = 0;
  for (int i = 0; i < N; i++) r += a[i] * b[i];
  return r;
}

// cuda/tools/linalg.dp.cpp:36-51: classical GS; the projection sum starts at
// zero for every vector (the reference re-zeroes it after each use).
template <int N, int KM>
__device__ __forceinline__ void ort_vecs(double (&v)[KM][N], int k) {
  for (int i = 1; i < KM; i++) {
    if (i >= k) break;
    double proj[N];
    for (int q = 0; q < N; q++) proj[q] = 0;
    for (int j = 0; j < i; j++) {
      double c = dot_seq<N>(v[j], v[i]) / dot_seq<N>(v[j], v[j]);
      for (int q = 0; q < N; q++) proj[q] += c * v[j][q];
    }
    for (int q = 0; q < N; q++) v[i][q] -= proj[q];
  }
}

// cuda/tools/linalg.dp.cpp:20-28
template <int N, int KM>
__device__ __forceinline__ void normalize_vecs(double (&v)[KM][N], int k, double eps) {
  for (int i = 0; i < KM; i++) {
    if (i >= k) break;
    double nr = sqrt(dot_seq<N>(v[i], v[i]));
    for (int q = 0; q < N; q++) v[i][q] = (v[i][q] / nr) * eps;
  }
}

// cuda/lyapunov.dp.cpp:182-225 (map branch): every iteration renormalises
// and adds its log-norms; the loop counters are doubles stepped by 1.
template <class M, int KM>
__device__ void point_var_map(const CompatArgs &a, const double *p, double *x,
                              double (&V)[KM][M::N], double *lyap, int k) {
  constexpr int N = M::N;
  DState<M> fs{p};
  DVar<M> fv{p, x};
  for (double t = 0; t < a.t_skip; t += 1) map_step<N>(x, fs);
  for (int i = 0; i < KM; i++)
    for (int q = 0; q < N; q++) V[i][q] = 0.;
  for (int i = 0; i < KM; i++)
    if (i < k) V[i][i] += a.eps;
  for (double t = 0; t < a.t_skip_clp; t += 1) {
    for (int i = 0; i < KM; i++)
      if (i < k) map_step<N>(V[i], fv);
    map_step<N>(x, fs);
    ort_vecs<N, KM>(V, k);
    normalize_vecs<N, KM>(V, k, a.eps);
  }
  for (double t = 0; t < a.calc_time; t += 1) {
    for (int i = 0; i < KM; i++)
      if (i < k) map_step<N>(V[i], fv);
    map_step<N>(x, fs);
    ort_vecs<N, KM>(V, k);
    for (int i = 0; i < KM; i++)
      if (i < k) lyap[i] += log(sqrt(dot_seq<N>(V[i], V[i])) / a.eps);
    normalize_vecs<N, KM>(V, k, a.eps);
  }
  for (int i = 0; i < KM; i++)
    if (i < k) lyap[i] = lyap[i] / a.calc_time;
}

// cuda/lyapunov.dp.cpp:70-128 (map branch): perturbed copies iterated beside
// the state; the loop counters are int32_t compared with the double times.
template <class M, int KM>
__device__ void point_fd_map(const CompatArgs &a, const double *p, double *x,
                             double (&S)[KM][M::N], double *lyap, int k) {
  constexpr int N = M::N;
  DState<M> fs{p};
  for (int32_t t = 0; t < a.t_skip; t++) map_step<N>(x, fs);
  for (int i = 0; i < KM; i++)
    if (i < k) {
      for (int q = 0; q < N; q++) S[i][q] = x[q];
      S[i][i] += a.eps;
    }
  for (int32_t t = 0; t < a.t_skip_clp; t++) {
    map_step<N>(x, fs);
    for (int i = 0; i < KM; i++)
      if (i < k) {
        map_step<N>(S[i], fs);
        for (int q = 0; q < N; q++) S[i][q] -= x[q];
      }
    ort_vecs<N, KM>(S, k);
    normalize_vecs<N, KM>(S, k, a.eps);
    for (int i = 0; i < KM; i++)
      if (i < k)
        for (int q = 0; q < N; q++) S[i][q] += x[q];
  }
  for (int32_t t = 0; t < a.calc_time; t++) {
    map_step<N>(x, fs);
    for (int i = 0; i < KM; i++)
      if (i < k) map_step<N>(S[i], fs);
    for (int i = 0; i < KM; i++)
      if (i < k)
        for (int q = 0; q < N; q++) S[i][q] -= x[q];
    ort_vecs<N, KM>(S, k);
    for (int i = 0; i < KM; i++)
      if (i < k) lyap[i] += log(sqrt(dot_seq<N>(S[i], S[i])) / a.eps);
    normalize_vecs<N, KM>(S, k, a.eps);
    for (int i = 0; i < KM; i++)
      if (i < k)
        for (int q = 0; q < N; q++) S[i][q] += x[q];
  }
  for (int i = 0; i < KM; i++)
    if (i < k) lyap[i] = lyap[i] / a.calc_time;
}

// cuda/lyapunov.dp.cpp:133-180, 224-225 (flow branch)
template <class M, int KM>
__device__ void point_var(const CompatArgs &a, const double *p, double *x, double (&V)[KM][M::N],
                          double *lyap, int k) {
  constexpr int N = M::N;
  const double h = a.step;
  DState<M> fs{p};
  DVar<M> fv{p, x};
  int32_t skip = 0;
  for (double t = 0; t < a.t_skip; t += h) dverk<N>(x, fs, h);
  for (int i = 0; i < KM; i++)
    for (int q = 0; q < N; q++) V[i][q] = 0.;
  for (int i = 0; i < KM; i++)
    if (i < k) V[i][i] += a.eps;
  for (double t = 0; t < a.t_skip_clp; t += h) {
    for (int i = 0; i < KM; i++)
      if (i < k) dverk<N>(V[i], fv, h);
    dverk<N>(x, fs, h);
    ort_vecs<N, KM>(V, k);
    normalize_vecs<N, KM>(V, k, a.eps);
  }
  for (double t = 0; t < a.calc_time; t += h) {
    skip++;
    for (int i = 0; i < KM; i++)
      if (i < k) dverk<N>(V[i], fv, h);
    dverk<N>(x, fs, h);
    if (skip == a.add_skip) {
      ort_vecs<N, KM>(V, k);
      for (int i = 0; i < KM; i++)
        if (i < k) lyap[i] += log(sqrt(dot_seq<N>(V[i], V[i])) / a.eps);
      normalize_vecs<N, KM>(V, k, a.eps);
      skip = 0;
    }
  }
  for (int i = 0; i < KM; i++)
    if (i < k) lyap[i] = lyap[i] / a.calc_time;
}

// cuda/lyapunov.dp.cpp:5-68, 127-128 (flow branch)
template <class M, int KM>
__device__ void point_fd(const CompatArgs &a, const double *p, double *x, double (&S)[KM][M::N],
                         double *lyap, int k) {
  constexpr int N = M::N;
  const double h = a.step;
  DState<M> fs{p};
  int32_t skip = 0;
  for (double t = 0; t < a.t_skip; t += h) dverk<N>(x, fs, h);
  for (int i = 0; i < KM; i++)
    if (i < k) {
      for (int q = 0; q < N; q++) S[i][q] = x[q];
      S[i][i] += a.eps;
    }
  for (double t = 0; t < a.t_skip_clp; t += h) {
    dverk<N>(x, fs, h);
    for (int i = 0; i < KM; i++)
      if (i < k) {
        dverk<N>(S[i], fs, h);
        for (int q = 0; q < N; q++) S[i][q] -= x[q];
      }
    ort_vecs<N, KM>(S, k);
    normalize_vecs<N, KM>(S, k, a.eps);
    for (int i = 0; i < KM; i++)
      if (i < k)
        for (int q = 0; q < N; q++) S[i][q] += x[q];
  }
  for (double t = 0; t < a.calc_time; t += h) {
    skip++;
    dverk<N>(x, fs, h);
    for (int i = 0; i < KM; i++)
      if (i < k) dverk<N>(S[i], fs, h);
    if (skip == a.add_skip) {
      for (int i = 0; i < KM; i++)
        if (i < k)
          for (int q = 0; q < N; q++) S[i][q] -= x[q];
      ort_vecs<N, KM>(S, k);
      for (int i = 0; i < KM; i++)
        if (i < k) lyap[i] += log(sqrt(dot_seq<N>(S[i], S[i])) / a.eps);
      normalize_vecs<N, KM>(S, k, a.eps);
      for (int i = 0; i < KM; i++)
        if (i < k)
          for (int q = 0; q < N; q++) S[i][q] += x[q];
      skip = 0;
    }
  }
  for (int i = 0; i < KM; i++)
    if (i < k) lyap[i] = lyap[i] / a.calc_time;
}

// cuda/lyapunov.dp.cpp:229-259 with qrDecomposition (linalg.dp.cpp:120-127)
// for square Q (k == n).  Q is kept column by column: column c of J*Q only
// involves column c of Q, so integrating columns separately is the same
// arithmetic as the reference's n*n-component DVERK step.
template <class M>
__device__ void point_qr(const CompatArgs &a, const double *p, double *x, double *lyap) {
  constexpr int N = M::N;
  const double h = a.step;
  DState<M> fs{p};
  DQcol<M> fq{p, x};
  double Qc[N][N];  // Qc[c][r] = Q[r][c]
  for (double t = 0; t < a.t_skip; t += h) dverk<N>(x, fs, h);
  for (int c = 0; c < N; c++)
    for (int r = 0; r < N; r++) Qc[c][r] = (r == c) ? 1. : 0.;
  for (double t = a.t_skip; t < a.t_skip + a.calc_time; t += h) {
    dverk<N>(x, fs, h);
    for (int c = 0; c < N; c++) dverk<N>(Qc[c], fq, h);
    double A[N][N];  // copy of the integrated matrix, column-major like Qc
    for (int c = 0; c < N; c++)
      for (int r = 0; r < N; r++) A[c][r] = Qc[c][r];
    // ortVecsColMaj: classical GS over the columns
    for (int i = 1; i < N; i++) {
      double proj[N];
      for (int r = 0; r < N; r++) proj[r] = 0;
      for (int j = 0; j < i; j++) {
        double c = dot_seq<N>(Qc[j], Qc[i]) / dot_seq<N>(Qc[j], Qc[j]);
        for (int r = 0; r < N; r++) proj[r] += c * Qc[j][r];
      }
      for (int r = 0; r < N; r++) Qc[i][r] -= proj[r];
    }
    // normalizeVecsColMaj(Q, rows, cols, 1)
    for (int i = 0; i < N; i++) {
      double nr = sqrt(dot_seq<N>(Qc[i], Qc[i]));
      for (int r = 0; r < N; r++) Qc[i][r] = (Qc[i][r] / nr) * 1;
    }
    // diagonal of R = Q^T A: R[i][i] = sum_q Q[q][i] A[q][i]
    for (int i = 0; i < N; i++) lyap[i] += log(fabs(dot_seq<N>(Qc[i], A[i])));
  }
  for (int i = 0; i < N; i++) lyap[i] = lyap[i] / a.calc_time;
}

template <class M, int KT>
__global__ void __launch_bounds__(128) compat_kernel(const CompatArgs a) {
  constexpr int N = M::N;
  constexpr int KM = KT > 0 ? KT : N;
  const int64_t pt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pt >= a.P) return;
  const int k = KT > 0 ? KT : a.k;
  double p[M::NP], x[N], lyap[KM];
  for (int i = 0; i < M::NP; i++) p[i] = a.params.base[pt * a.params.ps + i * a.params.cs];
  for (int i = 0; i < N; i++) x[i] = a.inits.base[pt * a.inits.ps + i * a.inits.cs];
  for (int i = 0; i < KM; i++)
    lyap[i] = (a.accumulate && i < k) ? a.lyap.base[pt * a.lyap.ps + i * a.lyap.cs] : 0.;

  double V[KM][N];
  if constexpr (IsMap<M>::value) {  // FD or VAR (the reference's QR has no map branch)
    if (a.method == 1) point_var_map<M, KM>(a, p, x, V, lyap, k);
    else point_fd_map<M, KM>(a, p, x, V, lyap, k);
    if (a.close)
      for (int i = 0; i < KM; i++)
        if (i < k)
          for (int q = 0; q < N; q++) a.close[(pt * k + i) * N + q] = V[i][q];
  } else if (a.method == 2) {
    point_qr<M>(a, p, x, lyap);
  } else {
    if (a.method == 1) point_var<M, KM>(a, p, x, V, lyap, k);
    else point_fd<M, KM>(a, p, x, V, lyap, k);
    if (a.close)
      for (int i = 0; i < KM; i++)
        if (i < k)
          for (int q = 0; q < N; q++) a.close[(pt * k + i) * N + q] = V[i][q];
  }
  bool finite = true;
  for (int i = 0; i < KM; i++)
    if (i < k) {
      a.lyap.base[pt * a.lyap.ps + i * a.lyap.cs] = lyap[i];
      finite = finite && isfinite(lyap[i]);
    }
  for (int i = 0; i < N; i++) a.inits.base[pt * a.inits.ps + i * a.inits.cs] = x[i];
  if (a.status) a.status[pt] = finite ? 0 : 1;
}

template <class M, int KT>
int launch_one(const CompatArgs &a, int block, cudaStream_t s) {
  const int64_t grid = (a.P + block - 1) / block;
  compat_kernel<M, KT><<<(unsigned)grid, block, 0, s>>>(a);
  return (int)cudaGetLastError();
}

template <class M>
int launch_model(const CompatArgs &a, int block, cudaStream_t s) {
  if constexpr (M::N <= 4) {
    switch (a.k) {
      case 1: return launch_one<M, 1>(a, block, s);
      case 2: return launch_one<M, 2>(a, block, s);
      case 3:
        if constexpr (M::N >= 3) return launch_one<M, 3>(a, block, s);
        return kErrUnsupported;
      case 4:
        if constexpr (M::N >= 4) return launch_one<M, 4>(a, block, s);
        return kErrUnsupported;
      default: return kErrUnsupported;
    }
  } else {
    return launch_one<M, 0>(a, block, s);  // runtime k, arrays sized n
  }
}

}  // namespace

int launch_compat(int model, const CompatArgs &a, int block, cudaStream_t s) {
  if (a.P <= 0) return 0;
  if (block <= 0 || block > 128) block = 128;
  switch (model) {
    case kShimizu: return launch_model<Shimizu>(a, block, s);
    case kLorenz: return launch_model<Lorenz>(a, block, s);
    case kRossler: return launch_model<Rossler>(a, block, s);
    case kChua: return launch_model<Chua>(a, block, s);
    case kHyperRossler: return launch_model<HyperRossler>(a, block, s);
    case kLorenz96: return launch_model<Lorenz96>(a, block, s);
    case kHenon: return launch_model<Henon>(a, block, s);
    default: return kErrUnsupported;
  }
}

}  // namespace chaos

// Test infrastructure only: runs the adaptive kernels' per-point integrator
// (chaos_oneapi_b200/csrc/adaptive.cuh: run_point, the host form of the
// lane state machine) for one point on the CPU, so that its algorithm --
// step control, renormalisation-interval policy, Gram-Schmidt, log sums --
// can be checked against the oracle without a GPU.  Built by
// tests/test_host_lane.py with nvcc; never linked into the library.
//
//   lane_driver MODEL PREC INTEG rtol h0 t_transient t_align t_avg dt_renorm p0 p1 [p2 [p3]] -- x0 x1 ...
//   MODEL: rossler | lorenz | chua | hyper_rossler; PREC: fp32 | fp64;
//   INTEG: dopri5 | dverk65, with the suffix "+mgs" for modified Gram-Schmidt
// Prints: status steps lambda_1 ... lambda_n
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../chaos_oneapi_b200/csrc/adaptive.cuh"

using namespace chaos;
using namespace chaos::adaptive;

template <class M, class R, int INTEG>
static int run(AdaptiveArgs &a) {
  run_point<M, M::N, R, INTEG>(a, 0);
  return 0;
}

template <class M>
static int dispatch(AdaptiveArgs &a, bool fp32, bool dopri) {
  if (fp32) return dopri ? run<M, float, kDopri5>(a) : run<M, float, kDverk65>(a);
  return dopri ? run<M, double, kDopri5>(a) : run<M, double, kDverk65>(a);
}

int main(int argc, char **argv) {
  if (argc < 12) return 2;
  const char *model = argv[1];
  const bool fp32 = !std::strcmp(argv[2], "fp32");
  const bool dopri = !std::strncmp(argv[3], "dopri5", 6);
  const bool mgs = std::strstr(argv[3], "+mgs") != nullptr;
  std::vector<double> p, x;
  int i = 10;
  for (; i < argc && std::strcmp(argv[i], "--"); i++) p.push_back(std::atof(argv[i]));
  for (i++; i < argc; i++) x.push_back(std::atof(argv[i]));
  const int n = (int)x.size();
  std::vector<double> spec(n, 0.0);
  int32_t status = -1;
  int64_t steps = 0;
  AdaptiveArgs a{};
  a.P = 1;
  a.k = n;
  a.gs = mgs ? 1 : 0;
  a.rtol = a.atol = std::atof(argv[4]);
  a.h0 = std::atof(argv[5]);
  a.t_transient = std::atof(argv[6]);
  a.t_align = std::atof(argv[7]);
  a.t_avg = std::atof(argv[8]);
  a.dt_renorm = std::atof(argv[9]);
  a.max_steps = 100000000;
  a.escape = 1e4;
  a.params = CView{p.data(), (int64_t)p.size(), 1};
  a.inits = CView{x.data(), n, 1};
  a.spectrum = View{spec.data(), n, 1};
  a.status = &status;
  a.steps = &steps;
  int rc = 2;
  if (!std::strcmp(model, "rossler") && n == 3) rc = dispatch<Rossler>(a, fp32, dopri);
  if (!std::strcmp(model, "lorenz") && n == 3) rc = dispatch<Lorenz>(a, fp32, dopri);
  if (!std::strcmp(model, "chua") && n == 3) rc = dispatch<Chua>(a, fp32, dopri);
  if (!std::strcmp(model, "hyper_rossler") && n == 4) rc = dispatch<HyperRossler>(a, fp32, dopri);
  if (rc) return rc;
  std::printf("%d %lld", status, (long long)steps);
  for (int q = 0; q < n; q++) std::printf(" %.17g", spec[q]);
  std::printf("\n");
  return 0;
}

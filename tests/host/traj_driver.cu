// Test infrastructure only: runs the trajectory kernels' per-point function
// (chaos_oneapi_b200/csrc/trajectory.cuh: run_trajectory, the state under the
// adaptive integrators with the sweep kernels' own step pass and controller)
// for one point on the CPU, so that its step sequence can be checked against
// the reference's dopriStep without a GPU.  Built by the tests with nvcc;
// never linked into the library.
//
//   traj_driver MODEL PREC INTEG rtol h0 hmax nsteps p0 p1 ... -- x0 x1 ...
// Prints: status, then one line per accepted step: t h x_0 .. x_{n-1}
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../chaos_oneapi_b200/csrc/trajectory.cuh"

using namespace chaos;
using namespace chaos::adaptive;

template <class M>
static int dispatch(TrajectoryArgs &ta, bool fp32, bool dopri) {
  if (fp32) dopri ? run_trajectory<M, float, kDopri5>(ta, 0) : run_trajectory<M, float, kDverk65>(ta, 0);
  else dopri ? run_trajectory<M, double, kDopri5>(ta, 0) : run_trajectory<M, double, kDverk65>(ta, 0);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 10) return 2;
  const char *model = argv[1];
  const bool fp32 = !std::strcmp(argv[2], "fp32");
  const bool dopri = !std::strcmp(argv[3], "dopri5");
  std::vector<double> p, x;
  int i = 8;
  for (; i < argc && std::strcmp(argv[i], "--"); i++) p.push_back(std::atof(argv[i]));
  for (i++; i < argc; i++) x.push_back(std::atof(argv[i]));
  const int n = (int)x.size(), nsteps = std::atoi(argv[7]);
  std::vector<double> t(nsteps), h(nsteps), xs((size_t)nsteps * n);
  int32_t status = -1;
  TrajectoryArgs ta{};
  AdaptiveArgs &a = ta.a;
  a.P = 1;
  a.k = n;
  a.rtol = a.atol = std::atof(argv[4]);
  a.h0 = std::atof(argv[5]);
  a.hmax = std::atof(argv[6]);
  a.max_steps = 100000000;
  a.escape = 1e4;
  a.params = CView{p.data(), (int64_t)p.size(), 1};
  a.inits = CView{x.data(), n, 1};
  ta.nsteps = nsteps;
  ta.t_out = t.data();
  ta.h_out = h.data();
  ta.x_out = xs.data();
  ta.status = &status;
  int rc = 2;
  if (!std::strcmp(model, "shimizu") && n == 3) rc = dispatch<Shimizu>(ta, fp32, dopri);
  if (!std::strcmp(model, "lorenz") && n == 3) rc = dispatch<Lorenz>(ta, fp32, dopri);
  if (!std::strcmp(model, "rossler") && n == 3) rc = dispatch<Rossler>(ta, fp32, dopri);
  if (!std::strcmp(model, "chua") && n == 3) rc = dispatch<Chua>(ta, fp32, dopri);
  if (!std::strcmp(model, "hyper_rossler") && n == 4) rc = dispatch<HyperRossler>(ta, fp32, dopri);
  if (rc) return rc;
  std::printf("%d\n", status);
  for (int s = 0; s < nsteps; s++) {
    std::printf("%.17g %.17g", t[s], h[s]);
    for (int j = 0; j < n; j++) std::printf(" %.17g", xs[(size_t)s * n + j]);
    std::printf("\n");
  }
  return 0;
}

// Test infrastructure only: checks, on the CPU, the float forms of the step
// limits and of the phase time that the FP32 steps use
// (chaos_oneapi_b200/csrc/adaptive.cuh: float_ru / float_rd / float_rz,
// step_at_least_hmin, step_above_hmax, time_left_as, make_ctl).  For random
// limits and random float steps near them, the float comparison must give
// the same answer as the double comparison it replaces, and the phase time
// left in float must never exceed the double time left; and a batch's
// launch arguments carry every segment's limits in the batch's precision
// (with_ctl).  Built by tests/test_host_lane.py with nvcc; never linked into
// the library.
//
//   limits_driver SEED N
// Prints "ok CASES" or the first failing case.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <random>

#include "../../chaos_oneapi_b200/csrc/adaptive.cuh"

using namespace chaos;
using namespace chaos::adaptive;

int main(int argc, char **argv) {
  const unsigned seed = argc > 1 ? (unsigned)atoi(argv[1]) : 1u;
  const long n = argc > 2 ? atol(argv[2]) : 100000;
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> expo(-14.0, 3.0), unit(0.5, 1.0);
  long cases = 0;
  for (long i = 0; i < n; i++) {
    // a limit of any magnitude the sweeps see, exactly representable or not
    const double lim = unit(rng) * std::pow(10.0, expo(rng));
    AdaptiveArgs a{};
    a.hmin = lim;
    a.hmax = lim * 1e3;
    a.rtol = a.atol = 1e-6;
    a.dt_renorm = 1.0;
    const Ctl c = make_ctl<float>(a);
    const double hmin = c.hmin, hmax = c.hmax;
    // floats around each limit: the nearest ones on both sides and a spread
    const float probes[] = {(float)hmin, nextafterf((float)hmin, 0.f),
                            nextafterf((float)hmin, INFINITY), (float)(hmin * 0.999999),
                            (float)(hmin * 1.000001), (float)hmax,
                            nextafterf((float)hmax, 0.f), nextafterf((float)hmax, INFINITY),
                            (float)(hmax * 0.9999999), (float)(hmax * 1.0000001)};
    for (float h : probes) {
      ++cases;
      if (step_at_least_hmin(h, c) != ((double)h >= hmin)) {
        printf("hmin %.17g h %.9g: float %d double %d\n", hmin, (double)h,
               (int)step_at_least_hmin(h, c), (int)((double)h >= hmin));
        return 1;
      }
      if (step_above_hmax(h, c) != ((double)h > hmax)) {
        printf("hmax %.17g h %.9g: float %d double %d\n", hmax, (double)h,
               (int)step_above_hmax(h, c), (int)((double)h > hmax));
        return 1;
      }
    }
    // phase time left: never above the exact value, and the nearest float
    // at or below it
    const double t = unit(rng) * std::pow(10.0, expo(rng) + 3.0);
    const float tr = time_left_as<float>(t);
    ++cases;
    if (!((double)tr <= t) || !((double)nextafterf(tr, INFINITY) > t)) {
      printf("t %.17g: float %.9g\n", t, (double)tr);
      return 1;
    }
  }
  // a batch's launch arguments: every segment gets the limits of its own
  // fields in the batch's precision (with_ctl), the others stay untouched
  BatchArgs b{};
  b.nseg = 3;
  for (int i = 0; i < kMaxSegments; i++) {
    b.seg[i].rtol = b.seg[i].atol = 1e-6 * (i + 1);
    b.seg[i].hmin = 1e-9 * (i + 1);
    b.seg[i].hmax = 0.5 * (i + 1);
    b.seg[i].max_steps = 1000 * (i + 1);
    b.seg[i].dt_renorm = 1.0;
  }
  for (int prec : {(int)kFP32, (int)kFP64}) {
    const BatchArgs w = with_ctl(b, prec);
    for (int i = 0; i < kMaxSegments; i++) {
      const Ctl want = i >= b.nseg ? Ctl{} : prec == kFP32 ? make_ctl<float>(b.seg[i])
                                                           : make_ctl<double>(b.seg[i]);
      const Ctl &got = w.seg[i].ctl;
      ++cases;
      if (got.rtol != want.rtol || got.tau != want.tau || got.hmin32 != want.hmin32 ||
          got.hmax32 != want.hmax32 || got.hmin != want.hmin || got.hmax != want.hmax ||
          got.max_steps != want.max_steps || got.escape != want.escape) {
        printf("batch segment %d precision %d: limits not filled\n", i, prec);
        return 1;
      }
    }
  }
  printf("ok %ld\n", cases);
  return 0;
}

// Host-side sweep inputs in the reference's conventions: the parameter grid
// of TaskLyapunov::allocate (tasklyapunov.cpp:45-63) and seeded per-point
// initial states (the reference copies one initial_state to every point,
// tasklyapunov.cpp:67-71; a per-point jitter makes neighbouring points
// independent samples).
#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/chaos_lyap.h"

namespace {

// Philox4x64-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): 10 rounds of two 64x64->128 multiplies with a
// Weyl-sequence key schedule.
void philox4x64(const uint64_t ctr[4], const uint64_t key[2], uint64_t out[4]) {
  uint64_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    const unsigned __int128 p0 = (unsigned __int128)0xD2E7470EE14C6C93ULL * c0;
    const unsigned __int128 p1 = (unsigned __int128)0xCA5A826395121157ULL * c2;
    const uint64_t hi0 = (uint64_t)(p0 >> 64), lo0 = (uint64_t)p0;
    const uint64_t hi1 = (uint64_t)(p1 >> 64), lo1 = (uint64_t)p1;
    c0 = hi1 ^ c1 ^ k0;
    c1 = lo1;
    c2 = hi0 ^ c3 ^ k1;
    c3 = lo0;
    k0 += 0x9E3779B97F4A7C15ULL;
    k1 += 0xBB67AE8584CAA73BULL;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

inline double unit53(uint64_t w) { return (double)(w >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" {

int64_t chaos_lyap_make_grid(int32_t m, const double *base, const double s1[4],
                             const double s2[4], double *out) {
  if (!s1 || !s2 || m <= 0) return -1;
  const int n1 = (int)s1[3], n2 = (int)s2[3];
  if (n1 <= 0 || n2 <= 0) return -1;
  const int64_t P = (int64_t)n1 * n2;
  if (!out) return P;
  if (!base) return -1;
  // A one-point axis has delta 0/0 in the reference; use the start value.
  const double d1 = n1 > 1 ? std::fabs(s1[2] - s1[1]) / (s1[3] - 1) : 0.0;
  const double d2 = n2 > 1 ? std::fabs(s2[2] - s2[1]) / (s2[3] - 1) : 0.0;
  int64_t c = 0;
  for (int a = 0; a < n1; ++a)
    for (int b = 0; b < n2; ++b) {
      const double v1 = s1[1] + a * d1, v2 = s2[1] + b * d2;
      for (int i = 0; i < m; ++i) {
        double v = base[i];
        if (i == (int)s1[0]) v = v1;
        else if (i == (int)s2[0]) v = v2;
        out[c * m + i] = v;
      }
      ++c;
    }
  return P;
}

int chaos_lyap_make_inits(int32_t n, int64_t P, const double *base, double amp, int32_t dist,
                          uint64_t seed, double *out) {
  if (n <= 0 || P < 0 || !base || !out || (dist != 0 && dist != 1)) return CHAOS_LYAP_EINVAL;
  const uint64_t key[2] = {seed, 0x6368616F735F6C79ULL};
  for (int64_t p = 0; p < P; ++p)
    for (int blk = 0; blk * 4 < n; ++blk) {
      const uint64_t ctr[4] = {(uint64_t)p, (uint64_t)blk, 0, 0};
      uint64_t r[4];
      philox4x64(ctr, key, r);
      for (int q = 0; q < 4 && blk * 4 + q < n; ++q) {
        double d;
        if (dist == 0) {
          d = (2.0 * unit53(r[q]) - 1.0) * amp;
        } else {  // Box-Muller on the word pair (r[q & ~1], r[q | 1])
          const double u1 = 1.0 - unit53(r[q & ~1]), u2 = unit53(r[q | 1]);
          const double rad = std::sqrt(-2.0 * std::log(u1));
          const double ang = 6.283185307179586 * u2;
          d = amp * ((q & 1) ? rad * std::sin(ang) : rad * std::cos(ang));
        }
        out[p * n + blk * 4 + q] = base[blk * 4 + q] + d;
      }
    }
  return CHAOS_LYAP_OK;
}

int chaos_lyap_make_inits_at(int32_t n, int64_t count, const int64_t *index, const double *base,
                             double amp, int32_t dist, uint64_t seed, double *out) {
  if (n <= 0 || count < 0 || !index || !base || !out || (dist != 0 && dist != 1))
    return CHAOS_LYAP_EINVAL;
  std::vector<double> one(n);
  for (int64_t i = 0; i < count; ++i) {
    // the point's own counter block, as chaos_lyap_make_inits would draw it
    const int64_t p = index[i];
    const uint64_t key[2] = {seed, 0x6368616F735F6C79ULL};
    for (int blk = 0; blk * 4 < n; ++blk) {
      const uint64_t ctr[4] = {(uint64_t)p, (uint64_t)blk, 0, 0};
      uint64_t r[4];
      philox4x64(ctr, key, r);
      for (int q = 0; q < 4 && blk * 4 + q < n; ++q) {
        double d;
        if (dist == 0) {
          d = (2.0 * unit53(r[q]) - 1.0) * amp;
        } else {
          const double u1 = 1.0 - unit53(r[q & ~1]), u2 = unit53(r[q | 1]);
          const double rad = std::sqrt(-2.0 * std::log(u1));
          const double ang = 6.283185307179586 * u2;
          d = amp * ((q & 1) ? rad * std::sin(ang) : rad * std::cos(ang));
        }
        out[i * n + blk * 4 + q] = base[blk * 4 + q] + d;
      }
    }
  }
  return CHAOS_LYAP_OK;
}

}  // extern "C"

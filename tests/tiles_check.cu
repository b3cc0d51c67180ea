// Host-side checks of the mixed grid kernels' tiling and of their expansion error bound, compiled and
// run by tests/test_tiles_cpu.py (no GPU needed: strip_tiles, strip_point and expansion_rest are
// host functions too).
//   1. Every grid of n1 x n2 <= 140 x 140 points: every point in exactly one tile, each tile's
//      anchor on the grid, |i1 - ca| <= ra <= 9 and |i2 - cb| <= rb <= 8 for every point.
//   2. Random geometries: the exact rest of D_j - D_c after its first two terms, computed in long
//      double from the cancellation-free form (2 g D_c + |Delta|^2)/(D_j + D_c), never exceeds
//      expansion_rest for the tile's reach, while dmax < D_c / 2.
//   3. Trajectory chunks of the launchers (aligned_chunk, used_chunks, splits_for).
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "mixed_tiles.cuh"

using namespace srs::tiles;

static int check_tiles() {
  int bad = 0;
  for (int n1 = 1; n1 <= 140; ++n1)
    for (int n2 = 1; n2 <= 140; ++n2) {
      const StripTiles m = strip_tiles(n1, n2);
      std::vector<int> seen((size_t)n1 * n2, 0);
      for (int t = 0; t < m.tiles; ++t)
        for (int tid = 0; tid < kThreads; ++tid) {
          const TilePoint P = strip_point(m, t, tid);
          if (!P.active) continue;
          if (P.i1 < 0 || P.i1 >= n1 || P.i2 < 0 || P.i2 >= n2 || P.ca < 0 || P.ca >= n1 || P.cb < 0 || P.cb >= n2 ||
              std::abs(P.i1 - P.ca) > P.ra || std::abs(P.i2 - P.cb) > P.rb || P.ra > 9 || P.rb > 8) {
            if (bad < 5) std::printf("tile bound violated: %d x %d tile %d thread %d\n", n1, n2, t, tid);
            ++bad;
            continue;
          }
          seen[(size_t)P.i1 * n2 + P.i2]++;
        }
      for (int v : seen)
        if (v != 1) ++bad;
    }
  return bad;
}

static int check_bound() {
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(-1.0, 1.0), L(0.0, 1.0);
  int bad = 0, tried = 0;
  double worst = 0;
  for (int trial = 0; trial < 20000; ++trial) {
    const double D = std::pow(10.0, 2.0 * L(rng) - 0.5);  // 0.3 m .. 30 m
    double n[3] = {U(rng), U(rng), U(rng)};
    const double nn = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    for (double &c : n) c /= nn;
    double u1[3], u2[3];
    const double s1 = std::pow(10.0, -5.0 + 3.0 * L(rng)), s2 = std::pow(10.0, -5.0 + 3.0 * L(rng));
    for (int c = 0; c < 3; ++c) {
      u1[c] = s1 * U(rng);
      u2[c] = s2 * U(rng);
    }
    const int ra = 1 + (int)(9 * L(rng)), rb = 1 + (int)(8 * L(rng));
    const double m1 = std::sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
    const double m2 = std::sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
    const double nu1 = n[0] * u1[0] + n[1] * u1[1] + n[2] * u1[2], nu2 = n[0] * u2[0] + n[1] * u2[1] + n[2] * u2[2];
    const double dmax = ra * m1 + rb * m2, gmax = ra * std::fabs(nu1) + rb * std::fabs(nu2);
    if (!(dmax < 0.5 * D)) continue;
    ++tried;
    const double bound = expansion_rest(1.0 / D, dmax, gmax);
    for (int da = -ra; da <= ra; ++da)
      for (int db = -rb; db <= rb; ++db) {
        long double d[3], dd = 0, g = 0;
        for (int c = 0; c < 3; ++c) {
          d[c] = (long double)da * u1[c] + (long double)db * u2[c];
          dd += d[c] * d[c];
          g += (long double)n[c] * d[c];
        }
        const long double Dc = D, Dj = std::sqrt(Dc * Dc + 2 * g * Dc + dd);
        const long double exact = (2 * g * Dc + dd) / (Dj + Dc);
        const long double rest = std::fabs(exact - (g + (dd - g * g) / (2 * Dc)));
        // the comparison allows for the long-double rounding of `exact` itself
        const long double tol = 1e-17L * std::fabs(exact);
        if (rest > bound + tol) {
          if (bad < 5)
            std::printf("bound violated: D %g dmax %g gmax %g rest %Lg bound %g\n", D, dmax, gmax, rest, bound);
          ++bad;
        }
        if (bound > 0 && rest / bound > worst) worst = (double)(rest / bound);
      }
  }
  std::printf("bound: %d geometries, worst rest / bound %.3f\n", tried, worst);
  return bad + (tried < 1000);
}

// 3. Trajectory chunking: for every split count the launchers can ask for, whole sub-tiles per chunk,
//    every point in exactly one chunk, no more chunks than asked for; the split model's choice is
//    within its range.
static int check_chunks() {
  int bad = 0;
  for (int64_t n : {1, 2, 127, 128, 129, 2001, 20001, 40001, 100000}) {
    for (int S = 1; S <= 300; ++S) {
      const int64_t chunk = aligned_chunk(n, S);
      const int used = used_chunks(n, chunk);
      if (chunk % kSub != 0 || chunk < kSub || used > S || used < 1 || (int64_t)(used - 1) * chunk >= n ||
          (int64_t)used * chunk < n)
        ++bad;
    }
    for (int64_t ctas : {1, 7, 81, 318, 1024, 100000}) {
      const int s = splits_for(ctas, n, 256, 888);
      if (s < 1 || s > std::max<int64_t>(1, n / 256)) ++bad;
    }
  }
  // the splits measured fastest on a B200: the config-1 map (81 strip tiles, 20001 points, 6 CTAs per
  // SM) in 32 chunks of 640 points, config 2's power density (318 tiles, 40001 points, 5 CTAs per SM)
  // in 16 chunks of 2560
  auto used_for = [](int64_t ctas, int64_t n, int64_t slots) {
    return used_chunks(n, aligned_chunk(n, splits_for(ctas, n, 256, slots)));
  };
  if (used_for(81, 20001, 148 * 6) != 32) {
    std::printf("config-1 split: %d chunks\n", used_for(81, 20001, 148 * 6));
    ++bad;
  }
  if (used_for(318, 40001, 148 * 5) != 16) {
    std::printf("config-2 split: %d chunks\n", used_for(318, 40001, 148 * 5));
    ++bad;
  }
  return bad;
}

int main() {
  const int a = check_tiles(), b = check_bound(), c = check_chunks();
  std::printf("tiles %d bound %d chunks %d\n", a, b, c);
  return a + b + c != 0;
}

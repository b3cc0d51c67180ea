// Device tile bodies of the mixed-precision sums, shared by the one-shot kernels (sums_mixed.cu) and
// the persistent work-queue kernel (queue.cu).  Every function here is executed by all kThreads
// threads of a CTA (it contains __syncthreads) and uses the shared-memory struct it is given.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include "srs_device.cuh"

namespace srs {
namespace tiles {

constexpr int kThreads = 128;
constexpr int kSub = 128;               // trajectory points per shared-memory tile
constexpr int kEnergiesPerThread = 4;

// Trajectory points per chunk for S chunks, rounded up to whole shared-memory sub-tiles: the FP32
// accumulators restart at every sub-tile, so with sub-tile-aligned chunks the result depends on S
// only through the FP64 order of the per-chunk sums.  The chunks actually used are ceil(n / chunk).
inline int64_t aligned_chunk(int64_t n, int S) {
  const int64_t c = (n + S - 1) / std::max(1, S);
  return (c + kSub - 1) / kSub * kSub;
}
inline int used_chunks(int64_t n, int64_t chunk) { return (int)((n + chunk - 1) / chunk); }

// Trajectory chunks S per tile for ctas tiles on a GPU with `slots` resident CTAs per wave, with chunks
// of at least min_chunk points.  Modelled time of a split: waves * (chunk + overhead) for the chunks
// the launch will actually use (aligned_chunk), waves = ceil(ctas * used / slots): a grid that
// overshoots a whole wave by a few CTAs leaves them to run alone at the end, so the model favours
// splits that fill the last wave.  The model does not see how a partly filled last wave drains, nor
// the per-chunk partial sums, so among splits within 2 % of the best: the finest when the best takes
// few waves (< 8: a long last CTA then decides the end), the coarsest otherwise (fewer partials).
// Measured on the config-1 map (81 tiles x 20001 points, 888 slots): 10 chunks 0.308 ms, 16 0.283,
// 20 0.276, 27 0.281, 32 0.269 (picked), 40 0.275; config 2 (318 tiles x 40001 points, 740 slots):
// 16 chunks 3.04 ms (picked), 9 chunks 3.11 ms.
inline int splits_for(int64_t ctas, int64_t n, int64_t min_chunk, int64_t slots) {
  ctas = std::max<int64_t>(1, ctas);
  slots = std::max<int64_t>(1, slots);
  const int64_t max_s = std::min<int64_t>(std::max<int64_t>(1, n / min_chunk), 4096);
  constexpr double kOverhead = 64.0;  // per-CTA set-up and output, in trajectory points
  constexpr double kTol = 0.02;
  auto model = [&](int64_t s, int64_t &used, int64_t &waves) {
    const int64_t chunk = aligned_chunk(n, (int)s);
    used = used_chunks(n, chunk);
    waves = (ctas * used + slots - 1) / slots;
    return (double)waves * ((double)chunk + kOverhead);
  };
  double best = 1e300;
  int64_t best_waves = 1, used = 0, waves = 0;
  for (int64_t s = 1; s <= max_s; ++s) {
    const double c = model(s, used, waves);
    if (c < best) {
      best = c;
      best_waves = waves;
    }
  }
  const bool finest = best_waves < 8;
  int best_s = 1;
  int64_t pick_used = finest ? 0 : INT64_MAX;
  for (int64_t s = 1; s <= max_s; ++s) {
    const double c = model(s, used, waves);
    if (c > best * (1.0 + kTol)) continue;
    if (finest ? used > pick_used : used < pick_used) {
      pick_used = used;
      best_s = (int)s;
    }
  }
  return best_s;
}

// Resident CTAs of `kernel` (kThreads threads, no dynamic shared memory) on the current device,
// queried once per (kernel, device): the launchers ask on every call.
template <typename K>
inline int64_t wave_slots(K kernel) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, int64_t> cache;
  int dev = 0, sms = 148, occ = 1;
  const bool have_dev = cudaGetDevice(&dev) == cudaSuccess;
  const auto key = std::make_pair(reinterpret_cast<const void *>(kernel), dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  if (have_dev) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kThreads, 0) != cudaSuccess || occ < 1) occ = 1;
  const int64_t slots = (int64_t)sms * occ;
  if (have_dev) {
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = slots;
  }
  return slots;
}

// Observation-grid tiles.  The u2 axis is cut into strips of balanced width (8 to 16 points when the
// grid is that wide), the points of a strip are taken row by row (u1 outer), and a CTA covers up to
// kThreads consecutive points of one strip: a compact block of at most 17 rows whose idle lanes are
// those of the last tile of each strip.  (A 101 x 101 map: 84 tiles with 5 % idle lanes, where
// rectangles of 8 x 16 points need 91 tiles with 12 % idle.)
struct StripTiles {
  int n1, n2;
  int wn, nwide;              // strips [0, nwide) are wn + 1 points wide, the others wn
  int per_wide, per_narrow;   // tiles per strip of each width
  int tiles;
};

// Points of one tile of a strip w points wide: kThreads, or 16 rows of a narrower strip.
__host__ __device__ inline int strip_tile_points(int w) { return 16 * w < kThreads ? 16 * w : kThreads; }

// wmax (8..16): the widest strip allowed (a tunable of the job queue; 16 elsewhere).
inline StripTiles strip_tiles(int n1, int n2, int wmax = 16) {
  StripTiles best{};
  wmax = std::min(16, std::max(8, wmax));
  const int lo = std::max(1, (n2 + wmax - 1) / wmax), hi = std::max(lo, n2 / 8);
  for (int ns = lo; ns <= hi; ++ns) {
    StripTiles m{};
    m.n1 = n1;
    m.n2 = n2;
    m.wn = n2 / ns;
    m.nwide = n2 % ns;
    auto per = [&](int w) {
      const int64_t p = strip_tile_points(w);
      return (int)(((int64_t)n1 * w + p - 1) / p);
    };
    m.per_wide = per(m.wn + 1);
    m.per_narrow = per(m.wn);
    m.tiles = m.nwide * m.per_wide + (ns - m.nwide) * m.per_narrow;
    if (ns == lo || m.tiles < best.tiles) best = m;
  }
  return best;
}
inline StripTiles strip_tiles(const srs_grid2d &g, int wmax = 16) { return strip_tiles(g.n1, g.n2, wmax); }

// Thread tid's grid point (i1, i2) in tile `tile`, whether it holds one, the tile's anchor point
// (ca, cb): the middle row of the tile's points and the middle column of its strip, and the largest
// |i1 - ca| and |i2 - cb| over the tile (ra, rb).
struct TilePoint {
  int i1, i2, ca, cb, ra, rb;
  bool active;
};
__host__ __device__ inline TilePoint strip_point(const StripTiles &m, int tile, int tid) {
  const int wide_tiles = m.nwide * m.per_wide;
  int w, c0, t;
  if (tile < wide_tiles) {
    const int s = tile / m.per_wide;
    t = tile - s * m.per_wide;
    w = m.wn + 1;
    c0 = s * w;
  } else {
    const int r = tile - wide_tiles, s = r / m.per_narrow;
    t = r - s * m.per_narrow;
    w = m.wn;
    c0 = m.nwide * (m.wn + 1) + s * w;
  }
  const int pts = strip_tile_points(w);
  const int64_t q0 = (int64_t)t * pts, qn = (int64_t)m.n1 * w;
  const int64_t qend = q0 + pts < qn ? q0 + pts : qn;
  const int64_t q = q0 + tid;
  TilePoint P;
  P.active = tid < pts && q < qend;
  P.i1 = (int)(q / w);
  P.i2 = c0 + (int)(q % w);
  const int r0 = (int)(q0 / w), r1 = (int)((qend - 1) / w);
  P.ca = (r0 + r1) / 2;
  P.cb = c0 + w / 2;
  P.ra = r1 - P.ca > P.ca - r0 ? r1 - P.ca : P.ca - r0;
  P.rb = c0 + w - 1 - P.cb > P.cb - c0 ? c0 + w - 1 - P.cb : P.cb - c0;
  return P;
}

// FP64 anchor common to flux and power density: the tile centre as seen from trajectory point i.
struct Anchor {
  double Dc, invDc;
  double nc[3];
  double dc[3];   // n_c - beta_hat
  double bhat[3];
  double bmag, omb;
};

__device__ inline Anchor make_anchor(const double Oc[3], const double *xp, const double *bp, int64_t n, int64_t i) {
  Anchor a;
  const double rx = Oc[0] - xp[i], ry = Oc[1] - xp[n + i], rz = Oc[2] - xp[2 * n + i];
  const double d2 = rx * rx + ry * ry + rz * rz;
  a.Dc = sqrt(d2);
  a.invDc = 1.0 / a.Dc;
  a.nc[0] = rx * a.invDc; a.nc[1] = ry * a.invDc; a.nc[2] = rz * a.invDc;
  const double bx = bp[i], by = bp[n + i], bz = bp[2 * n + i];
  const double b2 = bx * bx + by * by + bz * bz;
  a.bmag = sqrt(b2);
  const double ib = 1.0 / a.bmag;
  a.bhat[0] = bx * ib; a.bhat[1] = by * ib; a.bhat[2] = bz * ib;
  a.omb = (1.0 - b2) / (1.0 + a.bmag);  // 1 - |beta|, via 1 - |beta|^2 = 1/gamma^2
  for (int c = 0; c < 3; ++c) a.dc[c] = a.nc[c] - a.bhat[c];
  return a;
}

// What the anchor expansion of D_j - D_c leaves out, bounded for one trajectory point at distance
// D_c = 1/invD from a tile whose points lie within dmax of the anchor with |n_c . Delta| <= gmax:
// with h = |Delta|^2 - g^2, D_j - D_c = g + h/(2 D_c) - g h/(2 D_c^2) - h (|Delta|^2 - 5 g^2)/(8 D_c^3)
// + ...; the tiles keep the first two terms.  Returned (in metres): the third-order term's bound plus
// twice the fourth's, which covers the orders after it while dmax < D_c / 2 (checked against the exact
// rest on random geometries by tests/tiles_check.cu); callers treat dmax >= D_c / 2 as out of reach.
__host__ __device__ __forceinline__ double expansion_rest(double invD, double dmax, double gmax) {
  const double d2 = dmax * dmax, i2 = invD * invD;
  return 0.5 * gmax * d2 * i2 + 0.25 * d2 * (d2 + 4.0 * gmax * gmax) * i2 * invD;
}

// Limits of the expansion, per term: the phase error it leaves (radians, systematic), the rounding of
// the FP32 phase (radians: its magnitude in turns times 2^-24), and the relative error of the
// first-order 1/D_j.  A sub-tile that any trajectory point's bound exceeds is summed with exact FP64
// geometry per term instead.
constexpr double kRestPhase = 2e-6, kRoundPhase = 2e-5, kRestAmp = 1e-7;
// The power density's limits: relative errors of (1 - n.beta)^-5 from the expansion's rest and from
// the FP32 rounding of n_c . Delta.
constexpr double kRestPd = 1e-6, kRoundPd = 1e-5;


// Packed FP32x2 arithmetic (sm_100): one instruction performs the same operation on two values, each
// rounded as the scalar operation would be.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// Per trajectory point, 14 FP32 values anchored at the tile's anchor point, stored for PAIRS of
// consecutive points: record g of pair q is (field 2g of point 2q, of point 2q+1, field 2g+1 of 2q,
// of 2q+1), so one 16-byte broadcast load yields two fields of both points, ready for the packed
// instructions.  Signs are chosen so that the inner loop needs no negation.
//   0 phase (turns, mod 1)                        1 k1 (turns per grid step along u1, mod 1)
//   2 k2 (along u2)                               3 -(w/c)/(2 D_c)/2pi (turns per m^2)
//   4-6 n_c                                       7 1/(2 D_c)
//   8 1/D_c                                       9 1/D_c^2
//   10-12 (n_c - bhat) + bhat (1 - |beta|)        13 near-field z term -(c/w) n_cz / D_c^2
constexpr int kFluxFields = 14;
struct FluxShared {
  float4 r[2][kFluxFields / 2][kSub / 2];  // double-buffered: sub-tile k in r[k & 1]
};

// The flux terms of grid point (i1, i2) and trajectory points [base, base + cnt) with the geometry in
// FP64 per term (as the point-list kernel: R, 1/|R| from an FP32 reciprocal square root and two
// Newton steps, the retarded phase in turns reduced exactly, beta - n), the amplitude, sincos and
// sums in FP32; added to E (the field, not its negative).  For sub-tiles the anchor expansion does
// not reach (coarse grids, near distances).
__device__ __forceinline__ void flux_exact_terms(const double *__restrict__ xp, const double *__restrict__ bp,
                                              int64_t n, double dt, const srs_grid2d &g, int i1, int i2,
                                              double omega, int64_t base, int cnt, double E[6]) {
  double Pq[3];
  for (int c = 0; c < 3; ++c) Pq[c] = (g.origin[c] + g.u1[c] * (double)i1) + g.u2[c] * (double)i2;
  const double wt = omega * 0.15915494309189535, inv_c = 1.0 / kC;
  const float kap = (float)(-kC / omega), two_pi_f = 6.28318530717958647692f;
  float e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
  for (int k = 0; k < cnt; ++k) {
    const int64_t i = base + k;
    const double Rx = Pq[0] - __ldg(xp + i), Ry = Pq[1] - __ldg(xp + n + i), Rz = Pq[2] - __ldg(xp + 2 * n + i);
    const double R2 = fma(Rx, Rx, fma(Ry, Ry, Rz * Rz));
    const float yf = rsqrtf((float)R2);
    double y = (double)yf;
    double r = fma(-R2 * y, y, 1.0);
    y = fma(0.5 * y, r, y);
    r = fma(-R2 * y, y, 1.0);
    y = fma(0.5 * y, r, y);  // 1/|R| to FP64 accuracy
    const double ph = wt * fma(R2 * y, inv_c, dt * (double)i);
    const float fr = (float)(ph - rint(ph));
    const double nz = Rz * y;
    const float ax = (float)(__ldg(bp + i) - Rx * y) * yf, ay = (float)(__ldg(bp + n + i) - Ry * y) * yf,
                az = (float)(__ldg(bp + 2 * n + i) - nz) * yf;  // (beta - n)/D
    const float cz = kap * (float)nz * (yf * yf);              // near field: i kap n_z / D^2
    float sn, cs;
    __sincosf(fr * two_pi_f, &sn, &cs);
    e0 = fmaf(ax, cs, e0); e1 = fmaf(ax, sn, e1);
    e2 = fmaf(ay, cs, e2); e3 = fmaf(ay, sn, e3);
    e4 = fmaf(az, cs, fmaf(-cz, sn, e4)); e5 = fmaf(az, sn, fmaf(cz, cs, e5));
  }
  E[0] += e0; E[1] += e1; E[2] += e2; E[3] += e3; E[4] += e4; E[5] += e5;
}

// Flux: one strip tile (tile index `tile` of map m) against trajectory points [i0, iend); writes the six
// partial sums (Re/Im of E_x, E_y, E_z without the final constant) of every point of the tile to
// out6[c * np + j].
__device__ __forceinline__ void flux_tile(const double *__restrict__ xp, const double *__restrict__ bp, int64_t n,
                                          double dt, const srs_grid2d &g, const StripTiles &m, double omega,
                                          int tile, int64_t i0, int64_t iend, double *__restrict__ out6,
                                          FluxShared &sh) {
  // Expansion about the anchor point O_c (distance D_c, direction n_c from trajectory point i) for
  // the grid point O_c + Delta: with g = n_c . Delta and h = |Delta|^2 - g^2,
  //   D_j - D_c = g + h/(2 D_c)  (the third-order term g h/(2 D_c^2), < 1e-7 rad here, is dropped),
  //   1/D_j = (1/D_c)(1 - (D_j - D_c)/D_c)  (relative error ((D_j - D_c)/D_c)^2 < 1e-16),
  //   phase = w tau_c + k1 da + k2 db + (w/c) h/(2 D_c),
  // and the near-field term keeps its z part (its x, y parts are lambda/(2 pi D) times n_perp, < 1e-10
  // at 30 m).  Phases are kept in turns: the per-point phases and the grid-step phases k1, k2 are
  // reduced in FP64, and the FP32 phase of a tile point is reduced exactly (x - rint(x), rint by the
  // 1.5 * 2^23 shift, exact for |x| < 2^22 turns) before __sincosf.
  const int tid = threadIdx.x;
  const TilePoint P = strip_point(m, tile, tid);
  const bool active = P.active;
  const int da = P.i1 - P.ca, db = P.i2 - P.cb;
  const double wc = omega / kC;
  // the tile's reach from its anchor (a bound on |Delta|)
  const double dmax = P.ra * sqrt(g.u1[0] * g.u1[0] + g.u1[1] * g.u1[1] + g.u1[2] * g.u1[2]) +
                      P.rb * sqrt(g.u2[0] * g.u2[0] + g.u2[1] * g.u2[1] + g.u2[2] * g.u2[2]);
  double E[6] = {0, 0, 0, 0, 0, 0};

  // the records of trajectory points [base, base + kSub) into buffer b; returns whether this thread's
  // point needs the exact sum (the expansion's limits exceeded)
  auto fill = [&](int b, int64_t base) -> int {
    int bad = 0;
    float *rec = &sh.r[b][0][0].x;
    auto put = [&](int t, int f, float v) { rec[((f >> 1) * (kSub / 2) + (t >> 1)) * 4 + (f & 1) * 2 + (t & 1)] = v; };
    const int cnt = (int)imin64(kSub, iend - base);
    if (tid < cnt) {
      const int64_t i = base + tid;
      double Oc[3];
      for (int c = 0; c < 3; ++c) Oc[c] = g.origin[c] + (double)P.ca * g.u1[c] + (double)P.cb * g.u2[c];
      const Anchor A = make_anchor(Oc, xp, bp, n, i);
      const double tau = dt * (double)i + A.Dc / kC;
      const double inv2pi = 0.15915494309189535;  // 1/(2 pi)
      const double nu1 = A.nc[0] * g.u1[0] + A.nc[1] * g.u1[1] + A.nc[2] * g.u1[2];
      const double nu2 = A.nc[0] * g.u2[0] + A.nc[1] * g.u2[1] + A.nc[2] * g.u2[2];
      put(tid, 0, (float)(reduce_2pi(omega * tau) * inv2pi));
      put(tid, 1, (float)(reduce_2pi(wc * nu1) * inv2pi));
      put(tid, 2, (float)(reduce_2pi(wc * nu2) * inv2pi));
      {
        const double gmax = P.ra * fabs(nu1) + P.rb * fabs(nu2);
        const double curv = 0.5 * dmax * dmax * A.invDc;  // |h|/(2 D_c) <= this, metres
        const double turns = (wc * curv) * inv2pi + 0.5 * (1 + P.ra + P.rb);
        const double ramp = (gmax + curv) * A.invDc;       // |D_j - D_c| / D_c
        bad = dmax * A.invDc >= 0.5 || wc * expansion_rest(A.invDc, dmax, gmax) > kRestPhase ||
              turns * (6.283185307179586 * 0x1p-24) > kRoundPhase || ramp * ramp > kRestAmp;
      }
      put(tid, 3, (float)(-wc * 0.5 * A.invDc * inv2pi));
      put(tid, 4, (float)A.nc[0]);
      put(tid, 5, (float)A.nc[1]);
      put(tid, 6, (float)A.nc[2]);
      put(tid, 7, (float)(0.5 * A.invDc));
      put(tid, 8, (float)A.invDc);
      put(tid, 9, (float)(A.invDc * A.invDc));
      put(tid, 10, (float)(A.dc[0] + A.bhat[0] * A.omb));
      put(tid, 11, (float)(A.dc[1] + A.bhat[1] * A.omb));
      put(tid, 12, (float)(A.dc[2] + A.bhat[2] * A.omb));
      put(tid, 13, (float)(-(kC / omega) * A.invDc * A.invDc * A.nc[2]));
    } else if (tid == cnt && (cnt & 1)) {
      // the odd count's partner slot: all zero, so 1/D_j = 0 and its amplitude and near-field term vanish
      for (int f = 0; f < kFluxFields; ++f) put(tid, f, 0.0f);
    }
    return bad;
  };

  __syncthreads();  // the caller's previous use of sh is over
  int bad_cur = i0 < iend ? fill(0, i0) : 0;
  int b = 0;
  for (int64_t base = i0; base < iend; base += kSub, b ^= 1) {
    const int cnt = (int)imin64(kSub, iend - base);
    // records of this sub-tile complete; every thread is done with the other buffer
    const int exact = __syncthreads_or(bad_cur);
    bad_cur = base + kSub < iend ? fill(b ^ 1, base + kSub) : 0;
    if (!active) continue;
    if (exact) {
      flux_exact_terms(xp, bp, n, dt, g, P.i1, P.i2, omega, base, cnt, E);
      continue;
    }
    // this thread's offset from the anchor point (formed here, after the FP64 anchors, so that it does
    // not occupy registers while they are computed)
    float Dl[3];
    for (int c = 0; c < 3; ++c) Dl[c] = (float)((double)da * g.u1[c] + (double)db * g.u2[c]);
    const float2 Dx = f2(Dl[0], Dl[0]), Dy = f2(Dl[1], Dl[1]), Dz = f2(Dl[2], Dl[2]);
    const float2 Dxn = f2(-Dl[0], -Dl[0]), Dyn = f2(-Dl[1], -Dl[1]), Dzn = f2(-Dl[2], -Dl[2]);
    const float ddv = -(Dl[0] * Dl[0] + Dl[1] * Dl[1] + Dl[2] * Dl[2]);
    const float2 ddn = f2(ddv, ddv), fda = f2((float)da, (float)da), fdb = f2((float)db, (float)db);
    const float2 shift = f2(12582912.0f, 12582912.0f), nshift = f2(-12582912.0f, -12582912.0f),
                 mone = f2(-1.0f, -1.0f), two_pi = f2(6.28318530717958647692f, 6.28318530717958647692f);
    // The accumulators collect minus the field: the sum over points of amp (cos, sin) with amp =
    // ((n_c - bhat + bhat omb) + (Delta - n_c del)/D_j)/D_j, and for z of (amp - i nf)(cos + i sin).
    float2 acc[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[c] = f2(0.f, 0.f);
    const int pairs = (cnt + 1) >> 1;
    const float4(*r)[kSub / 2] = sh.r[b];
#pragma unroll 2
    for (int q = 0; q < pairs; ++q) {
      const float4 R0 = r[0][q], R1 = r[1][q], R2 = r[2][q], R3 = r[3][q], R4 = r[4][q], R5 = r[5][q],
                   R6 = r[6][q];
      const float2 ph0 = f2(R0.x, R0.y), k1 = f2(R0.z, R0.w), k2 = f2(R1.x, R1.y), qcn = f2(R1.z, R1.w);
      const float2 nx = f2(R2.x, R2.y), ny = f2(R2.z, R2.w), nz = f2(R3.x, R3.y), hinv = f2(R3.z, R3.w);
      const float2 w = f2(R4.x, R4.y), w2 = f2(R4.z, R4.w), bx = f2(R5.x, R5.y), by = f2(R5.z, R5.w);
      const float2 bz = f2(R6.x, R6.y), nf = f2(R6.z, R6.w);
      const float2 gqn = fma2(nz, Dzn, fma2(ny, Dyn, mul2(nx, Dxn)));  // -g
      const float2 hn = fma2(gqn, gqn, ddn);                          // -h
      const float2 deln = fma2(hn, hinv, gqn);                        // D_c - D_j
      const float2 rinv = fma2(deln, w2, w);                          // 1/D_j
      float2 ph = fma2(k1, fda, ph0);
      ph = fma2(k2, fdb, ph);
      ph = fma2(hn, qcn, ph);                                         // turns
      const float2 rn = add2(add2(ph, shift), nshift);                 // rint(ph)
      const float2 x = mul2(fma2(rn, mone, ph), two_pi);              // rad, in [-pi, pi]
      float2 sn, cs;
      __sincosf(x.x, &sn.x, &cs.x);
      __sincosf(x.y, &sn.y, &cs.y);
      const float2 ax = mul2(fma2(fma2(nx, deln, Dx), rinv, bx), rinv);
      const float2 ay = mul2(fma2(fma2(ny, deln, Dy), rinv, by), rinv);
      const float2 az = mul2(fma2(fma2(nz, deln, Dz), rinv, bz), rinv);
      acc[0] = fma2(ax, cs, acc[0]);
      acc[1] = fma2(ax, sn, acc[1]);
      acc[2] = fma2(ay, cs, acc[2]);
      acc[3] = fma2(ay, sn, acc[3]);
      acc[4] = fma2(az, cs, fma2(nf, sn, acc[4]));
      acc[5] = fma2(az, sn, fma2(neg2(nf), cs, acc[5]));
    }
#pragma unroll
    for (int c = 0; c < 6; ++c) E[c] -= (double)acc[c].x + (double)acc[c].y;
  }
  if (active) {
    const int64_t np = (int64_t)g.n1 * g.n2;
    double *o = out6 + (int64_t)P.i1 * g.n2 + P.i2;
#pragma unroll
    for (int c = 0; c < 6; ++c) o[c * np] = E[c];
  }
}

// ---- flux at an arbitrary list of observation points ----
//
// No grid to anchor on, so the geometry is FP64 per (point, trajectory point): R, |R| (an FP32
// reciprocal square root refined by two Newton steps to FP64 accuracy), the retarded time and the
// phase in turns reduced exactly (x - rint(x)), n and beta - n; the amplitude, sincos and accumulation
// are FP32 as in the grid tiles.  The near-field term keeps its z part only (its x, y parts are
// ~lambda/(2 pi D) of the amplitude, < 1e-10 at 30 m).
struct PointsShared {
  double x[3][kSub];
  double t[kSub];
  double b[3][kSub];
};

// One tile of kThreads observation points (points[3 j .. 3 j + 2], j = tile * kThreads + thread)
// against trajectory points [i0, iend); writes the six partial sums of every point to out6[c * np + j].
__device__ __forceinline__ void points_flux_tile(const double *__restrict__ xp, const double *__restrict__ bp,
                                                 int64_t n, double dt, const double *__restrict__ points, int64_t np,
                                                 double omega, int tile, int64_t i0, int64_t iend,
                                                 double *__restrict__ out6, PointsShared &sh) {
  const int tid = threadIdx.x;
  const int64_t j = (int64_t)tile * kThreads + tid;
  const bool active = j < np;
  const int64_t jj = active ? j : np - 1;
  const double Px = points[3 * jj], Py = points[3 * jj + 1], Pz = points[3 * jj + 2];
  const double wt = omega * 0.15915494309189535;  // turns per second
  const double inv_c = 1.0 / kC;
  const float kap = (float)(-kC / omega);
  const float two_pi_f = 6.28318530717958647692f;
  double E[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t base = i0; base < iend; base += kSub) {
    const int cnt = (int)imin64(kSub, iend - base);
    __syncthreads();
    if (tid < cnt) {
      const int64_t i = base + tid;
      sh.x[0][tid] = xp[i];
      sh.x[1][tid] = xp[n + i];
      sh.x[2][tid] = xp[2 * n + i];
      sh.t[tid] = dt * (double)i;
      sh.b[0][tid] = bp[i];
      sh.b[1][tid] = bp[n + i];
      sh.b[2][tid] = bp[2 * n + i];
    }
    __syncthreads();
    if (!active) continue;
    float e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
#pragma unroll 2
    for (int k = 0; k < cnt; ++k) {
      const double Rx = Px - sh.x[0][k], Ry = Py - sh.x[1][k], Rz = Pz - sh.x[2][k];
      const double R2 = fma(Rx, Rx, fma(Ry, Ry, Rz * Rz));
      const float yf = rsqrtf((float)R2);
      double y = (double)yf;
      double r = fma(-R2 * y, y, 1.0);
      y = fma(0.5 * y, r, y);
      r = fma(-R2 * y, y, 1.0);
      y = fma(0.5 * y, r, y);  // 1/|R| to FP64 accuracy
      const double D = R2 * y;
      const double ph = wt * fma(D, inv_c, sh.t[k]);
      const float fr = (float)(ph - rint(ph));
      const double nz = Rz * y;
      const float dx = (float)(sh.b[0][k] - Rx * y), dy = (float)(sh.b[1][k] - Ry * y), dz = (float)(sh.b[2][k] - nz);
      const float ax = dx * yf, ay = dy * yf, az = dz * yf;  // (beta - n)/D
      const float cz = kap * (float)nz * (yf * yf);          // near field: i kap n_z / D^2
      float sn, cs;
      __sincosf(fr * two_pi_f, &sn, &cs);
      e0 = fmaf(ax, cs, e0); e1 = fmaf(ax, sn, e1);
      e2 = fmaf(ay, cs, e2); e3 = fmaf(ay, sn, e3);
      e4 = fmaf(az, cs, fmaf(-cz, sn, e4)); e5 = fmaf(az, sn, fmaf(cz, cs, e5));
    }
    E[0] += e0; E[1] += e1; E[2] += e2; E[3] += e3; E[4] += e4; E[5] += e5;
  }
  if (active) {
    double *o = out6 + j;
#pragma unroll
    for (int c = 0; c < 6; ++c) o[c * np] = E[c];
  }
}

// Per trajectory point of a spectrum sub-tile, FP32 records whose signs are chosen so that the inner
// loops need no negation (a = (beta - n)/D, b = n/D^2; rot = exp(i dw tau), rot2 = exp(2 i dw tau)):
//   p0 = (a_x, a_y, a_z, b_z)     p1 = (-a_x, -a_y, -a_z, -Im rot)
//   p2 = (rot, rot2) as (re, im, re, im)     p3 = (-Im rot2, b_x, b_y, 0)
struct SpecShared {
  double tau[kSub];
  float4 p0[kSub], p1[kSub], p2[kSub], p3[kSub];
  float red[2][kThreads / 32];  // per-warp sums of the near-field bound of the current sub-tile
  float wmin[kThreads / 32];    // per-warp smallest angular frequency of the tile's energies
  // each thread's FP64 sums of its energies, [energy q * 6 + component][thread]: in shared memory rather
  // than registers (48 of them at four energies), so that more CTAs fit an SM
  double e[kEnergiesPerThread * 6][kThreads];
};

// The x and y near-field terms i kap b_perp of a sub-tile are left out when their sum can reach at most
// kNearPerp times the sub-tile's sum of |a| (kap = -c/w, |kap| largest at the tile's lowest energy).
// Over a trajectory the terms left out then add up to at most kNearPerp * sum |a|, below the FP32
// rounding of the sums themselves (~2^-24 sum |a| / sqrt(points) for random rounding, and the output
// |E| is a fraction of sum |a|).  At 30 m the ratio is ~1e-14 inside an undulator and lambda/(2 pi D)
// ~ 1e-11 in the drifts; observers a few metres away at low energies keep them.
constexpr float kNearPerp = 1e-10f;

// x modulo 2 pi for the spectrum's per-(point, thread) phase: the Cody-Waite steps of reduce_2pi
// without its third part, whose product k * P3 is below |x| * 1e-33 rad (1e-18 rad for |x| < 1e15
// rad, while the FP64 phase w tau itself carries |x| * 1.1e-16), so the result equals reduce_2pi's to
// within an ulp of pi.
__device__ __forceinline__ double reduce_2pi_short(double x) {
  const double kInv2Pi = 0.15915494309189535;
  const double P1 = 6.283185307179586, P2 = 2.4492935982947064e-16;
  const double k = rint(x * kInv2Pi);
  return __fma_rn(-k, P2, __fma_rn(-k, P1, x));
}

// Each thread owns K consecutive energies (kEnergiesPerThread, or 2 for spectra too small to fill
// the GPU otherwise).  On a uniform energy grid the phasors exp(i w_k tau) of a thread's energies are
// one reduced sincos per (trajectory point, thread) walked by the rotations exp(i dw tau) and
// exp(2 i dw tau) (dw = (w_last - w_first)/(ne - 1), formed in FP64 once per trajectory point per
// CTA): the walk is re-anchored every K energies.  A thread whose energies are not on that grid
// (|w_k - (w_0 + k dw)| * tau_max > 1e-3 rad) takes one reduced sincos per (point, energy) instead.
// No host synchronisation is needed to decide.  K = 4 is the measured optimum of the walk length: the
// kernel is bound by the FMA pipe, and every energy walked costs a complex multiply on it, while the
// sincos it replaces runs on the XU and FP64 pipes.
// One tile: energies of tile `etile` (kThreads * K of them, K per thread) against trajectory points
// [i0, iend); writes the six partial sums of every energy to out6[c * ne + k].
template <int K>
__device__ __forceinline__ void spectrum_tile(const double *__restrict__ xp, const double *__restrict__ bp,
                                              int64_t n, double dt, V3 obs, const double *__restrict__ omegas,
                                              int64_t ne, int etile, int64_t i0, int64_t iend,
                                              double *__restrict__ out6, SpecShared &sh) {
  static_assert(K == 2 || K == 4, "energies per thread: 2 or 4");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t k0 = ((int64_t)etile * kThreads + tid) * K;
  const bool active = k0 < ne;
  const double wfirst = omegas[0];
  const double dw = ne > 1 ? (omegas[ne - 1] - wfirst) / (double)(ne - 1) : 0.0;
  float kap[K];  // -c/w_k: the near-field term is i*kap*n/D^2
  double wkn[K];  // -w_k: sincos of the negated phase gives (cos, -sin) directly
  bool uniform = ne > 1;
  float wmin = 3.0e38f;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const int64_t k = imin64(k0 + q, ne - 1);
    const double w = omegas[k];
    wkn[q] = -w;
    kap[q] = (float)(-kC / w);
    const double dev = fabs(w - (wfirst + (double)k * dw));
    if (k0 + q < ne) {
      if (dev * (1e3 / kC) >= 1e-3) uniform = false;  // observers within 1 km
      wmin = fminf(wmin, (float)w);
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) wmin = fminf(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
  float2 kap2[K / 2];
#pragma unroll
  for (int pq = 0; pq < K / 2; ++pq) kap2[pq] = f2(kap[2 * pq], kap[2 * pq + 1]);
  double(*E)[kThreads] = sh.e;  // E[q * 6 + c][tid]: only this thread's column
#pragma unroll
  for (int q = 0; q < K * 6; ++q) E[q][tid] = 0;

  // whether every energy of the CTA is on the uniform grid: the fast loop below then has no branch
  const bool all_uniform = __syncthreads_and(uniform || !active);
  for (int64_t base = i0; base < iend; base += kSub) {
    const int cnt = (int)imin64(kSub, iend - base);
    __syncthreads();  // every thread is done with the previous sub-tile's records and sums
    float bsum = 0.f, asum = 0.f;
    if (tid < cnt) {
      const int64_t i = base + tid;
      const double rx = obs.x - xp[i], ry = obs.y - xp[n + i], rz = obs.z - xp[2 * n + i];
      const double D = sqrt(rx * rx + ry * ry + rz * rz), iD = 1.0 / D;
      const double nx = rx * iD, ny = ry * iD, nz = rz * iD;
      const double tau = dt * (double)i + D / kC;
      sh.tau[tid] = tau;
      const float ax = (float)((bp[i] - nx) * iD), ay = (float)((bp[n + i] - ny) * iD),
                  az = (float)((bp[2 * n + i] - nz) * iD);
      const double iD2 = iD * iD;
      const float bx = (float)(nx * iD2), by = (float)(ny * iD2), bz = (float)(nz * iD2);
      double sr, cr;
      sincos(reduce_2pi(dw * tau), &sr, &cr);
      const float rr = (float)cr, ri = (float)sr;
      // the rotation by two energy steps, squared in FP64
      const float r2r = K > 2 ? (float)((cr - sr) * (cr + sr)) : 0.f, r2i = K > 2 ? (float)(2.0 * cr * sr) : 0.f;
      sh.p0[tid] = make_float4(ax, ay, az, bz);
      sh.p1[tid] = make_float4(-ax, -ay, -az, -ri);
      sh.p2[tid] = make_float4(rr, ri, r2r, r2i);
      sh.p3[tid] = make_float4(-r2i, bx, by, 0.f);
      bsum = fabsf(bx) + fabsf(by);                          // >= |b_perp|
      asum = fmaxf(fabsf(ax), fmaxf(fabsf(ay), fabsf(az)));  // <= |a|
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      bsum += __shfl_xor_sync(0xffffffffu, bsum, o);
      asum += __shfl_xor_sync(0xffffffffu, asum, o);
    }
    if (lane == 0) {
      sh.red[0][warp] = bsum;
      sh.red[1][warp] = asum;
      sh.wmin[warp] = wmin;
    }
    __syncthreads();
    if (!active) continue;
    float Bs = 0.f, As = 0.f, wm = 3.0e38f;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      Bs += sh.red[0][w];
      As += sh.red[1][w];
      wm = fminf(wm, sh.wmin[w]);
    }
    // the same decision in every thread of the CTA: the same values added in the same order
    const bool perp_near = (float)kC / wm * Bs > kNearPerp * As;
    // accumulators packed by energy pairs (q, q+1): acc[p][c] = (e[2p][c], e[2p+1][c]), components
    // (Re, Im) of E_x, E_y, E_z
    float2 acc[K / 2][6];
#pragma unroll
    for (int pq = 0; pq < K / 2; ++pq)
#pragma unroll
      for (int c = 0; c < 6; ++c) acc[pq][c] = f2(0.f, 0.f);

    // z = exp(i w_q tau) as (zr, zin = -Im z) per energy pair
    auto phasors = [&](double tau, const float4 &P1, const float4 &P2, const float4 &P3, float2 *zr, float2 *zin,
                       bool uni) {
      float z0r, z0n;
      __sincosf((float)reduce_2pi_short(wkn[0] * tau), &z0n, &z0r);
      if (uni) {
        const float rr = P2.x, ri = P2.y, rin = P1.w;
        const float z1r = fmaf(z0n, ri, z0r * rr), z1n = fmaf(z0r, rin, z0n * rr);
        zr[0] = f2(z0r, z1r);
        zin[0] = f2(z0n, z1n);
        const float2 R2r = f2(P2.z, P2.z), R2i = f2(P2.w, P2.w), R2in = f2(P3.x, P3.x);
#pragma unroll
        for (int pq = 1; pq < K / 2; ++pq) {
          zr[pq] = fma2(zin[pq - 1], R2i, mul2(zr[pq - 1], R2r));
          zin[pq] = fma2(zr[pq - 1], R2in, mul2(zin[pq - 1], R2r));
        }
      } else {
        float cr[K], cn[K];
        cr[0] = z0r;
        cn[0] = z0n;
#pragma unroll
        for (int q = 1; q < K; ++q) __sincosf((float)reduce_2pi_short(wkn[q] * tau), &cn[q], &cr[q]);
#pragma unroll
        for (int pq = 0; pq < K / 2; ++pq) {
          zr[pq] = f2(cr[2 * pq], cr[2 * pq + 1]);
          zin[pq] = f2(cn[2 * pq], cn[2 * pq + 1]);
        }
      }
    };

    if (all_uniform && !perp_near) {
      // uniform grid, E_x and E_y without their near-field terms; E_z's near-field term summed apart,
      // sum b_z z, and multiplied by i kap once per sub-tile
      float2 nzr[K / 2], nzn[K / 2];  // sum b_z Re z, sum b_z (-Im z)
#pragma unroll
      for (int pq = 0; pq < K / 2; ++pq) nzr[pq] = nzn[pq] = f2(0.f, 0.f);
#pragma unroll 4
      for (int k = 0; k < cnt; ++k) {
        const double tau = sh.tau[k];
        const float4 P0 = sh.p0[k], P1 = sh.p1[k], P2 = sh.p2[k], P3 = sh.p3[k];
        float2 zr[K / 2], zin[K / 2];
        phasors(tau, P1, P2, P3, zr, zin, true);
        const float2 Ax = f2(P0.x, P0.x), Ay = f2(P0.y, P0.y), Az = f2(P0.z, P0.z), Bz = f2(P0.w, P0.w);
        const float2 Axn = f2(P1.x, P1.x), Ayn = f2(P1.y, P1.y), Azn = f2(P1.z, P1.z);
#pragma unroll
        for (int pq = 0; pq < K / 2; ++pq) {
          acc[pq][0] = fma2(Ax, zr[pq], acc[pq][0]);
          acc[pq][1] = fma2(Axn, zin[pq], acc[pq][1]);
          acc[pq][2] = fma2(Ay, zr[pq], acc[pq][2]);
          acc[pq][3] = fma2(Ayn, zin[pq], acc[pq][3]);
          acc[pq][4] = fma2(Az, zr[pq], acc[pq][4]);
          acc[pq][5] = fma2(Azn, zin[pq], acc[pq][5]);
          nzr[pq] = fma2(Bz, zr[pq], nzr[pq]);
          nzn[pq] = fma2(Bz, zin[pq], nzn[pq]);
        }
      }
      // E_z += i kap sum b_z z: Re += kap sum b_z (-Im z), Im += kap sum b_z Re z
#pragma unroll
      for (int pq = 0; pq < K / 2; ++pq) {
        acc[pq][4] = fma2(kap2[pq], nzn[pq], acc[pq][4]);
        acc[pq][5] = fma2(kap2[pq], nzr[pq], acc[pq][5]);
      }
    } else {
      // any energy grid, every component with its near-field term: e += (a + i kap b) z
#pragma unroll 2
      for (int k = 0; k < cnt; ++k) {
        const double tau = sh.tau[k];
        const float4 P0 = sh.p0[k], P1 = sh.p1[k], P2 = sh.p2[k], P3 = sh.p3[k];
        float2 zr[K / 2], zin[K / 2];
        phasors(tau, P1, P2, P3, zr, zin, uniform);
        const float2 Ax = f2(P0.x, P0.x), Ay = f2(P0.y, P0.y), Az = f2(P0.z, P0.z);
        const float2 Axn = f2(P1.x, P1.x), Ayn = f2(P1.y, P1.y), Azn = f2(P1.z, P1.z);
        const float2 Bx = f2(P3.y, P3.y), By = f2(P3.z, P3.z), Bz = f2(P0.w, P0.w);
#pragma unroll
        for (int pq = 0; pq < K / 2; ++pq) {
          const float2 cx = mul2(kap2[pq], Bx), cy = mul2(kap2[pq], By), cz = mul2(kap2[pq], Bz);
          acc[pq][0] = fma2(Ax, zr[pq], fma2(cx, zin[pq], acc[pq][0]));
          acc[pq][1] = fma2(Axn, zin[pq], fma2(cx, zr[pq], acc[pq][1]));
          acc[pq][2] = fma2(Ay, zr[pq], fma2(cy, zin[pq], acc[pq][2]));
          acc[pq][3] = fma2(Ayn, zin[pq], fma2(cy, zr[pq], acc[pq][3]));
          acc[pq][4] = fma2(Az, zr[pq], fma2(cz, zin[pq], acc[pq][4]));
          acc[pq][5] = fma2(Azn, zin[pq], fma2(cz, zr[pq], acc[pq][5]));
        }
      }
    }
#pragma unroll
    for (int pq = 0; pq < K / 2; ++pq)
#pragma unroll
      for (int c = 0; c < 6; ++c) {
        E[(2 * pq) * 6 + c][tid] += (double)acc[pq][c].x;
        E[(2 * pq + 1) * 6 + c][tid] += (double)acc[pq][c].y;
      }
  }
  if (active) {
#pragma unroll
    for (int q = 0; q < K; ++q) {
      const int64_t k = k0 + q;
      if (k >= ne) break;
      double *o = out6 + k;
#pragma unroll
      for (int c = 0; c < 6; ++c) o[c * ne] = E[q * 6 + c][tid];
    }
  }
}


}  // namespace tiles
}  // namespace srs

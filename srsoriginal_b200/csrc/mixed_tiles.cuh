// Device tile bodies of the mixed-precision sums, shared by the one-shot kernels (sums_mixed.cu) and
// the persistent work-queue kernel (queue.cu).  Every function here is executed by all kThreads
// threads of a CTA (it contains __syncthreads) and uses the shared-memory struct it is given.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "srs_device.cuh"

namespace srs {
namespace tiles {

constexpr int kThreads = 128;
constexpr int kTileA = 8, kTileB = 16;  // points of a CTA tile along u1 and u2 (kTileA * kTileB == kThreads)
constexpr int kSub = 128;               // trajectory points per shared-memory tile
constexpr int kEnergiesPerThread = 4;

// Trajectory chunks S per tile for ctas tiles on a GPU with `slots` resident CTAs per wave: the S
// minimising the modelled time waves(S) * (n/S + overhead), waves = ceil(ctas * S / slots), with
// chunks of at least min_chunk points.  A grid that overshoots a whole wave by a few CTAs leaves them
// to run alone at the end, so the model picks S that fills the last wave instead.
inline int splits_for(int64_t ctas, int64_t n, int64_t min_chunk, int64_t slots) {
  ctas = std::max<int64_t>(1, ctas);
  slots = std::max<int64_t>(1, slots);
  const int64_t max_s = std::min<int64_t>(std::max<int64_t>(1, n / min_chunk), 4096);
  constexpr double kOverhead = 64.0;  // per-CTA set-up and output, in trajectory points
  int best_s = 1;
  double best = 1e300;
  for (int64_t s = 1; s <= max_s; ++s) {
    const int64_t waves = (ctas * s + slots - 1) / slots;
    const double cost = (double)waves * ((double)((n + s - 1) / s) + kOverhead);
    if (cost < best * (1.0 - 1e-9)) {
      best = cost;
      best_s = (int)s;
    }
  }
  return best_s;
}

// Trajectory points per chunk for S chunks, rounded up to whole shared-memory sub-tiles: the FP32
// accumulators restart at every sub-tile, so with sub-tile-aligned chunks the result depends on S
// only through the FP64 order of the per-chunk sums.  The chunks actually used are ceil(n / chunk).
inline int64_t aligned_chunk(int64_t n, int S) {
  const int64_t c = (n + S - 1) / std::max(1, S);
  return (c + kSub - 1) / kSub * kSub;
}
inline int used_chunks(int64_t n, int64_t chunk) { return (int)((n + chunk - 1) / chunk); }

// Resident CTAs of `kernel` (kThreads threads, no dynamic shared memory) on the current device.
template <typename K>
inline int64_t wave_slots(K kernel) {
  int dev = 0, sms = 148, occ = 1;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kThreads, 0) != cudaSuccess || occ < 1) occ = 1;
  return (int64_t)sms * occ;
}

struct GridTiles {
  int t1, t2;  // tiles along n1 and n2
};
inline GridTiles tiles_of(const srs_grid2d &g) { return GridTiles{(g.n1 + kTileA - 1) / kTileA, (g.n2 + kTileB - 1) / kTileB}; }

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


struct FluxShared {
  float4 r[4][kSub];
};

// Flux: one tile of kTileA x kTileB grid points (tile T1, T2) against trajectory points [i0, iend);
// writes the six partial sums (Re/Im of E_x, E_y, E_z without the final constant) of every point of
// the tile to out6[c * np + j].
__device__ __forceinline__ void flux_tile(const double *__restrict__ xp, const double *__restrict__ bp, int64_t n,
                                          double dt, const srs_grid2d &g, double omega, int T1, int T2, int64_t i0,
                                          int64_t iend, double *__restrict__ out6, FluxShared &sh) {
  // Per trajectory point i (anchored at the tile centre), five float4 records read as broadcasts:
  //   r0 = (phase mod 1 turn, k1, k2 [turns per grid step, mod 1], (w/c)/(2 D_c) / 2pi [turns per m^2])
  //   r1 = (n_c, 1/D_c)
  //   r2 = ((n_c - bhat) + bhat (1 - |beta|), near-field z term -(c/w) n_cz / D_c^2)
  //   r3 = (1/(2 D_c), unused x3)
  // Phases are kept in turns so that the reduction to [-1/2, 1/2) is exact (x - rint(x)).
  // Terms below FP32 resolution are dropped: the third-order distance term g (|Delta|^2 - g^2)/(2 D_c^2)
  // (< 1e-7 rad here) and the near-field term's x, y parts (relative size lambda/(2 pi D) times
  // n_perp, < 1e-10 at 30 m); 1/D_j = (1/D_c)(1 - (D_j - D_c)/D_c) to first order (relative error
  // ((D_j - D_c)/D_c)^2 < 1e-16).
  float4 (*sm)[kSub] = sh.r;
  const int tid = threadIdx.x;
  const int a = tid / kTileB, b = tid % kTileB;
  const int i1 = T1 * kTileA + a, i2 = T2 * kTileB + b;
  const bool active = i1 < g.n1 && i2 < g.n2;
  const int64_t j = (int64_t)i1 * g.n2 + i2;
  const int64_t np = (int64_t)g.n1 * g.n2;
  // tile centre (a grid point) and this thread's integer offsets from it
  const int ca = T1 * kTileA + kTileA / 2, cb = T2 * kTileB + kTileB / 2;
  double Oc[3];
  for (int c = 0; c < 3; ++c) Oc[c] = g.origin[c] + (double)ca * g.u1[c] + (double)cb * g.u2[c];
  const int da = i1 - ca, db = i2 - cb;
  float Dl[3];
  for (int c = 0; c < 3; ++c) Dl[c] = (float)((double)da * g.u1[c] + (double)db * g.u2[c]);
  const float dd = Dl[0] * Dl[0] + Dl[1] * Dl[1] + Dl[2] * Dl[2];
  const float fda = (float)da, fdb = (float)db;
  const double wc = omega / kC;
  const double inv2pi = 0.15915494309189535;
  const float two_pi_f = 6.28318530717958647692f;
  double E[6] = {0, 0, 0, 0, 0, 0};

  for (int64_t base = i0; base < iend; base += kSub) {
    const int cnt = (int)imin64(kSub, iend - base);
    __syncthreads();
    if (tid < cnt) {
      const int64_t i = base + tid;
      const Anchor A = make_anchor(Oc, xp, bp, n, i);
      const double tau = dt * (double)i + A.Dc / kC;
      const double k1 = reduce_2pi(wc * (A.nc[0] * g.u1[0] + A.nc[1] * g.u1[1] + A.nc[2] * g.u1[2]));
      const double k2 = reduce_2pi(wc * (A.nc[0] * g.u2[0] + A.nc[1] * g.u2[1] + A.nc[2] * g.u2[2]));
      sm[0][tid] = make_float4((float)(reduce_2pi(omega * tau) * inv2pi), (float)(k1 * inv2pi), (float)(k2 * inv2pi),
                               (float)(wc * 0.5 * A.invDc * inv2pi));
      sm[1][tid] = make_float4((float)A.nc[0], (float)A.nc[1], (float)A.nc[2], (float)A.invDc);
      sm[2][tid] = make_float4((float)(A.dc[0] + A.bhat[0] * A.omb), (float)(A.dc[1] + A.bhat[1] * A.omb),
                               (float)(A.dc[2] + A.bhat[2] * A.omb),
                               (float)(-(kC / omega) * A.invDc * A.invDc * A.nc[2]));
      sm[3][tid] = make_float4((float)(0.5 * A.invDc), 0.f, 0.f, 0.f);
    }
    __syncthreads();
    if (!active) continue;
    float e0 = 0, e1 = 0, e2 = 0, e3 = 0, e4 = 0, e5 = 0;
#pragma unroll 4
    for (int k = 0; k < cnt; ++k) {
      const float4 r0 = sm[0][k], r1 = sm[1][k], r2 = sm[2][k];
      const float hinv = sm[3][k].x;
      const float gq = fmaf(r1.z, Dl[2], fmaf(r1.y, Dl[1], r1.x * Dl[0]));  // n_c . Delta
      const float h = fmaf(-gq, gq, dd);                                    // |Delta|^2 - g^2
      const float del = fmaf(h, hinv, gq);                                  // D_j - D_c
      const float t = del * r1.w;
      const float rinv = fmaf(-t, r1.w, r1.w);                              // 1/D_j
      float ph = fmaf(r0.y, fda, r0.x);
      ph = fmaf(r0.z, fdb, ph);
      ph = fmaf(h, r0.w, ph);                                               // turns
      const float fr = ph - rintf(ph);
      float sn, cs;
      __sincosf(fr * two_pi_f, &sn, &cs);
      // amplitude (beta - n_j)/D_j = -((n_c - bhat + bhat omb) + (Delta - n_c del)/D_j)/D_j
      const float ux = fmaf(fmaf(-r1.x, del, Dl[0]), rinv, r2.x);
      const float uy = fmaf(fmaf(-r1.y, del, Dl[1]), rinv, r2.y);
      const float uz = fmaf(fmaf(-r1.z, del, Dl[2]), rinv, r2.z);
      const float ax = ux * rinv, ay = uy * rinv, az = uz * rinv;  // minus the amplitude
      e0 = fmaf(-ax, cs, e0); e1 = fmaf(-ax, sn, e1);
      e2 = fmaf(-ay, cs, e2); e3 = fmaf(-ay, sn, e3);
      e4 = fmaf(-az, cs, fmaf(-r2.w, sn, e4)); e5 = fmaf(-az, sn, fmaf(r2.w, cs, e5));
    }
    E[0] += e0; E[1] += e1; E[2] += e2; E[3] += e3; E[4] += e4; E[5] += e5;
  }
  if (active) {
    double *o = out6 + j;
#pragma unroll
    for (int c = 0; c < 6; ++c) o[c * np] = E[c];
  }
}


struct SpecShared {
  double tau[kSub];
  float v[8][kSub];
};

// Each thread owns kEnergiesPerThread consecutive energies.  The rotation exp(i dw tau_i) is shared by
// all threads (dw = (w_last - w_first)/(ne - 1), computed once per trajectory point per CTA); a thread
// whose energies are not on that uniform grid (|w_k - (w_0 + k dw)| * tau_max > 1e-3 rad) takes one
// reduced sincos per (point, energy) instead.  No host synchronisation is needed to decide.
// One tile: energies of tile `etile` (kThreads * kEnergiesPerThread of them) against trajectory
// points [i0, iend); writes the six partial sums of every energy to out6[c * ne + k].
__device__ __forceinline__ void spectrum_tile(const double *__restrict__ xp, const double *__restrict__ bp,
                                              int64_t n, double dt, V3 obs, const double *__restrict__ omegas,
                                              int64_t ne, int etile, int64_t i0, int64_t iend,
                                              double *__restrict__ out6, SpecShared &sh) {
  double *stau = sh.tau;
  float (*sv)[kSub] = sh.v;  // a = (beta - n)/D (3), b' = n/D^2 (3), rotation exp(i dw tau) (2)
  constexpr int K = kEnergiesPerThread;
  const int tid = threadIdx.x;
  const int64_t k0 = ((int64_t)etile * kThreads + tid) * K;
  const bool active = k0 < ne;
  const double wfirst = omegas[0];
  const double dw = ne > 1 ? (omegas[ne - 1] - wfirst) / (double)(ne - 1) : 0.0;
  float kap[K];  // -c/w_k: the near-field term is i*kap*n/D^2
  double wk[K];
  bool uniform = ne > 1;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const int64_t k = imin64(k0 + q, ne - 1);
    wk[q] = omegas[k];
    kap[q] = (float)(-kC / wk[q]);
    const double dev = fabs(wk[q] - (wfirst + (double)k * dw));
    if (k0 + q < ne && dev * (1e3 / kC) >= 1e-3) uniform = false;  // observers within 1 km
  }
  double E[K][6];
#pragma unroll
  for (int q = 0; q < K; ++q)
#pragma unroll
    for (int c = 0; c < 6; ++c) E[q][c] = 0;

  for (int64_t base = i0; base < iend; base += kSub) {
    const int cnt = (int)imin64(kSub, iend - base);
    __syncthreads();
    if (tid < cnt) {
      const int64_t i = base + tid;
      const double rx = obs.x - xp[i], ry = obs.y - xp[n + i], rz = obs.z - xp[2 * n + i];
      const double D = sqrt(rx * rx + ry * ry + rz * rz), iD = 1.0 / D;
      const double nx = rx * iD, ny = ry * iD, nz = rz * iD;
      const double tau = dt * (double)i + D / kC;
      stau[tid] = tau;
      sv[0][tid] = (float)((bp[i] - nx) * iD);
      sv[1][tid] = (float)((bp[n + i] - ny) * iD);
      sv[2][tid] = (float)((bp[2 * n + i] - nz) * iD);
      const double iD2 = iD * iD;
      sv[3][tid] = (float)(nx * iD2);
      sv[4][tid] = (float)(ny * iD2);
      sv[5][tid] = (float)(nz * iD2);
      double sr, cr;
      sincos(reduce_2pi(dw * tau), &sr, &cr);
      sv[6][tid] = (float)cr;
      sv[7][tid] = (float)sr;
    }
    __syncthreads();
    if (!active) continue;
    float e[K][6];
#pragma unroll
    for (int q = 0; q < K; ++q)
#pragma unroll
      for (int c = 0; c < 6; ++c) e[q][c] = 0;
    for (int k = 0; k < cnt; ++k) {
      const double tau = stau[k];
      const float ax = sv[0][k], ay = sv[1][k], az = sv[2][k];
      const float bx = sv[3][k], by = sv[4][k], bz = sv[5][k];
      const float rr = sv[6][k], ri = sv[7][k];
      float zr, zi;
      __sincosf((float)reduce_2pi(wk[0] * tau), &zi, &zr);
#pragma unroll
      for (int q = 0; q < K; ++q) {
        if (q > 0) {
          if (uniform) {  // z <- z * exp(i dw tau)
            const float tr = zr * rr - zi * ri;
            zi = fmaf(zr, ri, zi * rr);
            zr = tr;
          } else {
            __sincosf((float)reduce_2pi(wk[q] * tau), &zi, &zr);
          }
        }
        // e += (a + i kap b') (zr + i zi)
        const float cx = kap[q] * bx, cy = kap[q] * by, cz = kap[q] * bz;
        e[q][0] = fmaf(ax, zr, fmaf(-cx, zi, e[q][0])); e[q][1] = fmaf(ax, zi, fmaf(cx, zr, e[q][1]));
        e[q][2] = fmaf(ay, zr, fmaf(-cy, zi, e[q][2])); e[q][3] = fmaf(ay, zi, fmaf(cy, zr, e[q][3]));
        e[q][4] = fmaf(az, zr, fmaf(-cz, zi, e[q][4])); e[q][5] = fmaf(az, zi, fmaf(cz, zr, e[q][5]));
      }
    }
#pragma unroll
    for (int q = 0; q < K; ++q)
#pragma unroll
      for (int c = 0; c < 6; ++c) E[q][c] += (double)e[q][c];
  }
  if (active) {
#pragma unroll
    for (int q = 0; q < K; ++q) {
      const int64_t k = k0 + q;
      if (k >= ne) break;
      double *o = out6 + k;
#pragma unroll
      for (int c = 0; c < 6; ++c) o[c * ne] = E[q][c];
    }
  }
}


}  // namespace tiles
}  // namespace srs

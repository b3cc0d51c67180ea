// Mixed-precision radiation sums: FP64 only where stability needs it (the retarded phase and its
// reduction modulo 2*pi, 1 - n.beta, the geometry anchors), FP32 for the bulk of the integrand
// (amplitude, per-pair phase increments, sincos on the SFU, accumulation), FP64 for the outer sums.
//
// Same physics as the plain kernels (src/OSCARSSR.cc:1154-1251 spectrum, :1989-2099 flux,
// :1477-1598 power density), reorganised for the B200:
//
// * Flux / power density on a regular grid of observation points (a rectangle surface): a CTA owns
//   an 8 x 16 tile of points and one chunk of the trajectory.  For each trajectory point i the CTA
//   computes ONCE, in FP64, an anchor at the tile's centre point c: distance D_c, direction n_c, the
//   reduced phase Phi_c = w (t_i + D_c/c) mod 2pi, the reduced per-grid-step phase increments
//   k1,k2 = (w/c) n_c.u1,u2 mod 2pi, and n_c - beta_hat.  Every point j = c + da*u1 + db*u2 of the
//   tile then needs only FP32 work on small quantities:
//       g = n_c . Delta_j,  h = |Delta_j|^2 - g^2,
//       D_j - D_c = g + h/(2 D_c) (1 - g/D_c) + O(|Delta|^4/D^3),
//       phase_j = Phi_c + k1 da + k2 db + (w/c) h/(2 D_c) (1 - g/D_c),
//       n_j - beta_hat = (n_c - beta_hat) + (Delta_j - n_c (D_j - D_c)) / D_j,
//   so no FP32 quantity is ever the difference of two nearly equal large numbers.
//   1 - n.beta = (1 - |beta|) + |beta| |n - beta_hat|^2 / 2 (both terms >= 0, no cancellation).
// * Spectrum on a uniform energy grid: a thread owns 4 consecutive energies; per trajectory point it
//   forms one FP64 anchor exp(i w_k0 tau_i) and walks the others with the per-point rotation
//   exp(i dw tau_i) (computed once per point per CTA in FP64), re-anchored at every point.  A
//   non-uniform grid gets one reduced sincos per (point, energy).
//
// Accumulation: FP32 within each 128-point shared-memory tile, then FP64 across tiles and chunks.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {

namespace {

constexpr int kThreads = 128;
constexpr int kTileA = 8, kTileB = 16;  // points of a CTA tile along u1 and u2 (kTileA * kTileB == kThreads)
constexpr int kSub = 128;               // trajectory points per shared-memory tile
constexpr int kTargetCtas = 148 * 6;
constexpr int kEnergiesPerThread = 4;

int splits_for(int64_t ctas, int64_t n, int64_t min_chunk) {
  int64_t s = (kTargetCtas + ctas - 1) / std::max<int64_t>(1, ctas);
  int64_t max_s = std::max<int64_t>(1, n / min_chunk);
  return (int)std::min<int64_t>(std::max<int64_t>(1, std::min(s, max_s)), 65535);
}

struct GridTiles {
  int t1, t2;  // tiles along n1 and n2
};
GridTiles tiles_of(const srs_grid2d &g) { return GridTiles{(g.n1 + kTileA - 1) / kTileA, (g.n2 + kTileB - 1) / kTileB}; }

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

// ---------------------------------------------------------------- flux on a grid

struct FluxRec {  // per trajectory point, per tile (FP32 unless noted)
  float phi, k1, k2, w1, invD, D;
  float nc[3], dc[3], bo[3], bim[3];
};

__global__ void __launch_bounds__(kThreads) flux_mixed_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                              int64_t n, double dt, srs_grid2d g, double omega,
                                                              int64_t chunk, double *__restrict__ partial) {
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
  __shared__ float4 sm[4][kSub];
  const int tid = threadIdx.x;
  const int T1 = blockIdx.x / ((g.n2 + kTileB - 1) / kTileB), T2 = blockIdx.x % ((g.n2 + kTileB - 1) / kTileB);
  const int a = tid / kTileB, b = tid % kTileB;
  const int i1 = T1 * kTileA + a, i2 = T2 * kTileB + b;
  const bool active = i1 < g.n1 && i2 < g.n2;
  const int64_t j = (int64_t)i1 * g.n2 + i2;
  const int64_t np = (int64_t)g.n1 * g.n2;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const double *xp = X + (int64_t)p * 3 * n, *bp = Bt + (int64_t)p * 3 * n;
  const int64_t i0 = (int64_t)s * chunk, iend = imin64(n, i0 + chunk);
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
    double *o = partial + ((int64_t)p * S + s) * 6 * np + j;
#pragma unroll
    for (int c = 0; c < 6; ++c) o[c * np] = E[c];
  }
}

// ---------------------------------------------------------------- power density on a grid

__global__ void __launch_bounds__(kThreads) pd_mixed_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                            const double *__restrict__ Ac, int64_t n, srs_grid2d g,
                                                            double nx_, double ny_, double nz_, int directional,
                                                            int64_t chunk, double *__restrict__ partial) {
  // (1 - n.beta)^5 ~ 1e-39 does not fit FP32, so the FP32 term is scaled: with omb = 1 - |beta|,
  // 1 - n.beta = omb_i * opn, opn = 1 + (|beta|/(2 omb_i)) |n - bhat|^2 >= 1, and
  // 1/(1 - n.beta)^5 = (omb_ref/omb_i)^5 / opn^5 / omb_ref^5; the last factor (~1e39) is applied in FP64.
  // Per trajectory point i, five float4 records read as broadcasts:
  //   r0 = (n_c, 1/D_c)                 r1 = (n_c - bhat, 1/(2 D_c))
  //   r2 = (bhat (1 - |beta|), omb_i)   r3 = (a/c, |beta|/(2 omb_i))
  //   r4 = (bhat . a, (omb_ref/omb_i)^5, n_c . normal, unused)
  __shared__ float4 sm[5][kSub];
  const int tid = threadIdx.x;
  const int nt2 = (g.n2 + kTileB - 1) / kTileB;
  const int T1 = blockIdx.x / nt2, T2 = blockIdx.x % nt2;
  const int a = tid / kTileB, b = tid % kTileB;
  const int i1 = T1 * kTileA + a, i2 = T2 * kTileB + b;
  const bool active = i1 < g.n1 && i2 < g.n2;
  const int64_t j = (int64_t)i1 * g.n2 + i2;
  const int64_t np = (int64_t)g.n1 * g.n2;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t off = (int64_t)p * 3 * n;
  const double *xp = X + off, *bp = Bt + off, *ap = Ac + off;
  const int64_t i0 = (int64_t)s * chunk, iend = imin64(n, i0 + chunk);
  const int ca = T1 * kTileA + kTileA / 2, cb = T2 * kTileB + kTileB / 2;
  double Oc[3];
  for (int c = 0; c < 3; ++c) Oc[c] = g.origin[c] + (double)ca * g.u1[c] + (double)cb * g.u2[c];
  const int da = i1 - ca, db = i2 - cb;
  float Dl[3];
  for (int c = 0; c < 3; ++c) Dl[c] = (float)((double)da * g.u1[c] + (double)db * g.u2[c]);
  const float dd = Dl[0] * Dl[0] + Dl[1] * Dl[1] + Dl[2] * Dl[2];
  const float nrx = (float)nx_, nry = (float)ny_, nrz = (float)nz_;
  double omb_ref;
  {
    const double bx = bp[0], by = bp[n], bz = bp[2 * n];
    const double b2 = bx * bx + by * by + bz * bz;
    omb_ref = (1.0 - b2) / (1.0 + sqrt(b2));
  }
  double sum = 0;
  for (int64_t base = i0; base < iend; base += kSub) {
    const int cnt = (int)imin64(kSub, iend - base);
    __syncthreads();
    if (tid < cnt) {
      const int64_t i = base + tid;
      const Anchor A = make_anchor(Oc, xp, bp, n, i);
      const double ax = ap[i], ay = ap[n + i], az = ap[2 * n + i];
      const double r = omb_ref / A.omb;
      sm[0][tid] = make_float4((float)A.nc[0], (float)A.nc[1], (float)A.nc[2], (float)A.invDc);
      sm[1][tid] = make_float4((float)A.dc[0], (float)A.dc[1], (float)A.dc[2], (float)(0.5 * A.invDc));
      sm[2][tid] = make_float4((float)(A.bhat[0] * A.omb), (float)(A.bhat[1] * A.omb), (float)(A.bhat[2] * A.omb),
                               (float)A.omb);
      sm[3][tid] = make_float4((float)ax, (float)ay, (float)az, (float)(0.5 * A.bmag / A.omb));
      sm[4][tid] = make_float4((float)(A.bhat[0] * ax + A.bhat[1] * ay + A.bhat[2] * az), (float)(r * r * r * r * r),
                               (float)(A.nc[0] * nx_ + A.nc[1] * ny_ + A.nc[2] * nz_), 0.f);
    }
    __syncthreads();
    if (!active) continue;
    float acc = 0;
#pragma unroll 4
    for (int k = 0; k < cnt; ++k) {
      const float4 r0 = sm[0][k], r1 = sm[1][k];
      const float gq = fmaf(r0.z, Dl[2], fmaf(r0.y, Dl[1], r0.x * Dl[0]));  // n_c . Delta
      const float h = fmaf(-gq, gq, dd);
      const float del = fmaf(h, r1.w, gq);                                    // D_j - D_c
      const float t = del * r0.w;
      const float rinv = fmaf(-t, r0.w, r0.w);                                // 1/D_j
      const float dnx = fmaf(-r0.x, del, Dl[0]) * rinv, dny = fmaf(-r0.y, del, Dl[1]) * rinv,
                  dnz = fmaf(-r0.z, del, Dl[2]) * rinv;                       // n_j - n_c
      const float4 r4 = sm[4][k];
      const float nd = fmaf(dnz, nrz, fmaf(dny, nry, fmaf(dnx, nrx, r4.z)));  // n_j . normal
      if (directional && nd <= 0.0f) continue;
      const float4 r2 = sm[2][k], r3 = sm[3][k];
      const float dx = r1.x + dnx, dy = r1.y + dny, dz = r1.z + dnz;           // n_j - bhat
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      const float opn = fmaf(r3.w, d2, 1.0f);  // (1 - n.beta) / omb_i
      const float opnb = r2.w * opn;           // 1 - n.beta
      const float na = fmaf(dz, r3.z, fmaf(dy, r3.y, fmaf(dx, r3.x, r4.x)));  // n . a
      // V = n x ((n - beta) x a) = (n - beta)(n.a) - a (1 - n.beta)
      const float Xx = dx + r2.x, Xy = dy + r2.y, Xz = dz + r2.z;
      const float Vx = fmaf(Xx, na, -r3.x * opnb), Vy = fmaf(Xy, na, -r3.y * opnb), Vz = fmaf(Xz, na, -r3.z * opnb);
      const float v2 = fmaf(Vz, Vz, fmaf(Vy, Vy, Vx * Vx));
      const float o2 = opn * opn;
      const float o5 = o2 * o2 * opn;
      acc = fmaf(v2 * rinv * rinv * nd * r4.y, __fdividef(1.0f, o5), acc);
    }
    sum += (double)acc;
  }
  const double r2 = 1.0 / (omb_ref * omb_ref);
  if (active) partial[((int64_t)p * S + s) * np + j] = sum * (r2 * r2 / omb_ref);
}

// ---------------------------------------------------------------- spectrum at one observer

// Each thread owns kEnergiesPerThread consecutive energies.  The rotation exp(i dw tau_i) is shared by
// all threads (dw = (w_last - w_first)/(ne - 1), computed once per trajectory point per CTA); a thread
// whose energies are not on that uniform grid (|w_k - (w_0 + k dw)| * tau_max > 1e-3 rad) takes one
// reduced sincos per (point, energy) instead.  No host synchronisation is needed to decide.
__global__ void __launch_bounds__(kThreads) spectrum_mixed_kernel(const double *__restrict__ X,
                                                                  const double *__restrict__ Bt, int64_t n, double dt,
                                                                  V3 obs, const double *__restrict__ omegas, int64_t ne,
                                                                  int64_t chunk, double *__restrict__ partial) {
  __shared__ double stau[kSub];
  __shared__ float sv[8][kSub];  // a = (beta - n)/D (3), b' = n/D^2 (3), rotation exp(i dw tau) (2)
  constexpr int K = kEnergiesPerThread;
  const int tid = threadIdx.x;
  const int64_t k0 = ((int64_t)blockIdx.x * kThreads + tid) * K;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const double *xp = X + (int64_t)p * 3 * n, *bp = Bt + (int64_t)p * 3 * n;
  const int64_t i0 = (int64_t)s * chunk, iend = imin64(n, i0 + chunk);
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
      double *o = partial + ((int64_t)p * S + s) * 6 * ne + k;
#pragma unroll
      for (int c = 0; c < 6; ++c) o[c * ne] = E[q][c];
    }
  }
}

__global__ void omega_kernel(const double *__restrict__ e, int64_t ne, double *__restrict__ w) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) w[i] = ev_to_omega(e[i]);
}

}  // namespace

// ---------------------------------------------------------------- launchers

static int flux_mixed_splits(int64_t n, const srs_grid2d &g, int nparticles) {
  GridTiles t = tiles_of(g);
  return splits_for((int64_t)t.t1 * t.t2 * nparticles, n, 512);
}

size_t mixed_flux_scratch_bytes(int64_t n, const srs_grid2d &g, int nparticles) {
  return sizeof(double) * 6 * (size_t)g.n1 * g.n2 * nparticles * flux_mixed_splits(n, g, nparticles);
}

static cudaError_t mixed_flux_splits(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                     double energy_ev, double *d_out, void *scratch, int S, cudaStream_t s) {
  const int64_t chunk = (t.n + S - 1) / S;
  GridTiles tl = tiles_of(g);
  const double omega = ev_to_omega(energy_ev);
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)(tl.t1 * tl.t2), S, t.nparticles);
  flux_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.n, t.dt, g, omega, chunk, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_flux_partials(partial, S, (int64_t)g.n1 * g.n2, t.nparticles, nullptr, omega, t.dt, flux_c0(b.charge),
                              flux_c2(b.charge, b.current), d_out, s);
}

cudaError_t mixed_flux(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g, double energy_ev,
                       double *d_out, void *scratch, cudaStream_t s) {
  return mixed_flux_splits(t, b, g, energy_ev, d_out, scratch, flux_mixed_splits(t.n, g, t.nparticles), s);
}

// ---------------------------------------------------------------- allocation-free flux entry point
//
// For callers that must not allocate device memory once they are running -- for example a host
// program whose device memory is entirely reserved up front by its own allocator, or a
// latency-critical loop that forbids cudaMalloc (which can synchronise the device and has no bounded
// latency).  The per-chunk partial sums that srs_flux keeps in a stream-ordered allocation live
// here in a fixed, file-scope device array instead.
//
// Every GPU that loads this library holds this array until the process exits.  All calls share it,
// and it keeps the last call's contents: calls that overlap on the GPU (different streams, or
// several host threads) race on it, so the caller must serialise them.  Nothing in it needs to start
// at zero: each call's main kernel writes every slot that its finishing kernel reads.
constexpr size_t kNoAllocScratchDoubles = (size_t)1 << 20;  // 8 MiB
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of g_noalloc_scratch, looked up once per device.  In host code the array's name is
// only a host-side stand-in, so the address must come from cudaGetSymbolAddress with the device
// current.
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[64];

static cudaError_t noalloc_scratch(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return cudaSuccess;
}

}  // namespace srs

extern "C" srs_status srs_flux_mixed_noalloc(srs_traj_view traj, srs_beam_consts beam, const srs_grid2d *grid,
                                             double energy_ev, double *d_out, void *stream) {
  using namespace srs;
  clear_error();
  if (!traj.x || !traj.beta || traj.n < 1 || traj.nparticles < 1 || !(traj.dt > 0))
    return fail(SRS_ERR_INVALID, "bad trajectory view");
  if (!grid || grid->n1 < 1 || grid->n2 < 1) return fail(SRS_ERR_INVALID, "the points must be given as a grid");
  if (!d_out) return fail(SRS_ERR_INVALID, "NULL output");
  if (!(energy_ev > 0)) return fail(SRS_ERR_INVALID, "energy_eV must be > 0");
  // partial sums: 6 doubles per (particle, point, trajectory chunk); use as many chunks as fit
  const size_t per_chunk = (size_t)6 * grid->n1 * grid->n2 * traj.nparticles;
  if (per_chunk > kNoAllocScratchDoubles)
    return fail(SRS_ERR_RANGE, "srs_flux_mixed_noalloc: nparticles * points = " +
                                   std::to_string((size_t)grid->n1 * grid->n2 * traj.nparticles) +
                                   " exceeds its fixed scratch (at most " +
                                   std::to_string(kNoAllocScratchDoubles / 6) + " particle-points); use srs_flux");
  const int S = (int)std::max<size_t>(1, std::min<size_t>((size_t)flux_mixed_splits(traj.n, *grid, traj.nparticles),
                                                          kNoAllocScratchDoubles / per_chunk));
  void *scratch = nullptr;
  SRS_CUDA(noalloc_scratch(&scratch));
  SRS_CUDA(mixed_flux_splits(traj, beam, *grid, energy_ev, d_out, scratch, S, static_cast<cudaStream_t>(stream)));
  return SRS_OK;
}

namespace srs {

size_t mixed_pd_scratch_bytes(int64_t n, const srs_grid2d &g, int nparticles) {
  GridTiles tl = tiles_of(g);
  return sizeof(double) * (size_t)g.n1 * g.n2 * nparticles *
         splits_for((int64_t)tl.t1 * tl.t2 * nparticles, n, 512);
}

cudaError_t mixed_power_density(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                int directional, double *d_out, void *scratch, cudaStream_t s) {
  GridTiles tl = tiles_of(g);
  const int S = splits_for((int64_t)tl.t1 * tl.t2 * t.nparticles, t.n, 512);
  const int64_t chunk = (t.n + S - 1) / S;
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)(tl.t1 * tl.t2), S, t.nparticles);
  pd_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.aoc, t.n, g, g.normal[0], g.normal[1], g.normal[2], directional, chunk,
                                            partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_pd_partials(partial, S, (int64_t)g.n1 * g.n2, t.nparticles, pd_const(b.charge, b.current) * t.dt,
                            directional, d_out, s);
}

size_t mixed_spectrum_scratch_bytes(int64_t n, int64_t ne, int nparticles) {
  const int64_t ctas = (ne + kThreads * kEnergiesPerThread - 1) / (kThreads * kEnergiesPerThread) * nparticles;
  return sizeof(double) * ((size_t)6 * ne * nparticles * splits_for(ctas, n, 256) + ne);
}

cudaError_t mixed_spectrum(const srs_traj_view &t, const srs_beam_consts &b, const double obs[3],
                           const double *d_energies, int64_t ne, double *d_out, void *scratch, cudaStream_t s) {
  const int64_t etiles = (ne + kThreads * kEnergiesPerThread - 1) / (kThreads * kEnergiesPerThread);
  const int S = splits_for(etiles * t.nparticles, t.n, 256);
  const int64_t chunk = (t.n + S - 1) / S;
  double *partial = static_cast<double *>(scratch);
  double *omegas = partial + (size_t)6 * ne * t.nparticles * S;
  omega_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(d_energies, ne, omegas);
  dim3 grid((unsigned)etiles, S, t.nparticles);
  spectrum_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.n, t.dt, v3(obs[0], obs[1], obs[2]), omegas, ne,
                                                  chunk, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_flux_partials(partial, S, ne, t.nparticles, omegas, 0.0, t.dt, flux_c0(b.charge),
                              flux_c2(b.charge, b.current), d_out, s);
}

}  // namespace srs

// Mixed-precision radiation sums: FP64 only where stability needs it (the retarded phase and its
// reduction modulo 2*pi, 1 - n.beta, the geometry anchors), FP32 for the bulk of the integrand
// (amplitude, per-pair phase increments, sincos on the SFU, accumulation), FP64 for the outer sums.
//
// Same physics as the plain kernels (src/OSCARSSR.cc:1154-1251 spectrum, :1989-2099 flux,
// :1477-1598 power density), reorganised for the B200:
//
// * Flux / power density on a regular grid of observation points (a rectangle surface): a CTA owns
//   a tile of up to 128 points (consecutive points of a strip 8-16 points wide, at most 17 rows) and
//   one chunk of the trajectory.  For each trajectory point i the CTA computes ONCE, in FP64, an
//   anchor at the tile's middle point c: distance D_c, direction n_c, the
//   reduced phase Phi_c = w (t_i + D_c/c) mod 2pi, the reduced per-grid-step phase increments
//   k1,k2 = (w/c) n_c.u1,u2 mod 2pi, and n_c - beta_hat.  Every point j = c + da*u1 + db*u2 of the
//   tile then needs only FP32 work on small quantities:
//       g = n_c . Delta_j,  h = |Delta_j|^2 - g^2,
//       D_j - D_c = g + h/(2 D_c) + O(g h/D_c^2)  (the dropped term is below FP32 resolution of the
//                                                   phase for the tiles' extent at metres of distance),
//       phase_j = Phi_c + k1 da + k2 db + (w/c) h/(2 D_c),
//       n_j - beta_hat = (n_c - beta_hat) + (Delta_j - n_c (D_j - D_c)) / D_j,
//   so no FP32 quantity is ever the difference of two nearly equal large numbers.
//   1 - n.beta = (1 - |beta|) + |beta| |n - beta_hat|^2 / 2 (both terms >= 0, no cancellation).
// * Spectrum on a uniform energy grid: a thread owns 4 (or 2) consecutive energies; per trajectory point it
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

#include "mixed_tiles.cuh"
#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {

using namespace tiles;

namespace {

// ---------------------------------------------------------------- flux on a grid

__global__ void __launch_bounds__(kThreads, 6) flux_mixed_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                              int64_t n, double dt, srs_grid2d g, StripTiles m,
                                                              double omega, int64_t chunk,
                                                              double *__restrict__ partial) {
  __shared__ tiles::FluxShared sh;
  wait_for_previous_grid();  // (launched with launch_after by the one-shot launcher)
  allow_next_grid();
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t np = (int64_t)g.n1 * g.n2;
  const int64_t i0 = (int64_t)s * chunk;
  tiles::flux_tile(X + (int64_t)p * 3 * n, Bt + (int64_t)p * 3 * n, n, dt, g, m, omega, blockIdx.x, i0,
                   imin64(n, i0 + chunk), partial + ((int64_t)p * S + s) * 6 * np, sh);
}

// ---------------------------------------------------------------- flux at a list of points

__global__ void __launch_bounds__(kThreads) flux_points_mixed_kernel(const double *__restrict__ X,
                                                                     const double *__restrict__ Bt, int64_t n,
                                                                     double dt, const double *__restrict__ points,
                                                                     int64_t np, double omega, int64_t chunk,
                                                                     double *__restrict__ partial) {
  __shared__ tiles::PointsShared sh;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t i0 = (int64_t)s * chunk;
  tiles::points_flux_tile(X + (int64_t)p * 3 * n, Bt + (int64_t)p * 3 * n, n, dt, points, np, omega, blockIdx.x, i0,
                          imin64(n, i0 + chunk), partial + ((int64_t)p * S + s) * 6 * np, sh);
}

// ---------------------------------------------------------------- power density on a grid

__global__ void __launch_bounds__(kThreads, 5) pd_mixed_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                            const double *__restrict__ Ac, int64_t n, srs_grid2d g,
                                                            StripTiles m, double nx_, double ny_, double nz_,
                                                            int directional, int64_t chunk,
                                                            double *__restrict__ partial) {
  // (1 - n.beta)^5 ~ 1e-39 does not fit FP32, so the FP32 term is scaled: with omb = 1 - |beta|,
  // 1 - n.beta = omb_i * opn, opn = 1 + (|beta|/(2 omb_i)) |n - bhat|^2 >= 1, and
  // 1/(1 - n.beta)^5 = (omb_ref/omb_i)^5 / opn^5 / omb_ref^5; the last factor (~1e39) is applied in FP64.
  // Per trajectory point, 20 FP32 values anchored at the tile's anchor point, stored for pairs of
  // consecutive points as in the flux tile (record g of pair q = fields 2g, 2g+1 of both points), with
  // signs chosen so that the inner loop needs no negation:
  //   0-2 n_c        3 1/D_c        4-6 n_c - bhat      7 1/(2 D_c)
  //   8-10 bhat (1 - |beta|)        11 -omb_i = -(1 - |beta_i|)
  //   12-14 a/c      15 |beta|/(2 omb_i)                16 bhat . a/c
  //   17 (omb_ref/omb_i)^5          18 n_c . normal     19 1/D_c^2
  // The records are double-buffered (sub-tile k in sm[k & 1]), so one barrier per sub-tile suffices.
  constexpr int kPdFields = 20;
  __shared__ float4 sm[2][kPdFields / 2][kSub / 2];
  const int tid = threadIdx.x;
  const TilePoint P = strip_point(m, blockIdx.x, tid);
  const bool active = P.active;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t off = (int64_t)p * 3 * n;
  const double *xp = X + off, *bp = Bt + off, *ap = Ac + off;
  const int64_t i0 = (int64_t)s * chunk, iend = imin64(n, i0 + chunk);
  const int da = P.i1 - P.ca, db = P.i2 - P.cb;
  // the tile's reach from its anchor (a bound on |Delta|)
  const double dmax = P.ra * sqrt(g.u1[0] * g.u1[0] + g.u1[1] * g.u1[1] + g.u1[2] * g.u1[2]) +
                      P.rb * sqrt(g.u2[0] * g.u2[0] + g.u2[1] * g.u2[1] + g.u2[2] * g.u2[2]);
  double omb_ref;
  {
    const double bx = bp[0], by = bp[n], bz = bp[2 * n];
    const double b2 = bx * bx + by * by + bz * bz;
    omb_ref = (1.0 - b2) / (1.0 + sqrt(b2));
  }

  // the records of trajectory points [base, base + kSub) into buffer buf; returns whether this thread's
  // point needs the exact sum.  An error e in D_j - D_c moves n.beta by ~e/D_c, which (1 - n.beta)^-5
  // amplifies by 5/(1 - |beta|) relative: the expansion's rest and the FP32 rounding of n_c . Delta are
  // bounded in those terms.
  auto fill = [&](int buf, int64_t base) -> int {
    int bad = 0;
    float *rec = &sm[buf][0][0].x;
    auto put = [&](int t, int f, float v) { rec[((f >> 1) * (kSub / 2) + (t >> 1)) * 4 + (f & 1) * 2 + (t & 1)] = v; };
    const int cnt = (int)imin64(kSub, iend - base);
    if (tid < cnt) {
      const int64_t i = base + tid;
      double Oc[3];
      for (int c = 0; c < 3; ++c) Oc[c] = g.origin[c] + (double)P.ca * g.u1[c] + (double)P.cb * g.u2[c];
      const Anchor A = make_anchor(Oc, xp, bp, n, i);
      {
        const double nu1 = A.nc[0] * g.u1[0] + A.nc[1] * g.u1[1] + A.nc[2] * g.u1[2];
        const double nu2 = A.nc[0] * g.u2[0] + A.nc[1] * g.u2[1] + A.nc[2] * g.u2[2];
        const double gmax = P.ra * fabs(nu1) + P.rb * fabs(nu2);
        const double gain = 5.0 * A.invDc / A.omb;
        const double ramp = (gmax + 0.5 * dmax * dmax * A.invDc) * A.invDc;
        bad = dmax * A.invDc >= 0.5 || gain * expansion_rest(A.invDc, dmax, gmax) > kRestPd ||
              gain * gmax * 0x1p-24 > kRoundPd || ramp * ramp > kRestAmp;
      }
      const double ax = ap[i], ay = ap[n + i], az = ap[2 * n + i];
      const double r = omb_ref / A.omb;
      put(tid, 0, (float)A.nc[0]); put(tid, 1, (float)A.nc[1]); put(tid, 2, (float)A.nc[2]);
      put(tid, 3, (float)A.invDc);
      put(tid, 4, (float)A.dc[0]); put(tid, 5, (float)A.dc[1]); put(tid, 6, (float)A.dc[2]);
      put(tid, 7, (float)(0.5 * A.invDc));
      put(tid, 8, (float)(A.bhat[0] * A.omb)); put(tid, 9, (float)(A.bhat[1] * A.omb));
      put(tid, 10, (float)(A.bhat[2] * A.omb));
      put(tid, 11, (float)(-A.omb));
      put(tid, 12, (float)ax); put(tid, 13, (float)ay); put(tid, 14, (float)az);
      put(tid, 15, (float)(0.5 * A.bmag / A.omb));
      put(tid, 16, (float)(A.bhat[0] * ax + A.bhat[1] * ay + A.bhat[2] * az));
      put(tid, 17, (float)(r * r * r * r * r));
      put(tid, 18, (float)(A.nc[0] * nx_ + A.nc[1] * ny_ + A.nc[2] * nz_));
      put(tid, 19, (float)(A.invDc * A.invDc));
    } else if (tid == cnt && (cnt & 1)) {
      // the odd count's partner slot: zero 1/D_c and (omb_ref/omb)^5 make its term 0; omb = 1 keeps
      // 1 - n.beta finite
      for (int f = 0; f < kPdFields; ++f) put(tid, f, f == 11 ? -1.0f : 0.0f);
    }
    return bad;
  };

  double sum = 0;
  int bad_cur = i0 < iend ? fill(0, i0) : 0;
  int buf = 0;
  for (int64_t base = i0; base < iend; base += kSub, buf ^= 1) {
    const int cnt = (int)imin64(kSub, iend - base);
    // records of this sub-tile complete; every thread is done with the other buffer
    const int exact = __syncthreads_or(bad_cur);
    bad_cur = base + kSub < iend ? fill(buf ^ 1, base + kSub) : 0;
    if (!active) continue;
    if (exact) {
      // FP64 geometry per term (R, 1/|R|, n, n - beta), the rest from the records, as the point-list kernel
      const float *rec = &sm[buf][0][0].x;
      auto get = [&](int f, int k) { return rec[((f >> 1) * (kSub / 2) + (k >> 1)) * 4 + (f & 1) * 2 + (k & 1)]; };
      double Pq[3];
      for (int c = 0; c < 3; ++c) Pq[c] = (g.origin[c] + g.u1[c] * (double)P.i1) + g.u2[c] * (double)P.i2;
      const float nrx = (float)nx_, nry = (float)ny_, nrz = (float)nz_;
      float acc = 0.f;
      for (int k = 0; k < cnt; ++k) {
        const int64_t i = base + k;
        const double Rx = Pq[0] - __ldg(xp + i), Ry = Pq[1] - __ldg(xp + n + i), Rz = Pq[2] - __ldg(xp + 2 * n + i);
        const double R2 = fma(Rx, Rx, fma(Ry, Ry, Rz * Rz));
        const float yf = rsqrtf((float)R2);
        double y = (double)yf;
        double e = fma(-R2 * y, y, 1.0);
        y = fma(0.5 * y, e, y);
        e = fma(-R2 * y, y, 1.0);
        y = fma(0.5 * y, e, y);  // 1/|R| to FP64 accuracy
        const double nx = Rx * y, ny = Ry * y, nz = Rz * y;
        const float mx = (float)(nx - __ldg(bp + i)), my = (float)(ny - __ldg(bp + n + i)),
                    mz = (float)(nz - __ldg(bp + 2 * n + i));  // n - beta
        const float dx = mx - get(8, k), dy = my - get(9, k), dz = mz - get(10, k);  // n - bhat
        const float nd = fmaf((float)nz, nrz, fmaf((float)ny, nry, (float)nx * nrx));
        const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
        const float opn = fmaf(get(15, k), d2, 1.0f);
        const float opnbn = get(11, k) * opn;  // -(1 - n.beta)
        const float acx = get(12, k), acy = get(13, k), acz = get(14, k);
        const float na = fmaf(dz, acz, fmaf(dy, acy, fmaf(dx, acx, get(16, k))));
        const float Vx = fmaf(mx, na, acx * opnbn), Vy = fmaf(my, na, acy * opnbn), Vz = fmaf(mz, na, acz * opnbn);
        const float v2 = fmaf(Vz, Vz, fmaf(Vy, Vy, Vx * Vx));
        const float o2 = opn * opn, o5 = o2 * o2 * opn;
        float term = v2 * (yf * yf) * nd * get(17, k) * __fdividef(1.0f, o5);
        if (directional && !(nd > 0.0f)) term = 0.0f;
        acc += term;
      }
      sum += (double)acc;
      continue;
    }
    // this thread's offset from the anchor point (formed after the FP64 anchors, off their registers)
    float Dl[3];
    for (int c = 0; c < 3; ++c) Dl[c] = (float)((double)da * g.u1[c] + (double)db * g.u2[c]);
    const float2 Dx = f2(Dl[0], Dl[0]), Dy = f2(Dl[1], Dl[1]), Dz = f2(Dl[2], Dl[2]);
    const float2 Dxn = f2(-Dl[0], -Dl[0]), Dyn = f2(-Dl[1], -Dl[1]), Dzn = f2(-Dl[2], -Dl[2]);
    const float ddv = -(Dl[0] * Dl[0] + Dl[1] * Dl[1] + Dl[2] * Dl[2]);
    const float2 ddn = f2(ddv, ddv), one = f2(1.0f, 1.0f);
    const float2 NRx = f2((float)nx_, (float)nx_), NRy = f2((float)ny_, (float)ny_), NRz = f2((float)nz_, (float)nz_);
    const float4(*sr)[kSub / 2] = sm[buf];
    float2 acc = f2(0.f, 0.f);
    const int pairs = (cnt + 1) >> 1;
#pragma unroll 2
    for (int q = 0; q < pairs; ++q) {
      const float4 R0 = sr[0][q], R1 = sr[1][q], R2 = sr[2][q], R3 = sr[3][q], R4 = sr[4][q];
      const float4 R5 = sr[5][q], R6 = sr[6][q], R7 = sr[7][q], R8 = sr[8][q], R9 = sr[9][q];
      const float2 ncx = f2(R0.x, R0.y), ncy = f2(R0.z, R0.w), ncz = f2(R1.x, R1.y), w = f2(R1.z, R1.w);
      const float2 dcx = f2(R2.x, R2.y), dcy = f2(R2.z, R2.w), dcz = f2(R3.x, R3.y), hinv = f2(R3.z, R3.w);
      const float2 box = f2(R4.x, R4.y), boy = f2(R4.z, R4.w), boz = f2(R5.x, R5.y), ombn = f2(R5.z, R5.w);
      const float2 acx = f2(R6.x, R6.y), acy = f2(R6.z, R6.w), acz = f2(R7.x, R7.y), bfac = f2(R7.z, R7.w);
      const float2 ba = f2(R8.x, R8.y), r5 = f2(R8.z, R8.w), ncn = f2(R9.x, R9.y), w2 = f2(R9.z, R9.w);
      const float2 gqn = fma2(ncz, Dzn, fma2(ncy, Dyn, mul2(ncx, Dxn)));  // -n_c . Delta
      const float2 hn = fma2(gqn, gqn, ddn);                              // -(|Delta|^2 - g^2)
      const float2 deln = fma2(hn, hinv, gqn);                            // D_c - D_j
      const float2 rinv = fma2(deln, w2, w);                              // 1/D_j
      const float2 dnx = mul2(fma2(ncx, deln, Dx), rinv);                 // n_j - n_c
      const float2 dny = mul2(fma2(ncy, deln, Dy), rinv);
      const float2 dnz = mul2(fma2(ncz, deln, Dz), rinv);
      const float2 nd = fma2(dnz, NRz, fma2(dny, NRy, fma2(dnx, NRx, ncn)));  // n_j . normal
      const float2 dx = add2(dcx, dnx), dy = add2(dcy, dny), dz = add2(dcz, dnz);  // n_j - bhat
      const float2 d2 = fma2(dz, dz, fma2(dy, dy, mul2(dx, dx)));
      const float2 opn = fma2(bfac, d2, one);                            // (1 - n.beta) / omb_i
      const float2 opnbn = mul2(ombn, opn);                              // -(1 - n.beta)
      const float2 na = fma2(dz, acz, fma2(dy, acy, fma2(dx, acx, ba)));  // n . a
      // V = n x ((n - beta) x a) = (n - beta)(n.a) - a (1 - n.beta)
      const float2 Vx = fma2(add2(dx, box), na, mul2(acx, opnbn));
      const float2 Vy = fma2(add2(dy, boy), na, mul2(acy, opnbn));
      const float2 Vz = fma2(add2(dz, boz), na, mul2(acz, opnbn));
      const float2 v2 = fma2(Vz, Vz, fma2(Vy, Vy, mul2(Vx, Vx)));
      const float2 o2 = mul2(opn, opn);
      const float2 o5 = mul2(mul2(o2, o2), opn);
      float2 term = mul2(mul2(mul2(v2, rinv), mul2(rinv, nd)), r5);
      term = mul2(term, f2(__fdividef(1.0f, o5.x), __fdividef(1.0f, o5.y)));
      if (directional) {  // the reference skips the terms that see the back of the surface
        term.x = nd.x > 0.0f ? term.x : 0.0f;
        term.y = nd.y > 0.0f ? term.y : 0.0f;
      }
      acc = add2(acc, term);
    }
    sum += (double)acc.x + (double)acc.y;
  }
  const double r2 = 1.0 / (omb_ref * omb_ref);
  if (active) partial[((int64_t)p * S + s) * ((int64_t)g.n1 * g.n2) + (int64_t)P.i1 * g.n2 + P.i2] = sum * (r2 * r2 / omb_ref);
}

// ---------------------------------------------------------------- power density at a list of points

// Each thread one observation point with its own normal; FP64 geometry per (point, trajectory point)
// -- R, |R| (FP32 reciprocal square root refined by two Newton steps), n and n - bhat -- and the
// rest in FP32 with the grid kernel's scaling of (1 - n.beta)^-5.
__global__ void __launch_bounds__(kThreads) pd_points_mixed_kernel(const double *__restrict__ X,
                                                                   const double *__restrict__ Bt,
                                                                   const double *__restrict__ Ac, int64_t n,
                                                                   const double *__restrict__ points,
                                                                   const double *__restrict__ normals, int64_t np,
                                                                   int directional, int64_t chunk,
                                                                   double *__restrict__ partial) {
  __shared__ double sx[3][kSub], sbh[3][kSub];
  __shared__ float sf[10][kSub];  // bhat omb (3), omb, a/c (3), |beta|/(2 omb), bhat.a, (omb_ref/omb)^5
  const int tid = threadIdx.x;
  const int64_t j = (int64_t)blockIdx.x * kThreads + tid;
  const bool active = j < np;
  const int64_t jj = active ? j : np - 1;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t off = (int64_t)p * 3 * n;
  const double *xp = X + off, *bp = Bt + off, *ap = Ac + off;
  const int64_t i0 = (int64_t)s * chunk, iend = imin64(n, i0 + chunk);
  const double Px = points[3 * jj], Py = points[3 * jj + 1], Pz = points[3 * jj + 2];
  const float nrx = (float)normals[3 * jj], nry = (float)normals[3 * jj + 1], nrz = (float)normals[3 * jj + 2];
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
      const double bx = bp[i], by = bp[n + i], bz = bp[2 * n + i];
      const double b2 = bx * bx + by * by + bz * bz, bm = sqrt(b2), ib = 1.0 / bm;
      const double omb = (1.0 - b2) / (1.0 + bm);
      const double hx = bx * ib, hy = by * ib, hz = bz * ib;
      const double ax = ap[i], ay = ap[n + i], az = ap[2 * n + i];
      const double r = omb_ref / omb;
      sx[0][tid] = xp[i]; sx[1][tid] = xp[n + i]; sx[2][tid] = xp[2 * n + i];
      sbh[0][tid] = hx; sbh[1][tid] = hy; sbh[2][tid] = hz;
      sf[0][tid] = (float)(hx * omb); sf[1][tid] = (float)(hy * omb); sf[2][tid] = (float)(hz * omb);
      sf[3][tid] = (float)omb;
      sf[4][tid] = (float)ax; sf[5][tid] = (float)ay; sf[6][tid] = (float)az;
      sf[7][tid] = (float)(0.5 * bm / omb);
      sf[8][tid] = (float)(hx * ax + hy * ay + hz * az);
      sf[9][tid] = (float)(r * r * r * r * r);
    }
    __syncthreads();
    if (!active) continue;
    float acc = 0.f;
#pragma unroll 2
    for (int k = 0; k < cnt; ++k) {
      const double Rx = Px - sx[0][k], Ry = Py - sx[1][k], Rz = Pz - sx[2][k];
      const double R2 = fma(Rx, Rx, fma(Ry, Ry, Rz * Rz));
      const float yf = rsqrtf((float)R2);
      double y = (double)yf;
      double e = fma(-R2 * y, y, 1.0);
      y = fma(0.5 * y, e, y);
      e = fma(-R2 * y, y, 1.0);
      y = fma(0.5 * y, e, y);  // 1/|R| to FP64 accuracy
      const double nx = Rx * y, ny = Ry * y, nz = Rz * y;
      const float dx = (float)(nx - sbh[0][k]), dy = (float)(ny - sbh[1][k]), dz = (float)(nz - sbh[2][k]);  // n - bhat
      const float nd = fmaf((float)nz, nrz, fmaf((float)ny, nry, (float)nx * nrx));                           // n . normal
      const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
      const float opn = fmaf(sf[7][k], d2, 1.0f);  // (1 - n.beta) / omb_i
      const float opnb = sf[3][k] * opn;           // 1 - n.beta
      const float acx = sf[4][k], acy = sf[5][k], acz = sf[6][k];
      const float na = fmaf(dz, acz, fmaf(dy, acy, fmaf(dx, acx, sf[8][k])));  // n . a
      // V = n x ((n - beta) x a) = (n - beta)(n.a) - a (1 - n.beta)
      const float Vx = fmaf(dx + sf[0][k], na, -acx * opnb), Vy = fmaf(dy + sf[1][k], na, -acy * opnb),
                  Vz = fmaf(dz + sf[2][k], na, -acz * opnb);
      const float v2 = fmaf(Vz, Vz, fmaf(Vy, Vy, Vx * Vx));
      const float o2 = opn * opn, o5 = o2 * o2 * opn;
      float term = v2 * (yf * yf) * nd * sf[9][k] * __fdividef(1.0f, o5);
      if (directional && !(nd > 0.0f)) term = 0.0f;  // the reference skips the terms that see the back
      acc += term;
    }
    sum += (double)acc;
  }
  const double r2 = 1.0 / (omb_ref * omb_ref);
  if (active) partial[((int64_t)p * S + s) * np + j] = sum * (r2 * r2 / omb_ref);
}

// ---------------------------------------------------------------- spectrum at one observer

template <int K>
__global__ void __launch_bounds__(kThreads) spectrum_mixed_kernel(const double *__restrict__ X,
                                                                  const double *__restrict__ Bt, int64_t n, double dt,
                                                                  V3 obs, const double *__restrict__ omegas, int64_t ne,
                                                                  int64_t chunk, double *__restrict__ partial) {
  __shared__ tiles::SpecShared sh;
  wait_for_previous_grid();  // (launched with launch_after by the one-shot launcher)
  allow_next_grid();
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t i0 = (int64_t)s * chunk;
  tiles::spectrum_tile<K>(X + (int64_t)p * 3 * n, Bt + (int64_t)p * 3 * n, n, dt, obs, omegas, ne, blockIdx.x, i0,
                          imin64(n, i0 + chunk), partial + ((int64_t)p * S + s) * 6 * ne, sh);
}

__global__ void omega_kernel(const double *__restrict__ e, int64_t ne, double *__restrict__ w) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) w[i] = ev_to_omega(e[i]);
}

}  // namespace

// ---------------------------------------------------------------- launchers

static int flux_mixed_splits(int64_t n, const srs_grid2d &g, int nparticles) {
  return splits_for((int64_t)strip_tiles(g).tiles * nparticles, n, 256, wave_slots(flux_mixed_kernel));
}

size_t mixed_flux_scratch_bytes(int64_t n, const srs_grid2d &g, int nparticles) {
  return sizeof(double) * 6 * (size_t)g.n1 * g.n2 * nparticles * flux_mixed_splits(n, g, nparticles);
}

static cudaError_t mixed_flux_splits(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                     double energy_ev, double *d_out, void *scratch, int S_max, cudaStream_t s) {
  const int64_t chunk = aligned_chunk(t.n, S_max);
  const int S = used_chunks(t.n, chunk);
  const StripTiles m = strip_tiles(g);
  const double omega = ev_to_omega(energy_ev);
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)m.tiles, S, t.nparticles);
  // set up while the trajectory's last kernel finishes (the kernel waits for its writes)
  cudaError_t e = launch_after(flux_mixed_kernel, grid, dim3(kThreads), 0, s, t.x, t.beta, t.n, t.dt, g, m, omega,
                               chunk, partial);
  if (e != cudaSuccess) return e;
  return finish_flux_partials(partial, S, (int64_t)g.n1 * g.n2, t.nparticles, nullptr, omega, t.dt, flux_c0(b.charge),
                              flux_c2(b.charge, b.current), d_out, s);
}

cudaError_t mixed_flux(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g, double energy_ev,
                       double *d_out, void *scratch, cudaStream_t s) {
  return mixed_flux_splits(t, b, g, energy_ev, d_out, scratch, flux_mixed_splits(t.n, g, t.nparticles), s);
}

static int flux_points_splits(int64_t n, int64_t np, int nparticles) {
  return splits_for((np + kThreads - 1) / kThreads * nparticles, n, 256, wave_slots(flux_points_mixed_kernel));
}

size_t mixed_flux_points_scratch_bytes(int64_t n, int64_t np, int nparticles) {
  return sizeof(double) * 6 * (size_t)np * nparticles * flux_points_splits(n, np, nparticles);
}

cudaError_t mixed_flux_points(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points, int64_t np,
                              double energy_ev, double *d_out, void *scratch, cudaStream_t s) {
  const int64_t chunk = aligned_chunk(t.n, flux_points_splits(t.n, np, t.nparticles));
  const int S = used_chunks(t.n, chunk);
  const double omega = ev_to_omega(energy_ev);
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)((np + kThreads - 1) / kThreads), S, t.nparticles);
  flux_points_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.n, t.dt, d_points, np, omega, chunk, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_flux_partials(partial, S, np, t.nparticles, nullptr, omega, t.dt, flux_c0(b.charge),
                              flux_c2(b.charge, b.current), d_out, s);
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
  return sizeof(double) * (size_t)g.n1 * g.n2 * nparticles *
         splits_for((int64_t)strip_tiles(g).tiles * nparticles, n, 256, wave_slots(pd_mixed_kernel));
}

cudaError_t mixed_power_density(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                int directional, double *d_out, void *scratch, cudaStream_t s) {
  const StripTiles m = strip_tiles(g);
  const int64_t chunk =
      aligned_chunk(t.n, splits_for((int64_t)m.tiles * t.nparticles, t.n, 256, wave_slots(pd_mixed_kernel)));
  const int S = used_chunks(t.n, chunk);
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)m.tiles, S, t.nparticles);
  pd_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.aoc, t.n, g, m, g.normal[0], g.normal[1], g.normal[2],
                                            directional, chunk, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_pd_partials(partial, S, (int64_t)g.n1 * g.n2, t.nparticles, pd_const(b.charge, b.current) * t.dt,
                            directional, d_out, s);
}

static int pd_points_splits(int64_t n, int64_t np, int nparticles) {
  return splits_for((np + kThreads - 1) / kThreads * nparticles, n, 256, wave_slots(pd_points_mixed_kernel));
}

size_t mixed_pd_points_scratch_bytes(int64_t n, int64_t np, int nparticles) {
  return sizeof(double) * (size_t)np * nparticles * pd_points_splits(n, np, nparticles);
}

cudaError_t mixed_power_density_points(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points,
                                       const double *d_normals, int64_t np, int directional, double *d_out,
                                       void *scratch, cudaStream_t s) {
  const int64_t chunk = aligned_chunk(t.n, pd_points_splits(t.n, np, t.nparticles));
  const int S = used_chunks(t.n, chunk);
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)((np + kThreads - 1) / kThreads), S, t.nparticles);
  pd_points_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.aoc, t.n, d_points, d_normals, np, directional,
                                                   chunk, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_pd_partials(partial, S, np, t.nparticles, pd_const(b.charge, b.current) * t.dt, directional, d_out, s);
}

// Energies per thread and trajectory chunks of a spectrum launch: kEnergiesPerThread with chunks of at
// least two sub-tiles when those CTAs fill one wave; otherwise (one observer's spectrum of a few
// thousand energies) two energies per thread and chunks down to one sub-tile, so that more CTAs share
// the work (a 1000-energy spectrum: 0.095 -> 0.083 ms per call against chunks of three sub-tiles; the
// partials, a few MB, stay in L2, and the reduction loads 24 chunks at a time).

struct SpecPlan {
  int K;
  int64_t etiles;
  int S_max;
};
static SpecPlan spectrum_plan(int64_t n, int64_t ne, int nparticles) {
  constexpr int K4 = kEnergiesPerThread;
  const int64_t slots4 = wave_slots(spectrum_mixed_kernel<K4>);
  const int64_t e4 = (ne + kThreads * K4 - 1) / (kThreads * K4);
  SpecPlan P;
  if (e4 * nparticles * std::max<int64_t>(1, n / 256) >= slots4) {
    P.K = K4;
    P.etiles = e4;
    P.S_max = splits_for(e4 * nparticles, n, 256, slots4);
  } else {
    P.K = 2;
    P.etiles = (ne + kThreads * 2 - 1) / (kThreads * 2);
    P.S_max = splits_for(P.etiles * nparticles, n, (int64_t)kSub, wave_slots(spectrum_mixed_kernel<2>));
  }
  return P;
}

size_t mixed_spectrum_scratch_bytes(int64_t n, int64_t ne, int nparticles) {
  return sizeof(double) * ((size_t)6 * ne * nparticles * spectrum_plan(n, ne, nparticles).S_max + ne);
}

cudaError_t mixed_spectrum(const srs_traj_view &t, const srs_beam_consts &b, const double obs[3],
                           const double *d_energies, int64_t ne, double *d_out, void *scratch, cudaStream_t s,
                           double *d_e6) {
  const SpecPlan plan = spectrum_plan(t.n, ne, t.nparticles);
  const int64_t etiles = plan.etiles;
  const int S_max = plan.S_max;
  const int64_t chunk = aligned_chunk(t.n, S_max);
  const int S = used_chunks(t.n, chunk);
  double *partial = static_cast<double *>(scratch);
  double *omegas = partial + (size_t)6 * ne * t.nparticles * S_max;  // after the S_max chunks sized for
  omega_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(d_energies, ne, omegas);
  dim3 grid((unsigned)etiles, S, t.nparticles);
  // set up while the angular frequencies are computed (the kernel waits for them)
  cudaError_t e = plan.K == 2 ? launch_after(spectrum_mixed_kernel<2>, grid, dim3(kThreads), 0, s, t.x, t.beta, t.n,
                                             t.dt, v3(obs[0], obs[1], obs[2]), (const double *)omegas, ne, chunk,
                                             partial)
                              : launch_after(spectrum_mixed_kernel<kEnergiesPerThread>, grid, dim3(kThreads), 0, s,
                                             t.x, t.beta, t.n, t.dt, v3(obs[0], obs[1], obs[2]),
                                             (const double *)omegas, ne, chunk, partial);
  if (e != cudaSuccess) return e;
  return finish_flux_partials(partial, S, ne, t.nparticles, omegas, 0.0, t.dt, flux_c0(b.charge),
                              flux_c2(b.charge, b.current), d_out, s, d_e6);
}

}  // namespace srs

// Plain FP64 radiation sums: the drop-in for the reference's GPU/CPU sums, in the reference's
// IEEE-double operation order (this file is compiled with -fmad=false).
//
//   spectrum  : OSCARSSR::CalculateSpectrum   src/OSCARSSR.cc:1154-1251 (energy loop :1202-1246)
//   flux      : OSCARSSR::CalculateFlux2      src/OSCARSSR.cc:1989-2099 (point loop :2054-2096)
//   power dens: OSCARSSR::CalculatePowerDensity src/OSCARSSR.cc:1477-1598 (loop :1533-1560)
//   total pow : OSCARSSR::CalculateTotalPower src/OSCARSSR.cc:1939-1978
//
// Per term the flux/spectrum integrand is (beta - n (1 + i c/(w D)))/D exp(i w (i dt + D/c)), summed
// over trajectory points; the phase w*(i*dt + D/c) is formed exactly as the reference forms it and
// reduced modulo 2*pi (Cody-Waite, three-part 2*pi, FMA) before the FP64 sincos, which is then
// evaluated on |r| <= pi.
//
// Divisions: every division of a term by the same distance D (or D^2, or (1 - n.beta)^5) is formed
// from one correctly rounded reciprocal (__drcp_rn) by Markstein's correction (div_rn), which gives
// the correctly rounded quotient, i.e. the IEEE division's result bit for bit, in three instructions
// instead of a division sequence each (normal operands: D, 1/D and the quotients of these sums are far
// from overflow and underflow).  The power density's (1 - n.beta)^5 is formed by multiplications
// (x^2 x^2 x, within two ulps of the reference's std::pow(x, 5)).
//
// Parallel layout (B200: 148 SMs): one thread per output (energy or observation point), 128 outputs
// per CTA, and the trajectory axis split into S contiguous chunks across CTAs so that small outputs
// (1000 energies) still fill every SM.  Each CTA stages its chunk through shared memory in 128-point
// tiles, read by all threads as broadcasts.  Partial complex sums go to scratch, and a second kernel
// adds the S partials in chunk order (deterministic) and applies the reference's final scaling.
#include <cuda_runtime.h>

#include <cuda_pipeline.h>

#include <algorithm>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {

namespace {

constexpr int kTile = 128;     // outputs per CTA and trajectory points per shared-memory tile

// a / b for the three components, from rb = RN(1/b)
__device__ __forceinline__ V3 div3_rn(V3 a, double b, double rb) {
  return v3(div_rn(a.x, b, rb), div_rn(a.y, b, rb), div_rn(a.z, b, rb));
}
// a / |a| (TVector3D::UnitVector), the three divisions from one reciprocal
__device__ __forceinline__ V3 unit_rn(V3 a) {
  const double m = mag(a);
  return div3_rn(a, m, __drcp_rn(m));
}
constexpr int kTargetCtas = 148 * 8;

int choose_splits(int64_t ctas_without_split, int64_t n) {
  int64_t s = (kTargetCtas + ctas_without_split - 1) / std::max<int64_t>(1, ctas_without_split);
  int64_t max_s = std::max<int64_t>(1, (n + 255) / 256);
  s = std::min<int64_t>(std::max<int64_t>(s, 1), std::min<int64_t>(max_s, 65535));
  return (int)s;
}

// ---------------------------------------------------------------- flux at observation points

__global__ void __launch_bounds__(kTile) flux_fp64_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                          int64_t n, double dt, const double *__restrict__ pts,
                                                          int64_t np, double omega, int64_t chunk,
                                                          double *__restrict__ partial) {
  __shared__ double sx[3][kTile], sb[3][kTile];
  const int tid = threadIdx.x;
  const int64_t j = (int64_t)blockIdx.x * kTile + tid;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const double *xp = X + (int64_t)p * 3 * n, *bp = Bt + (int64_t)p * 3 * n;
  const int64_t i0 = (int64_t)s * chunk, i1 = imin64(n, i0 + chunk);
  const bool active = j < np;
  V3 obs = active ? v3(pts[3 * j], pts[3 * j + 1], pts[3 * j + 2]) : v3(0, 0, 1);
  const double icow = kC / omega, rc = 1.0 / kC;
  double axr = 0, axi = 0, ayr = 0, ayi = 0, azr = 0, azi = 0;
  for (int64_t base = i0; base < i1; base += kTile) {
    const int cnt = (int)imin64(kTile, i1 - base);
    __syncthreads();
    if (tid < cnt) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sx[c][tid] = xp[c * n + base + tid];
        sb[c][tid] = bp[c * n + base + tid];
      }
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < cnt; ++k) {
      V3 R = obs - v3(sx[0][k], sx[1][k], sx[2][k]);
      double m = mag(R);
      const double rm = __drcp_rn(m);
      V3 N = div3_rn(R, m, rm);
      double ph = omega * (dt * (double)(int)(base + k) + div_rn(m, kC, rc));
      double sn, cs;
      sincos(reduce_2pi(ph), &sn, &cs);
      double f = div_rn(icow, m, rm);
      double ar, ai;
      ar = div_rn(sb[0][k] - N.x, m, rm); ai = div_rn(-(N.x * f), m, rm);
      axr += ar * cs - ai * sn; axi += ar * sn + ai * cs;
      ar = div_rn(sb[1][k] - N.y, m, rm); ai = div_rn(-(N.y * f), m, rm);
      ayr += ar * cs - ai * sn; ayi += ar * sn + ai * cs;
      ar = div_rn(sb[2][k] - N.z, m, rm); ai = div_rn(-(N.z * f), m, rm);
      azr += ar * cs - ai * sn; azi += ar * sn + ai * cs;
    }
  }
  if (active) {
    double *o = partial + ((int64_t)p * S + s) * 6 * np + j;
    o[0] = axr; o[np] = axi; o[2 * np] = ayr; o[3 * np] = ayi; o[4 * np] = azr; o[5 * np] = azi;
  }
}


// Block of kRedPoints x 6 threads: thread (c, k) adds component c of point j = block * kRedPoints + k
// over the S chunks in chunk order, then one thread per point applies the final scaling.  The loads of
// kRedBatch chunks are issued together as asynchronous copies into the thread's own shared-memory
// slots, so that a launch of a few thousand threads waits for memory once per kRedBatch chunks; the
// adds stay in chunk order (config 0's spectrum: 53 chunks, 6000 threads).
constexpr int kRedPoints = 32;
constexpr int kRedBatch = 24;
__global__ void __launch_bounds__(6 * kRedPoints) flux_fp64_reduce(const double *__restrict__ partial, int S,
                                                                   int64_t np, int nparticles,
                                                                   const double *__restrict__ omegas, double omega0,
                                                                   double dt, double C0, double C2,
                                                                   double *__restrict__ out, double *__restrict__ e6) {
  __shared__ double se[kRedPoints][7];
  __shared__ double sbuf[kRedBatch][6 * kRedPoints];  // [chunk in batch][thread]
  wait_for_previous_grid();  // (launched with launch_after by finish_flux_partials)
  const int k = threadIdx.x % kRedPoints, c = threadIdx.x / kRedPoints;
  const int64_t idx = (int64_t)blockIdx.x * kRedPoints + k;
  const bool valid = idx < np * nparticles;
  if (valid) {
    const int64_t p = idx / np, j = idx % np;
    const double *o = partial + (int64_t)p * S * 6 * np + c * np + j;
    const int64_t stride = 6 * np;
    double e = 0;
    int s = 0;
    double *const mine = &sbuf[0][threadIdx.x];
    for (; s < S; s += kRedBatch, o += kRedBatch * stride) {
      const int m = S - s < kRedBatch ? S - s : kRedBatch;
      for (int u = 0; u < m; ++u) __pipeline_memcpy_async(mine + u * 6 * kRedPoints, o + u * stride, sizeof(double));
      __pipeline_commit();
      __pipeline_wait_prior(0);
      for (int u = 0; u < m; ++u) e += mine[u * 6 * kRedPoints];
    }
    se[k][c] = e;
  }
  __syncthreads();
  if (c == 0 && valid) {
    double e[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) e[q] = se[k][q];
    const double omega = omegas ? omegas[idx % np] : omega0;
    out[idx] = finish_flux(e, omega, dt, C0, C2);
    if (e6) {
#pragma unroll
      for (int q = 0; q < 6; ++q) e6[6 * idx + q] = e[q];
    }
  }
}

// ---------------------------------------------------------------- spectrum at one observer

__global__ void __launch_bounds__(kTile) spectrum_fp64_kernel(const double *__restrict__ X,
                                                              const double *__restrict__ Bt, int64_t n, double dt,
                                                              V3 obs, const double *__restrict__ energies,
                                                              int64_t ne, int64_t chunk,
                                                              double *__restrict__ partial) {
  // Per trajectory point (energy independent): n = R/|R|, D, tau = i*dt + D/c, (beta - n)/D.
  __shared__ double sN[3][kTile], sD[kTile], sR[kTile], sT[kTile], sA[3][kTile];
  const int tid = threadIdx.x;
  const int64_t k = (int64_t)blockIdx.x * kTile + tid;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const double *xp = X + (int64_t)p * 3 * n, *bp = Bt + (int64_t)p * 3 * n;
  const int64_t i0 = (int64_t)s * chunk, i1 = imin64(n, i0 + chunk);
  const bool active = k < ne;
  const double omega = active ? ev_to_omega(energies[k]) : 1.0;
  const double icow = kC / omega;
  double axr = 0, axi = 0, ayr = 0, ayi = 0, azr = 0, azi = 0;
  for (int64_t base = i0; base < i1; base += kTile) {
    const int cnt = (int)imin64(kTile, i1 - base);
    __syncthreads();
    if (tid < cnt) {
      const int64_t i = base + tid;
      V3 R = obs - v3(xp[i], xp[n + i], xp[2 * n + i]);
      double m = mag(R);
      const double rm = __drcp_rn(m);
      V3 N = div3_rn(R, m, rm);
      sN[0][tid] = N.x; sN[1][tid] = N.y; sN[2][tid] = N.z;
      sD[tid] = m;
      sR[tid] = rm;
      sT[tid] = dt * (double)(int)i + div_rn(m, kC, 1.0 / kC);
      sA[0][tid] = div_rn(bp[i] - N.x, m, rm);
      sA[1][tid] = div_rn(bp[n + i] - N.y, m, rm);
      sA[2][tid] = div_rn(bp[2 * n + i] - N.z, m, rm);
    }
    __syncthreads();
    if (!active) continue;
    for (int q = 0; q < cnt; ++q) {
      const double m = sD[q], rm = sR[q];
      double sn, cs;
      sincos(reduce_2pi(omega * sT[q]), &sn, &cs);
      const double f = div_rn(icow, m, rm);
      double ar, ai;
      ar = sA[0][q]; ai = div_rn(-(sN[0][q] * f), m, rm);
      axr += ar * cs - ai * sn; axi += ar * sn + ai * cs;
      ar = sA[1][q]; ai = div_rn(-(sN[1][q] * f), m, rm);
      ayr += ar * cs - ai * sn; ayi += ar * sn + ai * cs;
      ar = sA[2][q]; ai = div_rn(-(sN[2][q] * f), m, rm);
      azr += ar * cs - ai * sn; azi += ar * sn + ai * cs;
    }
  }
  if (active) {
    double *o = partial + ((int64_t)p * S + s) * 6 * ne + k;
    o[0] = axr; o[ne] = axi; o[2 * ne] = ayr; o[3 * ne] = ayi; o[4 * ne] = azr; o[5 * ne] = azi;
  }
}

__global__ void omegas_kernel(const double *__restrict__ e, int64_t ne, double *__restrict__ w) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) w[i] = ev_to_omega(e[i]);
}

// ---------------------------------------------------------------- power density

__global__ void __launch_bounds__(kTile) pd_fp64_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                        const double *__restrict__ A, int64_t n,
                                                        const double *__restrict__ pts,
                                                        const double *__restrict__ nrms, int64_t np,
                                                        int directional, int64_t chunk,
                                                        double *__restrict__ partial) {
  __shared__ double sx[3][kTile], sb[3][kTile], sa[3][kTile];
  const int tid = threadIdx.x;
  const int64_t j = (int64_t)blockIdx.x * kTile + tid;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t off = (int64_t)p * 3 * n;
  const int64_t i0 = (int64_t)s * chunk, i1 = imin64(n, i0 + chunk);
  const bool active = j < np;
  V3 obs = active ? v3(pts[3 * j], pts[3 * j + 1], pts[3 * j + 2]) : v3(0, 0, 1);
  V3 nrm = active ? v3(nrms[3 * j], nrms[3 * j + 1], nrms[3 * j + 2]) : v3(0, 0, 1);
  double sum = 0;
  for (int64_t base = i0; base < i1; base += kTile) {
    const int cnt = (int)imin64(kTile, i1 - base);
    __syncthreads();
    if (tid < cnt) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        sx[c][tid] = X[off + c * n + base + tid];
        sb[c][tid] = Bt[off + c * n + base + tid];
        sa[c][tid] = A[off + c * n + base + tid];
      }
    }
    __syncthreads();
    if (!active) continue;
    for (int k = 0; k < cnt; ++k) {
      const V3 Xk = v3(sx[0][k], sx[1][k], sx[2][k]);
      const V3 B = v3(sb[0][k], sb[1][k], sb[2][k]);
      const V3 AC = v3(sa[0][k], sa[1][k], sa[2][k]);
      const V3 N1 = unit_rn(obs - Xk);
      const V3 N2 = unit_rn(orthogonal(N1));
      const V3 N3 = unit_rn(cross(N1, N2));
      const double nd = dot(N1, nrm);
      if (directional && nd <= 0) continue;
      const V3 num = cross(N1, cross(N1 - B, AC));
      const double omb = 1 - dot(B, N1), omb2 = omb * omb;
      const double den = omb2 * omb2 * omb;
      const double p2 = dot(num, N2), p3 = dot(num, N3);
      const double m2 = mag2(obs - Xk);
      const double rden = __drcp_rn(den), rm2 = __drcp_rn(m2);
      sum += div_rn(div_rn(p2 * p2, den, rden), m2, rm2) * nd;
      sum += div_rn(div_rn(p3 * p3, den, rden), m2, rm2) * nd;
    }
  }
  if (active) partial[((int64_t)p * S + s) * np + j] = sum;
}

__global__ void pd_fp64_reduce(const double *__restrict__ partial, int S, int64_t np, int nparticles, double cdt,
                               int directional, double *__restrict__ out) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= np * nparticles) return;
  const int64_t p = idx / np, j = idx % np;
  double sum = 0;
  const double *o = partial + (int64_t)p * S * np + j;
  int s = 0;
  for (; s + 8 <= S; s += 8, o += 8 * np) {  // chunk order, eight chunks' loads in flight at a time
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) v[u] = o[u * np];
#pragma unroll
    for (int u = 0; u < 8; ++u) sum += v[u];
  }
  for (; s < S; ++s, o += np) sum += *o;
  sum *= cdt;
  sum /= 1e6;
  if (!directional && sum < 0) sum *= -1;
  out[idx] = sum;
}

// ---------------------------------------------------------------- total power and accumulation

__global__ void total_power_kernel(const double *__restrict__ Bt, const double *__restrict__ A, int64_t n,
                                   int nparticles, double dt, double qi, const double *__restrict__ gamma,
                                   double *__restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nparticles) return;
  const double *bp = Bt + (int64_t)p * 3 * n, *ap = A + (int64_t)p * 3 * n;
  double tp = 0;
  for (int64_t i = 0; i < n; ++i) {
    V3 B = v3(bp[i], bp[n + i], bp[2 * n + i]), AC = v3(ap[i], ap[n + i], ap[2 * n + i]);
    tp += (mag2(AC) - mag2(cross(B, AC))) * dt;
  }
  tp *= fabs(qi) * pow(gamma[p], 6.0) / (6 * kPi * kEps0 * kC);
  out[p] = tp;
}

// The Lienard-Wiechert field of the trajectory point i at the observer and its arrival time
// (OSCARSSR::CalculateElectricFieldTimeDomain, OSCARSSR.cc:2646-2690; Duke, Synchrotron Radiation, p74):
//   E = q/(4 pi eps0) (1/(1 - n.beta))^3 [ (1 - beta^2)(n - beta)/R^2 + (1/c) n x ((n - beta) x a/c)/R ],
//   t = i dt + R/c, in the reference's vector operation order.
__global__ void efield_time_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                   const double *__restrict__ A, int64_t n, double dt, V3 obs, double C0,
                                   double *__restrict__ out_t, double *__restrict__ out_e) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const V3 x = v3(X[i], X[n + i], X[2 * n + i]);
  const V3 b = v3(Bt[i], Bt[n + i], Bt[2 * n + i]);
  const V3 ac = v3(A[i], A[n + i], A[2 * n + i]);
  const V3 R = obs - x;
  const double Rm = mag(R);
  const V3 N = R / Rm;  // TVector3D::UnitVector
  const double D = Rm;
  const double Mult = C0 * pow(1.0 / (1.0 - dot(N, b)), 3.0);
  const V3 nb = N - b;
  const double s1 = 1.0 - mag2(b);
  const V3 near = v3(s1 * nb.x, s1 * nb.y, s1 * nb.z) / mag2(R);
  const V3 c = cross(N, cross(nb, ac));
  const double ic = 1.0 / kC;
  const V3 far = v3(ic * c.x, ic * c.y, ic * c.z) / mag(R);
  const V3 sum = near + far;
  out_e[3 * i] = Mult * sum.x;
  out_e[3 * i + 1] = Mult * sum.y;
  out_e[3 * i + 2] = Mult * sum.z;
  out_t[i] = (double)i * dt + D / kC;
}

// Kahan accumulation over particles in order: T3DScalarContainer::AddToPoint (T3DScalarContainer.cc:31-47)
__global__ void accumulate_kernel(const double *__restrict__ vals, int nparticles, int64_t nout, double w,
                                  double *__restrict__ out, double *__restrict__ comp) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nout) return;
  double sum = out[j], c = comp[j];
  for (int p = 0; p < nparticles; ++p) {
    const double v = vals[(int64_t)p * nout + j] * w;
    const double y = v - c, t = sum + y;
    c = (t - sum) - y;
    sum = t;
  }
  out[j] = sum;
  comp[j] = c;
}

inline unsigned blocks_for(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

// ---------------------------------------------------------------- launchers

static int flux_splits(int64_t n, int64_t nout, int nparticles) {
  return choose_splits(((nout + kTile - 1) / kTile) * nparticles, n);
}

size_t fp64_flux_scratch_bytes(int64_t n, int64_t np, int nparticles) {
  return sizeof(double) * 6 * (size_t)np * nparticles * flux_splits(n, np, nparticles);
}

cudaError_t fp64_flux(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points, int64_t np,
                      double energy_ev, double *d_out, void *scratch, cudaStream_t s) {
  if (np <= 0 || t.nparticles <= 0) return cudaSuccess;
  const int S = flux_splits(t.n, np, t.nparticles);
  const int64_t chunk = (t.n + S - 1) / S;
  const double omega = ev_to_omega(energy_ev);
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)((np + kTile - 1) / kTile), S, t.nparticles);
  flux_fp64_kernel<<<grid, kTile, 0, s>>>(t.x, t.beta, t.n, t.dt, d_points, np, omega, chunk, partial);
  flux_fp64_reduce<<<blocks_for(np * t.nparticles, kRedPoints), 6 * kRedPoints, 0, s>>>(partial, S, np, t.nparticles, nullptr, omega,
                                                                      t.dt, flux_c0(b.charge),
                                                                      flux_c2(b.charge, b.current), d_out, nullptr);
  return cudaGetLastError();
}

size_t fp64_spectrum_scratch_bytes(int64_t n, int64_t ne, int nparticles) {
  return sizeof(double) * ((size_t)6 * ne * nparticles * flux_splits(n, ne, nparticles) + (size_t)ne);
}

cudaError_t fp64_spectrum(const srs_traj_view &t, const srs_beam_consts &b, const double obs[3],
                          const double *d_energies, int64_t ne, double *d_out, void *scratch, cudaStream_t s,
                          double *d_e6) {
  if (ne <= 0 || t.nparticles <= 0) return cudaSuccess;
  const int S = flux_splits(t.n, ne, t.nparticles);
  const int64_t chunk = (t.n + S - 1) / S;
  double *partial = static_cast<double *>(scratch);
  double *omegas = partial + (size_t)6 * ne * t.nparticles * S;
  dim3 grid((unsigned)((ne + kTile - 1) / kTile), S, t.nparticles);
  spectrum_fp64_kernel<<<grid, kTile, 0, s>>>(t.x, t.beta, t.n, t.dt, v3(obs[0], obs[1], obs[2]), d_energies, ne,
                                              chunk, partial);
  omegas_kernel<<<blocks_for(ne, 256), 256, 0, s>>>(d_energies, ne, omegas);
  flux_fp64_reduce<<<blocks_for(ne * t.nparticles, kRedPoints), 6 * kRedPoints, 0, s>>>(partial, S, ne, t.nparticles, omegas, 0.0,
                                                                      t.dt, flux_c0(b.charge),
                                                                      flux_c2(b.charge, b.current), d_out, d_e6);
  return cudaGetLastError();
}

size_t fp64_pd_scratch_bytes(int64_t n, int64_t np, int nparticles) {
  return sizeof(double) * (size_t)np * nparticles * flux_splits(n, np, nparticles);
}

cudaError_t fp64_power_density(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points,
                               const double *d_normals, int64_t np, int directional, double *d_out, void *scratch,
                               cudaStream_t s) {
  if (np <= 0 || t.nparticles <= 0) return cudaSuccess;
  const int S = flux_splits(t.n, np, t.nparticles);
  const int64_t chunk = (t.n + S - 1) / S;
  double *partial = static_cast<double *>(scratch);
  dim3 grid((unsigned)((np + kTile - 1) / kTile), S, t.nparticles);
  pd_fp64_kernel<<<grid, kTile, 0, s>>>(t.x, t.beta, t.aoc, t.n, d_points, d_normals, np, directional, chunk,
                                        partial);
  const double cdt = pd_const(b.charge, b.current) * t.dt;
  pd_fp64_reduce<<<blocks_for(np * t.nparticles, 256), 256, 0, s>>>(partial, S, np, t.nparticles, cdt, directional,
                                                                    d_out);
  return cudaGetLastError();
}

cudaError_t total_power(const srs_traj_view &t, const srs_beam_consts &b, const double *d_gamma, double *d_out,
                        cudaStream_t s) {
  if (t.nparticles <= 0) return cudaSuccess;
  total_power_kernel<<<blocks_for(t.nparticles, 64), 64, 0, s>>>(t.beta, t.aoc, t.n, t.nparticles, t.dt,
                                                                  b.charge * b.current, d_gamma, d_out);
  return cudaGetLastError();
}

cudaError_t finish_flux_partials(const double *partial, int S, int64_t nout, int nparticles, const double *omegas,
                                 double omega0, double dt, double C0, double C2, double *out, cudaStream_t s,
                                 double *e6) {
  // set up while the sums that wrote the partials finish (the kernel waits for their writes)
  return launch_after(flux_fp64_reduce, dim3((unsigned)blocks_for(nout * nparticles, kRedPoints)),
                      dim3(6 * kRedPoints), 0, s, partial, S, nout, nparticles, omegas, omega0, dt, C0, C2, out, e6);
}

cudaError_t finish_pd_partials(const double *partial, int S, int64_t np, int nparticles, double cdt, int directional,
                               double *out, cudaStream_t s) {
  pd_fp64_reduce<<<blocks_for(np * nparticles, 128), 128, 0, s>>>(partial, S, np, nparticles, cdt, directional, out);
  return cudaGetLastError();
}

cudaError_t accumulate_particles(const double *d_vals, int nparticles, int64_t nout, double weight, double *d_out,
                                 double *d_comp, cudaStream_t s) {
  if (nout <= 0) return cudaSuccess;
  accumulate_kernel<<<blocks_for(nout, 256), 256, 0, s>>>(d_vals, nparticles, nout, weight, d_out, d_comp);
  return cudaGetLastError();
}

cudaError_t efield_time(const srs_traj_view &t, double charge, const double obs[3], double *d_t, double *d_e,
                        cudaStream_t s) {
  if (t.n <= 0) return cudaSuccess;
  const double C0 = charge / (four_pi() * kEps0);  // OSCARSSR.cc:2662
  efield_time_kernel<<<(unsigned)((t.n + 127) / 128), 128, 0, s>>>(t.x, t.beta, t.aoc, t.n, t.dt, ld3(obs), C0, d_t,
                                                                    d_e);
  return cudaGetLastError();
}

}  // namespace srs

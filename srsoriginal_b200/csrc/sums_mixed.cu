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

#include "mixed_tiles.cuh"
#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {

using namespace tiles;

namespace {

// ---------------------------------------------------------------- flux on a grid

__global__ void __launch_bounds__(kThreads) flux_mixed_kernel(const double *__restrict__ X, const double *__restrict__ Bt,
                                                              int64_t n, double dt, srs_grid2d g, double omega,
                                                              int64_t chunk, double *__restrict__ partial) {
  __shared__ tiles::FluxShared sh;
  const int nt2 = (g.n2 + kTileB - 1) / kTileB;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t np = (int64_t)g.n1 * g.n2;
  const int64_t i0 = (int64_t)s * chunk;
  tiles::flux_tile(X + (int64_t)p * 3 * n, Bt + (int64_t)p * 3 * n, n, dt, g, omega, blockIdx.x / nt2,
                   blockIdx.x % nt2, i0, imin64(n, i0 + chunk), partial + ((int64_t)p * S + s) * 6 * np, sh);
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

__global__ void __launch_bounds__(kThreads) spectrum_mixed_kernel(const double *__restrict__ X,
                                                                  const double *__restrict__ Bt, int64_t n, double dt,
                                                                  V3 obs, const double *__restrict__ omegas, int64_t ne,
                                                                  int64_t chunk, double *__restrict__ partial) {
  __shared__ tiles::SpecShared sh;
  const int s = blockIdx.y, S = gridDim.y, p = blockIdx.z;
  const int64_t i0 = (int64_t)s * chunk;
  tiles::spectrum_tile(X + (int64_t)p * 3 * n, Bt + (int64_t)p * 3 * n, n, dt, obs, omegas, ne, blockIdx.x, i0,
                       imin64(n, i0 + chunk), partial + ((int64_t)p * S + s) * 6 * ne, sh);
}

__global__ void omega_kernel(const double *__restrict__ e, int64_t ne, double *__restrict__ w) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) w[i] = ev_to_omega(e[i]);
}

}  // namespace

// ---------------------------------------------------------------- launchers

static int flux_mixed_splits(int64_t n, const srs_grid2d &g, int nparticles) {
  GridTiles t = tiles_of(g);
  return splits_for((int64_t)t.t1 * t.t2 * nparticles, n, 256, wave_slots(flux_mixed_kernel));
}

size_t mixed_flux_scratch_bytes(int64_t n, const srs_grid2d &g, int nparticles) {
  return sizeof(double) * 6 * (size_t)g.n1 * g.n2 * nparticles * flux_mixed_splits(n, g, nparticles);
}

static cudaError_t mixed_flux_splits(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                     double energy_ev, double *d_out, void *scratch, int S_max, cudaStream_t s) {
  const int64_t chunk = aligned_chunk(t.n, S_max);
  const int S = used_chunks(t.n, chunk);
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
         splits_for((int64_t)tl.t1 * tl.t2 * nparticles, n, 256, wave_slots(pd_mixed_kernel));
}

cudaError_t mixed_power_density(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                int directional, double *d_out, void *scratch, cudaStream_t s) {
  GridTiles tl = tiles_of(g);
  const int64_t chunk =
      aligned_chunk(t.n, splits_for((int64_t)tl.t1 * tl.t2 * t.nparticles, t.n, 256, wave_slots(pd_mixed_kernel)));
  const int S = used_chunks(t.n, chunk);
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
  return sizeof(double) * ((size_t)6 * ne * nparticles * splits_for(ctas, n, 256, wave_slots(spectrum_mixed_kernel)) + ne);
}

cudaError_t mixed_spectrum(const srs_traj_view &t, const srs_beam_consts &b, const double obs[3],
                           const double *d_energies, int64_t ne, double *d_out, void *scratch, cudaStream_t s,
                           double *d_e6) {
  const int64_t etiles = (ne + kThreads * kEnergiesPerThread - 1) / (kThreads * kEnergiesPerThread);
  const int S_max = splits_for(etiles * t.nparticles, t.n, 256, wave_slots(spectrum_mixed_kernel));
  const int64_t chunk = aligned_chunk(t.n, S_max);
  const int S = used_chunks(t.n, chunk);
  double *partial = static_cast<double *>(scratch);
  double *omegas = partial + (size_t)6 * ne * t.nparticles * S_max;  // after the S_max chunks sized for
  omega_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(d_energies, ne, omegas);
  dim3 grid((unsigned)etiles, S, t.nparticles);
  spectrum_mixed_kernel<<<grid, kThreads, 0, s>>>(t.x, t.beta, t.n, t.dt, v3(obs[0], obs[1], obs[2]), omegas, ne,
                                                  chunk, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return finish_flux_partials(partial, S, ne, t.nparticles, omegas, 0.0, t.dt, flux_c0(b.charge),
                              flux_c2(b.charge, b.current), d_out, s, d_e6);
}

}  // namespace srs

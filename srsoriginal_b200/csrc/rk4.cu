// Fixed-step RK4 electron trajectories, one CUDA thread per particle (compiled with -fmad=false so
// every operation rounds like the reference's x86-64 build).
//
// Reference: OSCARSSR::CalculateTrajectory (src/OSCARSSR.cc:562-673), DerivativesB (:741-765),
// RK4 (:826-874).  State (x, vx, y, vy, z, vz) in m and m/s; dv/dt = (q/(m gamma)) v x B with gamma
// fixed.  Forward from t0 for nforward points, then backward for nbackward points; the stored a/c at
// a point is the derivative evaluated at the state of the previous step (the first forward point
// stores 0, which the reference reads from an uninitialised array).
//
// Layout written: [particle][component][point], point index = time order (the backward points come
// first, earliest at index 0), so no reversal pass is needed.
#include <cuda_runtime.h>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {

namespace {

constexpr int kMaxFieldsShared = 16;

__device__ inline void derivs(const srs_field *fields, int nf, const double x[6], double d[6], double qomg) {
  V3 B = field_sum(fields, nf, v3(x[0], x[2], x[4]));
  d[0] = x[1];
  d[1] = qomg * (-x[5] * B.y + x[3] * B.z);
  d[2] = x[3];
  d[3] = qomg * (x[5] * B.x - x[1] * B.z);
  d[4] = x[5];
  d[5] = qomg * (x[1] * B.y - x[3] * B.x);
}

__device__ inline void rk4_step(const srs_field *fields, int nf, double y[6], const double dydx[6], double h,
                                double qomg) {
  double dym[6], dyt[6], yt[6];
  const double hh = h * 0.5, h6 = h / 6.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dydx[i];
  derivs(fields, nf, yt, dyt, qomg);
#pragma unroll
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
  derivs(fields, nf, yt, dym, qomg);
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    yt[i] = y[i] + h * dym[i];
    dym[i] += dyt[i];
  }
  derivs(fields, nf, yt, dyt, qomg);
#pragma unroll
  for (int i = 0; i < 6; ++i) y[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
}

__global__ void rk4_kernel(const srs_field *__restrict__ gfields, int nfields,
                           const srs_particle *__restrict__ particles, int nparticles, double dt,
                           int64_t nfwd, int64_t nbwd, double *__restrict__ X, double *__restrict__ Bt,
                           double *__restrict__ A) {
  __shared__ srs_field sf[kMaxFieldsShared];
  const srs_field *fields = gfields;
  if (nfields <= kMaxFieldsShared) {
    for (int i = threadIdx.x; i < nfields; i += blockDim.x) sf[i] = gfields[i];
    __syncthreads();
    fields = sf;
  }
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nparticles) return;
  const srs_particle P = particles[p];
  const int64_t n = nfwd + nbwd;
  double *xp = X + (int64_t)p * 3 * n, *bp = Bt + (int64_t)p * 3 * n, *ap = A + (int64_t)p * 3 * n;
  const double C = kC;
  double x[6] = {P.x0[0], P.beta0[0] * C, P.x0[1], P.beta0[1] * C, P.x0[2], P.beta0[2] * C};
  double d[6] = {0, 0, 0, 0, 0, 0};
  auto store = [&](int64_t k) {
    xp[k] = x[0];
    xp[n + k] = x[2];
    xp[2 * n + k] = x[4];
    bp[k] = x[1] / C;
    bp[n + k] = x[3] / C;
    bp[2 * n + k] = x[5] / C;
    ap[k] = d[1] / C;
    ap[n + k] = d[3] / C;
    ap[2 * n + k] = d[5] / C;
  };
  x[0] = P.x0[0]; x[1] = P.beta0[0] * C; x[2] = P.x0[1]; x[3] = P.beta0[1] * C; x[4] = P.x0[2]; x[5] = P.beta0[2] * C;
  for (int64_t i = 0; i < nfwd; ++i) {
    store(nbwd + i);
    derivs(fields, nfields, x, d, P.qomg);
    rk4_step(fields, nfields, x, d, dt, P.qomg);
  }
  x[0] = P.x0[0]; x[1] = P.beta0[0] * C; x[2] = P.x0[1]; x[3] = P.beta0[1] * C; x[4] = P.x0[2]; x[5] = P.beta0[2] * C;
  const double mdt = -dt;
  for (int64_t i = 0; i < nbwd; ++i) {
    derivs(fields, nfields, x, d, P.qomg);
    rk4_step(fields, nfields, x, d, mdt, P.qomg);
    store(nbwd - 1 - i);
  }
}

__global__ void field_eval_kernel(const srs_field *__restrict__ fields, int nfields, const double *__restrict__ xyz,
                                  int64_t np, double *__restrict__ out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  V3 b = field_sum(fields, nfields, v3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
  out[3 * i] = b.x;
  out[3 * i + 1] = b.y;
  out[3 * i + 2] = b.z;
}

}  // namespace

cudaError_t launch_rk4(const srs_field *d_fields, int nfields, const srs_particle *d_particles, int nparticles,
                       double dt, int64_t nfwd, int64_t nbwd, double *d_x, double *d_b, double *d_a,
                       cudaStream_t s) {
  if (nparticles <= 0) return cudaSuccess;
  // Small blocks: a latency-bound serial loop per thread; spread particles over all SMs.
  const int threads = nparticles >= 148 * 64 ? 64 : 32;
  const int blocks = (nparticles + threads - 1) / threads;
  rk4_kernel<<<blocks, threads, 0, s>>>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a);
  return cudaGetLastError();
}

cudaError_t launch_field_eval(const srs_field *d_fields, int nfields, const double *d_xyz, int64_t np,
                              double *d_out, cudaStream_t s) {
  if (np <= 0) return cudaSuccess;
  const int threads = 128;
  field_eval_kernel<<<(unsigned)((np + threads - 1) / threads), threads, 0, s>>>(d_fields, nfields, d_xyz, np, d_out);
  return cudaGetLastError();
}

}  // namespace srs

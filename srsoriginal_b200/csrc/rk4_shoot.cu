// Parallel-in-time RK4 for one long trajectory: multiple shooting with Newton updates (compiled with
// -fmad=false; the steps are those of the serial kernels, rk4_fields.cuh).
//
// The serial chain of N RK4 steps costs ~0.9 us per step of latency on one SM, whatever the GPU's
// width.  Here the chain (each of the reference's two chains: forward from t0 with +dt, backward with
// -dt; OSCARSSR.cc:562-673) is cut into S segments of L steps.  Unknowns: the start state U_n of every
// segment (U_0 = the initial state, fixed).  One iteration is
//   (1) shoot_fine_kernel: every segment runs its L steps from U_n, all segments at once, and pushes
//       the six unit tangents of its start state along (eight lanes per segment: lane j carries
//       tangent j), giving the end state F_n(U_n) and the segment's 6 x 6 Jacobian Phi_n;
//   (2) shoot_update_kernel: one warp per chain sweeps the segments in order with Newton's update of
//       the matching conditions U_{n+1} = F_n(U_n):  U'_{n+1} = F_n(U_n) + Phi_n (U'_n - U_n).
// U'_{n+1} = F_n(U_n) holds exactly whenever U'_n = U_n, so after k iterations the first k segments
// start from the serial chain's exact states, and Newton's quadratic convergence brings all the others
// there up to the ulps by which a start state one ulp away rounds differently.  The iteration stops
// when the largest update is below the tolerance; every segment then integrates its points from its
// start state and stores them (shoot_store_kernel), the stored a/c lagged by one step as in the
// serial kernels.  When the iteration has not converged after its iteration limit (8 unless the caller
// sets one), the serial kernel runs instead (it exits at once otherwise): the sequence of launches
// needs no host synchronisation.
// Initial guess: straight flight from the initial state.
//
// The stored trajectory equals the serial one to ~1e-16 m (not bit for bit); the FP64 drop-in path
// keeps the serial kernel.
#include <cuda_runtime.h>

#include "rk4_fields.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

constexpr int kSegLanes = 8;   // lanes per segment: six tangents, two spare lanes (primal only)
constexpr int kFineThreads = 64;
constexpr int kMaxIters = 32;     // capacity of the per-iteration record
constexpr int kDefaultIters = 8;
// convergence: every update below 2^-48 of the trajectory's scale (position: its extent; velocity: |v0|)
constexpr double kTol = 3.552713678800501e-15;

// Segments: forward chain first (steps 0 .. mf-1 of +dt), then the backward chain (steps 0 .. mb-1
// of -dt), L steps each (the last of a chain shorter).
struct Plan {
  int64_t mf, mb;  // steps of each chain
  int sf, sb;      // segments of each chain
  int L;           // steps per segment
  double dt;
  int64_t nfwd, nbwd, n;  // stored points from t0 on, before t0; points per trajectory component
};

__device__ inline void seg_of(const Plan &P, int g, int &chain, int64_t &j0, int &len, double &h) {
  chain = g < P.sf ? 0 : 1;
  const int local = chain == 0 ? g : g - P.sf;
  const int64_t m = chain == 0 ? P.mf : P.mb;
  j0 = (int64_t)local * P.L;
  len = (int)imin64(P.L, m - j0);
  h = chain == 0 ? P.dt : -P.dt;
}

__device__ inline void load_fields(const srs_field *gfields, int nfields, srs_field *sf, Prepared *sp,
                                   int64_t stage_doubles) {
  for (int i = threadIdx.x; i < nfields; i += blockDim.x) {
    sf[i] = gfields[i];
    prepare(sf[i], sp[i]);
  }
  __syncthreads();
  if (stage_doubles > 0) stage_grids(sf, sp, nfields);
}

// flags[0]: converged; flags[1]: iterations run.  stats: [converged, iterations, last update, defect]
__global__ void shoot_init_kernel(Plan P, const srs_particle *__restrict__ part, double *__restrict__ U,
                                  int *__restrict__ flags, double *__restrict__ diag) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g == 0) {
    flags[0] = 0;
    flags[1] = 0;
    for (int k = 0; k < kMaxIters + 1; ++k) diag[k] = 0.0;
  }
  if (g >= P.sf + P.sb) return;
  int chain, len;
  int64_t j0;
  double h;
  seg_of(P, g, chain, j0, len, h);
  const double C = kC, t = (double)j0 * h;
  const double v[3] = {part->beta0[0] * C, part->beta0[1] * C, part->beta0[2] * C};
  for (int c = 0; c < 3; ++c) {
    U[6 * g + c] = j0 == 0 ? part->x0[c] : part->x0[c] + v[c] * t;
    U[6 * g + 3 + c] = v[c];
  }
}

__global__ void __launch_bounds__(kFineThreads) shoot_fine_kernel(const srs_field *__restrict__ gfields, int nfields,
                                                                  const srs_particle *__restrict__ part, Plan P,
                                                                  const double *__restrict__ U, double *__restrict__ F,
                                                                  double *__restrict__ Phi, const int *__restrict__ flags,
                                                                  int64_t stage_doubles) {
  if (flags[0]) return;  // converged: nothing left to do (uniform over the grid)
  __shared__ srs_field sf[kMaxFieldsShared];
  __shared__ Prepared sp[kMaxFieldsShared];
  load_fields(gfields, nfields, sf, sp, stage_doubles);
  const int g = blockIdx.x * (kFineThreads / kSegLanes) + threadIdx.x / kSegLanes;
  const int j = threadIdx.x % kSegLanes;
  if (g >= P.sf + P.sb) return;
  int chain, len;
  int64_t j0;
  double h;
  seg_of(P, g, chain, j0, len, h);
  const double qomg = part->qomg;
  V3 pos = ld3(U + 6 * g), vel = ld3(U + 6 * g + 3);
  V3 dp = v3(j == 0, j == 1, j == 2), dv = v3(j == 3, j == 4, j == 5);
  for (int s = 0; s < len; ++s) rk4_step_tangent(sp, sf, nfields, qomg, pos, vel, dp, dv, h);
  if (j == 0) {
    F[6 * g + 0] = pos.x; F[6 * g + 1] = pos.y; F[6 * g + 2] = pos.z;
    F[6 * g + 3] = vel.x; F[6 * g + 4] = vel.y; F[6 * g + 5] = vel.z;
  }
  if (j < 6) {  // column j of Phi (row-major [i][j])
    double *col = Phi + 36 * g + j;
    col[0] = dp.x; col[6] = dp.y; col[12] = dp.z; col[18] = dv.x; col[24] = dv.y; col[30] = dv.z;
  }
}

// One warp per chain; lane i < 6 owns component i of the update delta_n = U'_n - U_n (delta_0 = 0).
__global__ void __launch_bounds__(64) shoot_update_kernel(Plan P, double *__restrict__ U,
                                                          const double *__restrict__ F,
                                                          const double *__restrict__ Phi, int *__restrict__ flags,
                                                          double *__restrict__ diag, double scale_pos,
                                                          double scale_vel) {
  if (flags[0]) return;
  __shared__ double wmax[2];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = lane < 6 ? lane : 0;
  const unsigned full = 0xffffffffu;
  const int ns = w == 0 ? P.sf : P.sb, first = w == 0 ? 0 : P.sf;
  const double rscale = 1.0 / (i < 3 ? scale_pos : scale_vel);
  double d = 0.0, mx = 0.0;
  // the loads of segment n do not depend on the sweep: fetch them one segment ahead
  double phi[6], f = 0.0, uold = 0.0;
  auto fetch = [&](int n, double *ph, double &fv, double &uo) {
    const int g = first + n;
    for (int k = 0; k < 6; ++k) ph[k] = Phi[36 * g + 6 * i + k];
    fv = F[6 * g + i];
    uo = U[6 * (g + 1) + i];
  };
  if (ns > 1) fetch(0, phi, f, uold);
  for (int n = 0; n + 1 < ns; ++n) {
    double nphi[6], nf = 0.0, nu = 0.0;
    if (n + 2 < ns) fetch(n + 1, nphi, nf, nu);
    double dl[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) dl[k] = __shfl_sync(full, d, k);
    double acc = phi[0] * dl[0];
#pragma unroll
    for (int k = 1; k < 6; ++k) acc = acc + phi[k] * dl[k];
    const double unew = f + acc;  // = F_n exactly when delta_n = 0
    d = unew - uold;
    if (lane < 6) U[6 * (first + n + 1) + i] = unew;
    mx = fmax(mx, fabs(d) * rscale);
#pragma unroll
    for (int k = 0; k < 6; ++k) phi[k] = nphi[k];
    f = nf;
    uold = nu;
  }
  if (lane >= 6) mx = 0.0;
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(full, mx, o));
  if (lane == 0) wmax[w] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    const double m = fmax(wmax[0], wmax[1]);
    const int it = flags[1];
    diag[it < kMaxIters ? it : kMaxIters - 1] = m;
    flags[1] = it + 1;
    if (m <= kTol) flags[0] = 1;
  }
}

// After convergence: every segment integrates and stores its points (lane j of the segment's eight
// stores components j and j + 8 of each point); the end state's distance from the next segment's
// start (the defect) is reduced into diag[kMaxIters].
__global__ void __launch_bounds__(kFineThreads) shoot_store_kernel(const srs_field *__restrict__ gfields, int nfields,
                                                                   const srs_particle *__restrict__ part, Plan P,
                                                                   const double *__restrict__ U,
                                                                   const int *__restrict__ flags,
                                                                   double *__restrict__ diag, double scale_pos,
                                                                   double scale_vel, double *__restrict__ X,
                                                                   double *__restrict__ Bt, double *__restrict__ A,
                                                                   int64_t stage_doubles) {
  if (!flags[0]) return;  // not converged: the serial kernel writes the trajectory
  __shared__ srs_field sf[kMaxFieldsShared];
  __shared__ Prepared sp[kMaxFieldsShared];
  load_fields(gfields, nfields, sf, sp, stage_doubles);
  const int g = blockIdx.x * (kFineThreads / kSegLanes) + threadIdx.x / kSegLanes;
  const int j = threadIdx.x % kSegLanes;
  if (g >= P.sf + P.sb) return;
  int chain, len;
  int64_t j0;
  double h;
  seg_of(P, g, chain, j0, len, h);
  const double qomg = part->qomg, C = kC, rC = 1.0 / C;
  const int64_t n = P.n;
  auto store = [&](int64_t k, V3 pos, V3 vel, V3 acc) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int c = j + r * kSegLanes;
      if (c >= 9) break;
      const int l3 = c % 3;
      const V3 src = c < 3 ? pos : c < 6 ? vel : acc;
      const double v = l3 == 0 ? src.x : l3 == 1 ? src.y : src.z;
      double *const o = (c < 3 ? X : c < 6 ? Bt : A) + (int64_t)l3 * n + k;
      *o = c < 3 ? v : div_rn(v, C, rC);
    }
  };
  V3 pos = ld3(U + 6 * g), vel = ld3(U + 6 * g + 3);
  // the initial point (a/c = 0), stored when the forward chain has points; its first segment stores it,
  // or the backward chain's when the forward chain has no step
  if (j0 == 0 && P.nfwd >= 1 && (chain == 0 || P.sf == 0)) store(P.nbwd, pos, vel, v3(0, 0, 0));
  for (int s = 0; s < len; ++s) {
    const V3 acc = rk4_step_seq(sp, sf, nfields, qomg, pos, vel, h);
    const int64_t step = j0 + s;
    store(chain == 0 ? P.nbwd + step + 1 : P.nbwd - 1 - step, pos, vel, acc);
  }
  const int64_t m = chain == 0 ? P.mf : P.mb;
  if (j == 0 && j0 + len < m) {
    const double *nx = U + 6 * (g + 1);
    double e = fmax(fmax(fabs(pos.x - nx[0]), fabs(pos.y - nx[1])), fabs(pos.z - nx[2])) / scale_pos;
    e = fmax(e, fmax(fmax(fabs(vel.x - nx[3]), fabs(vel.y - nx[4])), fabs(vel.z - nx[5])) / scale_vel);
    atomicMax(reinterpret_cast<unsigned long long *>(diag + kMaxIters), (unsigned long long)__double_as_longlong(e));
  }
}

__global__ void shoot_stats_kernel(const int *__restrict__ flags, const double *__restrict__ diag,
                                   double *__restrict__ stats) {
  const int it = flags[1];
  stats[0] = flags[0];
  stats[1] = it;
  stats[2] = it > 0 ? diag[(it < kMaxIters ? it : kMaxIters) - 1] : 0.0;
  stats[3] = diag[kMaxIters];
}

}  // namespace

int shoot_default_steps(int64_t nsteps) {
  // per iteration: L steps of the fine kernel (~1.5 us each) against S = N / L segments of the serial
  // update (~0.07 us each): L ~ sqrt(N / 20)
  int L = 16;
  while ((int64_t)L * L * 20 < nsteps && L < 4096) L *= 2;
  return L;
}

size_t shoot_scratch_bytes(int64_t nfwd, int64_t nbwd, int steps_per_segment) {
  const int64_t mf = nfwd > 0 ? nfwd - 1 : 0, mb = nbwd;
  const int L = steps_per_segment > 0 ? steps_per_segment : shoot_default_steps(mf + mb);
  const int64_t segs = (mf + L - 1) / L + (mb + L - 1) / L + 1;
  return sizeof(double) * (size_t)(segs * (6 + 6 + 36) + kMaxIters + 1) + 64;
}

cudaError_t launch_rk4_shoot(const srs_field *d_fields, int nfields, const srs_particle *d_particle,
                             const srs_particle &host_particle, double dt, int64_t nfwd, int64_t nbwd, double *d_x,
                             double *d_b, double *d_a, cudaStream_t s, int64_t stage_doubles, int steps_per_segment,
                             int max_iterations, void *scratch, double *d_stats) {
  if (nfields > kMaxFieldsShared) return cudaErrorInvalidValue;
  if (max_iterations < 0 || max_iterations > kMaxIters) return cudaErrorInvalidValue;
  const int iters = max_iterations > 0 ? max_iterations : kDefaultIters;
  Plan P;
  P.mf = nfwd > 0 ? nfwd - 1 : 0;
  P.mb = nbwd;
  P.L = steps_per_segment > 0 ? steps_per_segment : shoot_default_steps(P.mf + P.mb);
  P.sf = (int)((P.mf + P.L - 1) / P.L);
  P.sb = (int)((P.mb + P.L - 1) / P.L);
  P.dt = dt;
  P.nfwd = nfwd;
  P.nbwd = nbwd;
  P.n = nfwd + nbwd;
  const int segs = P.sf + P.sb;
  double *U = static_cast<double *>(scratch);
  double *F = U + 6 * (size_t)(segs + 1);
  double *Phi = F + 6 * (size_t)(segs + 1);
  double *diag = Phi + 36 * (size_t)(segs + 1);
  int *flags = reinterpret_cast<int *>(diag + kMaxIters + 1);
  // scales of the convergence test: the trajectory's extent and speed
  const double C = kC;
  const double v0 = sqrt(host_particle.beta0[0] * host_particle.beta0[0] +
                         host_particle.beta0[1] * host_particle.beta0[1] +
                         host_particle.beta0[2] * host_particle.beta0[2]) * C;
  double xs = fmax(fmax(fabs(host_particle.x0[0]), fabs(host_particle.x0[1])), fabs(host_particle.x0[2]));
  const double scale_pos = fmax(fmax(xs, v0 * dt * (double)(P.mf > P.mb ? P.mf : P.mb)), 1e-300);
  const double scale_vel = fmax(v0, 1e-300);
  const size_t smem = sizeof(double) * (size_t)stage_doubles;
  if (smem > 0) {
    if (cudaError_t e = cudaFuncSetAttribute(shoot_fine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))
      return e;
    if (cudaError_t e = cudaFuncSetAttribute(shoot_store_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))
      return e;
  }
  if (segs > 0) {
    shoot_init_kernel<<<(segs + 127) / 128, 128, 0, s>>>(P, d_particle, U, flags, diag);
    const int blocks = (segs + kFineThreads / kSegLanes - 1) / (kFineThreads / kSegLanes);
    for (int it = 0; it < iters; ++it) {
      shoot_fine_kernel<<<blocks, kFineThreads, smem, s>>>(d_fields, nfields, d_particle, P, U, F, Phi, flags,
                                                           stage_doubles);
      shoot_update_kernel<<<1, 64, 0, s>>>(P, U, F, Phi, flags, diag, scale_pos, scale_vel);
    }
    shoot_store_kernel<<<blocks, kFineThreads, smem, s>>>(d_fields, nfields, d_particle, P, U, flags, diag, scale_pos,
                                                          scale_vel, d_x, d_b, d_a, stage_doubles);
    if (d_stats) shoot_stats_kernel<<<1, 1, 0, s>>>(flags, diag, d_stats);
    if (cudaError_t e = cudaGetLastError()) return e;
    // the serial kernel, which returns at once when the iteration converged
    return launch_rk4_unless(d_fields, nfields, d_particle, dt, nfwd, nbwd, d_x, d_b, d_a, s, stage_doubles, flags);
  }
  // nothing to integrate in parallel (a single point): the serial kernel
  return launch_rk4(d_fields, nfields, d_particle, 1, dt, nfwd, nbwd, d_x, d_b, d_a, s, stage_doubles);
}

}  // namespace srs

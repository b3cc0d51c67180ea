// Fixed-step RK4 electron trajectories (compiled with -fmad=false so every operation rounds like the
// reference's x86-64 build).
//
// Reference: OSCARSSR::CalculateTrajectory (src/OSCARSSR.cc:562-673), DerivativesB (:741-765),
// RK4 (:826-874).  State (x, vx, y, vy, z, vz) in m and m/s; dv/dt = (q/(m gamma)) v x B with gamma
// fixed.  Forward from t0 for nforward points, then backward for nbackward points; the stored a/c at
// a point is the derivative evaluated at the state of the previous step (the first forward point
// stores 0, which the reference reads from an uninitialised array).
//
// The trajectory is a serial chain, so its cost is latency.  Two things shorten the chain without
// changing a single rounding:
//  * Field constants that the reference recomputes on every call (period length and direction,
//    phase shift, region bounds, rotation sines/cosines) are computed once per launch, by the same
//    IEEE operations, into shared memory.
//  * Of the four field evaluations of an RK4 step, B(p0) and B(p0 + h/2 v0) need nothing but the
//    step's start state, and once B(p0) is known so does B(p3) while B(p4) needs only B(p0) and
//    B(p0 + h/2 v0): the step is two rounds of two independent evaluations.  In the warp-cooperative
//    kernel one warp owns one particle and lanes (position slot, field) evaluate them side by side;
//    warp shuffles gather the field sums in field order.  Every lane then advances the (identical)
//    state redundantly, and nine lanes store the nine trajectory components of a point.
// For very large batches one thread per particle (the plain kernel) gives better issue efficiency.
//
// Layout written: [particle][component][point], point index = time order (the backward points come
// first, earliest at index 0), so no reversal pass is needed.
#include <cuda_runtime.h>

#include "rk4_fields.cuh"
#include "srs_internal.h"

namespace srs {

namespace {

// ---------------------------------------------------------------- warp-cooperative kernel

// A group of G lanes (G = the power of two >= 2 * nfields) owns one particle; a warp holds 32/G
// particles.  Lane (slot, field) of a group evaluates one field at one of the two positions of a
// round; groups past the last particle recompute the last one and store nothing, so every lane stays
// in the shuffles.
// With specs != nullptr each particle has its own time step, point counts and output arrays (jobs of
// different trajectory lengths); a warp then runs its longest particle's step count, and groups whose
// trajectory is complete keep stepping without storing.
template <int G, bool kE>
__global__ void __launch_bounds__(128) rk4_warp_kernel(const srs_field *__restrict__ gfields, int nfields,
                                                       const srs_particle *__restrict__ particles, int nparticles,
                                                       double dt_all, int64_t nfwd_all, int64_t nbwd_all,
                                                       double *__restrict__ X, double *__restrict__ Bt,
                                                       double *__restrict__ A, const TrajSpec *__restrict__ specs,
                                                       int64_t stage_doubles, const int *__restrict__ skip) {
  wait_for_previous_grid();  // (launched with launch_after after the parallel-in-time passes)
  if (skip && *skip) return;  // the parallel-in-time integration already wrote this trajectory
  __shared__ srs_field sf[kMaxFieldsShared];
  __shared__ Prepared sp[kMaxFieldsShared];
  __shared__ double sink[128];  // target of the stores a lane does not make (no branch around them)
  for (int i = threadIdx.x; i < nfields; i += blockDim.x) {
    sf[i] = gfields[i];
    prepare(sf[i], sp[i]);
  }
  __syncthreads();
  if (stage_doubles > 0) stage_grids(sf, sp, nfields);
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1), gbase = lane - gl;
  // G == 32: the block's four warps all integrate the block's one particle (the same instruction
  // stream, so the same values) and take turns storing its points (point k by warp k mod 4): the
  // stores leave the serial chain of any one warp.  G < 32: one warp holds 32/G particles.
  const int pp = G == 32 ? (int)blockIdx.x
                         : (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 / G) + lane / G;
  const int store_turn = G == 32 ? (int)(threadIdx.x >> 5) : -1;
  const bool owner = pp < nparticles;
  const int p = owner ? pp : nparticles - 1;
  const srs_particle P = particles[p];
  const double dt = specs ? specs[p].dt : dt_all;
  const int64_t nfwd = specs ? specs[p].nfwd : nfwd_all, nbwd = specs ? specs[p].nbwd : nbwd_all;
  const int64_t n = nfwd + nbwd;
  double *const xp = specs ? specs[p].x : X + (int64_t)p * 3 * n;
  double *const bp = specs ? specs[p].beta : Bt + (int64_t)p * 3 * n;
  double *const ap = specs ? specs[p].aoc : A + (int64_t)p * 3 * n;
  int64_t fmax = nfwd, bmax = nbwd;  // the warp's longest forward / backward runs
  for (int o = 16; o > 0; o >>= 1) {
    fmax = max(fmax, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)fmax, o));
    bmax = max(bmax, (int64_t)__shfl_xor_sync(0xffffffffu, (long long)bmax, o));
  }
  // lane gl evaluates field gl % nfields at position (gl / nfields) % 2; lanes past 2 * nfields
  // repeat an evaluation (their results are not read), so no lane branches around the evaluation
  const int slot = nfields > 0 ? (gl / nfields) & 1 : 0, fidx = nfields > 0 ? gl % nfields : 0;
  const double C = kC, qomg = P.qomg;
  const unsigned full = 0xffffffffu;

  // G == 32 (one particle per block): this lane's field is held in registers across the loop, so the
  // serial chain reloads nothing from shared memory; narrower groups, which run many particles per SM,
  // keep it in shared memory to leave registers for occupancy
  Prepared myp;
  srs_field myf;
  if (G == 32) {
    myp = sp[fidx];
    myf = sf[fidx];
  }
  const Prepared &fp = G == 32 ? myp : sp[fidx];
  const srs_field &ff = G == 32 ? myf : sf[fidx];
  // B (and with kE, E) at two positions, one per slot, each summed over its fields in field order
  bool has_b = true;  // kE: whether the magnetic container has fields (DerivativesE / DerivativesEB)
  if (kE) {
    has_b = false;
    for (int f = 0; f < nfields; ++f) has_b = has_b || !field_electric(sf[f].kind);
  }
  auto fields2 = [&](V3 pa, V3 pb, V3 &Ba, V3 &Bb, V3 &Ea, V3 &Eb) {
    V3 mine = v3(0, 0, 0);
    if (nfields > 0) mine = field_one(fp, ff, slot == 0 ? pa : pb);
    Ba = v3(0, 0, 0);
    Bb = v3(0, 0, 0);
    Ea = v3(0, 0, 0);
    Eb = v3(0, 0, 0);
    for (int f = 0; f < nfields; ++f) {
      const int la = gbase + f, lb = gbase + nfields + f;
      const V3 va = v3(__shfl_sync(full, mine.x, la), __shfl_sync(full, mine.y, la), __shfl_sync(full, mine.z, la));
      const V3 vb = v3(__shfl_sync(full, mine.x, lb), __shfl_sync(full, mine.y, lb), __shfl_sync(full, mine.z, lb));
      if (kE && field_electric(sf[f].kind)) {
        Ea = Ea + va;
        Eb = Eb + vb;
      } else {
        Ba = Ba + va;
        Bb = Bb + vb;
      }
    }
  };
  // the velocity part of the derivative: DerivativesB, or with kE DerivativesE / DerivativesEB
  auto accel = [&](V3 v, V3 Bv, V3 Ev) -> V3 {
    if (!kE) return force(qomg, v, Bv);
    return has_b ? force_eb(qomg, v, Ev, Bv) : force_e(qomg, Ev);
  };
  // the group's lanes store the nine components of a point (x, y, z, beta = v/c, a/c), lane gl taking
  // components gl, gl + G, ...; selects, not branches
  const double rC = 1.0 / C;
  double *const my_sink = sink + (threadIdx.x & 127);
  auto store = [&](int64_t k, bool keep, V3 pos, V3 vel, V3 acc) {
    if (store_turn >= 0 && (int)(k & 3) != store_turn) return;  // warp-uniform
#pragma unroll
    for (int r = 0; r < (9 + G - 1) / G; ++r) {
      const int c = gl + r * G;
      const int l3 = c < 3 ? c : c < 6 ? c - 3 : c - 6;
      const V3 src = c < 3 ? pos : c < 6 ? vel : acc;
      const double v = l3 == 0 ? src.x : l3 == 1 ? src.y : src.z;
      double *const o = (keep && owner && c < 9) ? (c < 3 ? xp : c < 6 ? bp : ap) + (int64_t)l3 * n + k : my_sink;
      *o = c < 3 ? v : div_rn(v, C, rC);
    }
  };
  // one RK4 step of size h from (pos, vel); returns the derivative at the start state (its velocity part)
  auto step = [&](V3 &pos, V3 &vel, double h) -> V3 {
    const double hh = h * 0.5, h6 = h / 6.0;
    V3 B1, B2, B3, B4, E1, E2, E3, E4;
    const V3 p2 = vadd_scaled(pos, hh, vel);          // yt = y + hh*dydx (positions)
    fields2(pos, p2, B1, B2, E1, E2);
    const V3 a1 = accel(vel, B1, E1);                  // dydx (velocity part)
    const V3 v2 = vadd_scaled(vel, hh, a1);
    const V3 a2 = accel(v2, B2, E2);                   // dyt
    const V3 p3 = vadd_scaled(pos, hh, v2);            // yt = y + hh*dyt
    const V3 v3_ = vadd_scaled(vel, hh, a2);
    const V3 p4 = vadd_scaled(pos, h, v3_);            // yt = y + h*dym (positions need dym = dyt(p3) pos part = v3)
    // dym = f(yt3): position part v3_, velocity part a3 = force(v3_, B(p3))
    fields2(p3, p4, B3, B4, E3, E4);
    const V3 a3 = accel(v3_, B3, E3);
    const V3 v4 = vadd_scaled(vel, h, a3);             // yt = y + h*dym (velocities)
    const V3 m_pos = v3_ + v2, m_vel = a3 + a2;        // dym += dyt
    const V3 a4 = accel(v4, B4, E4);                   // dyt = f(yt4): position part v4
    // yout = y + h6*(dydx + dyt + 2.0*dym)
    const V3 npos = v3(pos.x + h6 * (vel.x + v4.x + 2.0 * m_pos.x), pos.y + h6 * (vel.y + v4.y + 2.0 * m_pos.y),
                       pos.z + h6 * (vel.z + v4.z + 2.0 * m_pos.z));
    const V3 nvel = v3(vel.x + h6 * (a1.x + a4.x + 2.0 * m_vel.x), vel.y + h6 * (a1.y + a4.y + 2.0 * m_vel.y),
                       vel.z + h6 * (a1.z + a4.z + 2.0 * m_vel.z));
    pos = npos;
    vel = nvel;
    return a1;
  };

  const V3 pos0 = v3(P.x0[0], P.x0[1], P.x0[2]);
  const V3 vel0 = v3(P.beta0[0] * C, P.beta0[1] * C, P.beta0[2] * C);
  V3 pos = pos0, vel = vel0, acc = v3(0, 0, 0);
  for (int64_t i = 0; i < fmax; ++i) {
    store(nbwd + i, i < nfwd, pos, vel, acc);
    acc = step(pos, vel, dt);
  }
  pos = pos0;
  vel = vel0;
  const double mdt = -dt;
  for (int64_t i = 0; i < bmax; ++i) {
    acc = step(pos, vel, mdt);
    store(nbwd - 1 - i, i < nbwd, pos, vel, acc);
  }
}

// ---------------------------------------------------------------- one thread per particle

template <bool kE>
__global__ void __launch_bounds__(64) rk4_thread_kernel(const srs_field *__restrict__ gfields, int nfields,
                                                        const srs_particle *__restrict__ particles, int nparticles,
                                                        double dt, int64_t nfwd, int64_t nbwd,
                                                        double *__restrict__ X, double *__restrict__ Bt,
                                                        double *__restrict__ A, int64_t stage_doubles) {
  __shared__ srs_field sf[kMaxFieldsShared];
  __shared__ Prepared sp[kMaxFieldsShared];
  for (int i = threadIdx.x; i < nfields; i += blockDim.x) {
    sf[i] = gfields[i];
    prepare(sf[i], sp[i]);
  }
  __syncthreads();
  if (stage_doubles > 0) stage_grids(sf, sp, nfields);
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nparticles) return;
  const srs_particle P = particles[p];
  const int64_t n = nfwd + nbwd;
  double *xp = X + (int64_t)p * 3 * n, *bp = Bt + (int64_t)p * 3 * n, *ap = A + (int64_t)p * 3 * n;
  const double C = kC, qomg = P.qomg;
  // the magnetic (electric = false) or electric container's sum at x
  auto Fsum = [&](V3 x, bool electric) {
    V3 s = v3(0, 0, 0);
    for (int f = 0; f < nfields; ++f)
      if (!kE || field_electric(sf[f].kind) == electric) s = s + field_one(sp[f], sf[f], x);
    return s;
  };
  bool has_b = true;
  if (kE) {
    has_b = false;
    for (int f = 0; f < nfields; ++f) has_b = has_b || !field_electric(sf[f].kind);
  }
  auto accel = [&](V3 v, V3 x) -> V3 {
    if (!kE) return force(qomg, v, Fsum(x, false));
    return has_b ? force_eb(qomg, v, Fsum(x, true), Fsum(x, false)) : force_e(qomg, Fsum(x, true));
  };
  auto step = [&](V3 &pos, V3 &vel, double h) -> V3 {
    const double hh = h * 0.5, h6 = h / 6.0;
    const V3 p2 = vadd_scaled(pos, hh, vel);
    const V3 a1 = accel(vel, pos);
    const V3 v2 = vadd_scaled(vel, hh, a1);
    const V3 a2 = accel(v2, p2);
    const V3 p3 = vadd_scaled(pos, hh, v2);
    const V3 v3_ = vadd_scaled(vel, hh, a2);
    const V3 a3 = accel(v3_, p3);
    const V3 p4 = vadd_scaled(pos, h, v3_);
    const V3 v4 = vadd_scaled(vel, h, a3);
    const V3 m_pos = v3_ + v2, m_vel = a3 + a2;
    const V3 a4 = accel(v4, p4);
    const V3 npos = v3(pos.x + h6 * (vel.x + v4.x + 2.0 * m_pos.x), pos.y + h6 * (vel.y + v4.y + 2.0 * m_pos.y),
                       pos.z + h6 * (vel.z + v4.z + 2.0 * m_pos.z));
    const V3 nvel = v3(vel.x + h6 * (a1.x + a4.x + 2.0 * m_vel.x), vel.y + h6 * (a1.y + a4.y + 2.0 * m_vel.y),
                       vel.z + h6 * (a1.z + a4.z + 2.0 * m_vel.z));
    pos = npos;
    vel = nvel;
    return a1;
  };
  const double rC = 1.0 / C;
  auto store = [&](int64_t k, V3 pos, V3 vel, V3 acc) {
    xp[k] = pos.x; xp[n + k] = pos.y; xp[2 * n + k] = pos.z;
    bp[k] = div_rn(vel.x, C, rC); bp[n + k] = div_rn(vel.y, C, rC); bp[2 * n + k] = div_rn(vel.z, C, rC);
    ap[k] = div_rn(acc.x, C, rC); ap[n + k] = div_rn(acc.y, C, rC); ap[2 * n + k] = div_rn(acc.z, C, rC);
  };
  const V3 pos0 = v3(P.x0[0], P.x0[1], P.x0[2]);
  const V3 vel0 = v3(P.beta0[0] * C, P.beta0[1] * C, P.beta0[2] * C);
  V3 pos = pos0, vel = vel0, acc = v3(0, 0, 0);
  for (int64_t i = 0; i < nfwd; ++i) {
    store(nbwd + i, pos, vel, acc);
    acc = step(pos, vel, dt);
  }
  pos = pos0;
  vel = vel0;
  for (int64_t i = 0; i < nbwd; ++i) {
    acc = step(pos, vel, -dt);
    store(nbwd - 1 - i, pos, vel, acc);
  }
}

__global__ void field_eval_kernel(const srs_field *__restrict__ fields, int nfields, const double *__restrict__ xyz,
                                  int64_t np, double *__restrict__ out, int electric) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  V3 b = field_sum(fields, nfields, v3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]), electric != 0);
  out[3 * i] = b.x;
  out[3 * i + 1] = b.y;
  out[3 * i + 2] = b.z;
}

}  // namespace

// Lanes per particle: at least 2 * nfields (two positions per round, one field per lane), rounded
// up to a power of two; then wider while the particles' groups still fit about one warp per
// scheduler (148 SMs x 4): wider groups store a point's nine components in parallel and shorten the
// per-step chain, but once every scheduler has a warp the batch is bound by the instructions issued
// per particle, which narrower groups save (4096 particles of 20001 points: 16 lanes 35.0 ms, 8
// lanes 26.3 ms, 4 lanes 25.3 ms, 2 lanes 26.9 ms; 2048: 16 lanes 25.0 ms, 8 lanes 23.1 ms).  G = 32
// gives a particle a whole block (four warps sharing the stores), taken while blocks of that kind fit
// 16 warps per SM.
static int group_size(int nparticles, int nfields) {
  constexpr int64_t kLanes = (int64_t)148 * 16 * 32;   // 16 warps per SM
  constexpr int64_t kOneWarpPerScheduler = (int64_t)148 * 4 * 32;
  int G = 2;
  while (G < 2 * nfields) G *= 2;
  while (G < 16 && (int64_t)nparticles * (2 * G) <= kOneWarpPerScheduler) G *= 2;
  if (G == 16 && (int64_t)nparticles * 4 * 32 <= kLanes) G = 32;
  return G;
}

int64_t grid_stage_doubles(const srs_field *host_fields, int nfields) {
  int64_t total = 0;
  for (int i = 0; i < nfields; ++i)
    if (field_shape(host_fields[i].kind) == SRS_FIELD_GRID)
      total += 3 * host_fields[i].n[0] * host_fields[i].n[1] * host_fields[i].n[2];
  return total <= kGridStageMaxDoubles ? total : 0;
}

namespace {
// The 48 KB default covers static plus dynamic shared memory; raise the kernel's dynamic limit
// whenever grid samples are staged.
template <typename K>
cudaError_t allow_smem(K kernel, size_t bytes) {
  if (bytes == 0) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}
}  // namespace

template <int G, bool kE>
static cudaError_t launch_warp_rk4_g(const srs_field *d_fields, int nfields, const srs_particle *d_particles, int nparticles,
                              double dt, int64_t nfwd, int64_t nbwd, double *d_x, double *d_b, double *d_a,
                              const TrajSpec *d_specs, int64_t stage_doubles, cudaStream_t s,
                              const int *d_skip = nullptr) {
  const size_t smem = sizeof(double) * (size_t)stage_doubles;
  if (cudaError_t e = allow_smem(rk4_warp_kernel<G, kE>, smem)) return e;
  const int warps = 4, per_block = G == 32 ? 1 : warps * (32 / G);
  const dim3 grid((nparticles + per_block - 1) / per_block), block(32 * warps);
  if (d_skip)  // the fallback after the parallel-in-time passes: set up while they finish
    return launch_after(rk4_warp_kernel<G, kE>, grid, block, smem, s, d_fields, nfields, d_particles, nparticles, dt,
                        nfwd, nbwd, d_x, d_b, d_a, d_specs, stage_doubles, d_skip);
  rk4_warp_kernel<G, kE><<<grid, block, smem, s>>>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x,
                                                   d_b, d_a, d_specs, stage_doubles, d_skip);
  return cudaGetLastError();
}

template <bool kE>
static cudaError_t launch_warp_rk4_e(int G, const srs_field *d_fields, int nfields, const srs_particle *d_particles,
                                     int nparticles, double dt, int64_t nfwd, int64_t nbwd, double *d_x, double *d_b,
                                     double *d_a, const TrajSpec *d_specs, int64_t stage_doubles, cudaStream_t s,
                                     const int *d_skip) {
  switch (G) {
    case 2: return launch_warp_rk4_g<2, kE>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a,
                                        d_specs, stage_doubles, s, d_skip);
    case 4: return launch_warp_rk4_g<4, kE>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a,
                                        d_specs, stage_doubles, s, d_skip);
    case 8: return launch_warp_rk4_g<8, kE>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a,
                                        d_specs, stage_doubles, s, d_skip);
    case 16: return launch_warp_rk4_g<16, kE>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a,
                                          d_specs, stage_doubles, s, d_skip);
    case 32: return launch_warp_rk4_g<32, kE>(d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a,
                                          d_specs, stage_doubles, s, d_skip);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t launch_warp_rk4(int G, const srs_field *d_fields, int nfields, const srs_particle *d_particles,
                                   int nparticles, double dt, int64_t nfwd, int64_t nbwd, double *d_x, double *d_b,
                                   double *d_a, const TrajSpec *d_specs, int64_t stage_doubles, cudaStream_t s,
                                   const int *d_skip = nullptr, bool electric = false) {
  return electric ? launch_warp_rk4_e<true>(G, d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b,
                                            d_a, d_specs, stage_doubles, s, d_skip)
                  : launch_warp_rk4_e<false>(G, d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b,
                                             d_a, d_specs, stage_doubles, s, d_skip);
}

bool has_electric(const srs_field *host_fields, int nfields) {
  for (int i = 0; i < nfields; ++i)
    if (field_electric(host_fields[i].kind)) return true;
  return false;
}

cudaError_t launch_rk4(const srs_field *d_fields, int nfields, const srs_particle *d_particles, int nparticles,
                       double dt, int64_t nfwd, int64_t nbwd, double *d_x, double *d_b, double *d_a,
                       cudaStream_t s, int64_t stage_doubles, bool electric) {
  if (nparticles <= 0) return cudaSuccess;
  if (nfields > kMaxFieldsShared) return cudaErrorInvalidValue;
  const size_t smem = sizeof(double) * (size_t)stage_doubles;
  const int G = group_size(nparticles, nfields);
  // grouped lanes while there are few particles per SM (the serial chain is the limit); one thread
  // per particle when there are enough particles to fill the SMs (issue rate is the limit)
  if (G <= 32 && (int64_t)nparticles * G <= 148 * 32 * 48) {
    if (cudaError_t e = launch_warp_rk4(G, d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a,
                                        nullptr, stage_doubles, s, nullptr, electric))
      return e;
  } else {
    const int threads = 64;
    if (electric) {
      if (cudaError_t e = allow_smem(rk4_thread_kernel<true>, smem)) return e;
      rk4_thread_kernel<true><<<(nparticles + threads - 1) / threads, threads, smem, s>>>(
          d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a, stage_doubles);
    } else {
      if (cudaError_t e = allow_smem(rk4_thread_kernel<false>, smem)) return e;
      rk4_thread_kernel<false><<<(nparticles + threads - 1) / threads, threads, smem, s>>>(
          d_fields, nfields, d_particles, nparticles, dt, nfwd, nbwd, d_x, d_b, d_a, stage_doubles);
    }
  }
  return cudaGetLastError();
}

cudaError_t launch_rk4_unless(const srs_field *d_fields, int nfields, const srs_particle *d_particles, double dt,
                              int64_t nfwd, int64_t nbwd, double *d_x, double *d_b, double *d_a, cudaStream_t s,
                              int64_t stage_doubles, const int *d_skip) {
  if (nfields > kMaxFieldsShared) return cudaErrorInvalidValue;
  return launch_warp_rk4(group_size(1, nfields), d_fields, nfields, d_particles, 1, dt, nfwd, nbwd, d_x, d_b, d_a,
                         nullptr, stage_doubles, s, d_skip);
}

cudaError_t launch_rk4_specs(const srs_field *d_fields, int nfields, const srs_particle *d_particles,
                             const TrajSpec *d_specs, int nparticles, cudaStream_t s, int64_t stage_doubles,
                             bool electric) {
  if (nparticles <= 0) return cudaSuccess;
  if (nfields > kMaxFieldsShared) return cudaErrorInvalidValue;
  const int G = group_size(nparticles, nfields);
  if (G > 32) return cudaErrorInvalidValue;
  if (cudaError_t e = launch_warp_rk4(G, d_fields, nfields, d_particles, nparticles, 0.0, 0, 0, nullptr, nullptr,
                                      nullptr, d_specs, stage_doubles, s, nullptr, electric))
    return e;
  return cudaGetLastError();
}

cudaError_t launch_field_eval(const srs_field *d_fields, int nfields, const double *d_xyz, int64_t np,
                              double *d_out, cudaStream_t s, bool electric) {
  if (np <= 0) return cudaSuccess;
  const int threads = 128;
  field_eval_kernel<<<(unsigned)((np + threads - 1) / threads), threads, 0, s>>>(d_fields, nfields, d_xyz, np, d_out,
                                                                                 electric ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace srs

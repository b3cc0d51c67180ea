// Parallel-in-time RK4 for one long trajectory: multiple shooting with Newton updates (compiled with
// -fmad=false; the steps round exactly as those of the serial warp kernel in rk4.cu).
//
// The serial chain of N RK4 steps costs ~0.9 us per step of latency on one SM, whatever the GPU's
// width.  Here each of the reference's two chains (forward from t0 with +dt, backward with -dt;
// OSCARSSR.cc:562-673) is cut into segments of L steps, and the start state U_n of every segment
// (U_0 = the initial state, fixed) is found by Newton's method on the matching conditions
// U_{n+1} = F_n(U_n), F_n = L serial steps.  One iteration is
//   (1) shoot_fine_kernel: all segments run their L steps from U_n at once, G lanes per segment as in
//       the serial warp kernel (two rounds of two field evaluations per step, shuffles to combine),
//       giving F_n(U_n).  While the updates are large, lanes 0..5 also carry the six unit tangents of
//       the start state (single precision, with the field's Jacobian shuffled from the lanes that
//       evaluate it), giving the segment's 6 x 6 Jacobian Phi_n.  Each block is a chunk of
//       consecutive segments and composes their affine maps delta_n -> delta_{n+1} =
//       (F_n - U_{n+1}) + Phi_n delta_n into one chunk map (M_c, b_c).
//   (2) shoot_update_kernel: one warp per chain carries delta across the chunk maps (delta = 0 at the
//       chain's start), then every chunk expands its segments: U'_{n+1} = F_n + Phi_n delta_n, exactly
//       F_n when delta_n = 0, so segments whose start is already exact stay exact.
// Once the largest update is small (2^-20 of the trajectory's scale) the Jacobians are kept (a chord
// step) and the fine kernel, without tangents, also stores the points of the trajectory it integrates;
// the iteration has converged when the largest update falls below 2^-48 of the scale, and the points
// stored in that iteration are the trajectory.  If it has not converged after the iteration limit the
// serial kernel writes the trajectory instead (it exits at once otherwise): no host synchronisation.
// Initial guess: straight flight from the initial state.
//
// The stored trajectory equals the serial one up to the ulps by which a start state a few ulps away
// rounds differently (~1e-16 m), not bit for bit; the FP64 drop-in path keeps the serial kernel.
#include <cuda_runtime.h>

#include "rk4_fields.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

constexpr int kShootThreads = 128;  // threads per fine block: 128 / G segments form one chunk
constexpr int kMaxIters = 32;       // capacity of the per-iteration record
constexpr int kDefaultIters = 8;
constexpr double kTol = 3.552713678800501e-15;  // 2^-48: converged
constexpr double kNear = 9.5367431640625e-07;   // 2^-20: keep the Jacobians, store the points
constexpr int kTile = 32;                        // chunk maps staged per chain in the update kernel

struct Plan {
  int64_t mf, mb;         // steps of each chain
  int sf, sb;             // segments of each chain
  int sfp, sbp;           // the same rounded up to whole chunks (the backward chain starts a chunk)
  int L, m;               // steps per segment, segments per chunk
  double dt;
  int64_t nfwd, nbwd, n;  // stored points from t0 on, before t0; points per trajectory component
};

struct Seg {
  int chain;
  bool active, last;  // a real segment; the last of its chain (no successor to match)
  int64_t j0;         // first step
  int len;            // steps
  double h;
};

__device__ inline Seg seg_of(const Plan &P, int g) {
  Seg s;
  s.chain = g < P.sfp ? 0 : 1;
  const int local = s.chain == 0 ? g : g - P.sfp;
  const int ns = s.chain == 0 ? P.sf : P.sb;
  const int64_t m = s.chain == 0 ? P.mf : P.mb;
  s.active = local < ns;
  s.last = local == ns - 1;
  s.j0 = (int64_t)local * P.L;
  s.len = s.active ? (int)imin64(P.L, m - s.j0) : 0;
  s.h = s.chain == 0 ? P.dt : -P.dt;
  return s;
}

// flags: [0] converged, [1] iterations run, [2] near (Jacobians kept, points stored), [3] the last fine
// run stored the points.  diag: [it] largest update of iteration it; [kMaxIters] largest mismatch
// |F_n(U_n) - U_{n+1}| of the last pass that stored points (both relative to the scales).
__global__ void shoot_init_kernel(Plan P, const srs_particle *__restrict__ part, double *__restrict__ U,
                                  int *__restrict__ flags, double *__restrict__ diag) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g == 0) {
    for (int k = 0; k < 4; ++k) flags[k] = 0;
    for (int k = 0; k < kMaxIters + 1; ++k) diag[k] = 0.0;
  }
  if (g >= P.sfp + P.sbp) return;
  const Seg s = seg_of(P, g);
  const double C = kC, t = (double)s.j0 * s.h;
  for (int c = 0; c < 3; ++c) {
    const double v = part->beta0[c] * C;
    U[6 * g + c] = !s.active ? 0.0 : s.j0 == 0 ? part->x0[c] : part->x0[c] + v * t;
    U[6 * g + 3 + c] = s.active ? v : 0.0;
  }
}

struct F3 {
  float x, y, z;
};
__device__ inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ inline F3 f3(V3 v) { return F3{(float)v.x, (float)v.y, (float)v.z}; }
__device__ inline F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ inline F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ inline F3 fcross(F3 a, F3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
__device__ inline F3 fmatvec(const float J[9], F3 d) {
  return f3(J[0] * d.x + J[1] * d.y + J[2] * d.z, J[3] * d.x + J[4] * d.y + J[5] * d.z,
            J[6] * d.x + J[7] * d.y + J[8] * d.z);
}

// One fine pass.  kTan: tangents and Jacobians (iterations far from convergence); otherwise the
// points are stored.  final_pass: the store pass after an iteration that converged without storing.
template <int G, bool kTan>
__global__ void __launch_bounds__(kShootThreads) shoot_fine_kernel(
    const srs_field *__restrict__ gfields, int nfields, const srs_particle *__restrict__ part, Plan P,
    const double *__restrict__ U, double *__restrict__ F, double *__restrict__ Phi, double *__restrict__ Mc,
    double *__restrict__ bc, int *__restrict__ flags, double *__restrict__ defect, double scale_pos, double scale_vel,
    double *__restrict__ X, double *__restrict__ Bt, double *__restrict__ A, int64_t stage_doubles, int final_pass) {
  if (final_pass) {
    if (!flags[0] || flags[3]) return;
  } else if (flags[0] || (flags[2] != 0) == kTan) {
    return;  // converged, or the other kind of pass is due (uniform over the grid)
  }
  constexpr int M = kShootThreads / G;  // segments per block (one chunk)
  __shared__ srs_field sf[kMaxFieldsShared];
  __shared__ Prepared sp[kMaxFieldsShared];
  __shared__ double sPhi[M][36], sR[M][6], sM[2][36], sB[2][6];
  for (int i = threadIdx.x; i < nfields; i += blockDim.x) {
    sf[i] = gfields[i];
    prepare(sf[i], sp[i]);
  }
  __syncthreads();
  if (stage_doubles > 0) stage_grids(sf, sp, nfields);
  const int lane = threadIdx.x & 31, gl = lane & (G - 1), gbase = lane - gl, grp = threadIdx.x / G;
  const int g = blockIdx.x * M + grp;
  const Seg S = seg_of(P, g);
  const int slot = nfields > 0 ? (gl / nfields) & 1 : 0, fidx = nfields > 0 ? gl % nfields : 0;
  const Prepared myp = sp[fidx];  // this lane's field constants, in registers for the serial chain
  const srs_field &ff = sf[fidx];
  const double C = kC, rC = 1.0 / C, qomg = part->qomg;
  const float qf = (float)qomg;
  const unsigned full = 0xffffffffu;

  // B (exact, summed in field order as the serial kernels do) and, with tangents, the FP32 Jacobian
  // at the two positions of a round
  auto fields2 = [&](V3 pa, V3 pb, V3 &Ba, V3 &Bb, float *Ja, float *Jb) {
    V3 mine = v3(0, 0, 0);
    float jm[9];
    const V3 at = slot == 0 ? pa : pb;
    if (nfields > 0) {
      mine = field_one(myp, ff, at);
      if (kTan) field_one_jac(myp, ff, at, jm);
    }
    Ba = v3(0, 0, 0);
    Bb = v3(0, 0, 0);
    if (kTan)
      for (int k = 0; k < 9; ++k) Ja[k] = Jb[k] = 0.f;
    for (int f = 0; f < nfields; ++f) {
      const int la = gbase + f, lb = gbase + nfields + f;
      Ba = Ba + v3(__shfl_sync(full, mine.x, la), __shfl_sync(full, mine.y, la), __shfl_sync(full, mine.z, la));
      Bb = Bb + v3(__shfl_sync(full, mine.x, lb), __shfl_sync(full, mine.y, lb), __shfl_sync(full, mine.z, lb));
      if (kTan)
        for (int k = 0; k < 9; ++k) {
          Ja[k] += __shfl_sync(full, jm[k], la);
          Jb[k] += __shfl_sync(full, jm[k], lb);
        }
    }
  };
  // lane gl stores components gl, gl + G of a point (x, y, z, beta, a/c); selects, not branches
  auto store = [&](int64_t k, V3 pos, V3 vel, V3 acc) {
#pragma unroll
    for (int r = 0; r < (9 + G - 1) / G; ++r) {
      const int c = gl + r * G;
      if (c >= 9) break;
      const int l3 = c % 3;
      const V3 src = c < 3 ? pos : c < 6 ? vel : acc;
      const double v = l3 == 0 ? src.x : l3 == 1 ? src.y : src.z;
      double *const o = (c < 3 ? X : c < 6 ? Bt : A) + (int64_t)l3 * P.n + k;
      *o = c < 3 ? v : div_rn(v, C, rC);
    }
  };

  V3 pos = ld3(U + 6 * g), vel = ld3(U + 6 * g + 3);
  F3 dp = f3(gl == 0, gl == 1, gl == 2), dv = f3(gl == 3, gl == 4, gl == 5);
  V3 opos = pos, ovel = vel;
  F3 odp = dp, odv = dv;
  // the initial point (a/c = 0) when the forward chain has points: stored by the forward chain's first
  // segment, or by the backward chain's when the forward chain has no step
  if (!kTan && S.active && S.j0 == 0 && P.nfwd >= 1 && (S.chain == 0 || P.sf == 0))
    store(P.nbwd, pos, vel, v3(0, 0, 0));
  const double h = S.h, hh = h * 0.5, h6 = h / 6.0;
  const float hf = (float)h, hhf = (float)hh, h6f = (float)h6;
  // every group of the block steps L times (the shuffles need the whole warp); a group keeps the
  // state reached after its own len steps
  for (int s = 0; s < P.L; ++s) {
    V3 B1, B2, B3, B4;
    float J1[9], J2[9], J3[9], J4[9];
    const V3 p2 = vadd_scaled(pos, hh, vel);
    fields2(pos, p2, B1, B2, J1, J2);
    const V3 a1 = force(qomg, vel, B1);
    const V3 v2 = vadd_scaled(vel, hh, a1);
    const V3 a2 = force(qomg, v2, B2);
    const V3 p3 = vadd_scaled(pos, hh, v2);
    const V3 v3_ = vadd_scaled(vel, hh, a2);
    const V3 p4 = vadd_scaled(pos, h, v3_);
    fields2(p3, p4, B3, B4, J3, J4);
    const V3 a3 = force(qomg, v3_, B3);
    const V3 v4 = vadd_scaled(vel, h, a3);
    const V3 m_pos = v3_ + v2, m_vel = a3 + a2;
    const V3 a4 = force(qomg, v4, B4);
    const V3 npos = v3(pos.x + h6 * (vel.x + v4.x + 2.0 * m_pos.x), pos.y + h6 * (vel.y + v4.y + 2.0 * m_pos.y),
                       pos.z + h6 * (vel.z + v4.z + 2.0 * m_pos.z));
    const V3 nvel = v3(vel.x + h6 * (a1.x + a4.x + 2.0 * m_vel.x), vel.y + h6 * (a1.y + a4.y + 2.0 * m_vel.y),
                       vel.z + h6 * (a1.z + a4.z + 2.0 * m_vel.z));
    if (kTan) {  // the same stages for the tangent (dp, dv), in FP32
      const F3 da1 = (fcross(dv, f3(B1)) + fcross(f3(vel), fmatvec(J1, dp))) * qf;
      const F3 dp2 = dp + dv * hhf, dv2 = dv + da1 * hhf;
      const F3 da2 = (fcross(dv2, f3(B2)) + fcross(f3(v2), fmatvec(J2, dp2))) * qf;
      const F3 dp3 = dp + dv2 * hhf, dv3 = dv + da2 * hhf;
      const F3 da3 = (fcross(dv3, f3(B3)) + fcross(f3(v3_), fmatvec(J3, dp3))) * qf;
      const F3 dp4 = dp + dv3 * hf, dv4 = dv + da3 * hf;
      const F3 da4 = (fcross(dv4, f3(B4)) + fcross(f3(v4), fmatvec(J4, dp4))) * qf;
      dp = dp + (dv + dv4 + (dv3 + dv2) * 2.f) * h6f;
      dv = dv + (da1 + da4 + (da3 + da2) * 2.f) * h6f;
    }
    pos = npos;
    vel = nvel;
    if (!kTan && s < S.len) {
      const int64_t step = S.j0 + s;
      store(S.chain == 0 ? P.nbwd + step + 1 : P.nbwd - 1 - step, pos, vel, a1);
    }
    if (s + 1 == S.len) {
      opos = pos;
      ovel = vel;
      odp = dp;
      odv = dv;
    }
  }
  if (final_pass) return;
  if (threadIdx.x == 0 && blockIdx.x == 0) flags[3] = kTan ? 0 : 1;

  // F_n; Phi_n (column gl from tangent lane gl); the chunk's map from them and r_n = F_n - U_{n+1}
  const bool link = S.active && !S.last;  // segment n has a successor to match
  double mis = 0.0;
  if (gl < 6) {
    const double fo[6] = {opos.x, opos.y, opos.z, ovel.x, ovel.y, ovel.z};
    F[6 * g + gl] = fo[gl];
    const double r = link ? fo[gl] - U[6 * (g + 1) + gl] : 0.0;
    sR[grp][gl] = r;
    mis = fabs(r) / (gl < 3 ? scale_pos : scale_vel);
    if (kTan) {
      const double col[6] = {odp.x, odp.y, odp.z, odv.x, odv.y, odv.z};
      for (int i = 0; i < 6; ++i) {
        const double v = link ? col[i] : (i == gl ? 1.0 : 0.0);
        Phi[36 * g + 6 * i + gl] = v;
        sPhi[grp][6 * i + gl] = v;
      }
    }
  }
  if (!kTan) {  // the mismatch of the stored trajectory's segments; the Jacobians of the last tangent pass
    for (int o = 16; o > 0; o >>= 1) mis = fmax(mis, __shfl_xor_sync(full, mis, o));
    if (lane == 0 && mis > 0.0)
      atomicMax(reinterpret_cast<unsigned long long *>(defect), (unsigned long long)__double_as_longlong(mis));
    for (int k = threadIdx.x; k < M * 36; k += blockDim.x) sPhi[k / 36][k % 36] = Phi[36 * (blockIdx.x * M) + k];
  }
  __syncthreads();
  // compose M <- Phi_n M, b <- r_n + Phi_n b over the chunk's segments in order (threads 0..35 own an
  // entry of M, threads 36..41 an entry of b; M is unchanged without new Jacobians)
  const int t = threadIdx.x;
  const int ti = t < 36 ? t / 6 : t - 36, tj = t % 6;
  if (t < 36) sM[0][t] = ti == tj ? 1.0 : 0.0;
  if (t >= 36 && t < 42) sB[0][ti] = 0.0;
  __syncthreads();
  int cur = 0;
  for (int n = 0; n < M; ++n) {
    if (kTan && t < 36) {
      double acc = sPhi[n][6 * ti] * sM[cur][tj];
      for (int k = 1; k < 6; ++k) acc = acc + sPhi[n][6 * ti + k] * sM[cur][6 * k + tj];
      sM[cur ^ 1][t] = acc;
    }
    if (t >= 36 && t < 42) {
      double acc = sPhi[n][6 * ti] * sB[cur][0];
      for (int k = 1; k < 6; ++k) acc = acc + sPhi[n][6 * ti + k] * sB[cur][k];
      sB[cur ^ 1][ti] = sR[n][ti] + acc;
    }
    __syncthreads();
    cur ^= 1;
  }
  if (kTan && t < 36) Mc[36 * blockIdx.x + t] = sM[cur][t];
  if (t >= 36 && t < 42) bc[6 * blockIdx.x + ti] = sB[cur][ti];
}

// Carries delta across the chunk maps (one warp per chain; delta = 0 at the start of a chain), then
// expands every chunk: U'_{n+1} = F_n + Phi_n delta_n, delta_{n+1} = U'_{n+1} - U_{n+1}.  The largest
// |delta| relative to the scales decides: converged (kTol), near (kNear).
__global__ void __launch_bounds__(1024) shoot_update_kernel(Plan P, double *__restrict__ U,
                                                            const double *__restrict__ F,
                                                            const double *__restrict__ Phi,
                                                            const double *__restrict__ Mc,
                                                            const double *__restrict__ bc, double *__restrict__ dstart,
                                                            int *__restrict__ flags, double *__restrict__ diag,
                                                            double scale_pos, double scale_vel) {
  if (flags[0]) return;
  __shared__ double tM[2][kTile][36], tb[2][kTile][6];
  __shared__ double wmax[32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const unsigned full = 0xffffffffu;
  const int c0 = P.sfp / P.m, c1 = P.sbp / P.m;  // chunks of each chain
  const int ntile = ((c0 > c1 ? c0 : c1) + kTile - 1) / kTile;
  double d = 0.0;  // warp w < 2: component `lane` (< 6) of delta at the current chunk start of chain w
  for (int tt = 0; tt < ntile; ++tt) {
    for (int k = threadIdx.x; k < 2 * kTile * 42; k += blockDim.x) {
      const int ch = k / (kTile * 42), r = k % (kTile * 42), q = r / 42, e = r % 42;
      const int cl = tt * kTile + q, cn = ch == 0 ? c0 : c1, cg = (ch == 0 ? 0 : c0) + cl;
      if (cl < cn) {
        if (e < 36) tM[ch][q][e] = Mc[36 * cg + e];
        else tb[ch][q][e - 36] = bc[6 * cg + e - 36];
      }
    }
    __syncthreads();
    if (w < 2) {
      const int cn = w == 0 ? c0 : c1, first = w == 0 ? 0 : c0;
      const int i = lane < 6 ? lane : 0;
      for (int q = 0; q < kTile && tt * kTile + q < cn; ++q) {
        const int cl = tt * kTile + q;
        if (lane < 6) dstart[6 * (first + cl) + lane] = d;
        double dl[6];
#pragma unroll
        for (int k = 0; k < 6; ++k) dl[k] = __shfl_sync(full, d, k);
        double acc = tM[w][q][6 * i] * dl[0];
#pragma unroll
        for (int k = 1; k < 6; ++k) acc = acc + tM[w][q][6 * i + k] * dl[k];
        d = tb[w][q][i] + acc;
      }
    }
    __syncthreads();
  }
  // expansion: a group of 8 threads per chunk, lane i < 6 owns component i
  const int gi = threadIdx.x & 7, gb = lane & ~7, i = gi < 6 ? gi : 0;
  const double rscale = 1.0 / (i < 3 ? scale_pos : scale_vel);
  double mx = 0.0;
  const int nchunks = c0 + c1, groups = blockDim.x / 8;
  for (int cb = 0; cb < nchunks; cb += groups) {  // warp-uniform trip count
    const int c = cb + (int)(threadIdx.x >> 3);
    const bool ok = c < nchunks;
    double dd = ok ? dstart[6 * c + i] : 0.0;
    for (int n = 0; n < P.m; ++n) {
      const int g = c * P.m + n;
      const Seg S = seg_of(P, ok ? g : 0);
      const bool link = ok && S.active && !S.last;
      double dl[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) dl[k] = __shfl_sync(full, dd, gb + k);
      if (link) {
        double acc = Phi[36 * g + 6 * i] * dl[0];
#pragma unroll
        for (int k = 1; k < 6; ++k) acc = acc + Phi[36 * g + 6 * i + k] * dl[k];
        const double unew = F[6 * g + i] + acc;  // = F_n exactly when delta_n = 0
        dd = unew - U[6 * (g + 1) + i];
        if (gi < 6) {
          U[6 * (g + 1) + i] = unew;
          mx = fmax(mx, fabs(dd) * rscale);
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(full, mx, o));
  if (lane == 0) wmax[w] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = fmax(m, wmax[k]);
    const int it = flags[1];
    diag[it < kMaxIters ? it : kMaxIters - 1] = m;
    flags[1] = it + 1;
    if (m <= kNear) flags[2] = 1;
    if (m <= kTol) flags[0] = 1;
    else diag[kMaxIters] = 0.0;  // the next storing pass records its own mismatch
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

int lanes_for(int nfields) {
  int G = 8;
  while (G < 2 * nfields) G *= 2;
  return G;
}

Plan make_plan(int64_t nfwd, int64_t nbwd, double dt, int steps_per_segment, int nfields) {
  Plan P;
  P.mf = nfwd > 0 ? nfwd - 1 : 0;
  P.mb = nbwd;
  P.L = steps_per_segment > 0 ? steps_per_segment : shoot_default_steps(P.mf + P.mb);
  P.m = kShootThreads / lanes_for(nfields);
  P.sf = (int)((P.mf + P.L - 1) / P.L);
  P.sb = (int)((P.mb + P.L - 1) / P.L);
  P.sfp = (P.sf + P.m - 1) / P.m * P.m;
  P.sbp = (P.sb + P.m - 1) / P.m * P.m;
  P.dt = dt;
  P.nfwd = nfwd;
  P.nbwd = nbwd;
  P.n = nfwd + nbwd;
  return P;
}

struct Scratch {
  double *U, *F, *Phi, *Mc, *bc, *dstart, *diag;
  int *flags;
  double scale_pos, scale_vel;
};

Scratch carve(void *scratch, const Plan &P) {
  const size_t segs = (size_t)(P.sfp + P.sbp) + 1, chunks = (size_t)(P.sfp + P.sbp) / P.m + 1;
  Scratch s;
  s.U = static_cast<double *>(scratch);
  s.F = s.U + 6 * segs;
  s.Phi = s.F + 6 * segs;
  s.Mc = s.Phi + 36 * segs;
  s.bc = s.Mc + 36 * chunks;
  s.dstart = s.bc + 6 * chunks;
  s.diag = s.dstart + 6 * chunks;
  s.flags = reinterpret_cast<int *>(s.diag + kMaxIters + 1);
  return s;
}

template <int G>
cudaError_t launch_fine(bool tan, int blocks, size_t smem, cudaStream_t s, const srs_field *d_fields, int nfields,
                        const srs_particle *d_particle, const Plan &P, const Scratch &W, double *d_x, double *d_b,
                        double *d_a, int64_t stage_doubles, int final_pass) {
  if (tan) {
    if (smem > 0)
      if (cudaError_t e = cudaFuncSetAttribute(shoot_fine_kernel<G, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem))
        return e;
    shoot_fine_kernel<G, true><<<blocks, kShootThreads, smem, s>>>(d_fields, nfields, d_particle, P, W.U, W.F, W.Phi,
                                                                   W.Mc, W.bc, W.flags, W.diag + kMaxIters,
                                                                   W.scale_pos, W.scale_vel, d_x, d_b, d_a,
                                                                   stage_doubles, final_pass);
  } else {
    if (smem > 0)
      if (cudaError_t e = cudaFuncSetAttribute(shoot_fine_kernel<G, false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem))
        return e;
    shoot_fine_kernel<G, false><<<blocks, kShootThreads, smem, s>>>(d_fields, nfields, d_particle, P, W.U, W.F,
                                                                    W.Phi, W.Mc, W.bc, W.flags, W.diag + kMaxIters,
                                                                    W.scale_pos, W.scale_vel, d_x, d_b, d_a,
                                                                    stage_doubles, final_pass);
  }
  return cudaGetLastError();
}

cudaError_t launch_fine_g(int G, bool tan, int blocks, size_t smem, cudaStream_t s, const srs_field *d_fields,
                          int nfields, const srs_particle *d_particle, const Plan &P, const Scratch &W, double *d_x,
                          double *d_b, double *d_a, int64_t stage_doubles, int final_pass) {
  switch (G) {
    case 8:
      return launch_fine<8>(tan, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a, stage_doubles,
                            final_pass);
    case 16:
      return launch_fine<16>(tan, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a, stage_doubles,
                             final_pass);
    case 32:
      return launch_fine<32>(tan, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a, stage_doubles,
                             final_pass);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace

int shoot_default_steps(int64_t nsteps) {
  // 16 steps per segment: each iteration costs ~16 serial steps plus a chunk sweep; long
  // trajectories keep the segment count near 4096
  int64_t L = 16;
  while (L * 4096 < nsteps && L < 4096) L *= 2;
  return (int)L;
}

size_t shoot_scratch_bytes(int64_t nfwd, int64_t nbwd, int steps_per_segment, int nfields) {
  const Plan P = make_plan(nfwd, nbwd, 1.0, steps_per_segment, nfields);
  const size_t segs = (size_t)(P.sfp + P.sbp) + 1, chunks = (size_t)(P.sfp + P.sbp) / P.m + 1;
  return sizeof(double) * (segs * 48 + chunks * 48 + kMaxIters + 1) + 64;
}

cudaError_t launch_rk4_shoot(const srs_field *d_fields, int nfields, const srs_particle *d_particle,
                             const srs_particle &host_particle, double dt, int64_t nfwd, int64_t nbwd, double *d_x,
                             double *d_b, double *d_a, cudaStream_t s, int64_t stage_doubles, int steps_per_segment,
                             int max_iterations, void *scratch, double *d_stats) {
  if (nfields > kMaxFieldsShared) return cudaErrorInvalidValue;
  if (max_iterations < 0 || max_iterations > kMaxIters) return cudaErrorInvalidValue;
  const int iters = max_iterations > 0 ? max_iterations : kDefaultIters;
  const Plan P = make_plan(nfwd, nbwd, dt, steps_per_segment, nfields);
  const int segs = P.sfp + P.sbp;
  if (segs == 0)  // nothing to integrate in parallel (a single point): the serial kernel
    return launch_rk4(d_fields, nfields, d_particle, 1, dt, nfwd, nbwd, d_x, d_b, d_a, s, stage_doubles);
  Scratch W = carve(scratch, P);
  // scales of the convergence test: the trajectory's extent and speed
  const double C = kC;
  const double v0 = sqrt(host_particle.beta0[0] * host_particle.beta0[0] +
                         host_particle.beta0[1] * host_particle.beta0[1] +
                         host_particle.beta0[2] * host_particle.beta0[2]) * C;
  const double xs = fmax(fmax(fabs(host_particle.x0[0]), fabs(host_particle.x0[1])), fabs(host_particle.x0[2]));
  const double scale_pos = fmax(fmax(xs, v0 * dt * (double)(P.mf > P.mb ? P.mf : P.mb)), 1e-300);
  const double scale_vel = fmax(v0, 1e-300);
  W.scale_pos = scale_pos;
  W.scale_vel = scale_vel;
  const size_t smem = sizeof(double) * (size_t)stage_doubles;
  const int G = lanes_for(nfields), blocks = segs / P.m;
  shoot_init_kernel<<<(segs + 127) / 128, 128, 0, s>>>(P, d_particle, W.U, W.flags, W.diag);
  for (int it = 0; it < iters; ++it) {
    for (bool tan : {true, false})
      if (cudaError_t e = launch_fine_g(G, tan, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a,
                                        stage_doubles, 0))
        return e;
    shoot_update_kernel<<<1, 1024, 0, s>>>(P, W.U, W.F, W.Phi, W.Mc, W.bc, W.dstart, W.flags, W.diag, scale_pos,
                                           scale_vel);
  }
  // converged after a pass with tangents: one more pass stores the points
  if (cudaError_t e = launch_fine_g(G, false, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a,
                                    stage_doubles, 1))
    return e;
  if (d_stats) shoot_stats_kernel<<<1, 1, 0, s>>>(W.flags, W.diag, d_stats);
  if (cudaError_t e = cudaGetLastError()) return e;
  // the serial kernel, which returns at once when the iteration converged
  return launch_rk4_unless(d_fields, nfields, d_particle, dt, nfwd, nbwd, d_x, d_b, d_a, s, stage_doubles, W.flags);
}

}  // namespace srs

// Parallel-in-time RK4 for one long trajectory: multiple shooting with Newton updates (compiled with
// -fmad=false; the steps round exactly as those of the serial warp kernel in rk4.cu).
//
// The serial chain of N RK4 steps costs ~0.9 us per step of latency on one SM, whatever the GPU's
// width.  Here each of the reference's two chains (forward from t0 with +dt, backward with -dt;
// OSCARSSR.cc:562-673) is cut into segments of L steps, and the start state U_n of every segment
// (U_0 = the initial state, fixed) is found by Newton's method on the matching conditions
// U_{n+1} = F_n(U_n), F_n = L serial steps.  One Newton iteration is one launch of shoot_pass_kernel,
// whose blocks are chunks of consecutive segments:
//   (1) each block first applies the previous iteration's update to its chunk: from the update
//       delta at the chunk's start (carried by the sweep, below), U'_{n+1} = F_n + Phi_n delta_n for
//       the chunk's segments in order (exactly F_n when delta_n = 0, so exact starts stay exact);
//   (2) all segments run their L steps from U_n at once, G lanes per segment as in the serial warp
//       kernel (two rounds of two field evaluations per step, shuffles to combine), giving F_n(U_n)
//       and the mismatch r_n = F_n(U_n) - U_{n+1}.  While the mismatches are large, lanes 0..5 also
//       carry the six unit tangents of the start state (single precision, with the field's Jacobian
//       shuffled from the lanes that evaluate it), giving the segment's 6 x 6 Jacobian Phi_n; then the
//       block composes its segments' affine maps delta_n -> delta_{n+1} = r_n + Phi_n delta_n into one
//       chunk map (M_c, b_c);
//   (3) the last block to finish (an atomic ticket; nothing waits) adds the mismatches at the chunk
//       boundaries, decides, and carries delta across the chunk maps (one warp per chain, delta = 0 at
//       the chain's start) for the next launch.
// Once the largest mismatch is small (2^-20 of the trajectory's scale) the Jacobians are kept (chord
// steps) and the passes, without tangents, store the points of the trajectory they integrate; the
// iteration has converged when a storing pass's largest mismatch is below 2^-51 of the scale (a
// velocity mismatch of a few ulps, left at every segment boundary, would drift the positions by
// ~1e-14 m): its stored points are the trajectory.  If it has not converged after the iteration limit the serial
// kernel writes the trajectory instead (it exits at once otherwise): no host synchronisation.
// Initial guess: straight flight from the initial state.
//
// The stored trajectory equals the serial one up to the ulps by which a start state a few ulps away
// rounds differently (~1e-15 m), not bit for bit; the FP64 drop-in path keeps the serial kernel.
#include <cuda_runtime.h>

#include <algorithm>

#include <cuda_pipeline.h>

#include "rk4_fields.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

constexpr int kShootThreads = 128;  // threads per block: 128 / G segments form one chunk
constexpr int kMaxIters = 32;       // capacity of the per-iteration record
constexpr int kDefaultIters = 8;
constexpr double kTol = 4.440892098500626e-16;  // 2^-51 (~2 ulps of the speed): converged
constexpr double kNear = 9.5367431640625e-07;   // 2^-20: keep the Jacobians, store the points
constexpr int kChunkDoubles = 132;               // per-chunk data staged for the sweep
constexpr int kMaxChunks = 192;                  // 192 x 132 doubles = 198 KB of shared memory
constexpr int kOneWaveChunks = 148;              // the B200's SMs: one pass block (chunk) per SM

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

// Device scratch of one integration.
struct Scratch {
  double *U, *F, *Phi;     // per segment: start state, end state, Jacobian (row-major 6 x 6)
  double *rec;             // per chunk, kChunkDoubles: the record the last block sweeps over (below)
  double *dstart;          // per chunk: delta at its start
  double *diag;            // [it]: largest mismatch of iteration it (relative to the scales)
  double *rmax;            // this launch's largest interior mismatch (reset by the last block)
  int *flags;              // [0] converged, [1] iterations, [2] near, [3] the last pass stored, [4] ticket
  Prepared *prep;          // [nfields]: the fields' constants, computed once by the init kernel
  double scale_pos, scale_vel;
};

__global__ void shoot_init_kernel(Plan P, const srs_particle *__restrict__ part, Scratch W,
                                  const srs_field *__restrict__ fields, int nfields) {
  allow_next_grid();  // the first pass may be set up meanwhile (it waits for this grid's writes)
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < nfields) prepare(fields[g], W.prep[g]);  // once per integration, not once per pass and block
  if (g == 0) {
    for (int k = 0; k < 5; ++k) W.flags[k] = 0;
    for (int k = 0; k < kMaxIters; ++k) W.diag[k] = 0.0;
    *W.rmax = 0.0;
  }
  if (g >= P.sfp + P.sbp) return;
  const Seg s = seg_of(P, g);
  const double C = kC, t = (double)s.j0 * s.h;
  for (int c = 0; c < 3; ++c) {
    const double v = part->beta0[c] * C;
    W.U[6 * g + c] = !s.active ? 0.0 : s.j0 == 0 ? part->x0[c] : part->x0[c] + v * t;
    W.U[6 * g + 3 + c] = s.active ? v : 0.0;
  }
}

// sum_k a[k * stride] b[k * bstride] over 6 terms as a tree (depth 4 instead of 6: the sweeps are
// chains of these, and a dependent FP64 operation costs tens of cycles)
__device__ __forceinline__ double dot6(const double *a, int stride, const double *b, int bstride) {
  const double p0 = a[0] * b[0], p1 = a[stride] * b[bstride], p2 = a[2 * stride] * b[2 * bstride];
  const double p3 = a[3 * stride] * b[3 * bstride], p4 = a[4 * stride] * b[4 * bstride];
  const double p5 = a[5 * stride] * b[5 * bstride];
  return ((p0 + p1) + (p2 + p3)) + (p4 + p5);
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

// One pass over all segments (see the file comment).  kTan: tangents and Jacobians (far from
// convergence), otherwise the points are stored.  final_pass: the store pass after an iteration that
// converged without storing (no update, no decision).
template <int M>
struct PassShared {
  srs_field sf[kMaxFieldsShared];
  Prepared sp[kMaxFieldsShared];
  double sPhi[M][36], sR[M][6], sU[M + 1][6], sF[M][6], sM[2][36], sB[2][6];
  double wred[kShootThreads / 32];
  int am_last, done;
};

template <int G, bool kTan>
__device__ __forceinline__ void shoot_pass(PassShared<kShootThreads / G> &sh, const srs_field *__restrict__ gfields,
                                           int nfields, const srs_particle *__restrict__ part, const Plan &P,
                                           const Scratch &W, double *__restrict__ X, double *__restrict__ Bt,
                                           double *__restrict__ A, int64_t stage_doubles, bool final_pass) {
  constexpr int M = kShootThreads / G;  // segments per block (one chunk)
  srs_field *const sf = sh.sf;
  Prepared *const sp = sh.sp;
  auto &sPhi = sh.sPhi;
  auto &sR = sh.sR;
  auto &sU = sh.sU;
  auto &sF = sh.sF;
  auto &sM = sh.sM;
  auto &sB = sh.sB;
  auto &wred = sh.wred;
  int &am_last = sh.am_last;
  int &done = sh.done;
  const int t = threadIdx.x, lane = t & 31, gl = lane & (G - 1), gbase = lane - gl, grp = t / G;
  const int c = blockIdx.x, g0 = c * M, g = g0 + grp;
  const int iter = W.flags[1];
  const unsigned full = 0xffffffffu;
  for (int i = t; i < nfields; i += blockDim.x) {
    sf[i] = gfields[i];
    sp[i] = W.prep[i];
  }
  // (1) this chunk's start states: the previous iteration's update, segment after segment (the first
  // segment's was set by the last block's sweep)
  for (int k = t; k < M * 6; k += blockDim.x) sU[k / 6][k % 6] = W.U[6 * g0 + k];
  if (iter > 0 && !final_pass) {
    for (int k = t; k < M * 36; k += blockDim.x) sPhi[k / 36][k % 36] = W.Phi[36 * g0 + k];
    for (int k = t; k < M * 6; k += blockDim.x) sF[k / 6][k % 6] = W.F[6 * g0 + k];
  }
  __syncthreads();
  if (iter > 0 && !final_pass && t < 32) {  // one warp; lane i < 6 owns component i of delta
    const int i = lane < 6 ? lane : 0;
    // (lane i reads sU[n + 1][i] before it writes it, and no lane reads a row that is written later in
    // the same step, so the warp needs no barrier)
    double d = W.dstart[6 * c + i];
    for (int n = 0; n + 1 < M; ++n) {
      const Seg S = seg_of(P, g0 + n);
      double dl[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) dl[k] = __shfl_sync(full, d, k);
      if (S.active && !S.last) {
        const double unew = sF[n][i] + dot6(&sPhi[n][6 * i], 1, dl, 1);  // = F_n exactly when delta_n = 0
        d = unew - sU[n + 1][i];
        if (lane < 6) sU[n + 1][i] = unew;
      }
    }
  }
  __syncthreads();
  // this chunk's record: [0, 36) M_c, [36, 42) b_c (without the boundary mismatch), [42, 84) the same
  // up to the last segment's start, [84, 120) Phi of the last segment, [120, 126) its end state,
  // [126, 132) the chunk's first start state
  double *const rec = W.rec + (size_t)kChunkDoubles * c;
  if (!final_pass) {
    for (int k = t; k < M * 6; k += blockDim.x) W.U[6 * g0 + k] = sU[k / 6][k % 6];
    if (t < 6) rec[126 + t] = sU[0][t];
  }
  if (stage_doubles > 0) stage_grids(sf, sp, nfields);  // (ends with a barrier)

  // (2) integrate
  const Seg S = seg_of(P, g);
  const int slot = nfields > 0 ? (gl / nfields) & 1 : 0, fidx = nfields > 0 ? gl % nfields : 0;
  const Prepared myp = sp[fidx];  // this lane's field constants, in registers for the serial chain
  const srs_field &ff = sf[fidx];
  const double C = kC, rC = 1.0 / C, qomg = part->qomg;
  const float qf = (float)qomg;
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
      const int cc = gl + r * G;
      if (cc >= 9) break;
      const int l3 = cc % 3;
      const V3 src = cc < 3 ? pos : cc < 6 ? vel : acc;
      const double v = l3 == 0 ? src.x : l3 == 1 ? src.y : src.z;
      double *const o = (cc < 3 ? X : cc < 6 ? Bt : A) + (int64_t)l3 * P.n + k;
      *o = cc < 3 ? v : div_rn(v, C, rC);
    }
  };
  V3 pos = ld3(&sU[grp][0]), vel = ld3(&sU[grp][3]);
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

  // (3) F_n, the interior mismatches r_n = F_n - U_{n+1} (the chunk's last segment's successor belongs
  // to the next chunk: the last block adds that one), Phi_n (column gl from tangent lane gl)
  const bool link = S.active && !S.last;  // segment n has a successor to match
  double mis = 0.0;
  if (gl < 6) {
    const double fo[6] = {opos.x, opos.y, opos.z, ovel.x, ovel.y, ovel.z};
    W.F[6 * g + gl] = fo[gl];
    if (grp == M - 1) rec[120 + gl] = fo[gl];
    const double r = link && grp + 1 < M ? fo[gl] - sU[grp + 1][gl] : 0.0;
    sR[grp][gl] = r;
    mis = fabs(r) / (gl < 3 ? W.scale_pos : W.scale_vel);
    if (kTan) {
      const double col[6] = {odp.x, odp.y, odp.z, odv.x, odv.y, odv.z};
      for (int i = 0; i < 6; ++i) {
        const double v = link ? col[i] : (i == gl ? 1.0 : 0.0);
        W.Phi[36 * g + 6 * i + gl] = v;
        sPhi[grp][6 * i + gl] = v;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) mis = fmax(mis, __shfl_xor_sync(full, mis, o));
  if (lane == 0 && mis > 0.0)
    atomicMax(reinterpret_cast<unsigned long long *>(W.rmax), (unsigned long long)__double_as_longlong(mis));
  if (!kTan)  // the Jacobians of the last pass with tangents
    for (int k = t; k < M * 36; k += blockDim.x) sPhi[k / 36][k % 36] = W.Phi[36 * g0 + k];
  __syncthreads();
  // compose M <- Phi_n M, b <- r_n + Phi_n b over the chunk's segments in order (threads 0..35 own an
  // entry of M, threads 36..41 an entry of b; M is unchanged without new Jacobians)
  const int ti = t < 36 ? t / 6 : t - 36, tj = t % 6;
  if (t < 36) sM[0][t] = ti == tj ? 1.0 : 0.0;
  if (t >= 36 && t < 42) sB[0][ti] = 0.0;
  __syncthreads();
  int cur = 0;
  for (int n = 0; n < M; ++n) {
    if (kTan && t < 36) {
      sM[cur ^ 1][t] = dot6(&sPhi[n][6 * ti], 1, &sM[cur][tj], 6);
    }
    if (t >= 36 && t < 42) {
      sB[cur ^ 1][ti] = sR[n][ti] + dot6(&sPhi[n][6 * ti], 1, sB[cur], 1);
    }
    __syncthreads();
    cur ^= 1;
    if (n == M - 2) {  // the map up to the last segment's start
      if (kTan && t < 36) rec[42 + t] = sM[cur][t];
      if (t >= 36 && t < 42) rec[78 + ti] = sB[cur][ti];
    }
  }
  if (kTan && t < 36) rec[t] = sM[cur][t];
  if (t >= 36 && t < 42) rec[36 + ti] = sB[cur][ti];
  if (kTan && t >= 64 && t < 100) rec[84 + t - 64] = sPhi[M - 1][t - 64];

  // the last block to finish decides and sweeps (the others' writes are fenced before their ticket)
  __threadfence();
  __syncthreads();
  if (t == 0) am_last = atomicAdd(&W.flags[4], 1) == (int)gridDim.x - 1;
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  const int c0 = P.sfp / P.m, c1 = P.sbp / P.m, nch = c0 + c1;  // chunks of each chain
  // every chunk's record, copied into the block's dynamic shared memory (the grid samples' area: this
  // block's integration is over) by asynchronous 16-byte copies, all in flight at once
  double *const sm = g_stage;
  {
    const int n16 = nch * kChunkDoubles / 2;
    for (int k = t; k < n16; k += blockDim.x) __pipeline_memcpy_async(sm + 2 * k, W.rec + 2 * k, 16);
    __pipeline_commit();
    __pipeline_wait_prior(0);
  }
  __syncthreads();
  // the boundary mismatches: chunk c's last segment against chunk c + 1's first start state, added to
  // b_c (the block left them out)
  double bm = 0.0;
  for (int k = t; k < nch * 6; k += blockDim.x) {
    const int cc = k / 6, i = k % 6;
    const Seg SL = seg_of(P, cc * M + M - 1);
    if (SL.active && !SL.last) {
      double *const ch = sm + kChunkDoubles * cc;
      const double r = ch[120 + i] - ch[kChunkDoubles + 126 + i];  // the next chunk's first start
      ch[36 + i] = ch[36 + i] + r;
      bm = fmax(bm, fabs(r) / (i < 3 ? W.scale_pos : W.scale_vel));
    }
  }
  for (int o = 16; o > 0; o >>= 1) bm = fmax(bm, __shfl_xor_sync(full, bm, o));
  if (lane == 0) wred[t >> 5] = bm;
  __syncthreads();
  if (t == 0) {
    double m = __longlong_as_double((long long)atomicAdd(reinterpret_cast<unsigned long long *>(W.rmax), 0ull));
    for (int k = 0; k < kShootThreads / 32; ++k) m = fmax(m, wred[k]);
    W.diag[iter < kMaxIters ? iter : kMaxIters - 1] = m;
    W.flags[1] = iter + 1;
    W.flags[3] = kTan ? 0 : 1;
    if (m <= kNear) W.flags[2] = 1;
    done = m <= kTol;
    if (done) W.flags[0] = 1;
    *W.rmax = 0.0;
    W.flags[4] = 0;
  }
  __syncthreads();
  if (done) return;
  // carry delta across the chunk maps: warp w < 2 sweeps chain w, lane i < 6 owning component i; delta
  // at each chunk's start replaces that chunk's [126, 132) slot and goes to global memory for the next
  // launch's expansion
  const int w = t >> 5;
  if (w < 2) {
    const int cn = w == 0 ? c0 : c1, first = w == 0 ? 0 : c0;
    const int i = lane < 6 ? lane : 0;
    double d = 0.0;
    for (int q = 0; q < cn; ++q) {
      double *const ch = sm + kChunkDoubles * (first + q);
      double dl[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) dl[k] = __shfl_sync(full, d, k);
      const double nd = ch[36 + i] + dot6(ch + 6 * i, 1, dl, 1);
      if (lane < 6) {
        W.dstart[6 * (first + q) + lane] = d;
        ch[126 + lane] = d;
      }
      d = nd;
    }
  }
  __syncthreads();
  // every chunk, in parallel: delta at its last segment's start (the map up to there; into the
  // chunk's [78, 84) slot), then the next chunk's first start state U' = F_last + Phi_last delta_last
  // (exactly F_last when delta_last = 0)
  for (int k = t; k < nch * 6; k += blockDim.x) {
    double *const ch = sm + kChunkDoubles * (k / 6);
    const int i = k % 6;
    ch[78 + i] = ch[78 + i] + dot6(ch + 42 + 6 * i, 1, ch + 126, 1);
  }
  __syncthreads();
  for (int k = t; k < nch * 6; k += blockDim.x) {
    const int cc = k / 6, i = k % 6, gl_ = cc * M + M - 1;
    const Seg SL = seg_of(P, gl_);
    if (SL.active && !SL.last) {
      const double *const ch = sm + kChunkDoubles * cc;
      W.U[6 * (gl_ + 1) + i] = ch[120 + i] + dot6(ch + 84 + 6 * i, 1, ch + 78, 1);
    }
  }
}

// One Newton iteration (pass kind from the flags: with tangents until the mismatches are small, then
// storing), or with final_pass the store pass after an iteration that converged without storing.
template <int G>
__global__ void __launch_bounds__(kShootThreads) shoot_pass_kernel(const srs_field *__restrict__ gfields, int nfields,
                                                                   const srs_particle *__restrict__ part, Plan P,
                                                                   Scratch W, double *__restrict__ X,
                                                                   double *__restrict__ Bt, double *__restrict__ A,
                                                                   int64_t stage_doubles, int final_pass) {
  __shared__ PassShared<kShootThreads / G> sh;
  // launched as a programmatic dependent of the previous kernel (launch_after): wait until that grid
  // has completed and its writes are visible, then let the next launch begin while this one runs
  wait_for_previous_grid();
  allow_next_grid();
  const int conv = W.flags[0], near = W.flags[2], stored = W.flags[3];
  if (final_pass) {
    if (conv && !stored) shoot_pass<G, false>(sh, gfields, nfields, part, P, W, X, Bt, A, stage_doubles, true);
  } else if (!conv) {
    if (near) shoot_pass<G, false>(sh, gfields, nfields, part, P, W, X, Bt, A, stage_doubles, false);
    else shoot_pass<G, true>(sh, gfields, nfields, part, P, W, X, Bt, A, stage_doubles, false);
  }
}

__global__ void shoot_stats_kernel(const int *__restrict__ flags, const double *__restrict__ diag,
                                   double *__restrict__ stats) {
  const int it = flags[1];
  stats[0] = flags[0];
  stats[1] = it;
  stats[2] = it > 0 ? diag[(it < kMaxIters ? it : kMaxIters) - 1] : 0.0;
  stats[3] = it > 1 ? diag[(it < kMaxIters ? it : kMaxIters) - 2] : 0.0;
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
  P.m = kShootThreads / lanes_for(nfields);
  auto chunks_for = [&](int64_t L) {
    return ((P.mf + L - 1) / L + P.m - 1) / P.m + ((P.mb + L - 1) / L + P.m - 1) / P.m;
  };
  if (steps_per_segment > 0) {
    P.L = steps_per_segment;
  } else {
    // A pass costs ~0.9 us per step of a segment (the blocks integrate their segments side by side)
    // plus ~0.09 us per chunk (the sequential sweep): L = sqrt(steps / 160) balances the two.  A pass
    // runs one block per chunk, one per SM (the sweep's shared memory), so longer segments when the
    // chunks would not fit one wave of kOneWaveChunks.
    int64_t L = shoot_default_steps(P.mf + P.mb);
    while (chunks_for(L) > kOneWaveChunks) ++L;
    P.L = (int)L;
  }
  // at most kMaxChunks chunks (their data are staged in shared memory for the sweep): longer segments
  // than asked for if needed
  while (((P.mf + P.L - 1) / P.L + (P.mb + P.L - 1) / P.L) > (int64_t)(kMaxChunks - 2) * P.m) P.L *= 2;
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

Scratch carve(void *scratch, const Plan &P) {
  const size_t segs = (size_t)(P.sfp + P.sbp) + 1, chunks = (size_t)(P.sfp + P.sbp) / P.m + 1;
  Scratch s;
  s.U = static_cast<double *>(scratch);
  s.F = s.U + 6 * segs;
  s.Phi = s.F + 6 * segs;
  s.rec = s.Phi + 36 * segs;
  s.dstart = s.rec + kChunkDoubles * chunks;
  s.diag = s.dstart + 6 * chunks;
  s.rmax = s.diag + kMaxIters;
  s.flags = reinterpret_cast<int *>(s.rmax + 1);
  s.prep = reinterpret_cast<Prepared *>(s.rmax + 5);  // after the 5 flags, 8-byte aligned
  s.scale_pos = s.scale_vel = 1.0;
  return s;
}

template <int G>
cudaError_t launch_pass(int blocks, size_t smem, cudaStream_t s, const srs_field *d_fields, int nfields,
                        const srs_particle *d_particle, const Plan &P, const Scratch &W, double *d_x, double *d_b,
                        double *d_a, int64_t stage_doubles, int final_pass) {
  if (smem > 0)
    if (cudaError_t e = cudaFuncSetAttribute(shoot_pass_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem))
      return e;
  return launch_after(shoot_pass_kernel<G>, dim3((unsigned)blocks), dim3(kShootThreads), smem, s, d_fields, nfields,
                      d_particle, P, W, d_x, d_b, d_a, stage_doubles, final_pass);
}

cudaError_t launch_pass_g(int G, int blocks, size_t smem, cudaStream_t s, const srs_field *d_fields, int nfields,
                          const srs_particle *d_particle, const Plan &P, const Scratch &W, double *d_x, double *d_b,
                          double *d_a, int64_t stage_doubles, int final_pass) {
  switch (G) {
    case 8:
      return launch_pass<8>(blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a, stage_doubles,
                            final_pass);
    case 16:
      return launch_pass<16>(blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a, stage_doubles,
                             final_pass);
    case 32:
      return launch_pass<32>(blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a, stage_doubles,
                             final_pass);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace

int shoot_default_steps(int64_t nsteps) {
  // steps per segment that balance a pass's integration (~0.9 us per step) against its sequential
  // chunk sweep (~0.09 us per chunk of 16 segments): L = sqrt(steps / 160), at least 4 (measured on
  // B200: 5001 to 40001 points, 14-25 % faster than 16 steps throughout)
  const int64_t L = llround(sqrt((double)std::max<int64_t>(nsteps, 1) / 160.0));
  return (int)std::max<int64_t>(4, L);
}

size_t shoot_scratch_bytes(int64_t nfwd, int64_t nbwd, int steps_per_segment, int nfields) {
  const Plan P = make_plan(nfwd, nbwd, 1.0, steps_per_segment, nfields);
  const size_t segs = (size_t)(P.sfp + P.sbp) + 1, chunks = (size_t)(P.sfp + P.sbp) / P.m + 1;
  return sizeof(double) * (segs * 48 + chunks * (kChunkDoubles + 6) + kMaxIters + 1) + 64 +
         sizeof(Prepared) * (size_t)nfields;
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
  W.scale_pos = fmax(fmax(xs, v0 * dt * (double)(P.mf > P.mb ? P.mf : P.mb)), 1e-300);
  W.scale_vel = fmax(v0, 1e-300);
  // dynamic shared memory: the grid samples during the integration, the chunk maps in the sweep
  const size_t smem = sizeof(double) * (size_t)std::max<int64_t>(stage_doubles, (int64_t)(segs / P.m) * kChunkDoubles);
  const int G = lanes_for(nfields), blocks = segs / P.m;
  shoot_init_kernel<<<(std::max(segs, nfields) + 127) / 128, 128, 0, s>>>(P, d_particle, W, d_fields, nfields);
  for (int it = 0; it < iters; ++it)
    if (cudaError_t e = launch_pass_g(G, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a,
                                      stage_doubles, 0))
      return e;
  // converged after a pass with tangents: one more pass stores the points
  if (cudaError_t e = launch_pass_g(G, blocks, smem, s, d_fields, nfields, d_particle, P, W, d_x, d_b, d_a,
                                    stage_doubles, 1))
    return e;
  if (d_stats) shoot_stats_kernel<<<1, 1, 0, s>>>(W.flags, W.diag, d_stats);
  if (cudaError_t e = cudaGetLastError()) return e;
  // the serial kernel, which returns at once when the iteration converged
  return launch_rk4_unless(d_fields, nfields, d_particle, dt, nfwd, nbwd, d_x, d_b, d_a, s, stage_doubles, W.flags);
}

}  // namespace srs

// Hand-written adjoint (reverse-mode derivative) of the on-axis spectrum and of the RK4 trajectory.
//
// The forward path is: initial state s0 = (x0, v0) and the fields -> RK4 states s_j (stored as the
// trajectory points x_j, beta_j = v_j / c) -> the sums E_k = Sum_i f_i(w_k) -> flux_k = C2 (C0 w_k dt)^2
// |E_k|^2 (OSCARSSR.cc:1154-1251).  Given dL/dflux_k this file computes dL/d(field parameters),
// dL/dx0, dL/dbeta0 and dL/d(q/(m gamma)).
//
// 1. Sum adjoint (spectrum_adjoint_kernel): one thread per trajectory point i, looping over the
//    energies, gives g_i = dL/d(x_i, beta_i) in closed form (derivatives of the amplitude
//    (beta - n(1 + i c/(w D)))/D and of the phase w (i dt + D/c) with respect to x and beta).
// 2. Trajectory adjoint: lambda_j = dL/ds_j obeys lambda_j = g_j + J_j^T lambda_{j+1}, where J_j is
//    the Jacobian of RK4 step j.  Instead of one serial sweep back through the N steps (the forward
//    RK4 is a serial chain; its adjoint need not be), the affine recurrence is solved as a scan:
//      (a) every step's 6 x 6 Jacobian is formed in parallel from the stored states, by forward-mode
//          tangents pushed through the four stages (step_jacobian_kernel);
//      (b) chunks of kAdjChunk steps are composed into one affine map lambda_j0 = M lambda_j1 + b
//          (chunk_compose_kernel);
//      (c) one warp carries lambda across the chunk maps from the last point back to the first
//          (carry_kernel);
//      (d) each chunk re-walks its steps backwards from its known end value, running the
//          reverse-mode step (VJP through the four stages, recomputed from the stored state) that
//          yields both lambda_j and the field-parameter and q/(m gamma) contributions
//          (chunk_finish_kernel).
//    The stored trajectory is itself the checkpoint set: the state at every step is in HBM (the sums
//    need every point anyway), so each step's stages are recomputed from its own stored state and
//    no sqrt(N) re-integration is needed.  The reverse pass does not re-run the forward integration.
// Both chains of the reference's trajectory are handled: forward from t0 with +dt (points nbwd ..
// n-1) and backward with -dt (points nbwd-1 .. 0), both starting from s0.
//
// States are in (x [m], beta) units so that the Jacobian entries are of comparable size.  All
// arithmetic is FP64.  Grid-sample gradients are accumulated with FP64 atomics (sub-ulp
// run-to-run differences); everything else is reduced in a fixed order.
#include <cuda_runtime.h>

#include <cuda_pipeline.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

constexpr int kAdjChunk = 16;     // steps per scan chunk
constexpr int kAdjMaxFields = 16;

__device__ inline void rot_matrix(const double r[3], double R[3][3]) {
  // R[i][j] = component i of rotate_xyz(e_j): the linear map the reference applies to the point
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    V3 e = v3(j == 0, j == 1, j == 2);
    rotate_xyz(e, r);
    R[0][j] = e.x;
    R[1][j] = e.y;
    R[2][j] = e.z;
  }
}
__device__ inline bool has_rotation(const double r[3]) { return r[0] != 0 || r[1] != 0 || r[2] != 0; }

// Corners of the grid interpolation at X: sample indices, weights and d(weight)/dX' per axis, where
// X' = R X - translation is the point in the grid's frame (TField3D_Grid.cc:124-243).  nc = 0 outside.
struct Corners {
  int nc;
  int64_t idx[8];
  double w[8];
  double dw[8][3];
};

__device__ void grid_corners(const srs_field &f, V3 XIN, Corners &C) {
  V3 X = XIN;
  if (has_rotation(f.rotations)) rotate_xyz(X, f.rotations);
  X = X - ld3(f.translation);
  const double xs[3] = {X.x, X.y, X.z};
  bool act[3];
  int64_t base[3];
  double t[3];
  C.nc = 0;
  for (int a = 0; a < 3; ++a) {
    act[a] = f.n[a] > 1;
    base[a] = 0;
    t[a] = 0;
    if (!act[a]) continue;
    if (xs[a] <= f.start[a] || xs[a] >= f.start[a] + (double)(f.n[a] - 1) * f.step[a]) return;
    uint64_t k = (uint64_t)((xs[a] - f.start[a]) / f.step[a]);
    if (k > (uint64_t)(f.n[a] - 2)) k = f.n[a] - 2;
    base[a] = (int64_t)k;
    t[a] = ((xs[a] - f.start[a]) - (double)k * f.step[a]) / f.step[a];
  }
  int na = 0, axes[3];
  for (int a = 0; a < 3; ++a)
    if (act[a]) axes[na++] = a;
  if (na == 0) return;
  C.nc = 1 << na;
  for (int c = 0; c < C.nc; ++c) {
    int64_t id[3] = {base[0], base[1], base[2]};
    double w = 1.0;
    double dwf[3] = {1.0, 1.0, 1.0};
    for (int q = 0; q < na; ++q) {
      const int a = axes[q];
      const int bit = (c >> q) & 1;
      id[a] += bit;
      const double fa = bit ? t[a] : 1.0 - t[a];
      const double da = (bit ? 1.0 : -1.0) / f.step[a];
      for (int r = 0; r < na; ++r) dwf[axes[r]] *= (r == q) ? da : fa;
      w *= fa;
    }
    C.idx[c] = id[0] * f.n[1] * f.n[2] + id[1] * f.n[2] + id[2];
    C.w[c] = w;
    for (int a = 0; a < 3; ++a) C.dw[c][a] = act[a] ? dwf[a] : 0.0;
  }
}

// Scalar profile of an amplitude field (B = field * shape) and its gradient in X.
__device__ double amp_shape(const srs_field &f, V3 X, V3 &grad) {
  grad = v3(0, 0, 0);
  if (f.kind == SRS_FIELD_UNDULATOR) {  // TField3D_IdealUndulator.cc:106-139
    const V3 per = ld3(f.period);
    const double plen = mag(per);
    const V3 u = unit(per);
    const double L = plen * (f.nperiods + 2);
    const double D = dot(X - ld3(f.center), u);
    const double ps = f.phase * plen / two_pi();
    if (D > L / 2. + ps || D < -L / 2. + ps) return 0.0;
    double a = 1.0;
    if (D < -L / 2. + ps + plen || D > L / 2. + ps - plen)
      a = (D < -L / 2. + ps + plen / 2. || D > L / 2. + ps - plen / 2.) ? 0.25 : 0.75;
    double s, c;
    sincos(two_pi() * (D - ps) / plen, &s, &c);
    const double tap = 1 + D * f.taper;
    const double dD = a * (c * (two_pi() / plen) * tap + s * f.taper);
    grad = u * dD;
    return a * s * tap;
  }
  if (f.kind == SRS_FIELD_GAUSSIAN) {  // TField3D_Gaussian.cc:88-113
    V3 xb = X;
    rotate_xyz(xb, f.rotations);
    const V3 rx = xb - ld3(f.center);
    const double r[3] = {rx.x, rx.y, rx.z};
    double frac = 1.0, g[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a)
      if (f.sigma_or_width[a] > 0) {
        const double tt = r[a] / f.sigma_or_width[a];
        frac *= exp(-(tt * tt) / 2.);
      }
    for (int a = 0; a < 3; ++a)
      if (f.sigma_or_width[a] > 0) g[a] = -frac * r[a] / (f.sigma_or_width[a] * f.sigma_or_width[a]);
    double R[3][3];
    rot_matrix(f.rotations, R);
    grad = v3(R[0][0] * g[0] + R[1][0] * g[1] + R[2][0] * g[2], R[0][1] * g[0] + R[1][1] * g[1] + R[2][1] * g[2],
              R[0][2] * g[0] + R[1][2] * g[1] + R[2][2] * g[2]);
    return frac;
  }
  if (f.kind == SRS_FIELD_UNIFORM_BOX) {  // TField3D_UniformBox.cc:93-111 (flat inside: no X gradient)
    V3 xb = X;
    rotate_xyz(xb, f.rotations);
    const V3 rx = xb - ld3(f.center);
    const double r[3] = {rx.x, rx.y, rx.z};
    for (int a = 0; a < 3; ++a)
      if (f.sigma_or_width[a] > 0 && fabs(r[a]) > fabs(f.sigma_or_width[a] / 2.)) return 0.0;
    return 1.0;
  }
  return 0.0;
}

// Sum of the fields at X and its Jacobian J[i][j] = dB_i / dX_j.
__device__ void field_jet(const srs_field *F, int nf, V3 X, V3 &B, double J[3][3]) {
  B = v3(0, 0, 0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) J[i][j] = 0.0;
  for (int q = 0; q < nf; ++q) {
    const srs_field &f = F[q];
    if (f.kind == SRS_FIELD_GRID) {
      Corners C;
      grid_corners(f, X, C);
      if (C.nc == 0) continue;
      double dBp[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};  // dB/dX' (grid frame)
      for (int c = 0; c < C.nc; ++c) {
        const V3 s = ld3(f.data + 3 * C.idx[c]);
        B = B + s * C.w[c];
        for (int a = 0; a < 3; ++a) {
          dBp[0][a] += s.x * C.dw[c][a];
          dBp[1][a] += s.y * C.dw[c][a];
          dBp[2][a] += s.z * C.dw[c][a];
        }
      }
      if (has_rotation(f.rotations)) {
        double R[3][3];
        rot_matrix(f.rotations, R);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[i][j] += dBp[i][0] * R[0][j] + dBp[i][1] * R[1][j] + dBp[i][2] * R[2][j];
      } else {
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) J[i][j] += dBp[i][j];
      }
    } else {
      V3 g;
      const double sh = amp_shape(f, X, g);
      const V3 A = ld3(f.field);
      B = B + A * sh;
      const double a[3] = {A.x, A.y, A.z}, gg[3] = {g.x, g.y, g.z};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J[i][j] += a[i] * gg[j];
    }
  }
}

// dL/d(field parameters) += (dB(X)/d parameters)^T Bbar: amplitude fields into amp[3 q + i] (a
// per-thread array), grid samples into the field's gradient array with atomics.
__device__ void field_param_vjp(const srs_field *F, int nf, V3 X, V3 Bbar, double *amp, double *const *grid_grads) {
  for (int q = 0; q < nf; ++q) {
    const srs_field &f = F[q];
    if (f.kind == SRS_FIELD_GRID) {
      double *gg = grid_grads ? grid_grads[q] : nullptr;
      if (!gg) continue;
      Corners C;
      grid_corners(f, X, C);
      for (int c = 0; c < C.nc; ++c) {
        atomicAdd(gg + 3 * C.idx[c] + 0, C.w[c] * Bbar.x);
        atomicAdd(gg + 3 * C.idx[c] + 1, C.w[c] * Bbar.y);
        atomicAdd(gg + 3 * C.idx[c] + 2, C.w[c] * Bbar.z);
      }
    } else if (q < kAdjMaxFields) {
      V3 g;
      const double sh = amp_shape(f, X, g);
      amp[3 * q + 0] += sh * Bbar.x;
      amp[3 * q + 1] += sh * Bbar.y;
      amp[3 * q + 2] += sh * Bbar.z;
    }
  }
}

__device__ inline V3 matvec(const double J[3][3], V3 d) {
  return v3(J[0][0] * d.x + J[0][1] * d.y + J[0][2] * d.z, J[1][0] * d.x + J[1][1] * d.y + J[1][2] * d.z,
            J[2][0] * d.x + J[2][1] * d.y + J[2][2] * d.z);
}
__device__ inline V3 matTvec(const double J[3][3], V3 d) {
  return v3(J[0][0] * d.x + J[1][0] * d.y + J[2][0] * d.z, J[0][1] * d.x + J[1][1] * d.y + J[2][1] * d.z,
            J[0][2] * d.x + J[1][2] * d.y + J[2][2] * d.z);
}

// The four stage states of RK4 step (pos, vel, h), with B and dB/dX at each (same stage structure as
// the forward integrator: OSCARSSR.cc:826-874).
struct Stages {
  V3 p[4], v[4], B[4];
  double J[4][3][3];
};

__device__ void make_stages(const srs_field *F, int nf, double q, V3 pos, V3 vel, double h, Stages &S) {
  const double hh = 0.5 * h;
  S.p[0] = pos;
  S.v[0] = vel;
  field_jet(F, nf, S.p[0], S.B[0], S.J[0]);
  V3 a = cross(S.v[0], S.B[0]) * q;
  S.p[1] = pos + S.v[0] * hh;
  S.v[1] = vel + a * hh;
  field_jet(F, nf, S.p[1], S.B[1], S.J[1]);
  a = cross(S.v[1], S.B[1]) * q;
  S.p[2] = pos + S.v[1] * hh;
  S.v[2] = vel + a * hh;
  field_jet(F, nf, S.p[2], S.B[2], S.J[2]);
  a = cross(S.v[2], S.B[2]) * q;
  S.p[3] = pos + S.v[2] * h;
  S.v[3] = vel + a * h;
  field_jet(F, nf, S.p[3], S.B[3], S.J[3]);
}

// Forward-mode: the tangent (dp, dv, dq) of the step's input -> tangent of its output.
__device__ void step_jvp(const Stages &S, double q, double h, V3 dp, V3 dv, double dq, V3 &odp, V3 &odv) {
  const double hh = 0.5 * h, coef[4] = {0.0, hh, hh, h}, wgt[4] = {1.0, 2.0, 2.0, 1.0};
  V3 sp = dp, sv = dv, accp = v3(0, 0, 0), accv = v3(0, 0, 0), da = v3(0, 0, 0);
  for (int s = 0; s < 4; ++s) {
    if (s > 0) {
      sp = dp + sv * coef[s];  // p_s = pos + coef_s v_{s-1}
      sv = dv + da * coef[s];  // v_s = vel + coef_s a_{s-1}
    }
    da = (cross(S.v[s], S.B[s]) * dq + cross(sv, S.B[s]) * q + cross(S.v[s], matvec(S.J[s], sp)) * q);
    accp = accp + sv * wgt[s];
    accv = accv + da * wgt[s];
  }
  odp = dp + accp * (h / 6.0);
  odv = dv + accv * (h / 6.0);
}

// Reverse-mode: adjoint (lp, lv) of the step's output -> adjoint of its input (pb, vb), q/(m gamma)
// adjoint qb, and the field-parameter contributions.
__device__ void step_vjp(const srs_field *F, int nf, const Stages &S, double q, double h, V3 lp, V3 lv, V3 &pb,
                         V3 &vb, double &qb, double *amp, double *const *grid_grads) {
  const double hh = 0.5 * h, coef[4] = {0.0, hh, hh, h}, wgt[4] = {1.0, 2.0, 2.0, 1.0};
  V3 vbar[4], abar[4];
  for (int s = 0; s < 4; ++s) {
    vbar[s] = lp * (h / 6.0 * wgt[s]);
    abar[s] = lv * (h / 6.0 * wgt[s]);
  }
  pb = lp;
  vb = lv;
  for (int s = 3; s >= 0; --s) {
    // a_s = q v_s x B_s
    vbar[s] = vbar[s] + cross(S.B[s], abar[s]) * q;
    const V3 Bbar = cross(abar[s], S.v[s]) * q;
    qb += dot(abar[s], cross(S.v[s], S.B[s]));
    const V3 pbar = matTvec(S.J[s], Bbar);
    field_param_vjp(F, nf, S.p[s], Bbar, amp, grid_grads);
    pb = pb + pbar;
    vb = vb + vbar[s];
    if (s > 0) {
      abar[s - 1] = abar[s - 1] + vbar[s] * coef[s];
      vbar[s - 1] = vbar[s - 1] + pbar * coef[s];
    }
  }
}

// ---------------------------------------------------------------- chains and scan

struct Chain {
  int64_t L;         // states in the chain (steps: L - 1)
  double h;          // step
  int64_t base;      // stored index of state 0
  int dir;           // stored index of state j: base + dir * j
  int64_t nch;       // chunks
  int64_t chunk_off; // first global chunk index
  int64_t step_off;  // first global step index (Jacobian storage)
  int skip_g0;       // state 0's g belongs to the other chain
};
struct Chains {
  Chain c[2];
  int n;
  int64_t total_chunks, total_steps;
};

struct Traj {
  const double *x, *beta, *gx, *gb;
  int64_t n;
};

__device__ inline void load_state(const Traj &T, int64_t k, V3 &pos, V3 &vel) {
  pos = v3(T.x[k], T.x[T.n + k], T.x[2 * T.n + k]);
  vel = v3(T.beta[k] * kC, T.beta[T.n + k] * kC, T.beta[2 * T.n + k] * kC);
}
// g of chain state j in (x, beta) units
__device__ inline void load_g(const Traj &T, const Chain &ch, int64_t j, double g[6]) {
  if (j == 0 && ch.skip_g0) {
    for (int r = 0; r < 6; ++r) g[r] = 0.0;
    return;
  }
  const int64_t k = ch.base + ch.dir * j;
  for (int c = 0; c < 3; ++c) {
    g[c] = T.gx[c * T.n + k];
    g[3 + c] = T.gb[c * T.n + k];
  }
}

__device__ inline int find_chain(const Chains &C, int64_t gidx, bool steps) {
  return (C.n > 1 && gidx >= (steps ? C.c[1].step_off : C.c[1].chunk_off)) ? 1 : 0;
}

// (a) J~_j (6 x 6, row = output, column = input, in (x, beta) units) of every step.
__global__ void __launch_bounds__(128) step_jacobian_kernel(const srs_field *__restrict__ gF, int nf, double q, Traj T,
                                                            Chains C, double *__restrict__ jac) {
  __shared__ srs_field F[kAdjMaxFields];
  for (int i = threadIdx.x; i < nf; i += blockDim.x) F[i] = gF[i];
  __syncthreads();
  const int64_t gs = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gs >= C.total_steps) return;
  const Chain &ch = C.c[find_chain(C, gs, true)];
  const int64_t j = gs - ch.step_off;
  V3 pos, vel;
  load_state(T, ch.base + ch.dir * j, pos, vel);
  Stages S;
  make_stages(F, nf, q, pos, vel, ch.h, S);
  double *Jo = jac + 36 * gs;
  for (int col = 0; col < 6; ++col) {
    V3 dp = v3(0, 0, 0), dv = v3(0, 0, 0);
    if (col < 3) dp = v3(col == 0, col == 1, col == 2);
    else dv = v3(col == 3, col == 4, col == 5) * kC;
    V3 op, ov;
    step_jvp(S, q, ch.h, dp, dv, 0.0, op, ov);
    const double out[6] = {op.x, op.y, op.z, ov.x / kC, ov.y / kC, ov.z / kC};
    for (int r = 0; r < 6; ++r) Jo[6 * r + col] = out[r];
  }
}

// (b) per chunk [j0, j1): lambda_j0 = M lambda_j1 + b, composed backwards from M = I, b = 0.
__global__ void chunk_compose_kernel(Traj T, Chains C, const double *__restrict__ jac, double *__restrict__ Mb) {
  const int64_t gc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gc >= C.total_chunks) return;
  const Chain &ch = C.c[find_chain(C, gc, false)];
  const int64_t c = gc - ch.chunk_off;
  const int64_t j0 = c * kAdjChunk, j1 = imin64(j0 + kAdjChunk, ch.L - 1);
  double M[6][6], b[6];
  for (int r = 0; r < 6; ++r) {
    b[r] = 0.0;
    for (int k = 0; k < 6; ++k) M[r][k] = r == k;
  }
  for (int64_t j = j1 - 1; j >= j0; --j) {
    const double *Jj = jac + 36 * (ch.step_off + j);
    double A[6][6];  // A = J^T
    for (int r = 0; r < 6; ++r)
      for (int k = 0; k < 6; ++k) A[r][k] = Jj[6 * k + r];
    double g[6];
    load_g(T, ch, j, g);
    double nb[6], nM[6][6];
    for (int r = 0; r < 6; ++r) {
      double s = g[r];
      for (int k = 0; k < 6; ++k) s += A[r][k] * b[k];
      nb[r] = s;
      for (int col = 0; col < 6; ++col) {
        double t = 0.0;
        for (int k = 0; k < 6; ++k) t += A[r][k] * M[k][col];
        nM[r][col] = t;
      }
    }
    for (int r = 0; r < 6; ++r) {
      b[r] = nb[r];
      for (int col = 0; col < 6; ++col) M[r][col] = nM[r][col];
    }
  }
  double *o = Mb + 42 * gc;
  for (int r = 0; r < 6; ++r) {
    for (int col = 0; col < 6; ++col) o[6 * r + col] = M[r][col];
    o[36 + r] = b[r];
  }
}

// (c) one warp per chain, lanes 0..5 own one component: lambda at every chunk start.  The sweep is
// sequential over the chunks, so the chunk maps come through shared memory in tiles of kCarryTile,
// the next tile's asynchronous copies in flight while the current one is swept (a step then waits on
// shared memory, not on a global load: 1250 chunks of config 4 took 0.63 ms with the maps read from
// global memory step by step).
constexpr int kCarryTile = 64;  // chunk maps per tile: 64 x 42 doubles = 21.5 KB, two buffers
__global__ void __launch_bounds__(32) carry_kernel(Traj T, Chains C, const double *__restrict__ Mb,
                                                   double *__restrict__ lam0) {
  __shared__ __align__(16) double tile[2][kCarryTile * 42];
  const int chain = blockIdx.x;
  if (chain >= C.n) return;
  const Chain &ch = C.c[chain];
  const int r = threadIdx.x;
  double g[6];
  load_g(T, ch, ch.L - 1, g);
  double lam = r < 6 ? g[r] : 0.0;  // lambda_{L-1} = g_{L-1}
  const int64_t nch = ch.nch, ntiles = (nch + kCarryTile - 1) / kCarryTile;
  // tile t: chunks [lo(t), hi(t)], hi(t) = nch - 1 - t * kCarryTile, swept from hi down to lo
  auto lo_of = [&](int64_t t) {
    const int64_t hi = nch - 1 - t * kCarryTile;
    return hi - kCarryTile + 1 > 0 ? hi - kCarryTile + 1 : (int64_t)0;
  };
  auto fetch = [&](int64_t t, int buf) {  // 16-byte copies: a chunk map is 21 of them, 16-byte aligned
    const int64_t hi = nch - 1 - t * kCarryTile, lo = lo_of(t);
    const double *src = Mb + 42 * (ch.chunk_off + lo);
    const int n16 = (int)(hi - lo + 1) * 21;
    for (int k = r; k < n16; k += 32) __pipeline_memcpy_async(&tile[buf][2 * k], src + 2 * k, 16);
    __pipeline_commit();
  };
  if (ntiles > 0) fetch(0, 0);
  for (int64_t t = 0; t < ntiles; ++t) {
    const int buf = (int)(t & 1);
    if (t + 1 < ntiles) fetch(t + 1, buf ^ 1);
    else __pipeline_commit();  // an empty group, so that "all but the newest" is always tile t
    __pipeline_wait_prior(1);
    __syncwarp();
    const int64_t hi = nch - 1 - t * kCarryTile, lo = lo_of(t);
    const int rr = r < 6 ? r : 0;
    for (int64_t c = hi; c >= lo; --c) {
      const double *o = &tile[buf][42 * (c - lo)];
      double l[6];
#pragma unroll
      for (int k = 0; k < 6; ++k) l[k] = __shfl_sync(0xffffffffu, lam, k);
      // b + M lambda as a tree (depth 4 instead of a chain of six multiply-adds: the sweep is a chain
      // of these, one per chunk)
      const double *m = o + 6 * rr;
      const double p0 = m[0] * l[0], p1 = m[1] * l[1], p2 = m[2] * l[2], p3 = m[3] * l[3], p4 = m[4] * l[4],
                   p5 = m[5] * l[5];
      lam = o[36 + rr] + (((p0 + p1) + (p2 + p3)) + (p4 + p5));
      if (r < 6) lam0[6 * (ch.chunk_off + c) + r] = lam;
    }
    __syncwarp();  // every lane is done with this buffer before the next iteration refills it
  }
}

// (d) per chunk: walk back from lambda_j1 with the reverse-mode step; field-parameter and q
// contributions go to per-chunk partials (amplitudes, q) or atomics (grid samples).
__global__ void __launch_bounds__(64) chunk_finish_kernel(const srs_field *__restrict__ gF, int nf, double q, Traj T,
                                                          Chains C, const double *__restrict__ lam0,
                                                          double *const *grid_grads, double *__restrict__ amp_part,
                                                          double *__restrict__ q_part, double *__restrict__ lam_init) {
  __shared__ srs_field F[kAdjMaxFields];
  for (int i = threadIdx.x; i < nf; i += blockDim.x) F[i] = gF[i];
  __syncthreads();
  const int64_t gc = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gc >= C.total_chunks) return;
  const int chain = find_chain(C, gc, false);
  const Chain &ch = C.c[chain];
  const int64_t c = gc - ch.chunk_off;
  const int64_t j0 = c * kAdjChunk, j1 = imin64(j0 + kAdjChunk, ch.L - 1);
  double lam[6];
  if (c == ch.nch - 1) {
    load_g(T, ch, ch.L - 1, lam);
  } else {
    for (int r = 0; r < 6; ++r) lam[r] = lam0[6 * (ch.chunk_off + c + 1) + r];
  }
  double amp[3 * kAdjMaxFields];
  for (int i = 0; i < 3 * kAdjMaxFields; ++i) amp[i] = 0.0;
  double qb = 0.0;
  for (int64_t j = j1 - 1; j >= j0; --j) {
    V3 pos, vel;
    load_state(T, ch.base + ch.dir * j, pos, vel);
    Stages S;
    make_stages(F, nf, q, pos, vel, ch.h, S);
    V3 pb, vb;
    step_vjp(F, nf, S, q, ch.h, v3(lam[0], lam[1], lam[2]), v3(lam[3], lam[4], lam[5]) * (1.0 / kC), pb, vb, qb, amp,
             grid_grads);
    double g[6];
    load_g(T, ch, j, g);
    lam[0] = g[0] + pb.x;
    lam[1] = g[1] + pb.y;
    lam[2] = g[2] + pb.z;
    lam[3] = g[3] + vb.x * kC;
    lam[4] = g[4] + vb.y * kC;
    lam[5] = g[5] + vb.z * kC;
  }
  for (int i = 0; i < 3 * nf && i < 3 * kAdjMaxFields; ++i) amp_part[(int64_t)3 * nf * gc + i] = amp[i];
  q_part[gc] = qb;
  if (c == 0)
    for (int r = 0; r < 6; ++r) lam_init[6 * chain + r] = lam[r];
}

// Fixed-order totals: out[0..2] dL/dx0, out[3..5] dL/dbeta0, out[6] dL/dq, out[7..] amplitudes.  The
// per-chunk partials of q and of each amplitude are added by the block: thread t adds a contiguous
// run of chunks in order, then a fixed tree over the 128 runs (a deterministic order; one thread
// adding all 1250 partials of config 4 one load after another took 0.12 ms).
__global__ void __launch_bounds__(128) adjoint_total_kernel(Chains C, int nf, const double *__restrict__ lam_init,
                                                            const double *__restrict__ amp_part,
                                                            const double *__restrict__ q_part,
                                                            double *__restrict__ out) {
  __shared__ double red[128];
  const int t = threadIdx.x;
  if (t < 6) {
    double s = 0.0;
    for (int k = 0; k < C.n; ++k) s += lam_init[6 * k + t];
    out[t] = s;
  }
  const int64_t total = C.total_chunks, per = (total + 127) / 128;
  const int64_t g0 = t * per, g1 = g0 + per < total ? g0 + per : total;
  for (int o = 0; o < 1 + 3 * nf; ++o) {  // o = 0: q; o = 1 + i: amplitude i
    double s = 0.0;
    for (int64_t g = g0; g < g1; ++g) s += o == 0 ? q_part[g] : amp_part[(int64_t)3 * nf * g + (o - 1)];
    red[t] = s;
    __syncthreads();
    for (int w = 64; w > 0; w >>= 1) {
      if (t < w) red[t] += red[t + w];
      __syncthreads();
    }
    if (t == 0) out[6 + o] = red[0];
    __syncthreads();
  }
}

// ---------------------------------------------------------------- sum adjoint

// Per energy k: W_k = 2 w_k conj(E_k) with w_k = dL/dflux_k * C2 (C0 w_k dt)^2.
__global__ void spectrum_weights_kernel(const double *__restrict__ energies, const double *__restrict__ e6,
                                        const double *__restrict__ gflux, int64_t ne, double dt, double C0, double C2,
                                        double *__restrict__ W) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const double om = ev_to_omega(energies[k]);
  const double g = C0 * om * dt;
  const double w = 2.0 * gflux[k] * C2 * g * g;
  W[8 * k + 0] = om;
  for (int c = 0; c < 3; ++c) {
    W[8 * k + 1 + 2 * c] = w * e6[6 * k + 2 * c];
    W[8 * k + 2 + 2 * c] = -w * e6[6 * k + 2 * c + 1];
  }
}

constexpr int kSumAdjThreads = 128, kSumAdjTile = 128;

__global__ void __launch_bounds__(kSumAdjThreads) spectrum_adjoint_kernel(const double *__restrict__ X,
                                                                          const double *__restrict__ Bt, int64_t n,
                                                                          double dt, V3 obs,
                                                                          const double *__restrict__ W, int64_t ne,
                                                                          double *__restrict__ gx,
                                                                          double *__restrict__ gb) {
  __shared__ double sW[kSumAdjTile][8];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  const int64_t ii = active ? i : n - 1;
  const V3 x = v3(X[ii], X[n + ii], X[2 * n + ii]);
  const V3 be = v3(Bt[ii], Bt[n + ii], Bt[2 * n + ii]);
  // D, n and the retarded time exactly as the plain FP64 sum forms them (this file is compiled
  // without FMA contraction): the phases w tau are ~1e10 rad, and the adjoint's e^{i w tau} must be
  // the forward's own to the last bit, or the gradient along the trajectory (the near-invariant
  // longitudinal direction, where the per-point terms cancel to ~1e-10) is lost in phase noise.
  const V3 R = obs - x;
  const double D = mag(R), iD = 1.0 / D;
  const V3 nv = R / D;
  const double tau = dt * (double)(int)ii + D / kC;
  const double nn[3] = {nv.x, nv.y, nv.z}, bb[3] = {be.x, be.y, be.z};
  double A[3] = {0, 0, 0}, Bc[3] = {0, 0, 0}, Tt = 0.0;
  for (int64_t k0 = 0; k0 < ne; k0 += kSumAdjTile) {
    const int cnt = (int)imin64(kSumAdjTile, ne - k0);
    __syncthreads();
    for (int t = threadIdx.x; t < cnt * 8; t += blockDim.x) sW[t / 8][t % 8] = W[8 * k0 + t];
    __syncthreads();
    for (int k = 0; k < cnt; ++k) {
      const double om = sW[k][0];
      double sn, cs;
      sincos(reduce_2pi(om * tau), &sn, &cs);
      const double cow = kC / om, woc = om / kC;
      double s1r = 0.0, s2i = 0.0, s3i = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double wr = sW[k][1 + 2 * c], wi = sW[k][2 + 2 * c];
        const double pr = wr * cs - wi * sn, pi = wr * sn + wi * cs;  // P = W e^{i a}
        A[c] += pr;
        Bc[c] += cow * pi;
        s1r += pr * (bb[c] - 2.0 * nn[c]);
        s2i += pi * nn[c];
        // (w/c) Im(P u) with u = (beta - n)/D - i (c/w) n / D^2
        s3i += -pr * nn[c] * iD * iD + woc * pi * (bb[c] - nn[c]) * iD;
      }
      Tt += s1r * iD * iD + 3.0 * cow * s2i * iD * iD * iD + s3i;
    }
  }
  if (!active) return;
  const double iD2 = iD * iD, iD3 = iD2 * iD;
  for (int c = 0; c < 3; ++c) {
    gb[c * n + i] = A[c] * iD;
    gx[c * n + i] = A[c] * iD2 - Bc[c] * iD3 + nn[c] * Tt;
  }
}

}  // namespace
}  // namespace srs

using namespace srs;

extern "C" {

srs_status srs_spectrum_efield(srs_traj_view traj, srs_beam_consts beam, const double obs[3],
                               const double *d_energies, int64_t ne, int32_t precision, double *d_flux,
                               double *d_e6, void *stream) {
  clear_error();
  if (!traj.x || !traj.beta || traj.n < 1 || traj.nparticles < 1 || !(traj.dt > 0))
    return fail(SRS_ERR_INVALID, "bad trajectory view");
  if (!obs || !d_energies || !d_flux || !d_e6 || ne < 1) return fail(SRS_ERR_INVALID, "bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer scratch;
  if (precision == SRS_PRECISION_FP64) {
    SRS_CUDA(scratch.alloc(fp64_spectrum_scratch_bytes(traj.n, ne, traj.nparticles), s));
    SRS_CUDA(fp64_spectrum(traj, beam, obs, d_energies, ne, d_flux, scratch.ptr, s, d_e6));
  } else if (precision == SRS_PRECISION_MIXED) {
    SRS_CUDA(scratch.alloc(mixed_spectrum_scratch_bytes(traj.n, ne, traj.nparticles), s));
    SRS_CUDA(mixed_spectrum(traj, beam, obs, d_energies, ne, d_flux, scratch.ptr, s, d_e6));
  } else {
    return fail(SRS_ERR_INVALID, "unknown precision");
  }
  return SRS_OK;
}

srs_status srs_spectrum_adjoint(srs_traj_view traj, srs_beam_consts beam, const double obs[3],
                                const double *d_energies, int64_t ne, const double *d_e6, const double *d_gflux,
                                double *d_gx, double *d_gbeta, void *stream) {
  clear_error();
  if (!traj.x || !traj.beta || traj.n < 1 || !(traj.dt > 0)) return fail(SRS_ERR_INVALID, "bad trajectory view");
  if (traj.nparticles != 1) return fail(SRS_ERR_INVALID, "the spectrum adjoint takes one particle");
  if (!obs || !d_energies || !d_e6 || !d_gflux || !d_gx || !d_gbeta || ne < 1)
    return fail(SRS_ERR_INVALID, "bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer W;
  SRS_CUDA(W.alloc(sizeof(double) * 8 * ne, s));
  spectrum_weights_kernel<<<(unsigned)((ne + 127) / 128), 128, 0, s>>>(
      d_energies, d_e6, d_gflux, ne, traj.dt, flux_c0(beam.charge), flux_c2(beam.charge, beam.current), W.as<double>());
  SRS_CUDA(cudaGetLastError());
  spectrum_adjoint_kernel<<<(unsigned)((traj.n + kSumAdjThreads - 1) / kSumAdjThreads), kSumAdjThreads, 0, s>>>(
      traj.x, traj.beta, traj.n, traj.dt, v3(obs[0], obs[1], obs[2]), W.as<double>(), ne, d_gx, d_gbeta);
  SRS_CUDA(cudaGetLastError());
  return SRS_OK;
}

srs_status srs_trajectory_adjoint(const srs_field *fields, int32_t nfields, const srs_particle *particle,
                                  double ctstart, double ctstop, double t0, int64_t npoints, const double *d_x,
                                  const double *d_beta, const double *d_gx, const double *d_gbeta,
                                  double *const *grid_grads, double *amp_grad, double *ic_grad, void *stream) {
  clear_error();
  if (!particle || !d_x || !d_beta || !d_gx || !d_gbeta || !ic_grad) return fail(SRS_ERR_INVALID, "NULL argument");
  if (nfields < 0 || nfields > kAdjMaxFields || (nfields > 0 && !fields))
    return fail(SRS_ERR_INVALID, "the adjoint takes 0.." + std::to_string(kAdjMaxFields) + " fields");
  if (has_electric(fields, nfields)) return fail(SRS_ERR_INVALID, "the adjoint takes magnetic fields only");
  double dt;
  int64_t nf, nb;
  if (srs_status st = srs_trajectory_counts(ctstart, ctstop, t0, npoints, &dt, &nf, &nb)) return st;
  if (nf < 1) return fail(SRS_ERR_INVALID, "empty forward trajectory");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Chains C;
  std::memset(&C, 0, sizeof C);
  int64_t chunks = 0, steps = 0;
  auto add = [&](int64_t L, double h, int64_t base, int dir, int skip) {
    Chain &ch = C.c[C.n++];
    ch.L = L;
    ch.h = h;
    ch.base = base;
    ch.dir = dir;
    ch.skip_g0 = skip;
    ch.nch = L > 1 ? (L - 1 + kAdjChunk - 1) / kAdjChunk : 0;
    ch.chunk_off = chunks;
    ch.step_off = steps;
    chunks += ch.nch;
    steps += L - 1;
  };
  add(nf, dt, nb, +1, 0);
  if (nb > 0) add(nb + 1, -dt, nb, -1, 1);
  C.total_chunks = chunks;
  C.total_steps = steps;
  const Traj T{d_x, d_beta, d_gx, d_gbeta, nf + nb};
  const double q = particle->qomg;

  // device copies: fields, grid-gradient pointer table
  DeviceBuffer dF, dG, jac, Mb, lam0, amp, qp, laminit, out;
  SRS_CUDA(dF.alloc(sizeof(srs_field) * std::max(1, nfields), s));
  SRS_CUDA(dG.alloc(sizeof(double *) * std::max(1, nfields), s));
  std::vector<double *> gg(std::max(1, nfields), nullptr);
  for (int i = 0; i < nfields; ++i) gg[i] = grid_grads ? grid_grads[i] : nullptr;
  if (nfields > 0)
    SRS_CUDA(cudaMemcpyAsync(dF.ptr, fields, sizeof(srs_field) * nfields, cudaMemcpyHostToDevice, s));
  SRS_CUDA(cudaMemcpyAsync(dG.ptr, gg.data(), sizeof(double *) * gg.size(), cudaMemcpyHostToDevice, s));
  SRS_CUDA(jac.alloc(sizeof(double) * 36 * std::max<int64_t>(1, steps), s));
  SRS_CUDA(Mb.alloc(sizeof(double) * 42 * std::max<int64_t>(1, chunks), s));
  SRS_CUDA(lam0.alloc(sizeof(double) * 6 * std::max<int64_t>(1, chunks), s));
  SRS_CUDA(amp.alloc(sizeof(double) * 3 * std::max(1, nfields) * std::max<int64_t>(1, chunks), s));
  SRS_CUDA(qp.alloc(sizeof(double) * std::max<int64_t>(1, chunks), s));
  SRS_CUDA(laminit.alloc(sizeof(double) * 12, s));
  SRS_CUDA(out.alloc(sizeof(double) * (7 + 3 * std::max(1, nfields)), s));
  SRS_CUDA(cudaMemsetAsync(laminit.ptr, 0, sizeof(double) * 12, s));
  const srs_field *Fd = dF.as<srs_field>();
  if (steps > 0) {
    step_jacobian_kernel<<<(unsigned)((steps + 127) / 128), 128, 0, s>>>(Fd, nfields, q, T, C, jac.as<double>());
    SRS_CUDA(cudaGetLastError());
    chunk_compose_kernel<<<(unsigned)((chunks + 63) / 64), 64, 0, s>>>(T, C, jac.as<double>(), Mb.as<double>());
    SRS_CUDA(cudaGetLastError());
    carry_kernel<<<C.n, 32, 0, s>>>(T, C, Mb.as<double>(), lam0.as<double>());
    SRS_CUDA(cudaGetLastError());
    chunk_finish_kernel<<<(unsigned)((chunks + 63) / 64), 64, 0, s>>>(
        Fd, nfields, q, T, C, lam0.as<double>(), reinterpret_cast<double *const *>(dG.ptr), amp.as<double>(),
        qp.as<double>(), laminit.as<double>());
    SRS_CUDA(cudaGetLastError());
  }
  // chains of a single state: lambda_0 = g_0
  for (int k = 0; k < C.n; ++k)
    if (C.c[k].L == 1 && !C.c[k].skip_g0) {
      for (int c = 0; c < 3; ++c) {
        SRS_CUDA(cudaMemcpyAsync(laminit.as<double>() + 6 * k + c, d_gx + c * T.n + C.c[k].base, sizeof(double),
                                 cudaMemcpyDeviceToDevice, s));
        SRS_CUDA(cudaMemcpyAsync(laminit.as<double>() + 6 * k + 3 + c, d_gbeta + c * T.n + C.c[k].base,
                                 sizeof(double), cudaMemcpyDeviceToDevice, s));
      }
    }
  adjoint_total_kernel<<<1, 128, 0, s>>>(C, nfields, laminit.as<double>(), amp.as<double>(), qp.as<double>(),
                                         out.as<double>());
  SRS_CUDA(cudaGetLastError());
  std::vector<double> h(7 + 3 * std::max(1, nfields));
  SRS_CUDA(cudaMemcpyAsync(h.data(), out.ptr, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, s));
  SRS_CUDA(cudaStreamSynchronize(s));
  for (int i = 0; i < 7; ++i) ic_grad[i] = h[i];
  if (amp_grad)
    for (int i = 0; i < 3 * nfields; ++i) amp_grad[i] = h[7 + i];
  return SRS_OK;
}

}  // extern "C"

// Field evaluation and RK4 steps shared by the trajectory kernels (rk4.cu, rk4_shoot.cu).  Both
// translation units are compiled with -fmad=false, so the steps below round exactly like the
// reference's x86-64 build (src/OSCARSSR.cc:741-765, 826-874).
#pragma once

#include <cuda_runtime.h>

#include "srs_device.cuh"

namespace srs {
namespace {

constexpr int kMaxFieldsShared = 16;
// grid samples staged in shared memory when all grid fields together fit (192 KB)
constexpr int64_t kGridStageMaxDoubles = 24576;


// Field constants the reference derives inside GetF (or in Init) from the descriptor.
struct Prepared {
  int kind;
  double F[3], C[3], u[3];
  double plen, rplen, ps, taper, b_lo, b_hi, e1_lo, e1_hi, e2_lo, e2_hi;  // undulator
  double rs[3], rc[3];                                                     // rotation sines / cosines
  const double *gd;                                                        // grid samples (shared or global)
  double rstep[3];                                                         // grid: 1 / step per axis
};

__device__ void prepare(const srs_field &f, Prepared &p) {
  p.kind = f.kind;
  p.gd = f.data;
  for (int c = 0; c < 3; ++c) p.rstep[c] = f.step[c] != 0 ? 1.0 / f.step[c] : 0.0;
  for (int c = 0; c < 3; ++c) {
    p.F[c] = f.field[c];
    p.C[c] = f.center[c];
    p.rs[c] = sin(f.rotations[c]);
    p.rc[c] = cos(f.rotations[c]);
  }
  if (f.kind == SRS_FIELD_UNDULATOR) {
    // TField3D_IdealUndulator::Init (:62-80) and the per-call expressions of GetF (:106-139)
    const V3 per = ld3(f.period);
    p.plen = mag(per);
    p.rplen = 1.0 / p.plen;
    const V3 u = unit(per);
    p.u[0] = u.x; p.u[1] = u.y; p.u[2] = u.z;
    const double L = mag(per) * (f.nperiods + 2);
    p.ps = f.phase * mag(per) / two_pi();
    p.taper = f.taper;
    p.b_hi = L / 2. + p.ps;
    p.b_lo = -L / 2. + p.ps;
    p.e1_lo = -L / 2. + p.ps + p.plen;
    p.e1_hi = L / 2. + p.ps - p.plen;
    p.e2_lo = -L / 2. + p.ps + p.plen / 2.;
    p.e2_hi = L / 2. + p.ps - p.plen / 2.;
  }
}

// RotateSelfXYZ with the angles' sines and cosines precomputed (TVector3D.cc:150-205)
__device__ inline V3 rotate_pre(V3 v, const Prepared &p) {
  double t = v.y;
  v.y = p.rc[0] * t - p.rs[0] * v.z;
  v.z = p.rs[0] * t + p.rc[0] * v.z;
  t = v.z;
  v.z = p.rc[1] * t - p.rs[1] * v.x;
  v.x = p.rs[1] * t + p.rc[1] * v.x;
  t = v.x;
  v.x = p.rc[2] * t - p.rs[2] * v.y;
  v.y = p.rs[2] * t + p.rc[2] * v.y;
  return v;
}

__device__ inline V3 field_one(const Prepared &p, const srs_field &f, V3 X) {
  switch (p.kind) {
    case SRS_FIELD_UNDULATOR: {
      const double D = (X.x - p.C[0]) * p.u[0] + (X.y - p.C[1]) * p.u[1] + (X.z - p.C[2]) * p.u[2];
      const double taper = 1 + D * p.taper;
      if (D > p.b_hi || D < p.b_lo) return v3(0, 0, 0);
      const double s = sin(div_rn(two_pi() * (D - p.ps), p.plen, p.rplen));
      // ends: 0.25 / 0.75 of the field; the centre multiplies by 1.0, which is exact
      const double fac = (D < p.e1_lo || D > p.e1_hi) ? ((D < p.e2_lo || D > p.e2_hi) ? 0.25 : 0.75) : 1.0;
      return v3(p.F[0] * fac * s * taper, p.F[1] * fac * s * taper, p.F[2] * fac * s * taper);
    }
    case SRS_FIELD_GAUSSIAN: {
      const V3 rx = rotate_pre(X, p) - ld3(p.C);
      double frac = 1;
      if (f.sigma_or_width[0] > 0) { double t = rx.x / f.sigma_or_width[0]; frac *= exp(-(t * t) / 2.); }
      if (f.sigma_or_width[1] > 0) { double t = rx.y / f.sigma_or_width[1]; frac *= exp(-(t * t) / 2.); }
      if (f.sigma_or_width[2] > 0) { double t = rx.z / f.sigma_or_width[2]; frac *= exp(-(t * t) / 2.); }
      return ld3(p.F) * frac;
    }
    case SRS_FIELD_UNIFORM_BOX: {
      const V3 rx = rotate_pre(X, p) - ld3(p.C);
      const double *w = f.sigma_or_width;
      if ((!(w[0] <= 0) && fabs(rx.x) > fabs(w[0] / 2.)) || (!(w[1] <= 0) && fabs(rx.y) > fabs(w[1] / 2.)) ||
          (!(w[2] <= 0) && fabs(rx.z) > fabs(w[2] / 2.)))
        return v3(0, 0, 0);
      return ld3(p.F);
    }
    case SRS_FIELD_GRID:  // grid_field with the rotation's sines and cosines precomputed
      return grid_interp(f, p.gd, rotate_pre(X, p) - ld3(f.translation), p.rstep);
    default:
      return v3(0, 0, 0);
  }
}

// DerivativesB (OSCARSSR.cc:741-765): the velocity part
__device__ inline V3 force(double qomg, V3 v, V3 B) {
  return v3(qomg * (-v.z * B.y + v.y * B.z), qomg * (v.z * B.x - v.x * B.z), qomg * (v.x * B.y - v.y * B.x));
}

__device__ inline V3 vadd_scaled(V3 a, double h, V3 b) { return v3(a.x + h * b.x, a.y + h * b.y, a.z + h * b.z); }

// Copies every grid field's samples into the block's dynamic shared memory (the launcher sizes it to
// the total when that fits) and points the prepared fields at the copies: the interpolation then
// reads shared memory instead of global memory inside the serial RK4 chain.
extern __shared__ double g_stage[];
__device__ void stage_grids(const srs_field *sf, Prepared *sp, int nfields) {
  int64_t off = 0;
  for (int i = 0; i < nfields; ++i) {
    if (sf[i].kind != SRS_FIELD_GRID) continue;
    const int64_t cnt = 3 * sf[i].n[0] * sf[i].n[1] * sf[i].n[2];
    for (int64_t k = threadIdx.x; k < cnt; k += blockDim.x) g_stage[off + k] = sf[i].data[k];
    off += cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    off = 0;
    for (int i = 0; i < nfields; ++i) {
      if (sf[i].kind != SRS_FIELD_GRID) continue;
      sp[i].gd = g_stage + off;
      off += 3 * sf[i].n[0] * sf[i].n[1] * sf[i].n[2];
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- directional field derivatives
// dB = (dB/dX) dX of one field at X.  Used only to push tangents through the RK4 stages (the Newton
// updates of the parallel-in-time trajectory): its accuracy steers the iteration, it never reaches a
// stored point.  The region factors of the undulator and the box edges are piecewise constant, so
// their derivative is taken as zero.

// Grid: X and dX in the grid's frame (a direction rotates like a point, without the translation).
__device__ inline V3 grid_dir(const srs_field &f, const double *data, V3 X, V3 dX, const double *rstep) {
  const double xs[3] = {X.x, X.y, X.z}, ds[3] = {dX.x, dX.y, dX.z};
  int64_t base[3] = {0, 0, 0};
  double t[3] = {0, 0, 0};
  bool act[3];
  for (int a = 0; a < 3; ++a) {
    act[a] = f.n[a] > 1;
    if (!act[a]) continue;
    if (xs[a] <= f.start[a] || xs[a] >= f.start[a] + (double)(f.n[a] - 1) * f.step[a]) return v3(0, 0, 0);
    uint64_t k = (uint64_t)((xs[a] - f.start[a]) * rstep[a]);
    if (k > (uint64_t)(f.n[a] - 2)) k = f.n[a] - 2;
    base[a] = (int64_t)k;
    t[a] = ((xs[a] - f.start[a]) - (double)k * f.step[a]) * rstep[a];
  }
  if (!act[0] && !act[1] && !act[2]) return v3(0, 0, 0);
  V3 out = v3(0, 0, 0);
  for (int c = 0; c < 8; ++c) {
    bool skip = false;
    int64_t id[3];
    for (int a = 0; a < 3; ++a) {
      const int bit = (c >> a) & 1;
      if (!act[a] && bit) skip = true;
      id[a] = base[a] + bit;
    }
    if (skip) continue;
    // d(weight of corner c) along dX: sum over active axes of (+-1/step) dX_a * prod_{b != a} (t_b or 1 - t_b)
    double dw = 0.0;
    for (int a = 0; a < 3; ++a) {
      if (!act[a]) continue;
      double w = (((c >> a) & 1) ? 1.0 : -1.0) * rstep[a] * ds[a];
      for (int b = 0; b < 3; ++b)
        if (b != a && act[b]) w *= ((c >> b) & 1) ? t[b] : 1.0 - t[b];
      dw += w;
    }
    out = out + ld3(data + 3 * (id[0] * f.n[1] * f.n[2] + id[1] * f.n[2] + id[2])) * dw;
  }
  return out;
}

__device__ inline V3 field_one_dir(const Prepared &p, const srs_field &f, V3 X, V3 dX) {
  switch (p.kind) {
    case SRS_FIELD_UNDULATOR: {
      const double D = (X.x - p.C[0]) * p.u[0] + (X.y - p.C[1]) * p.u[1] + (X.z - p.C[2]) * p.u[2];
      if (D > p.b_hi || D < p.b_lo) return v3(0, 0, 0);
      const double k = two_pi() * p.rplen;
      double s, c;
      sincos(k * (D - p.ps), &s, &c);
      const double fac = (D < p.e1_lo || D > p.e1_hi) ? ((D < p.e2_lo || D > p.e2_hi) ? 0.25 : 0.75) : 1.0;
      const double dD = dX.x * p.u[0] + dX.y * p.u[1] + dX.z * p.u[2];
      const double g = fac * (c * k * (1 + D * p.taper) + s * p.taper) * dD;
      return v3(p.F[0] * g, p.F[1] * g, p.F[2] * g);
    }
    case SRS_FIELD_GAUSSIAN: {
      const V3 rx = rotate_pre(X, p) - ld3(p.C);
      const V3 dr = rotate_pre(dX, p);
      const double r[3] = {rx.x, rx.y, rx.z}, d[3] = {dr.x, dr.y, dr.z};
      double frac = 1, lin = 0;
      for (int a = 0; a < 3; ++a) {
        const double sg = f.sigma_or_width[a];
        if (sg > 0) {
          const double tt = r[a] / sg;
          frac *= exp(-(tt * tt) / 2.);
          lin -= r[a] * d[a] / (sg * sg);
        }
      }
      return ld3(p.F) * (frac * lin);
    }
    case SRS_FIELD_GRID:
      return grid_dir(f, p.gd, rotate_pre(X, p) - ld3(f.translation), rotate_pre(dX, p), p.rstep);
    default:  // uniform box: flat inside, a jump at the edges
      return v3(0, 0, 0);
  }
}

// ---------------------------------------------------------------- one RK4 step, one lane

// B at X summed over the fields in field order (TFieldContainer.cc:92-103)
__device__ inline V3 field_sum_pre(const Prepared *sp, const srs_field *sf, int nfields, V3 X) {
  V3 s = v3(0, 0, 0);
  for (int f = 0; f < nfields; ++f) s = s + field_one(sp[f], sf[f], X);
  return s;
}
__device__ inline V3 field_dir_pre(const Prepared *sp, const srs_field *sf, int nfields, V3 X, V3 dX) {
  V3 s = v3(0, 0, 0);
  for (int f = 0; f < nfields; ++f) s = s + field_one_dir(sp[f], sf[f], X, dX);
  return s;
}

// One RK4 step of size h from (pos, vel), in the reference's operation order (OSCARSSR.cc:826-874);
// returns the velocity part of the derivative at the start state (the a/c the reference stores with
// the next point).  Identical roundings to the steps of the trajectory kernels in rk4.cu.
__device__ inline V3 rk4_step_seq(const Prepared *sp, const srs_field *sf, int nfields, double qomg, V3 &pos,
                                  V3 &vel, double h) {
  const double hh = h * 0.5, h6 = h / 6.0;
  const V3 p2 = vadd_scaled(pos, hh, vel);
  const V3 a1 = force(qomg, vel, field_sum_pre(sp, sf, nfields, pos));
  const V3 v2 = vadd_scaled(vel, hh, a1);
  const V3 a2 = force(qomg, v2, field_sum_pre(sp, sf, nfields, p2));
  const V3 p3 = vadd_scaled(pos, hh, v2);
  const V3 v3_ = vadd_scaled(vel, hh, a2);
  const V3 a3 = force(qomg, v3_, field_sum_pre(sp, sf, nfields, p3));
  const V3 p4 = vadd_scaled(pos, h, v3_);
  const V3 v4 = vadd_scaled(vel, h, a3);
  const V3 m_pos = v3_ + v2, m_vel = a3 + a2;
  const V3 a4 = force(qomg, v4, field_sum_pre(sp, sf, nfields, p4));
  const V3 npos = v3(pos.x + h6 * (vel.x + v4.x + 2.0 * m_pos.x), pos.y + h6 * (vel.y + v4.y + 2.0 * m_pos.y),
                     pos.z + h6 * (vel.z + v4.z + 2.0 * m_pos.z));
  const V3 nvel = v3(vel.x + h6 * (a1.x + a4.x + 2.0 * m_vel.x), vel.y + h6 * (a1.y + a4.y + 2.0 * m_vel.y),
                     vel.z + h6 * (a1.z + a4.z + 2.0 * m_vel.z));
  pos = npos;
  vel = nvel;
  return a1;
}

// The same step (same primal roundings) with a tangent (dp, dv) of the start state pushed through
// the four stages: on return (dp, dv) is the tangent of the end state.
__device__ inline void rk4_step_tangent(const Prepared *sp, const srs_field *sf, int nfields, double qomg, V3 &pos,
                                        V3 &vel, V3 &dp, V3 &dv, double h) {
  const double hh = h * 0.5, h6 = h / 6.0;
  const V3 p2 = vadd_scaled(pos, hh, vel), dp2 = vadd_scaled(dp, hh, dv);
  const V3 B1 = field_sum_pre(sp, sf, nfields, pos);
  const V3 a1 = force(qomg, vel, B1);
  const V3 da1 = force(qomg, dv, B1) + force(qomg, vel, field_dir_pre(sp, sf, nfields, pos, dp));
  const V3 v2 = vadd_scaled(vel, hh, a1), dv2 = vadd_scaled(dv, hh, da1);
  const V3 B2 = field_sum_pre(sp, sf, nfields, p2);
  const V3 a2 = force(qomg, v2, B2);
  const V3 da2 = force(qomg, dv2, B2) + force(qomg, v2, field_dir_pre(sp, sf, nfields, p2, dp2));
  const V3 p3 = vadd_scaled(pos, hh, v2), dp3 = vadd_scaled(dp, hh, dv2);
  const V3 v3_ = vadd_scaled(vel, hh, a2), dv3 = vadd_scaled(dv, hh, da2);
  const V3 B3 = field_sum_pre(sp, sf, nfields, p3);
  const V3 a3 = force(qomg, v3_, B3);
  const V3 da3 = force(qomg, dv3, B3) + force(qomg, v3_, field_dir_pre(sp, sf, nfields, p3, dp3));
  const V3 p4 = vadd_scaled(pos, h, v3_), dp4 = vadd_scaled(dp, h, dv3);
  const V3 v4 = vadd_scaled(vel, h, a3), dv4 = vadd_scaled(dv, h, da3);
  const V3 m_pos = v3_ + v2, m_vel = a3 + a2;
  const V3 B4 = field_sum_pre(sp, sf, nfields, p4);
  const V3 a4 = force(qomg, v4, B4);
  const V3 da4 = force(qomg, dv4, B4) + force(qomg, v4, field_dir_pre(sp, sf, nfields, p4, dp4));
  const V3 npos = v3(pos.x + h6 * (vel.x + v4.x + 2.0 * m_pos.x), pos.y + h6 * (vel.y + v4.y + 2.0 * m_pos.y),
                     pos.z + h6 * (vel.z + v4.z + 2.0 * m_pos.z));
  const V3 nvel = v3(vel.x + h6 * (a1.x + a4.x + 2.0 * m_vel.x), vel.y + h6 * (a1.y + a4.y + 2.0 * m_vel.y),
                     vel.z + h6 * (a1.z + a4.z + 2.0 * m_vel.z));
  dp = dp + (dv + dv4 + (dv3 + dv2) * 2.0) * h6;
  dv = dv + (da1 + da4 + (da3 + da2) * 2.0) * h6;
  pos = npos;
  vel = nvel;
}

}  // namespace
}  // namespace srs

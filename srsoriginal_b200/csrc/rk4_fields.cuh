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
  p.kind = field_shape(f.kind);
  p.gd = f.data;
  for (int c = 0; c < 3; ++c) p.rstep[c] = f.step[c] != 0 ? 1.0 / f.step[c] : 0.0;
  for (int c = 0; c < 3; ++c) {
    p.F[c] = f.field[c];
    p.C[c] = f.center[c];
    p.rs[c] = sin(f.rotations[c]);
    p.rc[c] = cos(f.rotations[c]);
  }
  if (p.kind == SRS_FIELD_UNDULATOR) {
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

// DerivativesE and DerivativesEB (OSCARSSR.cc:713-793): q/(m gamma) E, and q/(m gamma) (E + v x B) in the
// reference's operation order
__device__ inline V3 force_e(double qomg, V3 E) { return v3(qomg * E.x, qomg * E.y, qomg * E.z); }
__device__ inline V3 force_eb(double qomg, V3 v, V3 E, V3 B) {
  return v3(qomg * (E.x - v.z * B.y + v.y * B.z), qomg * (E.y + v.z * B.x - v.x * B.z),
            qomg * (E.z + v.x * B.y - v.y * B.x));
}

__device__ inline V3 vadd_scaled(V3 a, double h, V3 b) { return v3(a.x + h * b.x, a.y + h * b.y, a.z + h * b.z); }

// Copies every grid field's samples into the block's dynamic shared memory (the launcher sizes it to
// the total when that fits) and points the prepared fields at the copies: the interpolation then
// reads shared memory instead of global memory inside the serial RK4 chain.
extern __shared__ __align__(16) double g_stage[];
__device__ void stage_grids(const srs_field *sf, Prepared *sp, int nfields) {
  int64_t off = 0;
  for (int i = 0; i < nfields; ++i) {
    if (field_shape(sf[i].kind) != SRS_FIELD_GRID) continue;
    const int64_t cnt = 3 * sf[i].n[0] * sf[i].n[1] * sf[i].n[2];
    for (int64_t k = threadIdx.x; k < cnt; k += blockDim.x) g_stage[off + k] = sf[i].data[k];
    off += cnt;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    off = 0;
    for (int i = 0; i < nfields; ++i) {
      if (field_shape(sf[i].kind) != SRS_FIELD_GRID) continue;
      sp[i].gd = g_stage + off;
      off += 3 * sf[i].n[0] * sf[i].n[1] * sf[i].n[2];
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------- field Jacobians (FP32)
// J[3 i + k] = dB_i / dX_k of one field at X, in single precision.  Used only to push tangents through
// the RK4 stages (the Newton updates of the parallel-in-time trajectory): its accuracy sets how fast
// the iteration converges, it never reaches a stored point.  The undulator's region factors and the
// box's edges are piecewise constant, so their derivative is taken as zero.

// v -> R^T v for the rotation R of rotate_pre (R = Rz Ry Rx, so R^T applies Rz^T, then Ry^T, then Rx^T)
__device__ inline V3 rotate_pre_t(V3 v, const Prepared &p) {
  double t = v.x;
  v.x = p.rc[2] * t + p.rs[2] * v.y;
  v.y = -p.rs[2] * t + p.rc[2] * v.y;
  t = v.z;
  v.z = p.rc[1] * t + p.rs[1] * v.x;
  v.x = -p.rs[1] * t + p.rc[1] * v.x;
  t = v.y;
  v.y = p.rc[0] * t + p.rs[0] * v.z;
  v.z = -p.rs[0] * t + p.rc[0] * v.z;
  return v;
}

// grid: dB / dX' in the grid's frame (X' = R X - translation) into Jp
__device__ inline void grid_jac(const srs_field &f, const double *data, V3 X, const double *rstep, double Jp[9]) {
  for (int k = 0; k < 9; ++k) Jp[k] = 0.0;
  const double xs[3] = {X.x, X.y, X.z};
  int64_t base[3] = {0, 0, 0};
  double t[3] = {0, 0, 0};
  bool act[3];
  for (int a = 0; a < 3; ++a) {
    act[a] = f.n[a] > 1;
    if (!act[a]) continue;
    if (xs[a] <= f.start[a] || xs[a] >= f.start[a] + (double)(f.n[a] - 1) * f.step[a]) return;
    uint64_t k = (uint64_t)((xs[a] - f.start[a]) * rstep[a]);
    if (k > (uint64_t)(f.n[a] - 2)) k = f.n[a] - 2;
    base[a] = (int64_t)k;
    t[a] = ((xs[a] - f.start[a]) - (double)k * f.step[a]) * rstep[a];
  }
  if (!act[0] && !act[1] && !act[2]) return;
  for (int c = 0; c < 8; ++c) {
    bool skip = false;
    int64_t id[3];
    for (int a = 0; a < 3; ++a) {
      const int bit = (c >> a) & 1;
      if (!act[a] && bit) skip = true;
      id[a] = base[a] + bit;
    }
    if (skip) continue;
    const V3 smp = ld3(data + 3 * (id[0] * f.n[1] * f.n[2] + id[1] * f.n[2] + id[2]));
    for (int a = 0; a < 3; ++a) {
      if (!act[a]) continue;
      double w = (((c >> a) & 1) ? 1.0 : -1.0) * rstep[a];
      for (int b = 0; b < 3; ++b)
        if (b != a && act[b]) w *= ((c >> b) & 1) ? t[b] : 1.0 - t[b];
      Jp[0 + a] += smp.x * w;
      Jp[3 + a] += smp.y * w;
      Jp[6 + a] += smp.z * w;
    }
  }
}

__device__ inline void field_one_jac(const Prepared &p, const srs_field &f, V3 X, float J[9]) {
  for (int k = 0; k < 9; ++k) J[k] = 0.f;
  switch (p.kind) {
    case SRS_FIELD_UNDULATOR: {
      const double D = (X.x - p.C[0]) * p.u[0] + (X.y - p.C[1]) * p.u[1] + (X.z - p.C[2]) * p.u[2];
      if (D > p.b_hi || D < p.b_lo) return;
      const double k = two_pi() * p.rplen, a = k * (D - p.ps);
      const float r = (float)(a - two_pi() * rint(a * (0.5 / kPi)));  // |r| <= pi
      float s, c;
      __sincosf(r, &s, &c);
      const double fac = (D < p.e1_lo || D > p.e1_hi) ? ((D < p.e2_lo || D > p.e2_hi) ? 0.25 : 0.75) : 1.0;
      const float g = (float)fac * (c * (float)(k * (1 + D * p.taper)) + s * (float)p.taper);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J[3 * i + j] = (float)p.F[i] * g * (float)p.u[j];
      return;
    }
    case SRS_FIELD_GAUSSIAN: {
      const V3 rx = rotate_pre(X, p) - ld3(p.C);
      const double r[3] = {rx.x, rx.y, rx.z};
      double frac = 1, gr[3] = {0, 0, 0};
      for (int a = 0; a < 3; ++a) {
        const double sg = f.sigma_or_width[a];
        if (sg > 0) {
          const double tt = r[a] / sg;
          frac *= exp(-(tt * tt) / 2.);
        }
      }
      for (int a = 0; a < 3; ++a) {
        const double sg = f.sigma_or_width[a];
        if (sg > 0) gr[a] = -frac * r[a] / (sg * sg);
      }
      const V3 gx = rotate_pre_t(v3(gr[0], gr[1], gr[2]), p);  // gradient in X: R^T (gradient in the rotated frame)
      const double gv[3] = {gx.x, gx.y, gx.z};
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) J[3 * i + j] = (float)(p.F[i] * gv[j]);
      return;
    }
    case SRS_FIELD_GRID: {
      double Jp[9];
      grid_jac(f, p.gd, rotate_pre(X, p) - ld3(f.translation), p.rstep, Jp);
      for (int i = 0; i < 3; ++i) {  // row i: R^T (row i of dB/dX')
        const V3 row = rotate_pre_t(v3(Jp[3 * i], Jp[3 * i + 1], Jp[3 * i + 2]), p);
        J[3 * i] = (float)row.x;
        J[3 * i + 1] = (float)row.y;
        J[3 * i + 2] = (float)row.z;
      }
      return;
    }
    default:  // uniform box: flat inside
      return;
  }
}

}  // namespace
}  // namespace srs

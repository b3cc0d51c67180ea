// Device-side physics shared by the kernels: the reference's constants, 3-vector arithmetic in the
// reference's operation order, magnetic-field evaluation, and the phase reduction.
//
// Translation units that must reproduce the reference's IEEE-double results (the RK4 and the plain
// FP64 sums) are compiled with -fmad=false, so `a*b + c` below is a rounded multiply followed by a
// rounded add, exactly like the reference on x86-64.  Explicit __fma_rn calls are used only where a
// fused operation is wanted (the Cody-Waite reduction).
#pragma once

#include <cstdint>

#include "../../include/srs_b200.h"

namespace srs {

// ---- constants: include/TOSCARSSR.h:20-72 (same literals) ----
constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrt2Pi = 2.5066282746310002416123552393401;
constexpr double kC = 2.99792458e8;
constexpr double kH = 6.62606876e-34;
constexpr double kHbar = 1.054571596e-34;
constexpr double kQe = 1.602176462e-19;
constexpr double kMe = 9.10938356e-31;
constexpr double kEps0 = 8.854187817E-12;
constexpr double kMu0 = 1.2566370614E-6;
__host__ __device__ inline int64_t imin64(int64_t a, int64_t b) { return a < b ? a : b; }
__host__ __device__ inline double two_pi() { return 2.0 * kPi; }
__host__ __device__ inline double four_pi() { return 4.0 * kPi; }
__host__ __device__ inline double pi2() { return kPi * kPi; }
// eV -> angular frequency: e*Qe/Hbar (TOSCARSSR.h:66)
__host__ __device__ inline double ev_to_omega(double e) { return e * kQe / kHbar; }

// Flux constants of the frequency-domain sums (OSCARSSR.cc:1188-1194).
__host__ __device__ inline double flux_c0(double q) { return q / (four_pi() * kC * kEps0 * kSqrt2Pi); }
__host__ __device__ inline double flux_c2(double q, double current) {
  return four_pi() * current / (kH * (q < 0 ? -q : q) * kMu0 * kC) * 1e-6 * 0.001;
}
// Power-density constant without dt (OSCARSSR.cc:1577).
__host__ __device__ inline double pd_const(double q, double current) {
  double qi = q * current;
  return (qi < 0 ? -qi : qi) / (16 * pi2() * kEps0 * kC);
}

// ---- 3-vectors, TVector3D semantics (src/TVector3D.cc) ----
struct V3 {
  double x, y, z;
};
__host__ __device__ inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__host__ __device__ inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ inline V3 operator*(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ inline V3 operator/(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
__host__ __device__ inline double mag2(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
__host__ __device__ inline double mag(V3 a) { return sqrt(mag2(a)); }
__host__ __device__ inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ inline V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__host__ __device__ inline V3 unit(V3 a) { return a / mag(a); }
__host__ __device__ inline V3 ld3(const double *p) { return v3(p[0], p[1], p[2]); }
__host__ __device__ inline V3 orthogonal(V3 a) {  // include/TVector3D.h:120-131
  double xx = a.x < 0.0 ? -a.x : a.x, yy = a.y < 0.0 ? -a.y : a.y, zz = a.z < 0.0 ? -a.z : a.z;
  if (xx < yy) return xx < zz ? v3(0, a.z, -a.y) : v3(a.y, -a.x, 0);
  return yy < zz ? v3(-a.z, 0, a.x) : v3(a.y, -a.x, 0);
}
__host__ __device__ inline void rotate_xyz(V3 &v, const double r[3]) {  // TVector3D.cc:150-205
  double s = sin(r[0]), c = cos(r[0]), t = v.y;
  v.y = c * t - s * v.z;
  v.z = s * t + c * v.z;
  s = sin(r[1]); c = cos(r[1]); t = v.z;
  v.z = c * t - s * v.x;
  v.x = s * t + c * v.x;
  s = sin(r[2]); c = cos(r[2]); t = v.x;
  v.x = c * t - s * v.y;
  v.y = s * t + c * v.y;
}

// ---- fields ----

// TField3D_IdealUndulator::GetF (src/TField3D_IdealUndulator.cc:106-139)
__device__ inline V3 undulator_field(const srs_field &f, V3 X) {
  V3 per = ld3(f.period);
  double plen = mag(per);
  V3 u = unit(per);
  double L = mag(per) * (f.nperiods + 2);
  double D = dot(X - ld3(f.center), u);
  double taper = 1 + D * f.taper;
  double ps = f.phase * mag(per) / two_pi();
  if (D > L / 2. + ps || D < -L / 2. + ps) return v3(0, 0, 0);
  double s = sin(two_pi() * (D - ps) / plen);
  V3 F = ld3(f.field);
  if (D < -L / 2. + ps + plen || D > L / 2. + ps - plen) {
    if (D < -L / 2. + ps + plen / 2. || D > L / 2. + ps - plen / 2.) return F * 0.25 * s * taper;
    return F * 0.75 * s * taper;
  }
  return F * s * taper;
}

// TField3D_Gaussian::GetF (src/TField3D_Gaussian.cc:88-113)
__device__ inline V3 gaussian_field(const srs_field &f, V3 X) {
  V3 xb = X;
  rotate_xyz(xb, f.rotations);
  V3 rx = xb - ld3(f.center);
  double frac = 1;
  if (f.sigma_or_width[0] > 0) { double t = rx.x / f.sigma_or_width[0]; frac *= exp(-(t * t) / 2.); }
  if (f.sigma_or_width[1] > 0) { double t = rx.y / f.sigma_or_width[1]; frac *= exp(-(t * t) / 2.); }
  if (f.sigma_or_width[2] > 0) { double t = rx.z / f.sigma_or_width[2]; frac *= exp(-(t * t) / 2.); }
  return ld3(f.field) * frac;
}

// TField3D_UniformBox::GetF (src/TField3D_UniformBox.cc:93-111)
__device__ inline V3 box_field(const srs_field &f, V3 X) {
  V3 xb = X;
  rotate_xyz(xb, f.rotations);
  V3 rx = xb - ld3(f.center);
  const double *w = f.sigma_or_width;
  bool ix = w[0] <= 0, iy = w[1] <= 0, iz = w[2] <= 0;
  if ((!ix && fabs(rx.x) > fabs(w[0] / 2.)) || (!iy && fabs(rx.y) > fabs(w[1] / 2.)) ||
      (!iz && fabs(rx.z) > fabs(w[2] / 2.)))
    return v3(0, 0, 0);
  return ld3(f.field);
}

// RN(a / b) from the reciprocal rb = RN(1 / b): q = RN(a rb), r = a - b q (exact with an FMA),
// RN(q + r rb) (P. Markstein, IBM J. Res. Dev. 34(1), 1990; normal operands, no overflow or
// underflow).  A loop that divides by the same b many times saves the division's latency.
__device__ __forceinline__ double div_rn(double a, double b, double rb) {
  const double q = __dmul_rn(a, rb);
  const double r = __fma_rn(-q, b, a);
  return __fma_rn(r, rb, q);
}

__device__ inline V3 grid_at(const double *data, const srs_field &f, int64_t ix, int64_t iy, int64_t iz) {
  return ld3(data + 3 * (ix * f.n[1] * f.n[2] + iy * f.n[2] + iz));
}
// a + (b - a) d / step, with the division as a multiply-correct sequence when the reciprocal is known
__device__ inline V3 grid_lerp(V3 a, V3 b, double d, double step, const double *rstep, int axis) {
  const V3 t = (b - a) * d;
  if (rstep) {
    const double r = rstep[axis];
    return a + v3(div_rn(t.x, step, r), div_rn(t.y, step, r), div_rn(t.z, step, r));
  }
  return a + t / step;
}
// Interpolation at X, already in the grid's frame (rotated and translated); samples read from data
// (the field's own array, or a copy of it in shared memory).  rstep (optional): 1/step per axis, for
// the divisions by the step (same results: both are correctly rounded).
__device__ inline V3 grid_interp(const srs_field &f, const double *data, V3 X, const double *rstep = nullptr) {
  const bool hx = f.n[0] > 1, hy = f.n[1] > 1, hz = f.n[2] > 1;
  if (hx && (X.x <= f.start[0] || X.x >= f.start[0] + (double)(f.n[0] - 1) * f.step[0])) return v3(0, 0, 0);
  if (hy && (X.y <= f.start[1] || X.y >= f.start[1] + (double)(f.n[1] - 1) * f.step[1])) return v3(0, 0, 0);
  if (hz && (X.z <= f.start[2] || X.z >= f.start[2] + (double)(f.n[2] - 1) * f.step[2])) return v3(0, 0, 0);
  auto quot = [&](double a, int axis) { return rstep ? div_rn(a, f.step[axis], rstep[axis]) : a / f.step[axis]; };
  uint64_t nx = hx ? (uint64_t)quot(X.x - f.start[0], 0) : 0;
  double dx = hx ? (X.x - f.start[0]) - (double)nx * f.step[0] : 0;
  uint64_t ny = hy ? (uint64_t)quot(X.y - f.start[1], 1) : 0;
  double dy = hy ? (X.y - f.start[1]) - (double)ny * f.step[1] : 0;
  uint64_t nz = hz ? (uint64_t)quot(X.z - f.start[2], 2) : 0;
  double dz = hz ? (X.z - f.start[2]) - (double)nz * f.step[2] : 0;
  // Indices stay inside the map: X is strictly inside (start, stop) on every axis with n > 1, so
  // n? <= n-2 there up to rounding of the quotient; clamp that rounding case.
  if (hx && nx > (uint64_t)(f.n[0] - 2)) nx = f.n[0] - 2;
  if (hy && ny > (uint64_t)(f.n[1] - 2)) ny = f.n[1] - 2;
  if (hz && nz > (uint64_t)(f.n[2] - 2)) nz = f.n[2] - 2;
  const double *d = data;
  const double *rs = rstep;
  if (hx && hy && hz) {
    V3 v00 = grid_lerp(grid_at(d, f, nx, ny, nz), grid_at(d, f, nx + 1, ny, nz), dx, f.step[0], rs, 0);
    V3 v10 = grid_lerp(grid_at(d, f, nx, ny + 1, nz), grid_at(d, f, nx + 1, ny + 1, nz), dx, f.step[0], rs, 0);
    V3 v01 = grid_lerp(grid_at(d, f, nx, ny, nz + 1), grid_at(d, f, nx + 1, ny, nz + 1), dx, f.step[0], rs, 0);
    V3 v11 = grid_lerp(grid_at(d, f, nx, ny + 1, nz + 1), grid_at(d, f, nx + 1, ny + 1, nz + 1), dx, f.step[0], rs,
                       0);
    V3 v0 = grid_lerp(v00, v10, dy, f.step[1], rs, 1);
    V3 v1 = grid_lerp(v01, v11, dy, f.step[1], rs, 1);
    return grid_lerp(v0, v1, dz, f.step[2], rs, 2);
  } else if (hx && hy) {
    V3 v0 = grid_lerp(grid_at(d, f, nx, ny, 0), grid_at(d, f, nx + 1, ny, 0), dx, f.step[0], rs, 0);
    V3 v1 = grid_lerp(grid_at(d, f, nx, ny + 1, 0), grid_at(d, f, nx + 1, ny + 1, 0), dx, f.step[0], rs, 0);
    return grid_lerp(v0, v1, dy, f.step[1], rs, 1);
  } else if (hx && hz) {
    V3 v0 = grid_lerp(grid_at(d, f, nx, 0, nz), grid_at(d, f, nx + 1, 0, nz), dx, f.step[0], rs, 0);
    V3 v1 = grid_lerp(grid_at(d, f, nx, 0, nz + 1), grid_at(d, f, nx + 1, 0, nz + 1), dx, f.step[0], rs, 0);
    return grid_lerp(v0, v1, dz, f.step[2], rs, 2);
  } else if (hy && hz) {
    V3 v0 = grid_lerp(grid_at(d, f, 0, ny, nz), grid_at(d, f, 0, ny + 1, nz), dy, f.step[1], rs, 1);
    V3 v1 = grid_lerp(grid_at(d, f, 0, ny, nz + 1), grid_at(d, f, 0, ny + 1, nz + 1), dy, f.step[1], rs, 1);
    return grid_lerp(v0, v1, dz, f.step[2], rs, 2);
  } else if (hx) {
    return grid_lerp(ld3(d + 3 * nx), ld3(d + 3 * (nx + 1)), dx, f.step[0], rs, 0);
  } else if (hy) {
    return grid_lerp(ld3(d + 3 * ny), ld3(d + 3 * (ny + 1)), dy, f.step[1], rs, 1);
  } else if (hz) {
    return grid_lerp(ld3(d + 3 * nz), ld3(d + 3 * (nz + 1)), dz, f.step[2], rs, 2);
  }
  return v3(0, 0, 0);
}

// TField3D_Grid::GetF (src/TField3D_Grid.cc:124-243): rotate, translate, zero outside, then linear /
// bilinear / trilinear interpolation in x -> y -> z order with the reference's arithmetic.
__device__ inline V3 grid_field(const srs_field &f, V3 XIN) {
  V3 X = XIN;
  rotate_xyz(X, f.rotations);
  X = X - ld3(f.translation);
  return grid_interp(f, f.data, X);
}

// kind without the electric flag, and the flag
__host__ __device__ inline int field_shape(int kind) { return kind & SRS_FIELD_SHAPE_MASK; }
__host__ __device__ inline bool field_electric(int kind) { return (kind & SRS_FIELD_ELECTRIC) != 0; }

// TFieldContainer::GetF (src/TFieldContainer.cc:92-103): Sum(0,0,0) += each field of the magnetic
// (electric = false) or the electric container.
__device__ inline V3 field_sum(const srs_field *fields, int nfields, V3 X, bool electric = false) {
  V3 s = v3(0, 0, 0);
  for (int i = 0; i < nfields; ++i) {
    const srs_field &f = fields[i];
    if (field_electric(f.kind) != electric) continue;
    V3 b;
    switch (field_shape(f.kind)) {
      case SRS_FIELD_UNDULATOR: b = undulator_field(f, X); break;
      case SRS_FIELD_GAUSSIAN: b = gaussian_field(f, X); break;
      case SRS_FIELD_UNIFORM_BOX: b = box_field(f, X); break;
      case SRS_FIELD_GRID: b = grid_field(f, X); break;
      default: b = v3(0, 0, 0);
    }
    s = s + b;
  }
  return s;
}

// C2 |SumE * (0 + i C0 w dt)|^2 with libstdc++ complex arithmetic (OSCARSSR.cc:1241-1245); e holds
// Re/Im of SumE's x, y, z components.
__device__ inline double finish_flux(const double e[6], double omega, double dt, double C0, double C2) {
  const double g = (C0 * omega) * dt, z = 0.0 * dt;
  double parts[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double a = e[2 * c], b = e[2 * c + 1];
    const double pr = a * z - b * g, pi = a * g + b * z;
    parts[c] = pr * pr - pi * (-pi);
  }
  return C2 * ((parts[0] + parts[1]) + parts[2]);
}

// ---- phase reduction ----
// Cody-Waite additive reduction (Cody & Waite, "Software Manual for the Elementary Functions", 1980)
// of x modulo 2*pi with a three-part 2*pi (P1 + P2 + P3 = 2*pi to ~160 bits; P1, P2 are the double
// roundings of 2*pi and of the remainder).  Each step is one fused multiply-add, exact in the
// product, so for |x| < 2^46 the result is x - k*2*pi to within ~2 ulp of pi.
__device__ __forceinline__ double reduce_2pi(double x) {
  const double kInv2Pi = 0.15915494309189535;
  const double P1 = 6.283185307179586, P2 = 2.4492935982947064e-16, P3 = -5.989539619436679e-33;
  double k = rint(x * kInv2Pi);
  double r = __fma_rn(-k, P1, x);
  r = __fma_rn(-k, P2, r);
  r = __fma_rn(-k, P3, r);
  return r;
}

// The same reduction in FP32 arithmetic, for arguments of a few hundred radians at most.
__device__ __forceinline__ float reduce_2pi_f(float x) {
  const float kInv2Pi = 0.159154943f;
  const float P1 = 6.2831855f, P2 = -1.7484555e-07f, P3 = -6.860498e-15f;
  float k = rintf(x * kInv2Pi);
  float r = __fmaf_rn(-k, P1, x);
  r = __fmaf_rn(-k, P2, r);
  r = __fmaf_rn(-k, P3, r);
  return r;
}

}  // namespace srs

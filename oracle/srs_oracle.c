/*
 * ORACLE -- test infrastructure only (see srs_oracle.h).  Plain C99 restatement of the reference's
 * CPU algorithm, operation by operation, so that it reproduces the reference's IEEE-double results.
 * Each function cites the reference file:line it follows (paths inside dhidas/SRSOriginal).
 * Compiled with -ffp-contract=off: no fused multiply-add, like the reference on x86-64.
 */
#include "srs_oracle.h"

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ---- constants: include/TOSCARSSR.h:20-72 ---- */
#define K_PI 3.14159265358979323846
static double c_pi(void) { return K_PI; }
static double c_pi2(void) { return c_pi() * c_pi(); }
static double c_twopi(void) { return 2.0 * c_pi(); }
static double c_fourpi(void) { return 4.0 * c_pi(); }
static double c_sqrt2pi(void) { return 2.5066282746310002416123552393401; }
static double c_c(void) { return 2.99792458e8; }
static double c_h(void) { return 6.62606876e-34; }
static double c_hbar(void) { return 1.054571596e-34; }
static double c_qe(void) { return 1.602176462e-19; }
static double c_me(void) { return 9.10938356e-31; }
static double c_eps0(void) { return 8.854187817E-12; }
static double c_mu0(void) { return 1.2566370614E-6; }
static double ev_to_omega(double e) { return e * c_qe() / c_hbar(); }          /* TOSCARSSR.h:66 */
static double kg_to_gev(double m) { return 1e-9 * m * c_c() * c_c() / c_qe(); } /* TOSCARSSR.h:68 */
static double gev_to_kg(double m) { return c_qe() * m / (1e-9 * c_c() * c_c()); }

/* ---- 3-vector helpers: src/TVector3D.cc, include/TVector3D.h ---- */
typedef struct { double x, y, z; } v3;
static v3 mk(double x, double y, double z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static v3 vsub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }      /* :191-195 */
static v3 vadd(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3 vdiv(v3 a, double d) { return mk(a.x / d, a.y / d, a.z / d); }          /* :200-204 */
static v3 vmul(v3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }           /* TVector3D.h:140-153 */
static double mag2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }            /* :106-110 */
static double mag(v3 a) { return sqrt(mag2(a)); }                                  /* :98-102 */
static double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }        /* :114-118 */
static v3 cross(v3 a, v3 b) {                                                      /* :134-138 */
  return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static v3 unit(v3 a) { return vdiv(a, mag(a)); }                                   /* :142-146 */
static v3 orthogonal(v3 a) {                                                       /* TVector3D.h:120-131 */
  double xx = a.x < 0.0 ? -a.x : a.x;
  double yy = a.y < 0.0 ? -a.y : a.y;
  double zz = a.z < 0.0 ? -a.z : a.z;
  if (xx < yy) return xx < zz ? mk(0, a.z, -a.y) : mk(a.y, -a.x, 0);
  return yy < zz ? mk(-a.z, 0, a.x) : mk(a.y, -a.x, 0);
}
static void rot_x(v3 *v, double ang) {                                             /* :150-161 */
  double s = sin(ang), c = cos(ang), yy = v->y;
  v->y = c * yy - s * v->z;
  v->z = s * yy + c * v->z;
}
static void rot_y(v3 *v, double ang) {                                             /* :165-176 */
  double s = sin(ang), c = cos(ang), zz = v->z;
  v->z = c * zz - s * v->x;
  v->x = s * zz + c * v->x;
}
static void rot_z(v3 *v, double ang) {                                             /* :180-191 */
  double s = sin(ang), c = cos(ang), xx = v->x;
  v->x = c * xx - s * v->y;
  v->y = s * xx + c * v->y;
}
static void rot_xyz(v3 *v, const double r[3]) { rot_x(v, r[0]); rot_y(v, r[1]); rot_z(v, r[2]); }
static v3 ld(const double *p) { return mk(p[0], p[1], p[2]); }

/* ---- fields ---- */

/* src/TField3D_IdealUndulator.cc:106-139 (+ Init :62-80) */
static v3 undulator(const orc_field *f, v3 X) {
  v3 per = ld(f->period);
  double plen = mag(per);
  v3 u = unit(per);
  double L = mag(per) * (f->nperiods + 2);
  double D = dot(vsub(X, ld(f->center)), u);
  double taper = 1 + D * f->taper;
  double ps = f->phase * mag(per) / c_twopi();
  v3 F = ld(f->field);
  if (D > L / 2. + ps || D < -L / 2. + ps) return mk(0, 0, 0);
  double s = sin(c_twopi() * (D - ps) / plen);
  if (D < -L / 2. + ps + plen || D > L / 2. + ps - plen) {
    if (D < -L / 2. + ps + plen / 2. || D > L / 2. + ps - plen / 2.)
      return vmul(vmul(vmul(F, 0.25), s), taper);
    return vmul(vmul(vmul(F, 0.75), s), taper);
  }
  return vmul(vmul(F, s), taper);
}

/* src/TField3D_Gaussian.cc:88-113 */
static v3 gaussian(const orc_field *f, v3 X) {
  v3 xb = X;
  rot_xyz(&xb, f->rotations);
  v3 rx = vsub(xb, ld(f->center));
  double frac = 1;
  if (f->sigma_or_width[0] > 0) { double t = rx.x / f->sigma_or_width[0]; frac *= exp(-(t * t) / 2.); }
  if (f->sigma_or_width[1] > 0) { double t = rx.y / f->sigma_or_width[1]; frac *= exp(-(t * t) / 2.); }
  if (f->sigma_or_width[2] > 0) { double t = rx.z / f->sigma_or_width[2]; frac *= exp(-(t * t) / 2.); }
  return vmul(ld(f->field), frac);
}

/* src/TField3D_UniformBox.cc:93-111 */
static v3 ubox(const orc_field *f, v3 X) {
  v3 xb = X;
  rot_xyz(&xb, f->rotations);
  v3 rx = vsub(xb, ld(f->center));
  const double *w = f->sigma_or_width;
  int ix = w[0] <= 0, iy = w[1] <= 0, iz = w[2] <= 0;
  if ((!ix && fabs(rx.x) > fabs(w[0] / 2.)) || (!iy && fabs(rx.y) > fabs(w[1] / 2.)) ||
      (!iz && fabs(rx.z) > fabs(w[2] / 2.)))
    return mk(0, 0, 0);
  return ld(f->field);
}

/* src/TField3D_Grid.cc:124-243 */
static v3 gdat(const orc_field *f, int64_t ix, int64_t iy, int64_t iz) {
  return ld(f->data + 3 * (ix * f->n[1] * f->n[2] + iy * f->n[2] + iz));
}
static v3 lerp(v3 a, v3 b, double d, double step) {
  /* a + d * (b - a) / step, TVector3D ops left to right */
  return vadd(a, vdiv(vmul(vsub(b, a), d), step));
}
static v3 grid(const orc_field *f, v3 XIN) {
  v3 X = XIN;
  rot_xyz(&X, f->rotations);
  X = vsub(X, ld(f->translation));
  double st[3], sp[3];
  for (int k = 0; k < 3; ++k) st[k] = f->start[k] + (double)(f->n[k] - 1) * f->step[k];
  (void)sp;
  if (f->n[0] > 1 && (X.x <= f->start[0] || X.x >= st[0])) return mk(0, 0, 0);
  if (f->n[1] > 1 && (X.y <= f->start[1] || X.y >= st[1])) return mk(0, 0, 0);
  if (f->n[2] > 1 && (X.z <= f->start[2] || X.z >= st[2])) return mk(0, 0, 0);
  size_t nx = f->n[0] > 1 ? (size_t)((X.x - f->start[0]) / f->step[0]) : 0;
  double dx = f->n[0] > 1 ? (X.x - f->start[0]) - nx * f->step[0] : 0;
  size_t ny = f->n[1] > 1 ? (size_t)((X.y - f->start[1]) / f->step[1]) : 0;
  double dy = f->n[1] > 1 ? (X.y - f->start[1]) - ny * f->step[1] : 0;
  size_t nz = f->n[2] > 1 ? (size_t)((X.z - f->start[2]) / f->step[2]) : 0;
  double dz = f->n[2] > 1 ? (X.z - f->start[2]) - nz * f->step[2] : 0;
  int hx = f->n[0] > 1, hy = f->n[1] > 1, hz = f->n[2] > 1;
  if (hx && hy && hz) {
    v3 v00 = lerp(gdat(f, nx, ny, nz), gdat(f, nx + 1, ny, nz), dx, f->step[0]);
    v3 v10 = lerp(gdat(f, nx, ny + 1, nz), gdat(f, nx + 1, ny + 1, nz), dx, f->step[0]);
    v3 v01 = lerp(gdat(f, nx, ny, nz + 1), gdat(f, nx + 1, ny, nz + 1), dx, f->step[0]);
    v3 v11 = lerp(gdat(f, nx, ny + 1, nz + 1), gdat(f, nx + 1, ny + 1, nz + 1), dx, f->step[0]);
    v3 v0 = lerp(v00, v10, dy, f->step[1]);
    v3 v1 = lerp(v01, v11, dy, f->step[1]);
    return lerp(v0, v1, dz, f->step[2]);
  } else if (hx && hy) {
    v3 v0 = lerp(gdat(f, nx, ny, 0), gdat(f, nx + 1, ny, 0), dx, f->step[0]);
    v3 v1 = lerp(gdat(f, nx, ny + 1, 0), gdat(f, nx + 1, ny + 1, 0), dx, f->step[0]);
    return lerp(v0, v1, dy, f->step[1]);
  } else if (hx && hz) {
    v3 v0 = lerp(gdat(f, nx, 0, nz), gdat(f, nx + 1, 0, nz), dx, f->step[0]);
    v3 v1 = lerp(gdat(f, nx, 0, nz + 1), gdat(f, nx + 1, 0, nz + 1), dx, f->step[0]);
    return lerp(v0, v1, dz, f->step[2]);
  } else if (hy && hz) {
    v3 v0 = lerp(gdat(f, 0, ny, nz), gdat(f, 0, ny + 1, nz), dy, f->step[1]);
    v3 v1 = lerp(gdat(f, 0, ny, nz + 1), gdat(f, 0, ny + 1, nz + 1), dy, f->step[1]);
    return lerp(v0, v1, dz, f->step[2]);
  } else if (hx) {
    return lerp(ld(f->data + 3 * nx), ld(f->data + 3 * (nx + 1)), dx, f->step[0]);
  } else if (hy) {
    return lerp(ld(f->data + 3 * ny), ld(f->data + 3 * (ny + 1)), dy, f->step[1]);
  } else if (hz) {
    return lerp(ld(f->data + 3 * nz), ld(f->data + 3 * (nz + 1)), dz, f->step[2]);
  }
  return mk(0, 0, 0);
}

/* src/TFieldContainer.cc:92-103: Sum(0,0,0) += each field */
void orc_field_eval(const orc_field *fields, int nfields, const double x[3], double out[3]) {
  v3 X = ld(x), s = mk(0, 0, 0);
  for (int i = 0; i < nfields; ++i) {
    v3 f;
    switch (fields[i].kind) {
      case ORC_UNDULATOR: f = undulator(&fields[i], X); break;
      case ORC_GAUSSIAN: f = gaussian(&fields[i], X); break;
      case ORC_UNIFORM_BOX: f = ubox(&fields[i], X); break;
      case ORC_GRID: f = grid(&fields[i], X); break;
      default: f = mk(0, 0, 0);
    }
    s = vadd(s, f);
  }
  out[0] = s.x; out[1] = s.y; out[2] = s.z;
}

void orc_free(void *p) { free(p); }

/* src/TField3D_Grid.cc:318-509 (OSCARS format).  Header values are the first number on each line. */
int orc_grid_read_oscars(const char *path, const double rotations[3], const double translation[3],
                         const double *scaling, int nscaling, orc_field *out) {
  FILE *fp = fopen(path, "r");
  if (!fp) return -1;
  char line[4096];
  double hv[9];
  if (!fgets(line, sizeof line, fp)) { fclose(fp); return -2; }
  for (int k = 0; k < 9; ++k) {
    if (!fgets(line, sizeof line, fp)) { fclose(fp); return -2; }
    hv[k] = strtod(line, NULL);
  }
  int NX = (int)hv[2], NY = (int)hv[5], NZ = (int)hv[8];
  double xs_in = hv[0], xst_in = hv[1], ys_in = hv[3], yst_in = hv[4], zs_in = hv[6], zst_in = hv[7];
  double xst = nscaling > 0 ? xst_in * scaling[0] : xst_in;
  double yst = nscaling > 1 ? yst_in * scaling[1] : yst_in;
  double zst = nscaling > 2 ? zst_in * scaling[2] : zst_in;
  double fxs = nscaling > 3 ? scaling[3] : 1, fys = nscaling > 4 ? scaling[4] : 1,
         fzs = nscaling > 5 ? scaling[5] : 1;
  double mx = xs_in + xst_in * (NX - 1) / 2., xs = mx - xst * (NX - 1) / 2.;
  double my = ys_in + yst_in * (NY - 1) / 2., ys = my - yst * (NY - 1) / 2.;
  double mz = zs_in + zst_in * (NZ - 1) / 2., zs = mz - zst * (NZ - 1) / 2.;
  if (NX < 1 || NY < 1 || NZ < 1 || (NX == 1 && NY == 1 && NZ == 1)) { fclose(fp); return -3; }
  size_t n = (size_t)NX * NY * NZ;
  double *data = (double *)malloc(sizeof(double) * 3 * n);
  for (size_t i = 0; i < n; ++i) {
    if (!fgets(line, sizeof line, fp)) { free(data); fclose(fp); return -4; }
    char *e1, *e2, *e3;
    double fx = strtod(line, &e1), fy = strtod(e1, &e2), fz = strtod(e2, &e3);
    if (e3 == e2) { free(data); fclose(fp); return -4; }
    if (fxs != 1) fx *= fxs;
    if (fys != 1) fy *= fys;
    if (fzs != 1) fz *= fzs;
    v3 F = mk(fx, fy, fz);
    rot_xyz(&F, rotations);
    data[3 * i] = F.x; data[3 * i + 1] = F.y; data[3 * i + 2] = F.z;
  }
  fclose(fp);
  memset(out, 0, sizeof *out);
  out->kind = ORC_GRID;
  out->n[0] = NX; out->n[1] = NY; out->n[2] = NZ;
  out->start[0] = xs; out->start[1] = ys; out->start[2] = zs;
  out->step[0] = xst; out->step[1] = yst; out->step[2] = zst;
  memcpy(out->rotations, rotations, sizeof(double) * 3);
  memcpy(out->translation, translation, sizeof(double) * 3);
  out->data = data;
  return 0;
}

/* ---- trajectory: src/OSCARSSR.cc:562-673, DerivativesB :741-765, RK4 :826-874 ---- */

void orc_trajectory_counts(double ctstart, double ctstop, double t0, int64_t npts, double *dt,
                           int64_t *nf, int64_t *nb) {
  double DeltaT = ((ctstop - ctstart) / c_c() / (double)(size_t)(npts - 1));
  *dt = DeltaT;
  *nf = (int64_t)(size_t)(1 + (ctstop - t0) / c_c() / DeltaT);
  *nb = (int64_t)(size_t)((t0 - ctstart) / c_c() / DeltaT);
}

static void derivs_b(const orc_field *fields, int nf, const double x[6], double d[6], double qomg) {
  double p[3] = {x[0], x[2], x[4]}, B[3];
  orc_field_eval(fields, nf, p, B);
  d[0] = x[1];
  d[1] = qomg * (-x[5] * B[1] + x[3] * B[2]);
  d[2] = x[3];
  d[3] = qomg * (x[5] * B[0] - x[1] * B[2]);
  d[4] = x[5];
  d[5] = qomg * (x[1] * B[1] - x[3] * B[0]);
}

static void rk4(const orc_field *fields, int nf, double y[6], const double dydx[6], double h,
                double qomg) {
  double dym[6], dyt[6], yt[6];
  double hh = h * 0.5, h6 = h / 6.0;
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dydx[i];
  derivs_b(fields, nf, yt, dyt, qomg);
  for (int i = 0; i < 6; ++i) yt[i] = y[i] + hh * dyt[i];
  derivs_b(fields, nf, yt, dym, qomg);
  for (int i = 0; i < 6; ++i) { yt[i] = y[i] + h * dym[i]; dym[i] += dyt[i]; }
  derivs_b(fields, nf, yt, dyt, qomg);
  for (int i = 0; i < 6; ++i) y[i] = y[i] + h6 * (dydx[i] + dyt[i] + 2.0 * dym[i]);
}

int64_t orc_trajectory(const orc_field *fields, int nfields, const double x0[3], const double b0[3],
                       double qomg, double ctstart, double ctstop, double t0, int64_t npts, double *X,
                       double *B, double *A, double *dt_out) {
  double dt;
  int64_t nf, nb;
  orc_trajectory_counts(ctstart, ctstop, t0, npts, &dt, &nf, &nb);
  *dt_out = dt;
  int64_t n = nf + nb;
  const double C = c_c();
  double x[6], d[6] = {0, 0, 0, 0, 0, 0}; /* d starts at 0: the reference reads it uninitialised */
#define STORE(k)                                                                                \
  do {                                                                                          \
    X[k] = x[0]; X[n + (k)] = x[2]; X[2 * n + (k)] = x[4];                                      \
    B[k] = x[1] / C; B[n + (k)] = x[3] / C; B[2 * n + (k)] = x[5] / C;                          \
    A[k] = d[1] / C; A[n + (k)] = d[3] / C; A[2 * n + (k)] = d[5] / C;                          \
  } while (0)
  x[0] = x0[0]; x[1] = b0[0] * C; x[2] = x0[1]; x[3] = b0[1] * C; x[4] = x0[2]; x[5] = b0[2] * C;
  for (int64_t i = 0; i < nf; ++i) {
    STORE(nb + i);
    derivs_b(fields, nfields, x, d, qomg);
    rk4(fields, nfields, x, d, dt, qomg);
  }
  x[0] = x0[0]; x[1] = b0[0] * C; x[2] = x0[1]; x[3] = b0[1] * C; x[4] = x0[2]; x[5] = b0[2] * C;
  for (int64_t i = 0; i < nb; ++i) {
    derivs_b(fields, nfields, x, d, qomg);
    rk4(fields, nfields, x, d, -dt, qomg);
    STORE(nb - 1 - i);
  }
#undef STORE
  return n;
}

/* ---- radiation sums ---- */

static void kahan_add(double *out, double *comp, int64_t i, double v) { /* TSpectrumContainer.cc:159-175 */
  double sum = out[i], y = v - comp[i], t = sum + y;
  comp[i] = (t - sum) - y;
  out[i] = t;
}

/* The per-observer sum shared by the spectrum (OSCARSSR.cc:1202-1246) and flux (:2054-2096) paths:
 * SumE += (B - N*(1 + i(c/w)/D))/D * exp(i w (dt*iT + D/c)) with libstdc++ complex arithmetic,
 * then SumE *= i C0 w dt and |SumE|^2.  Returns the flux before C2 and weight. */
static double efield_sq(const double *x, const double *b, int64_t n, double dt, v3 obs, double omega,
                        double C0) {
  const double C = c_c();
  double icow = C / omega; /* imaginary part of I*C/Omega; real part 0 */
  double sxr = 0, sxi = 0, syr = 0, syi = 0, szr = 0, szi = 0;
  for (int64_t it = 0; it < n; ++it) {
    v3 X = mk(x[it], x[n + it], x[2 * n + it]);
    v3 R = vsub(obs, X);
    v3 N = unit(R);
    double D = mag(R);
    double ph = omega * (dt * (double)(int)it + D / C);
    double cs = cos(ph), sn = sin(ph);
    double f = icow / D; /* (One + ICoverOmega/D) = (1, f) */
    double nx[3] = {N.x, N.y, N.z}, bb[3] = {b[it], b[n + it], b[2 * n + it]};
    double re[3], im[3];
    for (int k = 0; k < 3; ++k) {
      /* N*(1, f) = (nx*1 - 0*f, nx*f + 0*1); B - that; / D */
      double pr = nx[k] * 1.0 - 0.0 * f, pi = nx[k] * f + 0.0 * 1.0;
      double ar = (bb[k] - pr) / D, ai = (0.0 - pi) / D;
      re[k] = ar * cs - ai * sn;
      im[k] = ar * sn + ai * cs;
    }
    sxr += re[0]; sxi += im[0];
    syr += re[1]; syi += im[1];
    szr += re[2]; szi += im[2];
  }
  /* SumE *= (0*dt, C0*w*dt): (a + ib)(0 + ig) = (a*0 - b*g, a*g + b*0) */
  double g = (C0 * omega) * dt, z = 0.0 * dt;
  double e[6] = {sxr, sxi, syr, syi, szr, szi};
  double s = 0;
  double parts[3];
  for (int k = 0; k < 3; ++k) {
    double a = e[2 * k], bq = e[2 * k + 1];
    double pr = a * z - bq * g, pi = a * g + bq * z;
    parts[k] = pr * pr - pi * (-pi); /* real part of p * conj(p) */
  }
  s = (parts[0] + parts[1]) + parts[2];
  return s;
}

static double flux_c0(double q) { return q / (c_fourpi() * c_c() * c_eps0() * c_sqrt2pi()); }
static double flux_c2(double q, double current) {
  return c_fourpi() * current / (c_h() * fabs(q) * c_mu0() * c_c()) * 1e-6 * 0.001;
}

/* OSCARSSR::CalculateSpectrum(TParticleA&, TVector3D const&, TSpectrumContainer&, double)
 * src/OSCARSSR.cc:1154-1251 */
void orc_spectrum(const double *x, const double *b, int64_t n, double dt, const double obs[3],
                  const double *energies_ev, int64_t ne, double charge, double current, double weight,
                  double *out, double *comp) {
  double C0 = flux_c0(charge), C2 = flux_c2(charge, current);
  for (int64_t k = 0; k < ne; ++k) {
    double om = ev_to_omega(energies_ev[k]);
    double s = efield_sq(x, b, n, dt, ld(obs), om, C0);
    kahan_add(out, comp, k, C2 * s * weight);
  }
}

/* OSCARSSR::CalculateFlux2, src/OSCARSSR.cc:1989-2099 */
void orc_flux(const double *x, const double *b, int64_t n, double dt, const double *points, int64_t np,
              double energy_ev, double charge, double current, double weight, double *out, double *comp) {
  double C0 = flux_c0(charge), C2 = flux_c2(charge, current);
  double om = ev_to_omega(energy_ev);
  for (int64_t j = 0; j < np; ++j) {
    double s = efield_sq(x, b, n, dt, ld(points + 3 * j), om, C0);
    kahan_add(out, comp, j, C2 * s * weight);
  }
}

/* The sum of efield_sq evaluated in long double (x86-64: a 64-bit significand) on the same FP64
 * inputs (trajectory, observer, w, dt).  The retarded phase w (dt i + D/c) is 1e10-1e11 rad here; FP64
 * keeps it to ~1e-5 rad per term, which is what any FP64 evaluation of src/OSCARSSR.cc:1154-1251 /
 * :1989-2099 (the reference's included) carries, while long double keeps ~1e-8 rad.  This is the
 * exact sum those FP64 evaluations approximate: the yardstick for outputs so weak (1e-6 of the map's
 * maximum) that the FP64 rounding of the phase dominates their error.  Returns the flux per unit
 * weight (C2 |C0 w dt SumE|^2). */
static double efield_sq_exact(const double *x, const double *b, int64_t n, double dt, v3 obs, double omega,
                              double C0, double C2) {
  const long double C = c_c(), w = omega, ldt = dt;
  long double s[6] = {0, 0, 0, 0, 0, 0};
  for (int64_t it = 0; it < n; ++it) {
    long double R[3] = {(long double)obs.x - x[it], (long double)obs.y - x[n + it], (long double)obs.z - x[2 * n + it]};
    long double D = sqrtl(R[0] * R[0] + R[1] * R[1] + R[2] * R[2]);
    long double ph = w * (ldt * (long double)it + D / C);
    long double cs = cosl(ph), sn = sinl(ph);
    long double f = C / w / D;
    for (int k = 0; k < 3; ++k) {
      long double nk = R[k] / D;
      long double ar = ((long double)b[k * n + it] - nk) / D, ai = -nk * f / D;
      s[2 * k] += ar * cs - ai * sn;
      s[2 * k + 1] += ar * sn + ai * cs;
    }
  }
  long double g = (long double)C0 * w * ldt, tot = 0;
  for (int k = 0; k < 6; ++k) tot += (s[k] * g) * (s[k] * g);
  return (double)(C2 * tot);
}

void orc_flux_exact(const double *x, const double *b, int64_t n, double dt, const double *points, int64_t np,
                    double energy_ev, double charge, double current, double *out) {
  double C0 = flux_c0(charge), C2 = flux_c2(charge, current), om = ev_to_omega(energy_ev);
  for (int64_t j = 0; j < np; ++j) out[j] = efield_sq_exact(x, b, n, dt, ld(points + 3 * j), om, C0, C2);
}

void orc_spectrum_exact(const double *x, const double *b, int64_t n, double dt, const double obs[3],
                        const double *energies_ev, int64_t ne, double charge, double current, double *out) {
  double C0 = flux_c0(charge), C2 = flux_c2(charge, current);
  for (int64_t k = 0; k < ne; ++k) out[k] = efield_sq_exact(x, b, n, dt, ld(obs), ev_to_omega(energies_ev[k]), C0, C2);
}

/* OSCARSSR::CalculatePowerDensity(TParticleA&, TSurfacePoints const&, T3DScalarContainer&, ...)
 * src/OSCARSSR.cc:1477-1598 (the weight is not applied on this path: :1583-1591) */
void orc_power_density(const double *x, const double *b, const double *a, int64_t n, double dt,
                       const double *points, const double *normals, int64_t np, int directional,
                       double charge, double current, double *out, double *comp) {
  for (int64_t j = 0; j < np; ++j) {
    v3 obs = ld(points + 3 * j), nrm = ld(normals + 3 * j);
    double sum = 0;
    for (int64_t it = 0; it < n; ++it) {
      v3 X = mk(x[it], x[n + it], x[2 * n + it]);
      v3 B = mk(b[it], b[n + it], b[2 * n + it]);
      v3 AC = mk(a[it], a[n + it], a[2 * n + it]);
      v3 N1 = unit(vsub(obs, X));
      v3 N2 = unit(orthogonal(N1));
      v3 N3 = unit(cross(N1, N2));
      double nd = dot(N1, nrm);
      if (directional && nd <= 0) continue;
      v3 num = cross(N1, cross(vsub(N1, B), AC));
      double den = pow(1 - dot(B, N1), 5);
      double p2 = dot(num, N2), p3 = dot(num, N3);
      sum += p2 * p2 / den / mag2(vsub(obs, X)) * nd;
      sum += p3 * p3 / den / mag2(vsub(obs, X)) * nd;
    }
    sum *= fabs(charge * current) / (16 * c_pi2() * c_eps0() * c_c()) * dt;
    sum /= 1e6;
    if (!directional && sum < 0) sum *= -1;
    kahan_add(out, comp, j, sum);
  }
}

/* OSCARSSR::CalculateTotalPower(TParticleA&), src/OSCARSSR.cc:1939-1978 */
double orc_total_power(const double *b, const double *a, int64_t n, double dt, double charge,
                       double current, double gamma) {
  double tp = 0;
  for (int64_t i = 0; i < n; ++i) {
    v3 B = mk(b[i], b[n + i], b[2 * n + i]), AC = mk(a[i], a[n + i], a[2 * n + i]);
    tp += (mag2(AC) - mag2(cross(B, AC))) * dt;
  }
  tp *= fabs(charge * current) * pow(gamma, 6) / (6 * c_pi() * c_eps0() * c_c());
  return tp;
}

/* TSpectrumContainer::Init(N, EFirst, ELast), src/TSpectrumContainer.cc:55-86 */
void orc_energy_grid(int64_t n, double e0, double e1, double *out) {
  if (n == 1) { out[0] = e0; return; }
  for (int64_t i = 0; i < n; ++i) out[i] = e0 + (e1 - e0) / (double)(size_t)(n - 1) * (double)(i + 1);
}

/* ---- surfaces: src/TSurfacePoints_Rectangle.cc ---- */
static void rect_emit(int nx1, int nx2, v3 start, v3 v1, v3 v2, double s1, double s2, v3 nv,
                      double *xyz, double *x12, double nrm[3]) {
  size_t np = (size_t)(nx1 * nx2);
  for (size_t i = 0; i < np; ++i) {
    int i1 = (int)(i / nx2), i2 = (int)(i % nx2);
    v3 p = vadd(vadd(start, vmul(v1, (double)i1)), vmul(v2, (double)i2)); /* :222-230 */
    xyz[3 * i] = p.x; xyz[3 * i + 1] = p.y; xyz[3 * i + 2] = p.z;
    x12[2 * i] = s1 * i1 - mag(v1) * (nx1 - 1) / 2.;                      /* :244-251 */
    x12[2 * i + 1] = s2 * i2 - mag(v2) * (nx2 - 1) / 2.;                  /* :252-259 */
  }
  v3 n = unit(nv); /* TSurfacePoint normalises the normal again (src/TSurfacePoint.cc:19-24) */
  nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
}

int orc_rectangle_plane(const char *plane, int nx1, int nx2, double w1, double w2, const double rot[3],
                        const double trans[3], int normal, double *xyz, double *x12, double nrm[3]) {
  char P[8] = {0};
  for (int i = 0; i < 7 && plane[i]; ++i) P[i] = (char)toupper((unsigned char)plane[i]);
  double s1 = w1 / (nx1 - 1), s2 = w2 / (nx2 - 1);                       /* :150-152 */
  v3 start, v1, v2;
  if (!strcmp(P, "XY")) { start = mk(-w1 / 2., -w2 / 2., 0); v1 = mk(s1, 0, 0); v2 = mk(0, s2, 0); }
  else if (!strcmp(P, "YX")) { start = mk(-w2 / 2., -w1 / 2., 0); v2 = mk(s2, 0, 0); v1 = mk(0, s1, 0); }
  else if (!strcmp(P, "XZ")) { start = mk(-w1 / 2., 0, -w2 / 2.); v1 = mk(s1, 0, 0); v2 = mk(0, 0, s2); }
  else if (!strcmp(P, "ZX")) { start = mk(-w2 / 2., 0, -w1 / 2.); v2 = mk(s2, 0, 0); v1 = mk(0, 0, s1); }
  else if (!strcmp(P, "YZ")) { start = mk(0, -w1 / 2., -w2 / 2.); v1 = mk(0, s1, 0); v2 = mk(0, 0, s2); }
  else if (!strcmp(P, "ZY")) { start = mk(0, -w2 / 2., -w1 / 2.); v2 = mk(0, s2, 0); v1 = mk(0, 0, s1); }
  else return -1;
  rot_xyz(&start, rot); rot_xyz(&v1, rot); rot_xyz(&v2, rot);
  start = vadd(start, ld(trans));
  v3 nv = unit(cross(v1, v2));
  if (normal == -1) nv = vmul(nv, -1);
  else if (normal != 0 && normal != 1) return -1;
  rect_emit(nx1, nx2, start, v1, v2, s1, s2, nv, xyz, x12, nrm);
  return 0;
}

int orc_rectangle_points(int nx1, int nx2, const double x0[3], const double x1[3], const double x2[3],
                         const double rot[3], const double trans[3], int normal, double *xyz,
                         double *x12, double nrm[3]) {
  v3 p0 = ld(x0), p1 = ld(x1), p2 = ld(x2);
  rot_xyz(&p0, rot); p0 = vadd(p0, ld(trans));  /* OSCARSSR_Python.cc:2712-2715 */
  rot_xyz(&p1, rot); p1 = vadd(p1, ld(trans));
  rot_xyz(&p2, rot); p2 = vadd(p2, ld(trans));
  double w1 = mag(vsub(p1, p0)), w2 = mag(vsub(p2, p0)); /* TSurfacePoints_Rectangle.cc:95-103 */
  double s1 = w1 / (nx1 - 1), s2 = w2 / (nx2 - 1);
  v3 v1 = vdiv(vsub(p1, p0), (double)(nx1 - 1)), v2 = vdiv(vsub(p2, p0), (double)(nx2 - 1));
  v3 nv = unit(cross(v1, v2));
  if (normal == -1) nv = vmul(nv, -1);
  else if (normal != 0 && normal != 1) return -1;
  rect_emit(nx1, nx2, p0, v1, v2, s1, s2, nv, xyz, x12, nrm);
  return 0;
}

/* ---- random numbers: src/TRandomA.cc (std::mt19937 + std::normal_distribution<double> +
 * std::uniform_real_distribution<double>).  Restated from the published algorithms:
 * MT19937 (Matsumoto & Nishimura, 1998), libstdc++'s generate_canonical<double,53> (two 32-bit
 * draws), and the Marsaglia polar method with one cached value, which a reseed does not clear. ---- */
static uint32_t mt[624];
static int mti = 625;
static int nsaved = 0;
static double saved;

void orc_rng_seed(uint32_t s) {
  mt[0] = s;
  for (int i = 1; i < 624; ++i) mt[i] = 1812433253u * (mt[i - 1] ^ (mt[i - 1] >> 30)) + (uint32_t)i;
  mti = 624;
}
static uint32_t mt_next(void) {
  if (mti >= 624) {
    if (mti == 625) orc_rng_seed(5489u);
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (mt[i] & 0x80000000u) | (mt[(i + 1) % 624] & 0x7fffffffu);
      mt[i] = mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    mti = 0;
  }
  uint32_t y = mt[mti++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}
static double canonical(void) {
  const double r = 4294967296.0;
  double sum = (double)mt_next();
  double tmp = r;
  sum += (double)mt_next() * tmp;
  tmp *= r;
  double ret = sum / tmp;
  if (ret >= 1.0) ret = nextafter(1.0, 0.0);
  return ret;
}
void orc_rng_clear_cache(void) { nsaved = 0; }
double orc_rng_uniform(void) { return canonical() * (1.0 - 0.0) + 0.0; }
double orc_rng_normal(void) {
  double ret;
  if (nsaved) {
    nsaved = 0;
    ret = saved;
  } else {
    double x, y, r2;
    do {
      x = 2.0 * canonical() - 1.0;
      y = 2.0 * canonical() - 1.0;
      r2 = x * x + y * y;
    } while (r2 > 1.0 || r2 == 0.0);
    double mult = sqrt(-2 * log(r2) / r2);
    saved = x * mult;
    nsaved = 1;
    ret = y * mult;
  }
  return ret * 1.0 + 0.0;
}

/* ---- particle beam: src/OSCARSSR_Python.cc:1661-1870, src/TParticleBeam.cc, src/TParticleA.cc ---- */
int orc_beam_init(orc_beam *bm, const char *type, double energy_gev, const double d0[3],
                  const double x0[3], double sigma_energy_gev, double t0, double current,
                  const double rot[3], const double trans[3], const double *hdir, const double *beta,
                  const double *emittance, const double lattice_ref[3], double mass, double charge) {
  memset(bm, 0, sizeof *bm);
  char t[32] = {0};
  for (int i = 0; i < 31 && type[i]; ++i) t[i] = (char)tolower((unsigned char)type[i]);
  if (!strcmp(type, "custom")) { bm->q = charge; bm->m = mass; }
  else if (!strcmp(t, "electron") || !strcmp(t, "anti-positron")) { bm->q = -c_qe(); bm->m = c_me(); }
  else if (!strcmp(t, "positron") || !strcmp(t, "anti-electron")) { bm->q = c_qe(); bm->m = c_me(); }
  else if (!strcmp(t, "muon")) { bm->q = -c_qe(); bm->m = gev_to_kg(0.1056583715); }
  else if (!strcmp(t, "anti-muon")) { bm->q = c_qe(); bm->m = gev_to_kg(0.1056583715); }
  else if (!strcmp(t, "proton")) { bm->q = c_qe(); bm->m = gev_to_kg(0.938272046); }
  else if (!strcmp(t, "anti-proton")) { bm->q = -c_qe(); bm->m = gev_to_kg(0.938272046); }
  else if (!strcmp(t, "pi+")) { bm->q = c_qe(); bm->m = gev_to_kg(0.13957018); }
  else if (!strcmp(t, "pi-")) { bm->q = -c_qe(); bm->m = gev_to_kg(0.13957018); }
  else return -1;
  v3 pos = ld(x0), dir = ld(d0);
  v3 h = hdir ? ld(hdir) : unit(orthogonal(dir));
  h = unit(h);
  double su0 = 0, su1 = 0, sp0 = 0, sp1 = 0;
  if (beta && emittance) {
    su0 = sqrt(emittance[0] * beta[0]); su1 = sqrt(emittance[1] * beta[1]);
    sp0 = sqrt(emittance[0] / beta[0]); sp1 = sqrt(emittance[1] / beta[1]);
  }
  rot_xyz(&pos, rot);
  pos = vadd(pos, ld(trans));
  bm->current = current != 0 ? current : bm->q; /* TParticleA::SetCurrent */
  bm->x0[0] = pos.x; bm->x0[1] = pos.y; bm->x0[2] = pos.z;
  v3 u = unit(dir);
  bm->u0[0] = u.x; bm->u0[1] = u.y; bm->u0[2] = u.z;
  bm->e0 = energy_gev;
  bm->t0 = t0;
  /* TParticleBeam::SetSigma, src/TParticleBeam.cc:137-158 */
  v3 hh = unit(h);
  v3 vv = unit(cross(u, hh));
  if (fabs(dot(hh, u)) > 0.00000001) return -2;
  bm->hdir[0] = hh.x; bm->hdir[1] = hh.y; bm->hdir[2] = hh.z;
  bm->vdir[0] = vv.x; bm->vdir[1] = vv.y; bm->vdir[2] = vv.z;
  bm->sigma_u[0] = su0; bm->sigma_u[1] = su1;
  bm->sigma_up[0] = sp0; bm->sigma_up[1] = sp1;
  bm->sigma_at[0] = lattice_ref[0]; bm->sigma_at[1] = lattice_ref[1]; bm->sigma_at[2] = lattice_ref[2];
  bm->sigma_e = sigma_energy_gev;
  return 0;
}

/* TParticleBeam::GetNewParticle("ideal") :200-222 / GetNewParticle() :228-265, then
 * TParticleA::SetInitialParticleConditions -> SetGamma -> SetQoverMGamma (TParticleA.cc:353-382) */
void orc_beam_particle(const orc_beam *bm, int random, double x0[3], double b0[3], double *gamma,
                       double *qomg) {
  v3 X, Bv;
  v3 u = ld(bm->u0);
  if (!random) {
    double g = bm->e0 / kg_to_gev(bm->m);
    double beta = sqrt(1.0 - 1.0 / (g * g));
    X = ld(bm->x0);
    Bv = vmul(u, beta);
  } else {
    double enew = bm->e0 + bm->sigma_e * orc_rng_normal();
    double g = enew / kg_to_gev(bm->m);
    double beta = sqrt(1.0 - 1.0 / (g * g));
    double dmid = dot(vsub(ld(bm->sigma_at), ld(bm->x0)), u);
    X = ld(bm->x0);
    X = vadd(X, vmul(vmul(vmul(ld(bm->hdir), bm->sigma_u[0]), 1 + dmid), orc_rng_normal()));
    X = vadd(X, vmul(vmul(vmul(ld(bm->vdir), bm->sigma_u[1]), 1 + dmid), orc_rng_normal()));
    Bv = vmul(u, beta);
    rot_y(&Bv, bm->sigma_up[0] * orc_rng_normal());
    rot_x(&Bv, -bm->sigma_up[1] * orc_rng_normal());
  }
  double b2 = mag2(Bv);
  double g = 1.0 / sqrt(1.0 - b2);
  x0[0] = X.x; x0[1] = X.y; x0[2] = X.z;
  b0[0] = Bv.x; b0[1] = Bv.y; b0[2] = Bv.z;
  *gamma = g;
  *qomg = bm->q / bm->m / g;
}

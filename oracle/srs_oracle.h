/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C99 restatement of the reference's (dhidas/SRSOriginal, OSCARS SR 1.31.05) CPU algorithm
 * for the radiation hot path, in the reference's own IEEE-double operation order.  Only the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it, and only as the checker; nothing
 * in the shipped library links or calls it.
 *
 * Pinned against the reference itself: tests/golden/make_golden.py runs the reference (built from
 * its own sources by oracle/Makefile) and stores its outputs as fixtures, and
 * tests/test_oracle_golden.py checks this restatement against them.
 */
#ifndef SRS_ORACLE_H
#define SRS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Field kinds (same numbering as the product's include/srs_b200.h). */
enum { ORC_UNDULATOR = 1, ORC_GAUSSIAN = 2, ORC_UNIFORM_BOX = 3, ORC_GRID = 4 };

/* One magnetic-field object, already in the form the reference stores after construction. */
typedef struct {
  int kind;
  /* undulator: field (rotated), period (rotated), center, nperiods, phase, taper */
  double field[3];
  double period[3];
  double center[3];
  int nperiods;
  double phase;
  double taper;
  /* gaussian / box: field (rotated), center, sigma-or-width, rotations applied to the point */
  double sigma_or_width[3];
  double rotations[3];
  /* grid: rotations, translation, start/step/n per axis, data (n = nx*ny*nz rotated vectors) */
  double translation[3];
  double start[3];
  double step[3];
  int64_t n[3];
  const double *data; /* 3 doubles per sample, ix*ny*nz + iy*nz + iz */
} orc_field;

/* Sum of all fields at x (TFieldContainer::GetF). */
void orc_field_eval(const orc_field *fields, int nfields, const double x[3], double out[3]);

/* Reads an OSCARS-format grid file (TField3D_Grid::ReadFile); data is malloc'ed, free with
 * orc_free.  Returns 0 on success. */
int orc_grid_read_oscars(const char *path, const double rotations[3], const double translation[3],
                         const double *scaling, int nscaling, orc_field *out);
void orc_free(void *p);

/* Trajectory point counts and time step (OSCARSSR::CalculateTrajectory). */
void orc_trajectory_counts(double ctstart, double ctstop, double t0, int64_t npoints_setting,
                           double *dt, int64_t *nforward, int64_t *nbackward);

/* Fixed-step RK4 trajectory.  x/b/a are SoA arrays of 3*(nf+nb) doubles (x[0..n), x[n..2n) ...).
 * Returns the number of points written. */
int64_t orc_trajectory(const orc_field *fields, int nfields, const double x0[3], const double b0[3],
                       double qomg, double ctstart, double ctstop, double t0, int64_t npoints_setting,
                       double *x, double *b, double *a, double *dt_out);

/* Radiation sums; trajectory SoA as above with n points.  Results are *added* (Kahan) into out
 * with compensation array comp (both length nout), as the reference's containers do. */
void orc_spectrum(const double *x, const double *b, int64_t n, double dt, const double obs[3],
                  const double *energies_ev, int64_t ne, double charge, double current, double weight,
                  double *out, double *comp);
void orc_flux(const double *x, const double *b, int64_t n, double dt, const double *points, int64_t np,
              double energy_ev, double charge, double current, double weight, double *out, double *comp);
void orc_power_density(const double *x, const double *b, const double *a, int64_t n, double dt,
                       const double *points, const double *normals, int64_t np, int directional,
                       double charge, double current, double *out, double *comp);
double orc_total_power(const double *b, const double *a, int64_t n, double dt, double charge,
                       double current, double gamma);

/* The same flux / spectrum sums in long double on the same FP64 inputs (written, not added): the exact
 * values that FP64 evaluations of the retarded phase approximate (see srs_oracle.c). */
void orc_flux_exact(const double *x, const double *b, int64_t n, double dt, const double *points, int64_t np,
                    double energy_ev, double charge, double current, double *out);
void orc_spectrum_exact(const double *x, const double *b, int64_t n, double dt, const double obs[3],
                        const double *energies_ev, int64_t ne, double charge, double current, double *out);

/* Spectrum energy grid (TSpectrumContainer::Init(N, EFirst, ELast)). */
void orc_energy_grid(int64_t n, double efirst, double elast, double *out);

/* Rectangle surfaces (TSurfacePoints_Rectangle).  plane: "XY","YX","XZ","ZX","YZ","ZY".
 * xyz: 3*np point coordinates (AoS), x12: 2*np in-plane coordinates (GetX1, GetX2), normal[3] is
 * the per-point unit normal (TSurfacePoint normalises it again).  Returns 0 or -1 on bad input. */
int orc_rectangle_plane(const char *plane, int nx1, int nx2, double w1, double w2, const double rot[3],
                        const double trans[3], int normal, double *xyz, double *x12, double nrm[3]);
int orc_rectangle_points(int nx1, int nx2, const double x0[3], const double x1[3], const double x2[3],
                         const double rot[3], const double trans[3], int normal, double *xyz,
                         double *x12, double nrm[3]);

/* Process-wide random generator (TRandomA): MT19937 + libstdc++'s normal and uniform draws. */
void orc_rng_seed(uint32_t seed);
double orc_rng_normal(void);
double orc_rng_uniform(void);
void orc_rng_clear_cache(void); /* a fresh process's state: no cached normal */

/* Particle physics helpers (TParticleA / TParticleBeam). */
typedef struct {
  double q, m, current;   /* charge [C], mass [kg], beam current [A] */
  double x0[3], u0[3];    /* beam position, unit direction */
  double e0, t0;          /* energy [GeV], t0 [m] */
  double hdir[3], vdir[3];/* horizontal / vertical unit directions */
  double sigma_u[2], sigma_up[2], sigma_at[3], sigma_e;
} orc_beam;

/* Fills beam from the set_particle_beam arguments (OSCARSSR_Python.cc:1661-1870). */
int orc_beam_init(orc_beam *bm, const char *type, double energy_gev, const double d0[3],
                  const double x0[3], double sigma_energy_gev, double t0, double current,
                  const double rot[3], const double trans[3], const double *hdir /* or NULL */,
                  const double *beta /* [2] or NULL */, const double *emittance /* or NULL */,
                  const double lattice_ref[3], double mass, double charge);
/* Ideal or random particle: writes x0, beta0, gamma and q/(m gamma). */
void orc_beam_particle(const orc_beam *bm, int random, double x0[3], double b0[3], double *gamma,
                       double *qomg);

#ifdef __cplusplus
}
#endif
#endif

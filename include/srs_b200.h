/*
 * srs_b200 -- B200-native radiation hot path of the SRS / OSCARS synchrotron-radiation simulator:
 * the RK4 electron trajectory through magnetic fields and the frequency-domain Lienard-Wiechert sums
 * (on-axis spectrum, flux on a surface, power density on a surface).
 *
 * Plain C ABI: POD structs, plain pointers and sizes, no C++ or torch types.  Every call returns an
 * srs_status; srs_last_error() returns the message of the calling thread's last failure.  No
 * exception crosses this boundary.
 *
 * Reference interfaces replaced (paths inside dhidas/SRSOriginal):
 *   include/OSCARSSR_Cuda.h:25  OSCARSSR_Cuda_GetDeviceCount            -> srs_device_count
 *   include/OSCARSSR_Cuda.h:27  OSCARSSR_Cuda_CalculateSpectrumGPU      -> srs_spectrum
 *   include/OSCARSSR_Cuda.h:26  OSCARSSR_Cuda_CalculateFluxGPU          -> srs_flux
 *   include/OSCARSSR_Cuda.h:28  OSCARSSR_Cuda_CalculatePowerDensityGPU  -> srs_power_density
 *   src/OSCARSSR.cc:562-874     OSCARSSR::CalculateTrajectory + RK4     -> srs_trajectory
 *   src/OSCARSSR.cc:1939-1978   OSCARSSR::CalculateTotalPower           -> srs_total_power
 * and, for the Python-facing calls of src/OSCARSSR_Python.cc, the srs_sim_* object API below.
 *
 * Units follow the reference: SI, energies in eV (photons) and GeV (beam), times as c*t in metres,
 * flux in photons/s/0.1%bw/mm^2, power density in W/mm^2.
 */
#ifndef SRS_B200_H
#define SRS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int srs_status;
enum {
  SRS_OK = 0,
  SRS_ERR_INVALID = 1,   /* bad argument (reference: ValueError / std::invalid_argument) */
  SRS_ERR_RANGE = 2,     /* out of range / length (reference: std::out_of_range, length_error) */
  SRS_ERR_CUDA = 3,      /* a CUDA runtime error; the message names the call */
  SRS_ERR_NO_DEVICE = 4, /* no CUDA device */
  SRS_ERR_TIMEOUT = 5,   /* a bounded device-side wait gave up */
  SRS_ERR_IO = 6         /* a field file could not be read */
};

/* Message of the calling thread's last failed call ("" if none). */
const char *srs_last_error(void);
/* Library version string. */
const char *srs_version(void);

/* Number of CUDA devices (OSCARSSR_Cuda_GetDeviceCount, src/OSCARSSR_Cuda.cu:30-36). */
int srs_device_count(void);

/* The library's temporary device buffers come from its own stream-ordered memory pool on each device,
 * which keeps freed blocks for the next call (no counterpart in the reference, which allocates host
 * memory only).  This returns the current device's unused blocks to the driver. */
srs_status srs_trim_memory(void);

/* ------------------------------------------------------------------ fields */

enum { SRS_FIELD_UNDULATOR = 1, SRS_FIELD_GAUSSIAN = 2, SRS_FIELD_UNIFORM_BOX = 3, SRS_FIELD_GRID = 4 };
/* kind | SRS_FIELD_ELECTRIC: an electric field [V/m] of the same shape, in the reference's separate
 * electric-field container (OSCARSSR.cc:202-234).  With electric fields the RK4 derivative is
 * q/(m gamma) E alone or q/(m gamma) (E + v x B) (DerivativesE / DerivativesEB, OSCARSSR.cc:690-793). */
enum { SRS_FIELD_ELECTRIC = 0x100, SRS_FIELD_SHAPE_MASK = 0xff };

/* One magnetic-field object in the form the reference keeps after construction:
 *  undulator (TField3D_IdealUndulator.cc): field and period already rotated, center, nperiods,
 *            phase [rad], taper [1/m];
 *  gaussian  (TField3D_Gaussian.cc): field already rotated, center, sigma (axes with sigma<=0 are
 *            ignored), rotations applied to the evaluation point;
 *  uniform box (TField3D_UniformBox.cc): field rotated, center, width (<=0: unbounded axis),
 *            rotations applied to the point;
 *  grid (TField3D_Grid.cc): rotations and translation applied to the point, start/step/n per axis,
 *            data = 3 doubles per sample at index ix*ny*nz + iy*nz + iz, already rotated.  For
 *            srs_trajectory the data pointer must be DEVICE memory; the srs_sim_* API owns its copy. */
typedef struct srs_field {
  int32_t kind;
  int32_t nperiods;
  double field[3];
  double period[3];
  double center[3];
  double phase;
  double taper;
  double sigma_or_width[3];
  double rotations[3];
  double translation[3];
  double start[3];
  double step[3];
  int64_t n[3];
  const double *data;
} srs_field;

/* Initial conditions of one particle: position [m], beta = v/c, q/(m gamma) [C/kg]. */
typedef struct srs_particle {
  double x0[3];
  double beta0[3];
  double qomg;
} srs_particle;

/* ------------------------------------------------------------------ trajectory */

/* Time step and point counts of the reference's forward/backward RK4 (OSCARSSR.cc:592-598):
 * dt = (ctstop-ctstart)/c/(npoints-1), nforward = (size_t)(1 + (ctstop-t0)/c/dt),
 * nbackward = (size_t)((t0-ctstart)/c/dt); a trajectory has nforward+nbackward points. */
srs_status srs_trajectory_counts(double ctstart, double ctstop, double t0, int64_t npoints, double *dt,
                                 int64_t *nforward, int64_t *nbackward);

/* Fixed-step RK4 of nparticles particles through the sum of the fields, one CUDA thread per
 * particle, in the reference's IEEE-double operation order (OSCARSSR.cc:562-874).  particles and
 * fields are HOST arrays; d_x, d_beta, d_aoc are DEVICE arrays of nparticles*3*n doubles laid out
 * [particle][component][point] (n = nforward+nbackward).  The stored a/c of a point is the derivative
 * at the previous step's state, as in the reference (0 at the first forward point).  stream: a
 * cudaStream_t or NULL. */
srs_status srs_trajectory(const srs_field *fields, int32_t nfields, const srs_particle *particles,
                          int32_t nparticles, double ctstart, double ctstop, double t0, int64_t npoints,
                          double *d_x, double *d_beta, double *d_aoc, void *stream);

/* The trajectory of ONE particle, integrated parallel in time: the serial RK4 chain is cut into
 * segments of steps_per_segment steps (0 = automatic) whose start states are found by Newton
 * iterations of multiple shooting, every segment stepping with the same arithmetic as srs_trajectory.
 * The result equals srs_trajectory's to a few ulps of the positions (~1e-16 m), not bit for bit: it
 * feeds the mixed-precision sums, while the FP64 drop-in keeps srs_trajectory.  When the iteration
 * has not converged after max_iterations iterations (0 = 8; at most 32) the serial kernel writes the
 * trajectory instead (no host synchronisation either way).  d_stats (optional, DEVICE, 4 doubles): converged (1 or 0),
 * iterations, and the largest mismatch between a segment's end and the next one's start in the last
 * and in the previous iteration, relative to the trajectory's extent (positions) or speed (velocities);
 * the stored trajectory's is the last one's (below 2^-51 when converged).
 * No reference counterpart: the reference integrates serially (OSCARSSR.cc:562-673). */
srs_status srs_trajectory_shoot(const srs_field *fields, int32_t nfields, const srs_particle *particle,
                                double ctstart, double ctstop, double t0, int64_t npoints,
                                int32_t steps_per_segment, int32_t max_iterations, double *d_x,
                                double *d_beta, double *d_aoc, double *d_stats, void *stream);

/* ------------------------------------------------------------------ radiation sums */

/* Arithmetic of the sums. */
enum {
  SRS_PRECISION_FP64 = 0, /* plain IEEE double, the reference's operation order: the drop-in */
  SRS_PRECISION_MIXED = 1 /* FP32 amplitude/sincos/accumulation, FP64 phase and reduction */
};

/* Trajectory of one or more particles on the DEVICE, layout as written by srs_trajectory. */
typedef struct srs_traj_view {
  const double *x;
  const double *beta;
  const double *aoc;
  int64_t n;          /* points per particle */
  int32_t nparticles; /* particles, consecutive blocks of 3*n doubles */
  double dt;          /* time step [s] */
} srs_traj_view;

/* Beam constants of the sums: particle charge [C] and beam current [A]. */
typedef struct srs_beam_consts {
  double charge;
  double current;
} srs_beam_consts;

/* Flux spectrum at one observer (OSCARSSR_Cuda_CalculateSpectrumGPU / OSCARSSR.cc:1154-1251):
 * d_energies (DEVICE, ne photon energies in eV).  d_out (DEVICE) receives nparticles*ne values,
 * particle-major: flux of each particle (weight 1).  Mixed precision walks uniform energy grids with
 * a complex-rotation recurrence; non-uniform grids get one sincos per term. */
srs_status srs_spectrum(srs_traj_view traj, srs_beam_consts beam, const double obs[3],
                        const double *d_energies, int64_t ne, int32_t precision, double *d_out,
                        void *stream);

/* Flux at np observation points at one photon energy (OSCARSSR_Cuda_CalculateFluxGPU /
 * OSCARSSR.cc:1989-2099).  d_points: DEVICE, 3*np doubles (x,y,z per point).  d_out: DEVICE,
 * nparticles*np values.  For SRS_PRECISION_MIXED, points that form a regular grid are best given as
 * grid (see srs_grid2d; d_points may then be NULL): the tiles anchor the FP64 geometry on it.  With
 * grid NULL any list of points is accepted; the geometry and phase are then FP64 per term and the
 * amplitude, sincos and accumulation FP32. */
typedef struct srs_grid2d {
  double origin[3]; /* point (0,0) */
  double u1[3];     /* step to point (1,0) */
  double u2[3];     /* step to point (0,1) */
  double normal[3]; /* unit surface normal (power density) */
  int32_t n1, n2;   /* point i is (i / n2, i % n2), as TSurfacePoints_Rectangle::GetXYZ */
} srs_grid2d;

srs_status srs_flux(srs_traj_view traj, srs_beam_consts beam, const double *d_points, int64_t np,
                    const srs_grid2d *grid, double energy_ev, int32_t precision, double *d_out,
                    void *stream);

/* srs_flux with SRS_PRECISION_MIXED on a grid, allocating nothing.  No counterpart in the
 * reference.  For callers that must not allocate device memory while they run (their device memory
 * is reserved up front by their own allocator, or a loop that may not call cudaMalloc, whose latency
 * is unbounded and which can synchronise the device).  srs_flux takes its scratch (per-chunk partial
 * sums) from a stream-ordered allocation; this entry point uses a fixed 8 MiB array that the library
 * defines in device memory instead, which every GPU that loads the library holds until the process
 * exits.  Limit: nparticles * grid->n1 * grid->n2 <= 174762 (SRS_ERR_RANGE beyond that, with a
 * message).  The caller still passes the trajectory and the output (DEVICE memory).  All calls share
 * the array and it keeps the last call's contents, so calls that overlap on the GPU (other streams,
 * other host threads) race: serialise them.  The first call on each device looks up the array's
 * device address (cudaGetSymbolAddress) with that device current; make that first call before any
 * stream capture.  Results equal srs_flux's to rounding (the partial sums may be split into fewer
 * trajectory chunks). */
srs_status srs_flux_mixed_noalloc(srs_traj_view traj, srs_beam_consts beam, const srs_grid2d *grid,
                                  double energy_ev, double *d_out, void *stream);

/* Power density at np points with unit normals (OSCARSSR.cc:1477-1598; the reference's CPU
 * semantics: with directional != 0 the terms with n.normal <= 0 are skipped, otherwise the result is
 * made non-negative).  d_points, d_normals: DEVICE 3*np doubles.  d_out: DEVICE nparticles*np values
 * in W/mm^2 (weight 1).  For SRS_PRECISION_MIXED a regular grid with one normal is best given as
 * `grid` (d_points/d_normals may then be NULL); with grid NULL any points with their own normals are
 * accepted (FP64 geometry per term, FP32 for the rest). */
srs_status srs_power_density(srs_traj_view traj, srs_beam_consts beam, const double *d_points,
                             const double *d_normals, int64_t np, const srs_grid2d *grid,
                             int32_t directional, int32_t precision, double *d_out, void *stream);

/* Host-buffer forms of the three sums for one particle, synchronous on the default stream: the
 * trajectory (x, beta, aoc: HOST SoA arrays of 3*n doubles, [component][point]), points, normals and
 * energies are HOST arrays, out (HOST) receives one value per output at weight 1.  These are what an
 * adapter for the reference's seam calls (include/OSCARSSR_Cuda.h:26-28 copy the particle's trajectory
 * and the surface to the device, sum, and copy back the same way).  Spectrum: precision as
 * srs_spectrum; flux and power density: plain FP64 on any point list. */
srs_status srs_spectrum_host(const double *x, const double *beta, int64_t n, double dt, srs_beam_consts beam,
                             const double obs[3], const double *energies, int64_t ne, int32_t precision,
                             double *out);
srs_status srs_flux_host(const double *x, const double *beta, int64_t n, double dt, srs_beam_consts beam,
                         const double *points, int64_t np, double energy_ev, double *out);
srs_status srs_power_density_host(const double *x, const double *beta, const double *aoc, int64_t n, double dt,
                                  srs_beam_consts beam, const double *points, const double *normals, int64_t np,
                                  int32_t directional, double *out);

/* Total radiated power of each particle (OSCARSSR.cc:1939-1978); gamma is per particle (HOST array).
 * out: HOST, nparticles values [W]. */
srs_status srs_total_power(srs_traj_view traj, srs_beam_consts beam, const double *gamma, double *out,
                           void *stream);

/* Deterministic weighted sum over particles: out[j] (HOST) += w * Kahan-accumulated values
 * d_vals[p*nout + j] in particle order, with the reference containers' compensation array comp
 * (HOST, nout), i.e. exactly the reference's per-particle AddToFlux/AddToPoint sequence. */
srs_status srs_accumulate(const double *d_vals, int32_t nparticles, int64_t nout, double weight,
                          double *out, double *comp, void *stream);

/* ------------------------------------------------------------------ derivatives
 * No counterpart in the reference (it has no derivatives): the hand-written adjoint of
 * flux_k = C2 (C0 w_k dt)^2 |E_k|^2 on a spectrum (OSCARSSR.cc:1154-1251) back through the RK4
 * trajectory (OSCARSSR.cc:562-874) to the field parameters and the initial conditions. */

/* srs_spectrum that also returns the sums E_k: d_e6 (DEVICE, nparticles*ne*6) receives Re/Im of
 * E_x, E_y, E_z of every output, before the final scaling.  d_flux as srs_spectrum's d_out. */
srs_status srs_spectrum_efield(srs_traj_view traj, srs_beam_consts beam, const double obs[3],
                               const double *d_energies, int64_t ne, int32_t precision, double *d_flux,
                               double *d_e6, void *stream);

/* Adjoint of the spectrum sum for one particle: given E_k (d_e6, from srs_spectrum_efield) and
 * d_gflux = dL/dflux_k (DEVICE, ne), writes dL/dx_i and dL/dbeta_i of every trajectory point to d_gx,
 * d_gbeta (DEVICE, 3*n each, layout as the trajectory).  FP64. */
srs_status srs_spectrum_adjoint(srs_traj_view traj, srs_beam_consts beam, const double obs[3],
                                const double *d_energies, int64_t ne, const double *d_e6,
                                const double *d_gflux, double *d_gx, double *d_gbeta, void *stream);

/* Adjoint of the RK4 trajectory of one particle (the same arguments as srs_trajectory, with the
 * trajectory it wrote in d_x, d_beta): given dL/dx_i, dL/dbeta_i (d_gx, d_gbeta), accumulates
 *   grid_grads[f] (HOST array of nfields DEVICE pointers, entries may be NULL; for grid fields:
 *       3*nsamples values, dL/d(sample), ADDED to what is there),
 *   amp_grad (HOST, 3*nfields, may be NULL; dL/d(field vector) of undulator, Gaussian and uniform
 *       fields, 0 for grids),
 *   ic_grad (HOST, 7): dL/dx0[3], dL/dbeta0[3], dL/d(q/(m gamma)).
 * At most 16 fields.  The recurrence lambda_j = g_j + J_j^T lambda_{j+1} is solved as a parallel
 * scan over the stored states (no serial sweep).  Synchronises the stream (host outputs). */
srs_status srs_trajectory_adjoint(const srs_field *fields, int32_t nfields, const srs_particle *particle,
                                  double ctstart, double ctstop, double t0, int64_t npoints,
                                  const double *d_x, const double *d_beta, const double *d_gx,
                                  const double *d_gbeta, double *const *grid_grads, double *amp_grad,
                                  double *ic_grad, void *stream);

/* ------------------------------------------------------------------ heterogeneous work queue
 * No counterpart in the reference (which runs one calculation per call, each with its own launch
 * and host synchronisation, OSCARSSR.cc:1154-1251 and 1989-2099): a set of mixed-precision flux and
 * spectrum jobs of different sizes, each with its own trajectory, run as ONE persistent launch.
 * The jobs are cut into (tile, trajectory chunk) work items, ordered longest first; resident CTAs
 * take items from an atomic ticket.  srs_queue_run replays a CUDA graph captured on its first call
 * (ticket reset, queue kernel, chunk-order reduction).  Results equal srs_spectrum / srs_flux
 * (SRS_PRECISION_MIXED, one particle) to rounding of the per-chunk partial sums. */
enum { SRS_JOB_FLUX = 0, SRS_JOB_SPECTRUM = 1 };

typedef struct srs_job {
  int32_t kind;          /* SRS_JOB_FLUX or SRS_JOB_SPECTRUM */
  srs_traj_view traj;    /* one particle (nparticles is ignored); DEVICE arrays */
  srs_beam_consts beam;
  srs_grid2d grid;       /* flux: the observation grid */
  double energy_ev;      /* flux: photon energy */
  double obs[3];         /* spectrum: observer */
  const double *d_energies; /* spectrum: DEVICE, ne photon energies [eV], read at srs_queue_create */
  int64_t ne;
  double *d_out;         /* DEVICE: n1*n2 (flux) or ne (spectrum) values, weight 1 */
} srs_job;

typedef struct srs_queue srs_queue;

/* Plan the jobs: chunk = trajectory points per work item (>= 128), ctas_per_sm = resident CTAs per
 * SM of the persistent grid (0: as many as fit).  The trajectories and outputs must stay valid and
 * at the same addresses for the queue's lifetime.  Synchronises the device (it reads the
 * spectrum jobs' energies once). */
srs_status srs_queue_create(srs_queue **out, const srs_job *jobs, int32_t njobs, int32_t chunk,
                            int32_t ctas_per_sm);

/* The tile shape of a queue's work items (the autotuner's search space). */
typedef struct srs_queue_shape {
  int32_t chunk;               /* trajectory points per work item (>= 128; rounded up to 128s) */
  int32_t ctas_per_sm;         /* resident CTAs per SM of the persistent grid (0: as many as fit) */
  int32_t energies_per_thread; /* spectrum items: 2 or 4 energies per thread (0: 4) */
  int32_t strip_width;         /* flux items: widest strip of grid points in a tile, 8..16 (0: 16) */
  int32_t groups;              /* with trajectories: groups of jobs by trajectory length (0: 16) */
  int32_t steps_per_segment;   /* with trajectories: RK4 steps per segment of the parallel-in-time
                                  integrations (0: 16; longer segments use less shared memory, so more
                                  integrations run side by side) */
} srs_queue_shape;

/* srs_queue_create with a tile shape and, optionally, the jobs' trajectories integrated inside the
 * queue's graph (no counterpart in the reference, whose calls each integrate and sum one particle).
 * particles == NULL: the jobs' trajectories are given, as for srs_queue_create.  Otherwise particle j
 * (HOST array of njobs) is integrated through the HOST field list (the same fields for every job, at
 * most 16) with ctstart[j], ctstop[j], t0[j], npoints[j] (as srs_trajectory) into job j's trajectory
 * view -- its x, beta and aoc arrays must hold exactly that many points -- by every srs_queue_run:
 * the jobs are split into `groups` groups by trajectory length, and each group is one branch of the
 * graph: its trajectories integrated parallel in time (as srs_trajectory_shoot: within ~1e-15 m of the
 * serial RK4, magnetic fields only), then its work items, so the sums of some groups overlap the
 * integration of the others. */
srs_status srs_queue_create_shaped(srs_queue **out, const srs_job *jobs, int32_t njobs, const srs_queue_shape *shape,
                                   const srs_field *fields, int32_t nfields, const srs_particle *particles,
                                   const double *ctstart, const double *ctstop, const double *t0,
                                   const int64_t *npoints);
/* Run every job once, ordered after the work already queued on stream; later work on stream waits
 * for the results. */
srs_status srs_queue_run(srs_queue *q, void *stream);
/* Work items, field evaluations (points x trajectory points) per run, scratch bytes, CTAs. */
srs_status srs_queue_info(srs_queue *q, int64_t *nitems, double *evals, size_t *scratch_bytes,
                          int32_t *grid);
void srs_queue_destroy(srs_queue *q);

/* RK4 trajectories of nparticles particles with per-particle ctstart/ctstop/t0/npoints (HOST
 * arrays) in one launch, each written to its own DEVICE arrays d_x[p], d_beta[p], d_aoc[p] (3*n_p
 * doubles each, layout as srs_trajectory).  Same arithmetic as srs_trajectory. */
srs_status srs_trajectory_batch(const srs_field *fields, int32_t nfields, const srs_particle *particles,
                                int32_t nparticles, const double *ctstart, const double *ctstop,
                                const double *t0, const int64_t *npoints, double *const *d_x,
                                double *const *d_beta, double *const *d_aoc, void *stream);

/* ------------------------------------------------------------------ simulation object
 * The state and calls behind the reference's Python type oscars.sr.sr (src/OSCARSSR_Python.cc),
 * for the hot-path methods.  One object per thread; calls on one object are serialised. */
typedef struct srs_sim srs_sim;

srs_status srs_sim_create(srs_sim **out);
void srs_sim_destroy(srs_sim *sim);

srs_status srs_sim_set_ctstartstop(srs_sim *sim, double start, double stop);       /* :282 */
srs_status srs_sim_set_npoints_trajectory(srs_sim *sim, int64_t n);                 /* :315 */
srs_status srs_sim_get_ctstartstop(srs_sim *sim, double *start, double *stop);
int64_t srs_sim_get_npoints_trajectory(srs_sim *sim);
srs_status srs_sim_set_nthreads_global(srs_sim *sim, int32_t n);                    /* :239 */
srs_status srs_sim_set_gpu_global(srs_sim *sim, int32_t g);                         /* :200 */

/* Fields (:736 undulator, :561 gaussian, :640 uniform, :337 file).  Vectors are 3 doubles. */
srs_status srs_sim_add_bfield_undulator(srs_sim *sim, const double bfield[3], const double period[3],
                                        int32_t nperiods, double phase, const double rotations[3],
                                        const double translation[3], double taper);
srs_status srs_sim_add_bfield_gaussian(srs_sim *sim, const double bfield[3], const double sigma[3],
                                       const double rotations[3], const double translation[3]);
srs_status srs_sim_add_bfield_uniform(srs_sim *sim, const double bfield[3], const double width[3],
                                      const double rotations[3], const double translation[3]);
/* Field map file (OSCARSSR::AddMagneticField, OSCARSSR.cc:68-90; TField3D_Grid.cc:25-45) in one of
 * the reference's formats (case-insensitive): "OSCARS" (regular grid; scale[0..2] step scaling,
 * [3..5] field scaling), "OSCARS1D <columns>" (irregular samples along one axis, columns named
 * X|Y|Z and Bx|By|Bz (or Ex.., Fx..) in file order, scale factors per column, regridded at 10000
 * points per metre), "SRW" or "SPECTRA" (no scaling).  nscale may be 0. */
srs_status srs_sim_add_bfield_file(srs_sim *sim, const char *path, const char *format,
                                   const double rotations[3], const double translation[3],
                                   const double *scale, int32_t nscale);
/* Field map interpolated between OSCARS-format files (add_bfield_interpolated,
 * OSCARSSR_Python.cc:419-510; TField3D_Grid.cc:1150-1420): nmap pairs (parameter, path), identical
 * headers, the map at `parameter` by linear interpolation between the two files around it.  At
 * exactly the smallest mapping parameter the reference's result is NaN, reproduced. */
srs_status srs_sim_add_bfield_interpolated(srs_sim *sim, const double *parameters, const char *const *paths,
                                           int32_t nmap, const char *format, double parameter,
                                           const double rotations[3], const double translation[3],
                                           const double *scale, int32_t nscale);
/* The same readers without a simulation object (host only, no GPU): the grid descriptor (its data
 * pointer NULL) and the rotated samples, 3 doubles each, into data when *ndata is large enough;
 * *ndata returns the number of doubles.  No reference counterpart (the reference reads inside
 * add_bfield_file / add_bfield_interpolated). */
srs_status srs_read_field_file(const char *path, const char *format, const double rotations[3],
                               const double translation[3], const double *scale, int32_t nscale, srs_field *out,
                               double *data, int64_t *ndata);
srs_status srs_read_field_interpolated(const double *parameters, const char *const *paths, int32_t nmap,
                                       const char *format, double parameter, const double rotations[3],
                                       const double translation[3], const double *scale, int32_t nscale,
                                       srs_field *out, double *data, int64_t *ndata);
/* Field map given as arrays (same meaning as the file's header and body). */
srs_status srs_sim_add_bfield_grid(srs_sim *sim, const double start[3], const double step[3],
                                   const int64_t n[3], const double *data, const double rotations[3],
                                   const double translation[3]);
/* Remove the magnetic fields (OSCARSSR::ClearMagneticFields); the electric fields stay. */
srs_status srs_sim_clear_bfields(srs_sim *sim);
/* Electric fields [V/m] (OSCARSSR_Python.cc:876-1390): the same shapes and arguments as the magnetic
 * ones (the undulator without taper, the file without scaling); they enter the RK4 as
 * q/(m gamma) E (DerivativesE / DerivativesEB, OSCARSSR.cc:690-793).  Trajectories with electric
 * fields are always integrated serially. */
srs_status srs_sim_add_efield_undulator(srs_sim *sim, const double efield[3], const double period[3],
                                        int32_t nperiods, double phase, const double rotations[3],
                                        const double translation[3]);
srs_status srs_sim_add_efield_gaussian(srs_sim *sim, const double efield[3], const double sigma[3],
                                       const double rotations[3], const double translation[3]);
srs_status srs_sim_add_efield_uniform(srs_sim *sim, const double efield[3], const double width[3],
                                      const double rotations[3], const double translation[3]);
srs_status srs_sim_add_efield_file(srs_sim *sim, const char *path, const char *format,
                                   const double rotations[3], const double translation[3]);
srs_status srs_sim_clear_efields(srs_sim *sim);
/* Electric field at points (device evaluation), HOST arrays of 3*np doubles. */
srs_status srs_sim_get_efield(srs_sim *sim, const double *xyz, int64_t np, double *out);
/* The time-domain electric field of the current particle at obs
 * (OSCARSSR::CalculateElectricFieldTimeDomain, OSCARSSR.cc:2646-2690): for every trajectory point, in
 * time order, the arrival time t [s] (HOST, *n doubles) and the field [V/m] (HOST, 3 * *n doubles).
 * With t or e NULL, *n returns the number of points. */
srs_status srs_sim_calculate_efield_time(srs_sim *sim, const double obs[3], double *t, double *e, int64_t *n);
/* The object keeps the device trajectory of its last single-particle calculation and reuses it
 * while the particle, the fields and the trajectory settings are unchanged (the reference recomputes
 * the identical trajectory on every call).  enabled = 0 turns this off; every call drops the kept
 * trajectory.  No counterpart in the reference. */
srs_status srs_sim_set_trajectory_cache(srs_sim *sim, int32_t enabled);
/* How the object integrates single-particle trajectories: SRS_TRAJ_AUTO (default) parallel in time
 * (srs_trajectory_shoot) for the mixed-precision sums and serially (srs_trajectory, the reference's
 * roundings) for everything else; SRS_TRAJ_SERIAL always serially; SRS_TRAJ_PARALLEL always parallel
 * in time.  Trajectories shorter than 1024 points and multi-particle batches are always serial.
 * No counterpart in the reference. */
enum { SRS_TRAJ_AUTO = 0, SRS_TRAJ_SERIAL = 1, SRS_TRAJ_PARALLEL = 2 };
srs_status srs_sim_set_trajectory_mode(srs_sim *sim, int32_t mode);
int32_t srs_sim_get_nfields(srs_sim *sim);
/* Field at points (evaluated on the device): xyz and out are HOST arrays of 3*np doubles. */
srs_status srs_sim_get_bfield(srs_sim *sim, const double *xyz, int64_t np, double *out);
/* Replace field k's grid samples (DEVICE or HOST pointer, 3*nsamples doubles): used by the adjoint. */
srs_status srs_sim_set_field_grid_data(srs_sim *sim, int32_t k, const double *data, int32_t on_device);

/* Particle beams (:1661 add_particle_beam; set_particle_beam = clear + add + ideal particle).
 * hdir/beta/emittance may be NULL (not given); type "custom" uses mass [kg] and charge [C]. */
typedef struct srs_beam_args {
  const char *type;
  const char *name;
  double energy_gev;
  double d0[3];
  double x0[3];
  double sigma_energy_gev;
  double t0;
  double current;
  double weight;
  double rotations[3];
  double translation[3];
  const double *horizontal_direction; /* 3 or NULL */
  const double *beta;                 /* 2 or NULL */
  const double *emittance;            /* 2 or NULL */
  double lattice_reference[3];
  double mass;
  double charge;
} srs_beam_args;
srs_status srs_sim_add_particle_beam(srs_sim *sim, const srs_beam_args *args);
srs_status srs_sim_clear_particle_beams(srs_sim *sim);
int32_t srs_sim_get_nparticle_beams(srs_sim *sim);
/* beam "" = chosen by weight; which "ideal", "random" or "" (random). */
srs_status srs_sim_set_new_particle(srs_sim *sim, const char *beam, const char *which);
/* Current particle: x0, beta0, E0 [GeV], gamma, q/(m gamma), t0, q, current. */
srs_status srs_sim_get_particle(srs_sim *sim, double x0[3], double beta0[3], double *e0, double *gamma);

/* Process-wide generator (TRandomA: std::mt19937 + std::normal_distribution<double>). */
void srs_set_seed(double seed);
double srs_random_uniform(void);
double srs_random_normal(void);
/* Reseed AND forget the normal distribution's cached value: the generator state of a freshly
 * started process after set_seed(seed).  (srs_set_seed, like the reference's set_seed, keeps it.) */
void srs_random_reset(double seed);

/* Trajectory of the current particle: first call with x == NULL returns n; then x and beta (HOST,
 * 3*n doubles each, point-major x,y,z) are filled (OSCARSSR_Python.cc:1988-2037). */
srs_status srs_sim_calculate_trajectory(srs_sim *sim, int64_t *n, double *x, double *beta);

/* The sums for the current particle (nparticles == 0) or nparticles sampled particles with weight
 * 1/nparticles; results are Kahan-added into out/comp (HOST, length nout), as the reference's
 * containers.  comp == NULL: the sums start from zero and are written to out (its contents are not
 * read), and the compensation stays on the device.  For the power density, weighted != 0 applies the
 * weight (the reference's GPU path) and 0 does not (its CPU paths). */
srs_status srs_sim_calculate_spectrum(srs_sim *sim, const double obs[3], const double *energies,
                                      int64_t ne, int32_t nparticles, int32_t precision, double *out,
                                      double *comp);
srs_status srs_sim_calculate_flux(srs_sim *sim, const double *points, int64_t np,
                                  const srs_grid2d *grid, double energy_ev, int32_t nparticles,
                                  int32_t precision, double *out, double *comp);
/* The flux on a rectangle given as srs_rectangle_plane takes it (calculate_flux_rectangle with
 * plane and width, OSCARSSR_Python.cc:3009-3233), in one call: out, comp as srs_sim_calculate_flux;
 * xyz (3*n1*n2), x12 (2*n1*n2) and nrm receive the surface (each may be NULL).  With
 * SRS_PRECISION_MIXED the sums walk the grid and the points are written while the GPU computes;
 * otherwise they are built first and uploaded.  rotations / translation NULL: zero. */
srs_status srs_sim_calculate_flux_plane(srs_sim *sim, const char *plane, int32_t n1, int32_t n2, double w1,
                                        double w2, const double rotations[3], const double translation[3],
                                        int32_t normal, double energy_ev, int32_t nparticles, int32_t precision,
                                        double *out, double *comp, double *xyz, double *x12, double nrm[3]);
srs_status srs_sim_calculate_power_density(srs_sim *sim, const double *points, const double *normals,
                                           int64_t np, const srs_grid2d *grid, int32_t directional,
                                           int32_t nparticles, int32_t weighted, int32_t precision,
                                           double *out, double *comp);
srs_status srs_sim_calculate_total_power(srs_sim *sim, double *out);

/* ------------------------------------------------------------------ measurement */

/* Instruction throughput of one pipe of the current device, all SMs, from a timed launch of
 * independent dependency chains: kind 0 = FP32 FFMA, 1 = FP64 DFMA, 2 = SFU sine (MUFU).
 * ops_per_s receives instructions per second (an FMA counts as one).  Used as roofline denominators
 * for the compute-bound sums.  No counterpart in the reference. */
srs_status srs_measure_peak(int32_t kind, double *ops_per_s, void *stream);

/* ------------------------------------------------------------------ host-side geometry */

/* Spectrum energy grid (TSpectrumContainer::Init, TSpectrumContainer.cc:55-86): e0 + (e1-e0)/(n-1)*(i+1). */
srs_status srs_energy_grid(int64_t n, double e0, double e1, double *out);

/* Rectangle surfaces (TSurfacePoints_Rectangle.cc).  xyz: 3*n1*n2, x12: 2*n1*n2 (GetX1/GetX2),
 * normal: the unit normal, grid: the same points as a regular grid (for SRS_PRECISION_MIXED). */
srs_status srs_rectangle_plane(const char *plane, int32_t n1, int32_t n2, double w1, double w2,
                               const double rotations[3], const double translation[3], int32_t normal,
                               double *xyz, double *x12, double nrm[3], srs_grid2d *grid);
srs_status srs_rectangle_points(int32_t n1, int32_t n2, const double x0[3], const double x1[3],
                                const double x2[3], const double rotations[3],
                                const double translation[3], int32_t normal, double *xyz, double *x12,
                                double nrm[3], srs_grid2d *grid);

#ifdef __cplusplus
}
#endif
#endif

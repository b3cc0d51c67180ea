// C ABI of the kernels (include/srs_b200.h): argument checks, stream-ordered scratch, dispatch.
#include <cuda_runtime.h>

#include <mutex>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {

static thread_local std::string g_error;

void set_error(const std::string &msg) { g_error = msg; }
void clear_error() { g_error.clear(); }
srs_status fail(srs_status code, const std::string &msg) {
  g_error = msg;
  return code;
}
srs_status cuda_fail(cudaError_t e, const char *what) {
  g_error = std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e);
  return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? SRS_ERR_NO_DEVICE : SRS_ERR_CUDA;
}

cudaError_t library_pool(cudaMemPool_t *pool) {
  static std::mutex mu;
  static cudaMemPool_t pools[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    e = cudaMemPoolCreate(&p, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = ~0ull;  // keep freed blocks for reuse until srs_trim_memory
    e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    pools[dev] = p;
  }
  *pool = pools[dev];
  return cudaSuccess;
}

static srs_status check_view(const srs_traj_view &t, bool need_aoc) {
  if (!t.x || !t.beta || (need_aoc && !t.aoc)) return fail(SRS_ERR_INVALID, "trajectory pointers are NULL");
  if (t.n < 1) return fail(SRS_ERR_RANGE, "no points in trajectory.  Is particle or beam defined?");
  if (t.nparticles < 1) return fail(SRS_ERR_INVALID, "nparticles must be >= 1");
  if (!(t.dt > 0) || !std::isfinite(t.dt)) return fail(SRS_ERR_INVALID, "trajectory time step must be > 0");
  return SRS_OK;
}

}  // namespace srs

using namespace srs;

extern "C" {

const char *srs_last_error(void) { return g_error.c_str(); }
const char *srs_version(void) { return "srs_b200 1.0.0 (sm_100a)"; }

srs_status srs_trim_memory(void) {
  clear_error();
  cudaMemPool_t pool;
  SRS_CUDA(library_pool(&pool));
  SRS_CUDA(cudaMemPoolTrimTo(pool, 0));
  return SRS_OK;
}

int srs_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

srs_status srs_trajectory_counts(double ctstart, double ctstop, double t0, int64_t npoints, double *dt,
                                 int64_t *nforward, int64_t *nbackward) {
  clear_error();
  if (ctstart > t0) return fail(SRS_ERR_RANGE, "start time is greater than T0");
  if (ctstart >= ctstop)
    return fail(SRS_ERR_RANGE, "start time is greater than stop time.  check that set_ctstartstop is set");
  if (npoints < 2) return fail(SRS_ERR_RANGE, "npoints_trajectory must be >= 2");
  // OSCARSSR.cc:592-598, same expressions (size_t truncation included)
  const double DeltaT = ((ctstop - ctstart) / kC / (double)(size_t)(npoints - 1));
  const double f = 1 + (ctstop - t0) / kC / DeltaT;
  const double b = (t0 - ctstart) / kC / DeltaT;
  if (!(f >= 0) || !(b >= 0) || f > 4e9 || b > 4e9) return fail(SRS_ERR_RANGE, "trajectory point count out of range");
  if (dt) *dt = DeltaT;
  if (nforward) *nforward = (int64_t)(size_t)f;
  if (nbackward) *nbackward = (int64_t)(size_t)b;
  return SRS_OK;
}

srs_status srs_trajectory(const srs_field *fields, int32_t nfields, const srs_particle *particles,
                          int32_t nparticles, double ctstart, double ctstop, double t0, int64_t npoints,
                          double *d_x, double *d_beta, double *d_aoc, void *stream) {
  clear_error();
  double dt;
  int64_t nf, nb;
  srs_status st = srs_trajectory_counts(ctstart, ctstop, t0, npoints, &dt, &nf, &nb);
  if (st) return st;
  if (nfields < 0 || (nfields > 0 && !fields)) return fail(SRS_ERR_INVALID, "bad field array");
  if (nparticles < 1 || !particles) return fail(SRS_ERR_INVALID, "bad particle array");
  if (!d_x || !d_beta || !d_aoc) return fail(SRS_ERR_INVALID, "output pointers are NULL");
  for (int i = 0; i < nfields; ++i)
    if (field_shape(fields[i].kind) == SRS_FIELD_GRID && !fields[i].data)
      return fail(SRS_ERR_INVALID, "grid field without data");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer df, dp;
  SRS_CUDA(df.alloc(sizeof(srs_field) * (nfields > 0 ? nfields : 1), s));
  SRS_CUDA(dp.alloc(sizeof(srs_particle) * nparticles, s));
  if (nfields > 0) SRS_CUDA(cudaMemcpyAsync(df.ptr, fields, sizeof(srs_field) * nfields, cudaMemcpyHostToDevice, s));
  SRS_CUDA(cudaMemcpyAsync(dp.ptr, particles, sizeof(srs_particle) * nparticles, cudaMemcpyHostToDevice, s));
  SRS_CUDA(launch_rk4(df.as<srs_field>(), nfields, dp.as<srs_particle>(), nparticles, dt, nf, nb, d_x, d_beta, d_aoc, s,
                      nfields > 0 ? grid_stage_doubles(fields, nfields) : 0, has_electric(fields, nfields)));
  return SRS_OK;
}

srs_status srs_trajectory_shoot(const srs_field *fields, int32_t nfields, const srs_particle *particle,
                                double ctstart, double ctstop, double t0, int64_t npoints,
                                int32_t steps_per_segment, int32_t max_iterations, double *d_x, double *d_beta,
                                double *d_aoc, double *d_stats, void *stream) {
  clear_error();
  double dt;
  int64_t nf, nb;
  srs_status st = srs_trajectory_counts(ctstart, ctstop, t0, npoints, &dt, &nf, &nb);
  if (st) return st;
  if (nfields < 0 || (nfields > 0 && !fields)) return fail(SRS_ERR_INVALID, "bad field array");
  if (!particle) return fail(SRS_ERR_INVALID, "bad particle");
  if (!d_x || !d_beta || !d_aoc) return fail(SRS_ERR_INVALID, "output pointers are NULL");
  if (steps_per_segment < 0) return fail(SRS_ERR_INVALID, "steps_per_segment must be >= 0");
  if (max_iterations < 0 || max_iterations > 32) return fail(SRS_ERR_INVALID, "max_iterations must be in [0, 32]");
  for (int i = 0; i < nfields; ++i)
    if (field_shape(fields[i].kind) == SRS_FIELD_GRID && !fields[i].data)
      return fail(SRS_ERR_INVALID, "grid field without data");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer df, dp, scratch;
  SRS_CUDA(df.alloc(sizeof(srs_field) * (nfields > 0 ? nfields : 1), s));
  SRS_CUDA(dp.alloc(sizeof(srs_particle), s));
  SRS_CUDA(scratch.alloc(shoot_scratch_bytes(nf, nb, steps_per_segment, nfields), s));
  if (nfields > 0) SRS_CUDA(cudaMemcpyAsync(df.ptr, fields, sizeof(srs_field) * nfields, cudaMemcpyHostToDevice, s));
  SRS_CUDA(cudaMemcpyAsync(dp.ptr, particle, sizeof(srs_particle), cudaMemcpyHostToDevice, s));
  if (has_electric(fields, nfields)) {  // electric fields: the serial kernel (its statistics say 0 iterations)
    SRS_CUDA(launch_rk4(df.as<srs_field>(), nfields, dp.as<srs_particle>(), 1, dt, nf, nb, d_x, d_beta, d_aoc, s,
                        grid_stage_doubles(fields, nfields), true));
    if (d_stats) SRS_CUDA(cudaMemsetAsync(d_stats, 0, sizeof(double) * 4, s));
    return SRS_OK;
  }
  SRS_CUDA(launch_rk4_shoot(df.as<srs_field>(), nfields, dp.as<srs_particle>(), *particle, dt, nf, nb, d_x, d_beta,
                            d_aoc, s, nfields > 0 ? grid_stage_doubles(fields, nfields) : 0, steps_per_segment,
                            max_iterations, scratch.ptr, d_stats));
  return SRS_OK;
}

srs_status srs_spectrum(srs_traj_view traj, srs_beam_consts beam, const double obs[3], const double *d_energies,
                        int64_t ne, int32_t precision, double *d_out, void *stream) {
  clear_error();
  if (srs_status st = check_view(traj, false)) return st;
  if (!obs || !d_out || (ne > 0 && !d_energies)) return fail(SRS_ERR_INVALID, "NULL argument");
  if (ne < 1) return fail(SRS_ERR_INVALID, "'npoints' must be > 0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer scratch;
  if (precision == SRS_PRECISION_FP64) {
    SRS_CUDA(scratch.alloc(fp64_spectrum_scratch_bytes(traj.n, ne, traj.nparticles), s));
    SRS_CUDA(fp64_spectrum(traj, beam, obs, d_energies, ne, d_out, scratch.ptr, s));
  } else if (precision == SRS_PRECISION_MIXED) {
    SRS_CUDA(scratch.alloc(mixed_spectrum_scratch_bytes(traj.n, ne, traj.nparticles), s));
    SRS_CUDA(mixed_spectrum(traj, beam, obs, d_energies, ne, d_out, scratch.ptr, s));
  } else {
    return fail(SRS_ERR_INVALID, "unknown precision");
  }
  return SRS_OK;
}

srs_status srs_flux(srs_traj_view traj, srs_beam_consts beam, const double *d_points, int64_t np,
                    const srs_grid2d *grid, double energy_ev, int32_t precision, double *d_out, void *stream) {
  clear_error();
  if (srs_status st = check_view(traj, false)) return st;
  if (!d_out) return fail(SRS_ERR_INVALID, "NULL output");
  if (np < 1) return fail(SRS_ERR_INVALID, "no observation points");
  if (!(energy_ev > 0)) return fail(SRS_ERR_INVALID, "energy_eV must be > 0");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer scratch;
  if (precision == SRS_PRECISION_FP64) {
    if (!d_points) return fail(SRS_ERR_INVALID, "NULL points");
    SRS_CUDA(scratch.alloc(fp64_flux_scratch_bytes(traj.n, np, traj.nparticles), s));
    SRS_CUDA(fp64_flux(traj, beam, d_points, np, energy_ev, d_out, scratch.ptr, s));
  } else if (precision == SRS_PRECISION_MIXED) {
    if (grid) {  // a regular grid: the tiles anchor on it
      if ((int64_t)grid->n1 * grid->n2 != np || grid->n1 < 1 || grid->n2 < 1)
        return fail(SRS_ERR_INVALID, "grid size does not match the number of points");
      SRS_CUDA(scratch.alloc(mixed_flux_scratch_bytes(traj.n, *grid, traj.nparticles), s));
      SRS_CUDA(mixed_flux(traj, beam, *grid, energy_ev, d_out, scratch.ptr, s));
    } else {  // any list of points
      if (!d_points) return fail(SRS_ERR_INVALID, "NULL points");
      SRS_CUDA(scratch.alloc(mixed_flux_points_scratch_bytes(traj.n, np, traj.nparticles), s));
      SRS_CUDA(mixed_flux_points(traj, beam, d_points, np, energy_ev, d_out, scratch.ptr, s));
    }
  } else {
    return fail(SRS_ERR_INVALID, "unknown precision");
  }
  return SRS_OK;
}

srs_status srs_power_density(srs_traj_view traj, srs_beam_consts beam, const double *d_points,
                             const double *d_normals, int64_t np, const srs_grid2d *grid, int32_t directional,
                             int32_t precision, double *d_out, void *stream) {
  clear_error();
  if (srs_status st = check_view(traj, true)) return st;
  if (!d_out) return fail(SRS_ERR_INVALID, "NULL output");
  if (np < 1) return fail(SRS_ERR_INVALID, "no observation points");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer scratch;
  if (precision == SRS_PRECISION_FP64) {
    if (!d_points || !d_normals) return fail(SRS_ERR_INVALID, "NULL points or normals");
    SRS_CUDA(scratch.alloc(fp64_pd_scratch_bytes(traj.n, np, traj.nparticles), s));
    SRS_CUDA(fp64_power_density(traj, beam, d_points, d_normals, np, directional, d_out, scratch.ptr, s));
  } else if (precision == SRS_PRECISION_MIXED) {
    if (grid) {  // a regular grid (one normal): the tiles anchor on it
      if ((int64_t)grid->n1 * grid->n2 != np || grid->n1 < 1 || grid->n2 < 1)
        return fail(SRS_ERR_INVALID, "grid size does not match the number of points");
      SRS_CUDA(scratch.alloc(mixed_pd_scratch_bytes(traj.n, *grid, traj.nparticles), s));
      SRS_CUDA(mixed_power_density(traj, beam, *grid, directional, d_out, scratch.ptr, s));
    } else {  // any points, each with its own normal
      if (!d_points || !d_normals) return fail(SRS_ERR_INVALID, "NULL points or normals");
      SRS_CUDA(scratch.alloc(mixed_pd_points_scratch_bytes(traj.n, np, traj.nparticles), s));
      SRS_CUDA(mixed_power_density_points(traj, beam, d_points, d_normals, np, directional, d_out, scratch.ptr, s));
    }
  } else {
    return fail(SRS_ERR_INVALID, "unknown precision");
  }
  return SRS_OK;
}

// ---- host-buffer forms: what the reference's GPU seam does per call (copy in, sum, copy out) ----

namespace {
// Uploads a one-particle trajectory given as HOST SoA arrays (3*n each; aoc may be NULL).
struct HostTraj {
  DeviceBuffer buf;
  srs_traj_view view{};
  srs_status up(const double *x, const double *beta, const double *aoc, int64_t n, double dt, cudaStream_t s) {
    if (!x || !beta || n < 1) return fail(SRS_ERR_INVALID, "bad trajectory");
    const size_t arr = sizeof(double) * 3 * (size_t)n;
    SRS_CUDA(buf.alloc(arr * (aoc ? 3 : 2), s));
    double *d = buf.as<double>();
    SRS_CUDA(cudaMemcpyAsync(d, x, arr, cudaMemcpyHostToDevice, s));
    SRS_CUDA(cudaMemcpyAsync(d + 3 * n, beta, arr, cudaMemcpyHostToDevice, s));
    if (aoc) SRS_CUDA(cudaMemcpyAsync(d + 6 * n, aoc, arr, cudaMemcpyHostToDevice, s));
    view = srs_traj_view{d, d + 3 * n, aoc ? d + 6 * n : nullptr, n, 1, dt};
    return SRS_OK;
  }
};
srs_status upload(DeviceBuffer &b, const double *h, size_t count, cudaStream_t s) {
  SRS_CUDA(b.alloc(sizeof(double) * std::max<size_t>(1, count), s));
  if (count) SRS_CUDA(cudaMemcpyAsync(b.ptr, h, sizeof(double) * count, cudaMemcpyHostToDevice, s));
  return SRS_OK;
}
srs_status download(double *h, const DeviceBuffer &b, size_t count, cudaStream_t s) {
  SRS_CUDA(cudaMemcpyAsync(h, b.ptr, sizeof(double) * count, cudaMemcpyDeviceToHost, s));
  SRS_CUDA(cudaStreamSynchronize(s));
  return SRS_OK;
}
}  // namespace

srs_status srs_spectrum_host(const double *x, const double *beta, int64_t n, double dt, srs_beam_consts beam,
                             const double obs[3], const double *energies, int64_t ne, int32_t precision,
                             double *out) {
  clear_error();
  if (!energies || !out || !obs || ne < 1) return fail(SRS_ERR_INVALID, "bad argument");
  cudaStream_t s = nullptr;
  HostTraj t;
  DeviceBuffer de, dout;
  if (srs_status st = t.up(x, beta, nullptr, n, dt, s)) return st;
  if (srs_status st = upload(de, energies, ne, s)) return st;
  SRS_CUDA(dout.alloc(sizeof(double) * ne, s));
  if (srs_status st = srs_spectrum(t.view, beam, obs, de.as<double>(), ne, precision, dout.as<double>(), s)) return st;
  return download(out, dout, ne, s);
}

srs_status srs_flux_host(const double *x, const double *beta, int64_t n, double dt, srs_beam_consts beam,
                         const double *points, int64_t np, double energy_ev, double *out) {
  clear_error();
  if (!points || !out || np < 1) return fail(SRS_ERR_INVALID, "bad argument");
  cudaStream_t s = nullptr;
  HostTraj t;
  DeviceBuffer dp, dout;
  if (srs_status st = t.up(x, beta, nullptr, n, dt, s)) return st;
  if (srs_status st = upload(dp, points, 3 * np, s)) return st;
  SRS_CUDA(dout.alloc(sizeof(double) * np, s));
  if (srs_status st = srs_flux(t.view, beam, dp.as<double>(), np, nullptr, energy_ev, SRS_PRECISION_FP64,
                               dout.as<double>(), s))
    return st;
  return download(out, dout, np, s);
}

srs_status srs_power_density_host(const double *x, const double *beta, const double *aoc, int64_t n, double dt,
                                  srs_beam_consts beam, const double *points, const double *normals, int64_t np,
                                  int32_t directional, double *out) {
  clear_error();
  if (!points || !normals || !out || !aoc || np < 1) return fail(SRS_ERR_INVALID, "bad argument");
  cudaStream_t s = nullptr;
  HostTraj t;
  DeviceBuffer dp, dn, dout;
  if (srs_status st = t.up(x, beta, aoc, n, dt, s)) return st;
  if (srs_status st = upload(dp, points, 3 * np, s)) return st;
  if (srs_status st = upload(dn, normals, 3 * np, s)) return st;
  SRS_CUDA(dout.alloc(sizeof(double) * np, s));
  if (srs_status st = srs_power_density(t.view, beam, dp.as<double>(), dn.as<double>(), np, nullptr, directional,
                                        SRS_PRECISION_FP64, dout.as<double>(), s))
    return st;
  return download(out, dout, np, s);
}

srs_status srs_total_power(srs_traj_view traj, srs_beam_consts beam, const double *gamma, double *out, void *stream) {
  clear_error();
  if (srs_status st = check_view(traj, true)) return st;
  if (!gamma || !out) return fail(SRS_ERR_INVALID, "NULL argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer dg, dout;
  SRS_CUDA(dg.alloc(sizeof(double) * traj.nparticles, s));
  SRS_CUDA(dout.alloc(sizeof(double) * traj.nparticles, s));
  SRS_CUDA(cudaMemcpyAsync(dg.ptr, gamma, sizeof(double) * traj.nparticles, cudaMemcpyHostToDevice, s));
  SRS_CUDA(total_power(traj, beam, dg.as<double>(), dout.as<double>(), s));
  SRS_CUDA(cudaMemcpyAsync(out, dout.ptr, sizeof(double) * traj.nparticles, cudaMemcpyDeviceToHost, s));
  SRS_CUDA(cudaStreamSynchronize(s));
  return SRS_OK;
}

srs_status srs_accumulate(const double *d_vals, int32_t nparticles, int64_t nout, double weight, double *out,
                          double *comp, void *stream) {
  clear_error();
  if (!d_vals || !out || !comp || nparticles < 1 || nout < 0) return fail(SRS_ERR_INVALID, "bad argument");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer dout;
  SRS_CUDA(dout.alloc(sizeof(double) * 2 * nout, s));
  double *o = dout.as<double>(), *c = o + nout;
  SRS_CUDA(cudaMemcpyAsync(o, out, sizeof(double) * nout, cudaMemcpyHostToDevice, s));
  SRS_CUDA(cudaMemcpyAsync(c, comp, sizeof(double) * nout, cudaMemcpyHostToDevice, s));
  SRS_CUDA(accumulate_particles(d_vals, nparticles, nout, weight, o, c, s));
  SRS_CUDA(cudaMemcpyAsync(out, o, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
  SRS_CUDA(cudaMemcpyAsync(comp, c, sizeof(double) * nout, cudaMemcpyDeviceToHost, s));
  SRS_CUDA(cudaStreamSynchronize(s));
  return SRS_OK;
}

}  // extern "C"

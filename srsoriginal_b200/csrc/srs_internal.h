// Internal declarations shared by the library's translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "../../include/srs_b200.h"

namespace srs {

// ---- error reporting: a thread-local message behind srs_last_error() ----
void set_error(const std::string &msg);
void clear_error();
srs_status fail(srs_status code, const std::string &msg);
srs_status cuda_fail(cudaError_t e, const char *what);

#define SRS_CUDA(call)                                              \
  do {                                                              \
    cudaError_t srs_e_ = (call);                                    \
    if (srs_e_ != cudaSuccess) return ::srs::cuda_fail(srs_e_, #call); \
  } while (0)

// ---- programmatic dependent launch ----
// A kernel launched by launch_after may be set up on the GPU while the stream's previous kernel is
// still running; it must call wait_for_previous_grid() before it reads or writes any memory that
// kernel touches (the wait ends when that grid has completed and its writes are visible; in a kernel
// launched the ordinary way it returns at once).  allow_next_grid() lets the stream's next such launch
// begin early.  Used on chains of short dependent kernels (the parallel-in-time passes, then the sums),
// where the launch latency between kernels is a visible part of the time.
__device__ __forceinline__ void wait_for_previous_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_next_grid() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline cudaError_t launch_after(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                Args &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// The library's stream-ordered memory pool of the current device (created on first use, kept for the
// process).  Freed blocks stay in it for the next call instead of going back to the driver at every
// synchronisation (a pool's default release threshold is 0, which makes a call that needs the 5.9 GB
// trajectory batch of a 4096-electron beam map it again every time); srs_trim_memory returns them.
cudaError_t library_pool(cudaMemPool_t *pool);

// Stream-ordered device buffer (from the library's pool, freed on the caller's stream).
struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0;
  cudaStream_t stream = nullptr;
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  ~DeviceBuffer() { release(); }
  cudaError_t alloc(size_t n, cudaStream_t s) {
    release();
    stream = s;
    bytes = n;
    if (n == 0) return cudaSuccess;
    cudaMemPool_t pool;
    cudaError_t e = library_pool(&pool);
    if (e != cudaSuccess) return e;
    return cudaMallocFromPoolAsync(&ptr, n, pool, s);
  }
  void release() {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    bytes = 0;
  }
  template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Per-particle trajectory parameters for batches of different lengths (device array).
struct TrajSpec {
  double dt;
  int64_t nfwd, nbwd;
  double *x, *beta, *aoc;  // 3 * (nfwd + nbwd) doubles each, [component][point]
};

// ---- field maps from files (field_files.cpp): the grid descriptor and its samples (host) ----
srs_status read_field_file(const std::string &path, const std::string &format, const double rot[3],
                           const double trans[3], const double *scale, int nscale, srs_field &f,
                           std::vector<double> &data);
srs_status read_field_interpolated(std::vector<std::pair<double, std::string>> mapping, const std::string &format,
                                   double parameter, const double rot[3], const double trans[3],
                                   const double *scale, int nscale, srs_field &f, std::vector<double> &data);

// ---- kernel launchers ----
// Time-domain electric field of one trajectory (first particle of the view) at obs: arrival times (n)
// and fields (3 n, point-major).
cudaError_t efield_time(const srs_traj_view &t, double charge, const double obs[3], double *d_t, double *d_e,
                        cudaStream_t s);
// Grid samples (doubles) to stage in shared memory for these fields (HOST array): their total, or 0
// when they do not fit.  Pass it to the RK4 launchers.
int64_t grid_stage_doubles(const srs_field *host_fields, int nfields);
// electric: some of the fields are electric (SRS_FIELD_ELECTRIC); has_electric tells from a HOST array
bool has_electric(const srs_field *host_fields, int nfields);
cudaError_t launch_rk4(const srs_field *d_fields, int nfields, const srs_particle *d_particles, int nparticles,
                       double dt, int64_t nfwd, int64_t nbwd, double *d_x, double *d_b, double *d_a,
                       cudaStream_t s, int64_t stage_doubles, bool electric = false);
cudaError_t launch_rk4_specs(const srs_field *d_fields, int nfields, const srs_particle *d_particles,
                             const TrajSpec *d_specs, int nparticles, cudaStream_t s, int64_t stage_doubles,
                             bool electric = false);
// One particle with the serial warp kernel, which returns at once when *d_skip != 0.
cudaError_t launch_rk4_unless(const srs_field *d_fields, int nfields, const srs_particle *d_particles, double dt,
                              int64_t nfwd, int64_t nbwd, double *d_x, double *d_b, double *d_a, cudaStream_t s,
                              int64_t stage_doubles, const int *d_skip);
// One particle parallel in time (rk4_shoot.cu); scratch of shoot_scratch_bytes bytes.
int shoot_default_steps(int64_t nsteps);
size_t shoot_scratch_bytes(int64_t nfwd, int64_t nbwd, int steps_per_segment, int nfields);
cudaError_t launch_rk4_shoot(const srs_field *d_fields, int nfields, const srs_particle *d_particle,
                             const srs_particle &host_particle, double dt, int64_t nfwd, int64_t nbwd, double *d_x,
                             double *d_b, double *d_a, cudaStream_t s, int64_t stage_doubles, int steps_per_segment,
                             int max_iterations, void *scratch, double *d_stats);
cudaError_t launch_field_eval(const srs_field *d_fields, int nfields, const double *d_xyz, int64_t np,
                              double *d_out, cudaStream_t s, bool electric = false);

// Plain FP64 sums.  Scratch is caller-provided (size from the *_scratch_bytes functions).
size_t fp64_spectrum_scratch_bytes(int64_t n, int64_t ne, int nparticles);
// d_e6 (optional): the reduced sums SumE (Re/Im of x, y, z) of every output, 6 per output.
cudaError_t fp64_spectrum(const srs_traj_view &t, const srs_beam_consts &b, const double obs[3],
                          const double *d_energies, int64_t ne, double *d_out, void *scratch, cudaStream_t s,
                          double *d_e6 = nullptr);
size_t fp64_flux_scratch_bytes(int64_t n, int64_t np, int nparticles);
cudaError_t fp64_flux(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points, int64_t np,
                      double energy_ev, double *d_out, void *scratch, cudaStream_t s);
size_t fp64_pd_scratch_bytes(int64_t n, int64_t np, int nparticles);
cudaError_t fp64_power_density(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points,
                               const double *d_normals, int64_t np, int directional, double *d_out, void *scratch,
                               cudaStream_t s);
cudaError_t total_power(const srs_traj_view &t, const srs_beam_consts &b, const double *d_gamma, double *d_out,
                        cudaStream_t s);
cudaError_t accumulate_particles(const double *d_vals, int nparticles, int64_t nout, double weight, double *d_out,
                                 double *d_comp, cudaStream_t s);

// Mixed-precision sums.
size_t mixed_spectrum_scratch_bytes(int64_t n, int64_t ne, int nparticles);
cudaError_t mixed_spectrum(const srs_traj_view &t, const srs_beam_consts &b, const double obs[3],
                           const double *d_energies, int64_t ne, double *d_out, void *scratch, cudaStream_t s,
                           double *d_e6 = nullptr);
size_t mixed_flux_scratch_bytes(int64_t n, const srs_grid2d &g, int nparticles);
cudaError_t mixed_flux(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g, double energy_ev,
                       double *d_out, void *scratch, cudaStream_t s);
// Mixed-precision flux at an arbitrary list of points (FP64 geometry and phase, FP32 amplitude).
size_t mixed_flux_points_scratch_bytes(int64_t n, int64_t np, int nparticles);
cudaError_t mixed_flux_points(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points, int64_t np,
                              double energy_ev, double *d_out, void *scratch, cudaStream_t s);
size_t mixed_pd_points_scratch_bytes(int64_t n, int64_t np, int nparticles);
cudaError_t mixed_power_density_points(const srs_traj_view &t, const srs_beam_consts &b, const double *d_points,
                                       const double *d_normals, int64_t np, int directional, double *d_out,
                                       void *scratch, cudaStream_t s);
size_t mixed_pd_scratch_bytes(int64_t n, const srs_grid2d &g, int nparticles);
cudaError_t mixed_power_density(const srs_traj_view &t, const srs_beam_consts &b, const srs_grid2d &g,
                                int directional, double *d_out, void *scratch, cudaStream_t s);

// Finishing kernels shared by both precisions: add the S per-chunk partial sums in chunk order and
// apply the reference's final scaling.
cudaError_t finish_flux_partials(const double *partial, int S, int64_t nout, int nparticles, const double *omegas,
                                 double omega0, double dt, double C0, double C2, double *out, cudaStream_t s,
                                 double *e6 = nullptr);
cudaError_t finish_pd_partials(const double *partial, int S, int64_t np, int nparticles, double cdt, int directional,
                               double *out, cudaStream_t s);

}  // namespace srs

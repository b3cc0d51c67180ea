// Host-side simulation object behind the srs_sim_* C ABI: the state and dispatch of the reference's
// Python type oscars.sr.sr (src/OSCARSSR_Python.cc, src/OSCARSSR.cc) for the hot-path calls.
//
// Everything numeric runs on the GPU (trajectories, sums, accumulation, field evaluation).  The
// host keeps the objects the reference keeps on the host: field descriptors, particle beams, the
// process-wide random generator (std::mt19937 + std::normal_distribution<double>, exactly as
// src/TRandomA.cc uses them, so sampled particles are bit-identical), surfaces and settings.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <functional>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

// Shortest single-particle trajectory integrated parallel in time (below it the serial chain, at
// ~0.9 us per step, costs about what the shooting iterations' launches do).
constexpr int64_t kShootMinPoints = 1024;

// ---------------------------------------------------------------- global random generator
// TRandomA (src/TRandomA.cc): one process-wide engine seeded from std::random_device; SetSeed
// replaces the engine but keeps the distributions, so a cached second normal value survives a reseed.
struct GlobalRandom {
  std::mutex mu;
  std::unique_ptr<std::mt19937> mt;
  std::normal_distribution<double> normal{0, 1};
  std::uniform_real_distribution<double> uniform{0, 1};
  GlobalRandom() {
    std::random_device rd;
    mt.reset(new std::mt19937(rd()));
  }
};
GlobalRandom &rng() {
  static GlobalRandom g;
  return g;
}

// ---------------------------------------------------------------- small vector helpers (host)
V3 rot(V3 v, const double r[3]) {
  rotate_xyz(v, r);
  return v;
}
V3 vec(const double *p) { return v3(p[0], p[1], p[2]); }
void put(double *o, V3 v) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
}
std::string lower(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  return s;
}
std::string upper(std::string s) {
  std::transform(s.begin(), s.end(), s.begin(), ::toupper);
  return s;
}
double gev_to_kg(double m) { return kQe * m / (1e-9 * kC * kC); }
double kg_to_gev(double m) { return 1e-9 * m * kC * kC / kQe; }

// ---------------------------------------------------------------- particles and beams
struct Particle {
  bool set = false;
  double q = 0, m = 0, current = 0;
  V3 x0{0, 0, 0}, b0{0, 0, 0};
  double t0 = 0, gamma = 0, qomg = 0;
};

// TParticleBeam (src/TParticleBeam.cc) with the Python-side sigma setup (OSCARSSR_Python.cc:1818-1866)
struct Beam {
  std::string name;
  double q = 0, m = 0, current = 0;
  V3 x0{0, 0, 0}, u0{0, 0, 1};
  double e0 = 0, t0 = 0;
  V3 hdir{1, 0, 0}, vdir{0, 1, 0};
  double su[2] = {0, 0}, sup[2] = {0, 0};
  V3 sigma_at{0, 0, 0};
  double sigma_e = 0;

  // TParticleA::SetInitialParticleConditions -> SetGamma -> SetQoverMGamma (TParticleA.cc:323-382)
  Particle make(V3 X, V3 B) const {
    Particle p;
    p.set = true;
    p.q = q;
    p.m = m;
    p.current = current;
    p.x0 = X;
    p.b0 = B;
    p.t0 = t0;
    const double b2 = mag2(B);
    p.gamma = 1.0 / sqrt(1.0 - b2);
    p.qomg = q / m / p.gamma;
    return p;
  }
  // GetNewParticle("ideal"), TParticleBeam.cc:200-222
  Particle ideal() const {
    const double g = e0 / kg_to_gev(m);
    const double beta = sqrt(1.0 - 1.0 / (g * g));
    return make(x0, u0 * beta);
  }
  // GetNewParticle(), TParticleBeam.cc:228-265: draws E, x, y, x', y' in this order
  Particle random() const {
    GlobalRandom &r = rng();
    std::lock_guard<std::mutex> lk(r.mu);
    const double enew = e0 + sigma_e * r.normal(*r.mt);
    const double g = enew / kg_to_gev(m);
    const double beta = sqrt(1.0 - 1.0 / (g * g));
    const double dmid = dot(sigma_at - x0, u0);
    V3 X = x0;
    X = X + hdir * su[0] * (1 + dmid) * r.normal(*r.mt);
    X = X + vdir * su[1] * (1 + dmid) * r.normal(*r.mt);
    V3 B = u0 * beta;
    {
      const double a = sup[0] * r.normal(*r.mt);  // RotateSelfY
      const double s = sin(a), c = cos(a), zz = B.z;
      B.z = c * zz - s * B.x;
      B.x = s * zz + c * B.x;
    }
    {
      const double a = -sup[1] * r.normal(*r.mt);  // RotateSelfX
      const double s = sin(a), c = cos(a), yy = B.y;
      B.y = c * yy - s * B.z;
      B.z = s * yy + c * B.z;
    }
    return make(X, B);
  }
};

}  // namespace
}  // namespace srs

using namespace srs;

// ---------------------------------------------------------------- the object
struct srs_sim {
  std::mutex mu;
  cudaStream_t stream = nullptr;
  double ctstart = 0, ctstop = 0;
  int64_t npoints = 0;
  int64_t npoints_per_meter = 10000;
  int32_t nthreads_global = 2, gpu_global = 0;
  std::vector<srs_field> fields;             // host descriptors (grid data pointers are device)
  std::vector<std::vector<double>> grid_host; // host copy of each grid's samples (empty otherwise)
  std::vector<double *> grid_dev;             // device samples per field (nullptr otherwise)
  double *d_fields = nullptr;                 // device copy of `fields`
  bool fields_dirty = true;
  uint64_t fields_version = 0;                // bumped by every field change (trajectory cache key)
  // Device trajectory of the last single-particle calculation.  The reference recomputes the same
  // trajectory on every call; keeping it lets later calls (other energies, maps, spectra) skip the
  // RK4 when the particle, the fields and the trajectory settings are unchanged.
  struct TrajCache {
    bool valid = false;
    double key[12] = {0};
    uint64_t fields_version = 0;
    double *x = nullptr, *b = nullptr, *a = nullptr;
    int64_t capacity = 0;
    srs_traj_view view{};
  } cache;
  bool cache_enabled = true;
  int32_t traj_mode = SRS_TRAJ_AUTO;
  // pinned staging of the caller's accumulator arrays (grow-only)
  double *pinned = nullptr;
  size_t pinned_doubles = 0;
  std::vector<Beam> beams;
  std::vector<double> weight_sums;
  std::map<std::string, size_t> beam_index;
  Particle particle;

  ~srs_sim() {
    for (double *p : grid_dev)
      if (p) cudaFree(p);
    if (d_fields) cudaFree(d_fields);
    if (cache.x) cudaFree(cache.x);
    if (cache.b) cudaFree(cache.b);
    if (cache.a) cudaFree(cache.a);
    if (pinned) cudaFreeHost(pinned);
    if (stream) cudaStreamDestroy(stream);
  }

  srs_status upload_fields() {
    if (!fields_dirty) return SRS_OK;
    if (d_fields) cudaFree(d_fields);
    d_fields = nullptr;
    SRS_CUDA(cudaMalloc(&d_fields, sizeof(srs_field) * std::max<size_t>(1, fields.size())));
    if (!fields.empty())
      SRS_CUDA(cudaMemcpy(d_fields, fields.data(), sizeof(srs_field) * fields.size(), cudaMemcpyHostToDevice));
    fields_dirty = false;
    return SRS_OK;
  }

  // Removes the magnetic (electric = false) or the electric fields, keeping the others in order.
  void remove_fields(bool electric) {
    size_t k = 0;
    for (size_t i = 0; i < fields.size(); ++i) {
      if (field_electric(fields[i].kind) == electric) {
        if (grid_dev[i]) cudaFree(grid_dev[i]);
        continue;
      }
      fields[k] = fields[i];
      grid_host[k] = std::move(grid_host[i]);
      grid_dev[k] = grid_dev[i];
      ++k;
    }
    fields.resize(k);
    grid_host.resize(k);
    grid_dev.resize(k);
    fields_dirty = true;
    ++fields_version;
  }

  // The magnetic or electric field at np points (HOST arrays of 3 np doubles), evaluated on the device.
  srs_status eval_fields(const double *xyz, int64_t np, double *out, bool electric) {
    if (!xyz || !out || np < 0) return fail(SRS_ERR_INVALID, "bad argument");
    if (np == 0) return SRS_OK;
    if (srs_status st = upload_fields()) return st;
    DeviceBuffer dx, dout;
    SRS_CUDA(dx.alloc(sizeof(double) * 3 * np, stream));
    SRS_CUDA(dout.alloc(sizeof(double) * 3 * np, stream));
    SRS_CUDA(cudaMemcpyAsync(dx.ptr, xyz, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, stream));
    SRS_CUDA(launch_field_eval(reinterpret_cast<const srs_field *>(d_fields), (int)fields.size(), dx.as<double>(), np,
                               dout.as<double>(), stream, electric));
    SRS_CUDA(cudaMemcpyAsync(out, dout.ptr, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, stream));
    SRS_CUDA(cudaStreamSynchronize(stream));
    return SRS_OK;
  }

  srs_status add_field(const srs_field &f, std::vector<double> &&host_grid) {
    double *dev = nullptr;
    srs_field g = f;
    if (field_shape(f.kind) == SRS_FIELD_GRID) {
      SRS_CUDA(cudaMalloc(&dev, sizeof(double) * host_grid.size()));
      SRS_CUDA(cudaMemcpy(dev, host_grid.data(), sizeof(double) * host_grid.size(), cudaMemcpyHostToDevice));
      g.data = dev;
    }
    fields.push_back(g);
    grid_host.push_back(std::move(host_grid));
    grid_dev.push_back(dev);
    fields_dirty = true;
    ++fields_version;
    return SRS_OK;
  }

  // TParticleBeamContainer::GetRandomBeamIndexByWeight (TParticleBeamContainer.cc:109-142)
  srs_status random_beam_index(size_t &idx) {
    const size_t N = weight_sums.size();
    if (N == 0) return fail(SRS_ERR_RANGE, "no beam defined");
    if (N == 1) {
      idx = 0;
      return SRS_OK;
    }
    double u;
    {
      GlobalRandom &r = rng();
      std::lock_guard<std::mutex> lk(r.mu);
      u = r.uniform(*r.mt);
    }
    const double R = u * weight_sums[N - 1];
    for (size_t i = 0; i != N; ++i)
      if (R < weight_sums[i]) {
        idx = i;
        return SRS_OK;
      }
    return fail(SRS_ERR_RANGE, "random weight out of range.  SERIOUS ERROR");
  }

  srs_status new_random_particle(Particle &p) {
    size_t i;
    if (srs_status st = random_beam_index(i)) return st;
    p = beams[i].random();
    return SRS_OK;
  }

  srs_status ensure_particle() {
    if (particle.set) return SRS_OK;
    if (beams.empty()) return fail(SRS_ERR_RANGE, "no beam defined");
    return new_random_particle(particle);
  }

  // The particles of one calculation: the current one, or nparticles new random ones (the last of
  // which becomes the current particle, as OSCARSSR::SetNewParticle leaves it).
  srs_status particles_for(int32_t nparticles, std::vector<Particle> &out, double &weight) {
    out.clear();
    if (srs_status st = ensure_particle()) return st;
    if (nparticles == 0) {
      out.push_back(particle);
      weight = 1;
      return SRS_OK;
    }
    weight = 1.0 / (double)nparticles;
    for (int i = 0; i < nparticles; ++i) {
      Particle p;
      if (srs_status st = new_random_particle(p)) return st;
      out.push_back(p);
    }
    particle = out.back();
    return SRS_OK;
  }

  // Whether the single-particle trajectory of a calculation in this precision is integrated parallel
  // in time: for the mixed-precision sums in the automatic mode (their error budget, 1e-4, dwarfs the
  // shooting trajectory's ~1e-16 m), always in the parallel mode, never for the FP64 drop-in path
  // unless the caller asked for it.
  bool shoot_for(int32_t precision) const {
    if (traj_mode == SRS_TRAJ_PARALLEL) return true;
    return traj_mode == SRS_TRAJ_AUTO && precision == SRS_PRECISION_MIXED;
  }

  // RK4 trajectories of a batch of particles that share t0 into device arrays (layout of srs_trajectory).
  // shoot: one particle, parallel in time (long trajectories only; short ones are cheaper serially).
  srs_status integrate(const Particle *ps, int np, double *X, double *B, double *A, srs_traj_view &view,
                       bool shoot = false) {
    double dt;
    int64_t nf, nb;
    if (srs_status st = srs_trajectory_counts(ctstart, ctstop, ps[0].t0, npoints, &dt, &nf, &nb)) return st;
    const int64_t n = nf + nb;
    if (n < 1) return fail(SRS_ERR_RANGE, "no points in trajectory.  Is particle or beam defined?");
    if (srs_status st = upload_fields()) return st;
    std::vector<srs_particle> hp(np);
    for (int i = 0; i < np; ++i) {
      put(hp[i].x0, ps[i].x0);
      put(hp[i].beta0, ps[i].b0);
      hp[i].qomg = ps[i].qomg;
    }
    DeviceBuffer dp;
    SRS_CUDA(dp.alloc(sizeof(srs_particle) * np, stream));
    SRS_CUDA(cudaMemcpyAsync(dp.ptr, hp.data(), sizeof(srs_particle) * np, cudaMemcpyHostToDevice, stream));
    const int64_t stage = fields.empty() ? 0 : grid_stage_doubles(fields.data(), (int)fields.size());
    const bool electric = has_electric(fields.data(), (int)fields.size());
    if (shoot && !electric && np == 1 && n >= kShootMinPoints) {
      DeviceBuffer scratch;
      SRS_CUDA(scratch.alloc(shoot_scratch_bytes(nf, nb, 0, (int)fields.size()), stream));
      SRS_CUDA(launch_rk4_shoot(reinterpret_cast<const srs_field *>(d_fields), (int)fields.size(),
                                dp.as<srs_particle>(), hp[0], dt, nf, nb, X, B, A, stream, stage, 0, 0, scratch.ptr,
                                nullptr));
    } else {
      SRS_CUDA(launch_rk4(reinterpret_cast<const srs_field *>(d_fields), (int)fields.size(), dp.as<srs_particle>(), np,
                          dt, nf, nb, X, B, A, stream, stage, electric));
    }
    view.x = X;
    view.beta = B;
    view.aoc = A;
    view.n = n;
    view.nparticles = np;
    view.dt = dt;
    return SRS_OK;
  }

  srs_status point_count(const Particle &p, int64_t &n) {
    double dt;
    int64_t nf, nb;
    if (srs_status st = srs_trajectory_counts(ctstart, ctstop, p.t0, npoints, &dt, &nf, &nb)) return st;
    n = nf + nb;
    return SRS_OK;
  }

  // A batch into stream-ordered buffers owned by the caller.
  srs_status trajectories(const Particle *ps, int np, DeviceBuffer &X, DeviceBuffer &B, DeviceBuffer &A,
                          srs_traj_view &view) {
    int64_t n;
    if (srs_status st = point_count(ps[0], n)) return st;
    const size_t bytes = sizeof(double) * 3 * (size_t)std::max<int64_t>(n, 1) * np;
    SRS_CUDA(X.alloc(bytes, stream));
    SRS_CUDA(B.alloc(bytes, stream));
    SRS_CUDA(A.alloc(bytes, stream));
    return integrate(ps, np, X.as<double>(), B.as<double>(), A.as<double>(), view);
  }

  // The trajectory of one particle, from the cache when nothing it depends on has changed.
  srs_status single(const Particle &p, srs_traj_view &view, bool shoot = false) {
    const double key[12] = {p.x0.x, p.x0.y, p.x0.z, p.b0.x, p.b0.y, p.b0.z, p.qomg, p.t0, ctstart, ctstop,
                            (double)npoints, shoot ? 1.0 : 0.0};
    if (cache_enabled && cache.valid && cache.fields_version == fields_version && cache.view.n > 0 &&
        std::memcmp(key, cache.key, sizeof key) == 0) {
      int64_t n;
      if (srs_status st = point_count(p, n)) return st;
      if (n == cache.view.n) {
        view = cache.view;
        return SRS_OK;
      }
    }
    cache.valid = false;
    int64_t n;
    if (srs_status st = point_count(p, n)) return st;
    if (n > cache.capacity) {
      for (double **q : {&cache.x, &cache.b, &cache.a}) {
        if (*q) cudaFree(*q);
        *q = nullptr;
      }
      cache.capacity = 0;
      for (double **q : {&cache.x, &cache.b, &cache.a}) SRS_CUDA(cudaMalloc(q, sizeof(double) * 3 * (size_t)n));
      cache.capacity = n;
    }
    if (srs_status st = integrate(&p, 1, cache.x, cache.b, cache.a, cache.view, shoot)) return st;
    std::memcpy(cache.key, key, sizeof key);
    cache.fields_version = fields_version;
    cache.valid = cache_enabled;
    view = cache.view;
    return SRS_OK;
  }

  // Particles per device batch: trajectories of at most ~8 GB at a time.
  int batch_size(int total) const {
    double dt;
    int64_t nf = 0, nb = 0;
    const double t0 = particle.set ? particle.t0 : 0.0;
    if (srs_trajectory_counts(ctstart, ctstop, t0, npoints, &dt, &nf, &nb) != SRS_OK) return std::max(1, total);
    const double per = 72.0 * (double)std::max<int64_t>(1, nf + nb);
    const int cap = (int)std::max(1.0, std::floor(8e9 / per));
    return std::max(1, std::min(total, cap));
  }

  // The common driver: sample particles, integrate in batches, run `sum` on each batch (writing
  // per-particle values to d_vals), then Kahan-accumulate them in particle order into out/comp.
  // host_work, when given, runs after all device work of the call is queued and before the host
  // waits for it (host-side preparation of the call's other outputs, overlapped with the GPU)
  template <class SumFn>
  srs_status run(int32_t nparticles, int64_t nout, double *out, double *comp, bool apply_weight, int32_t precision,
                 SumFn sum, const std::function<void()> &host_work = {}) {
    std::vector<Particle> ps;
    double weight;
    if (srs_status st = particles_for(nparticles, ps, weight)) return st;
    if (!apply_weight) weight = 1.0;
    DeviceBuffer dacc;
    SRS_CUDA(dacc.alloc(sizeof(double) * 2 * nout, stream));
    double *d_out = dacc.as<double>(), *d_comp = d_out + nout;
    if ((size_t)(2 * nout) > pinned_doubles) {
      if (pinned) SRS_CUDA(cudaFreeHost(pinned));
      pinned = nullptr;
      pinned_doubles = 0;
      SRS_CUDA(cudaMallocHost(&pinned, sizeof(double) * 2 * nout));
      pinned_doubles = 2 * nout;
    }
    // the caller's accumulators go up after the first batch's sums are queued: the host copies them
    // into pinned memory while the GPU computes.  Without comp the sums start from zero on the device.
    const bool fresh = comp == nullptr;
    bool uploaded = false;
    auto upload = [&]() -> srs_status {
      if (fresh) {
        SRS_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * 2 * nout, stream));
      } else {
        std::memcpy(pinned, out, sizeof(double) * nout);
        std::memcpy(pinned + nout, comp, sizeof(double) * nout);
        SRS_CUDA(cudaMemcpyAsync(d_out, pinned, sizeof(double) * 2 * nout, cudaMemcpyHostToDevice, stream));
      }
      uploaded = true;
      return SRS_OK;
    };
    const int bs = batch_size((int)ps.size());
    for (size_t b0 = 0; b0 < ps.size();) {
      // a batch shares t0 (particles of different beams may not)
      size_t b1 = b0 + 1;
      while (b1 < ps.size() && (int)(b1 - b0) < bs && ps[b1].t0 == ps[b0].t0 && ps[b1].q == ps[b0].q &&
             ps[b1].current == ps[b0].current)
        ++b1;
      const int np = (int)(b1 - b0);
      DeviceBuffer X, B, A, vals;
      srs_traj_view view;
      if (nparticles == 0) {
        if (srs_status st = single(ps[b0], view, shoot_for(precision))) return st;
      } else if (srs_status st = trajectories(&ps[b0], np, X, B, A, view)) {
        return st;
      }
      srs_beam_consts bc{ps[b0].q, ps[b0].current};
      // one particle with weight 1 into outputs that start from zero: its sums are the result (a
      // compensated add of v to zero gives v), so they are written straight into the output
      if (fresh && ps.size() == 1 && weight == 1.0) {
        if (srs_status st = sum(view, bc, d_out)) return st;
        uploaded = true;
        b0 = b1;
        continue;
      }
      SRS_CUDA(vals.alloc(sizeof(double) * (size_t)nout * np, stream));
      if (srs_status st = sum(view, bc, vals.as<double>())) return st;
      if (!uploaded)
        if (srs_status st = upload()) return st;
      SRS_CUDA(accumulate_particles(vals.as<double>(), np, nout, weight, d_out, d_comp, stream));
      b0 = b1;
    }
    if (!uploaded)
      if (srs_status st = upload()) return st;
    SRS_CUDA(cudaMemcpyAsync(pinned, d_out, sizeof(double) * (fresh ? 1 : 2) * nout, cudaMemcpyDeviceToHost, stream));
    if (host_work) host_work();
    SRS_CUDA(cudaStreamSynchronize(stream));
    std::memcpy(out, pinned, sizeof(double) * nout);
    if (!fresh) std::memcpy(comp, pinned + nout, sizeof(double) * nout);
    return SRS_OK;
  }
};

#define SIM_GUARD(sim)                                                     \
  if (!(sim)) return fail(SRS_ERR_INVALID, "NULL simulation object");     \
  std::lock_guard<std::mutex> srs_lk_((sim)->mu);                         \
  clear_error()

extern "C" {

srs_status srs_sim_create(srs_sim **out) {
  clear_error();
  if (!out) return fail(SRS_ERR_INVALID, "NULL output");
  std::unique_ptr<srs_sim> s(new srs_sim());
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev < 1) {
    cudaGetLastError();
    return fail(SRS_ERR_NO_DEVICE, "You are requesting the GPU, but none were found");
  }
  SRS_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  *out = s.release();
  return SRS_OK;
}

void srs_sim_destroy(srs_sim *sim) { delete sim; }

srs_status srs_sim_set_ctstartstop(srs_sim *sim, double start, double stop) {
  SIM_GUARD(sim);
  // OSCARSSR::SetCTStartStop (OSCARSSR.cc:448-458): npoints = size_t(points_per_meter * (stop - start))
  sim->npoints = (int64_t)(size_t)((double)sim->npoints_per_meter * (stop - start));
  sim->ctstart = start;
  sim->ctstop = stop;
  return SRS_OK;
}
srs_status srs_sim_set_npoints_trajectory(srs_sim *sim, int64_t n) {
  SIM_GUARD(sim);
  sim->npoints = n;
  return SRS_OK;
}
srs_status srs_sim_get_ctstartstop(srs_sim *sim, double *start, double *stop) {
  SIM_GUARD(sim);
  if (start) *start = sim->ctstart;
  if (stop) *stop = sim->ctstop;
  return SRS_OK;
}
int64_t srs_sim_get_npoints_trajectory(srs_sim *sim) { return sim ? sim->npoints : 0; }
srs_status srs_sim_set_nthreads_global(srs_sim *sim, int32_t n) {
  SIM_GUARD(sim);
  sim->nthreads_global = n;
  return SRS_OK;
}
srs_status srs_sim_set_gpu_global(srs_sim *sim, int32_t g) {
  SIM_GUARD(sim);
  sim->gpu_global = g;
  return SRS_OK;
}

srs_status srs_sim_add_bfield_undulator(srs_sim *sim, const double bfield[3], const double period[3], int32_t nperiods,
                                        double phase, const double rotations[3], const double translation[3],
                                        double taper) {
  SIM_GUARD(sim);
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_UNDULATOR;
  put(f.field, rot(vec(bfield), rotations));   // OSCARSSR_Python.cc:809-810
  put(f.period, rot(vec(period), rotations));
  std::memcpy(f.center, translation, sizeof(double) * 3);
  f.nperiods = nperiods;
  f.phase = phase;
  f.taper = taper;
  return sim->add_field(f, {});
}

srs_status srs_sim_add_bfield_gaussian(srs_sim *sim, const double bfield[3], const double sigma[3],
                                       const double rotations[3], const double translation[3]) {
  SIM_GUARD(sim);
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_GAUSSIAN;  // TField3D_Gaussian(BField, Center=translation, Sigma, Rotations)
  put(f.field, rot(vec(bfield), rotations));
  std::memcpy(f.center, translation, sizeof(double) * 3);
  std::memcpy(f.sigma_or_width, sigma, sizeof(double) * 3);
  std::memcpy(f.rotations, rotations, sizeof(double) * 3);
  return sim->add_field(f, {});
}

srs_status srs_sim_add_bfield_uniform(srs_sim *sim, const double bfield[3], const double width[3],
                                      const double rotations[3], const double translation[3]) {
  SIM_GUARD(sim);
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_UNIFORM_BOX;  // TField3D_UniformBox(BField, Width, Center=translation, Rotations)
  put(f.field, rot(vec(bfield), rotations));
  std::memcpy(f.center, translation, sizeof(double) * 3);
  std::memcpy(f.sigma_or_width, width, sizeof(double) * 3);
  std::memcpy(f.rotations, rotations, sizeof(double) * 3);
  return sim->add_field(f, {});
}

srs_status srs_sim_add_bfield_file(srs_sim *sim, const char *path, const char *format, const double rotations[3],
                                   const double translation[3], const double *scale, int32_t nscale) {
  SIM_GUARD(sim);
  if (!path || !format || !*path || !*format) return fail(SRS_ERR_INVALID, "'ifile' or 'iformat' is blank");
  srs_field f;
  std::vector<double> data;
  if (srs_status st = read_field_file(path, format, rotations, translation, scale, nscale, f, data)) return st;
  return sim->add_field(f, std::move(data));
}

srs_status srs_read_field_file(const char *path, const char *format, const double rotations[3],
                               const double translation[3], const double *scale, int32_t nscale, srs_field *out,
                               double *data, int64_t *ndata) {
  clear_error();
  if (!path || !format || !*path || !*format) return fail(SRS_ERR_INVALID, "'ifile' or 'iformat' is blank");
  if (!out || !ndata || !rotations || !translation) return fail(SRS_ERR_INVALID, "NULL argument");
  srs_field f;
  std::vector<double> d;
  if (srs_status st = read_field_file(path, format, rotations, translation, scale, nscale, f, d)) return st;
  *out = f;
  out->data = nullptr;
  if (data && *ndata >= (int64_t)d.size()) std::memcpy(data, d.data(), sizeof(double) * d.size());
  *ndata = (int64_t)d.size();
  return SRS_OK;
}

srs_status srs_read_field_interpolated(const double *parameters, const char *const *paths, int32_t nmap,
                                       const char *format, double parameter, const double rotations[3],
                                       const double translation[3], const double *scale, int32_t nscale,
                                       srs_field *out, double *data, int64_t *ndata) {
  clear_error();
  if (!format || !*format) return fail(SRS_ERR_INVALID, "'iformat' is blank");
  if (!out || !ndata || !rotations || !translation || nmap < 0 || (nmap > 0 && (!parameters || !paths)))
    return fail(SRS_ERR_INVALID, "NULL argument");
  std::vector<std::pair<double, std::string>> mapping;
  for (int i = 0; i < nmap; ++i) {
    if (!paths[i]) return fail(SRS_ERR_INVALID, "Incorrect format in 'mapping'");
    mapping.emplace_back(parameters[i], paths[i]);
  }
  srs_field f;
  std::vector<double> d;
  if (srs_status st = read_field_interpolated(mapping, format, parameter, rotations, translation, scale, nscale, f, d))
    return st;
  *out = f;
  out->data = nullptr;
  if (data && *ndata >= (int64_t)d.size()) std::memcpy(data, d.data(), sizeof(double) * d.size());
  *ndata = (int64_t)d.size();
  return SRS_OK;
}

srs_status srs_sim_add_bfield_interpolated(srs_sim *sim, const double *parameters, const char *const *paths,
                                           int32_t nmap, const char *format, double parameter,
                                           const double rotations[3], const double translation[3],
                                           const double *scale, int32_t nscale) {
  SIM_GUARD(sim);
  if (!format || !*format) return fail(SRS_ERR_INVALID, "'iformat' is blank");
  if (nmap < 0 || (nmap > 0 && (!parameters || !paths))) return fail(SRS_ERR_INVALID, "Incorrect format in 'mapping'");
  std::vector<std::pair<double, std::string>> mapping;
  for (int i = 0; i < nmap; ++i) {
    if (!paths[i]) return fail(SRS_ERR_INVALID, "Incorrect format in 'mapping'");
    mapping.emplace_back(parameters[i], paths[i]);
  }
  srs_field f;
  std::vector<double> data;
  if (srs_status st = read_field_interpolated(mapping, format, parameter, rotations, translation, scale, nscale, f,
                                              data))
    return st;
  return sim->add_field(f, std::move(data));
}

srs_status srs_sim_add_bfield_grid(srs_sim *sim, const double start[3], const double step[3], const int64_t n[3],
                                   const double *data, const double rotations[3], const double translation[3]) {
  SIM_GUARD(sim);
  if (!data || n[0] < 1 || n[1] < 1 || n[2] < 1 || (n[0] == 1 && n[1] == 1 && n[2] == 1))
    return fail(SRS_ERR_RANGE, "invalid dimensions");
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_GRID;
  for (int k = 0; k < 3; ++k) {
    f.start[k] = start[k];
    f.step[k] = step[k];
    f.n[k] = n[k];
    f.rotations[k] = rotations[k];
    f.translation[k] = translation[k];
  }
  const size_t cnt = (size_t)(n[0] * n[1] * n[2]);
  std::vector<double> d(3 * cnt);
  for (size_t i = 0; i < cnt; ++i) {
    V3 F = rot(v3(data[3 * i], data[3 * i + 1], data[3 * i + 2]), rotations);
    d[3 * i] = F.x;
    d[3 * i + 1] = F.y;
    d[3 * i + 2] = F.z;
  }
  return sim->add_field(f, std::move(d));
}

srs_status srs_sim_clear_bfields(srs_sim *sim) {
  SIM_GUARD(sim);
  sim->remove_fields(false);
  return SRS_OK;
}

srs_status srs_sim_clear_efields(srs_sim *sim) {
  SIM_GUARD(sim);
  sim->remove_fields(true);
  return SRS_OK;
}

// ---------------------------------------------------------------- electric fields
// The reference's electric-field container (OSCARSSR.cc:202-234, OSCARSSR_Python.cc:876-1390): the same
// shapes as the magnetic ones, marked SRS_FIELD_ELECTRIC.

srs_status srs_sim_add_efield_undulator(srs_sim *sim, const double efield[3], const double period[3], int32_t nperiods,
                                        double phase, const double rotations[3], const double translation[3]) {
  SIM_GUARD(sim);
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_UNDULATOR | SRS_FIELD_ELECTRIC;  // OSCARSSR_Python.cc:1156-1240 (no taper)
  put(f.field, rot(vec(efield), rotations));
  put(f.period, rot(vec(period), rotations));
  std::memcpy(f.center, translation, sizeof(double) * 3);
  f.nperiods = nperiods;
  f.phase = phase;
  return sim->add_field(f, {});
}

srs_status srs_sim_add_efield_gaussian(srs_sim *sim, const double efield[3], const double sigma[3],
                                       const double rotations[3], const double translation[3]) {
  SIM_GUARD(sim);
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_GAUSSIAN | SRS_FIELD_ELECTRIC;
  put(f.field, rot(vec(efield), rotations));
  std::memcpy(f.center, translation, sizeof(double) * 3);
  std::memcpy(f.sigma_or_width, sigma, sizeof(double) * 3);
  std::memcpy(f.rotations, rotations, sizeof(double) * 3);
  return sim->add_field(f, {});
}

srs_status srs_sim_add_efield_uniform(srs_sim *sim, const double efield[3], const double width[3],
                                      const double rotations[3], const double translation[3]) {
  SIM_GUARD(sim);
  srs_field f;
  std::memset(&f, 0, sizeof f);
  f.kind = SRS_FIELD_UNIFORM_BOX | SRS_FIELD_ELECTRIC;
  put(f.field, rot(vec(efield), rotations));
  std::memcpy(f.center, translation, sizeof(double) * 3);
  std::memcpy(f.sigma_or_width, width, sizeof(double) * 3);
  std::memcpy(f.rotations, rotations, sizeof(double) * 3);
  return sim->add_field(f, {});
}

srs_status srs_sim_add_efield_file(srs_sim *sim, const char *path, const char *format, const double rotations[3],
                                   const double translation[3]) {
  SIM_GUARD(sim);
  if (!path || !format || !*path || !*format) return fail(SRS_ERR_INVALID, "'ifile' or 'iformat' is blank");
  srs_field f;
  std::vector<double> data;
  // OSCARSSR::AddElectricField (OSCARSSR.cc:202-211): the grid reader without scaling
  if (srs_status st = read_field_file(path, format, rotations, translation, nullptr, 0, f, data)) return st;
  f.kind |= SRS_FIELD_ELECTRIC;
  return sim->add_field(f, std::move(data));
}

srs_status srs_sim_get_efield(srs_sim *sim, const double *xyz, int64_t np, double *out) {
  SIM_GUARD(sim);
  return sim->eval_fields(xyz, np, out, true);
}

srs_status srs_sim_calculate_efield_time(srs_sim *sim, const double obs[3], double *t, double *e, int64_t *n) {
  SIM_GUARD(sim);
  if (!obs || !n) return fail(SRS_ERR_INVALID, "NULL argument");
  if (srs_status st = sim->ensure_particle()) return st;
  double dt;
  int64_t nf, nb;
  if (srs_status st = srs_trajectory_counts(sim->ctstart, sim->ctstop, sim->particle.t0, sim->npoints, &dt, &nf, &nb))
    return st;
  if (!t || !e) {
    *n = nf + nb;
    return SRS_OK;
  }
  if (*n != nf + nb) return fail(SRS_ERR_INVALID, "output size does not match the trajectory");
  srs_traj_view v;
  if (srs_status st = sim->single(sim->particle, v, sim->shoot_for(SRS_PRECISION_FP64))) return st;
  DeviceBuffer dt_, de;
  SRS_CUDA(dt_.alloc(sizeof(double) * v.n, sim->stream));
  SRS_CUDA(de.alloc(sizeof(double) * 3 * v.n, sim->stream));
  SRS_CUDA(efield_time(v, sim->particle.q, obs, dt_.as<double>(), de.as<double>(), sim->stream));
  SRS_CUDA(cudaMemcpyAsync(t, dt_.ptr, sizeof(double) * v.n, cudaMemcpyDeviceToHost, sim->stream));
  SRS_CUDA(cudaMemcpyAsync(e, de.ptr, sizeof(double) * 3 * v.n, cudaMemcpyDeviceToHost, sim->stream));
  SRS_CUDA(cudaStreamSynchronize(sim->stream));
  return SRS_OK;
}

srs_status srs_sim_set_trajectory_mode(srs_sim *sim, int32_t mode) {
  SIM_GUARD(sim);
  if (mode != SRS_TRAJ_AUTO && mode != SRS_TRAJ_SERIAL && mode != SRS_TRAJ_PARALLEL)
    return fail(SRS_ERR_INVALID, "unknown trajectory mode");
  sim->traj_mode = mode;
  return SRS_OK;
}

srs_status srs_sim_set_trajectory_cache(srs_sim *sim, int32_t enabled) {
  SIM_GUARD(sim);
  sim->cache_enabled = enabled != 0;
  sim->cache.valid = false;
  return SRS_OK;
}

int32_t srs_sim_get_nfields(srs_sim *sim) { return sim ? (int32_t)sim->fields.size() : 0; }

srs_status srs_sim_get_bfield(srs_sim *sim, const double *xyz, int64_t np, double *out) {
  SIM_GUARD(sim);
  return sim->eval_fields(xyz, np, out, false);
}

srs_status srs_sim_set_field_grid_data(srs_sim *sim, int32_t k, const double *data, int32_t on_device) {
  SIM_GUARD(sim);
  if (k < 0 || k >= (int32_t)sim->fields.size() || field_shape(sim->fields[k].kind) != SRS_FIELD_GRID || !data)
    return fail(SRS_ERR_INVALID, "field is not a grid");
  const size_t cnt = sim->grid_host[k].size();
  SRS_CUDA(cudaMemcpyAsync(sim->grid_dev[k], data, sizeof(double) * cnt,
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, sim->stream));
  SRS_CUDA(cudaStreamSynchronize(sim->stream));
  if (!on_device) std::memcpy(sim->grid_host[k].data(), data, sizeof(double) * cnt);
  ++sim->fields_version;
  return SRS_OK;
}

srs_status srs_sim_add_particle_beam(srs_sim *sim, const srs_beam_args *a) {
  SIM_GUARD(sim);
  if (!a || !a->type || !a->name || !*a->type || !*a->name) return fail(SRS_ERR_INVALID, "'type' or 'name' is blank");
  if (a->sigma_energy_gev < 0) return fail(SRS_ERR_INVALID, "'sigma_energy_GeV' cannot be less than zero");
  if (sim->beam_index.count(a->name))
    return fail(SRS_ERR_INVALID, "invalid argument in adding particle beam.  possibly 'name' already exists");
  Beam b;
  b.name = a->name;
  const std::string type = a->type, t = lower(a->type);
  if (type == "custom") {
    if (a->mass == 0 || a->charge == 0) return fail(SRS_ERR_INVALID, "'mass' or 'charge' is zero");
    b.q = a->charge;
    b.m = a->mass;
  } else if (t == "electron" || t == "anti-positron") { b.q = -kQe; b.m = kMe; }
  else if (t == "positron" || t == "anti-electron") { b.q = kQe; b.m = kMe; }
  else if (t == "muon") { b.q = -kQe; b.m = gev_to_kg(0.1056583715); }
  else if (t == "anti-muon") { b.q = kQe; b.m = gev_to_kg(0.1056583715); }
  else if (t == "proton") { b.q = kQe; b.m = gev_to_kg(0.938272046); }
  else if (t == "anti-proton") { b.q = -kQe; b.m = gev_to_kg(0.938272046); }
  else if (t == "pi+") { b.q = kQe; b.m = gev_to_kg(0.13957018); }
  else if (t == "pi-") { b.q = -kQe; b.m = gev_to_kg(0.13957018); }
  else return fail(SRS_ERR_INVALID, "particle type not found: " + type);
  const V3 dir = vec(a->d0);
  V3 h = a->horizontal_direction ? vec(a->horizontal_direction) : unit(orthogonal(dir));
  h = unit(h);
  double su0 = 0, su1 = 0, sp0 = 0, sp1 = 0;
  if (a->beta && a->emittance) {
    su0 = sqrt(a->emittance[0] * a->beta[0]);
    su1 = sqrt(a->emittance[1] * a->beta[1]);
    sp0 = sqrt(a->emittance[0] / a->beta[0]);
    sp1 = sqrt(a->emittance[1] / a->beta[1]);
  }
  V3 pos = rot(vec(a->x0), a->rotations) + vec(a->translation);
  b.current = a->current != 0 ? a->current : b.q;  // TParticleA::SetCurrent
  b.x0 = pos;
  b.u0 = unit(dir);
  b.e0 = a->energy_gev;
  b.t0 = a->t0;
  // TParticleBeam::SetSigma (TParticleBeam.cc:137-158)
  b.hdir = unit(h);
  b.vdir = unit(cross(b.u0, b.hdir));
  if (fabs(dot(b.hdir, b.u0)) > 0.00000001)
    return fail(SRS_ERR_INVALID, "horizontal_direction is not perpendicular to the beam direction");
  b.su[0] = su0; b.su[1] = su1;
  b.sup[0] = sp0; b.sup[1] = sp1;
  b.sigma_at = vec(a->lattice_reference);
  b.sigma_e = a->sigma_energy_gev;
  sim->weight_sums.push_back(sim->weight_sums.empty() ? a->weight : sim->weight_sums.back() + a->weight);
  sim->beams.push_back(b);
  sim->beam_index[b.name] = sim->beams.size() - 1;
  return SRS_OK;
}

srs_status srs_sim_clear_particle_beams(srs_sim *sim) {
  SIM_GUARD(sim);
  sim->beams.clear();
  sim->weight_sums.clear();
  sim->beam_index.clear();
  return SRS_OK;
}

int32_t srs_sim_get_nparticle_beams(srs_sim *sim) { return sim ? (int32_t)sim->beams.size() : 0; }

// OSCARSSR::SetNewParticle(BeamName, IdealOrRandom) (OSCARSSR.cc:398-412) / SetNewParticle() (:386-394)
srs_status srs_sim_set_new_particle(srs_sim *sim, const char *beam, const char *which) {
  SIM_GUARD(sim);
  const std::string b = beam ? beam : "", w = lower(which ? which : "");
  if (sim->beams.empty()) return fail(SRS_ERR_RANGE, "no beam defined");
  if (b.empty() && w.empty()) return sim->new_random_particle(sim->particle);
  size_t idx;
  if (b.empty()) {
    if (srs_status st = sim->random_beam_index(idx)) return st;
  } else {
    auto it = sim->beam_index.find(b);
    if (it == sim->beam_index.end()) return fail(SRS_ERR_RANGE, "'beam' name not found");
    idx = it->second;
  }
  sim->particle = w == "ideal" ? sim->beams[idx].ideal() : sim->beams[idx].random();
  return SRS_OK;
}

srs_status srs_sim_get_particle(srs_sim *sim, double x0[3], double beta0[3], double *e0, double *gamma) {
  SIM_GUARD(sim);
  if (!sim->particle.set) return fail(SRS_ERR_RANGE, "particle not initialized.  make sure you have a particle or beam defined");
  if (x0) put(x0, sim->particle.x0);
  if (beta0) put(beta0, sim->particle.b0);
  if (e0) *e0 = kg_to_gev(sim->particle.m) * sim->particle.gamma;
  if (gamma) *gamma = sim->particle.gamma;
  return SRS_OK;
}

void srs_set_seed(double seed) {
  GlobalRandom &r = rng();
  std::lock_guard<std::mutex> lk(r.mu);
  r.mt.reset(new std::mt19937((int)seed));  // TRandomA::SetSeed(int)
}
void srs_random_reset(double seed) {
  GlobalRandom &r = rng();
  std::lock_guard<std::mutex> lk(r.mu);
  r.mt.reset(new std::mt19937((int)seed));
  r.normal.reset();
}
double srs_random_uniform(void) {
  GlobalRandom &r = rng();
  std::lock_guard<std::mutex> lk(r.mu);
  return r.uniform(*r.mt);
}
double srs_random_normal(void) {
  GlobalRandom &r = rng();
  std::lock_guard<std::mutex> lk(r.mu);
  return r.normal(*r.mt);
}

srs_status srs_sim_calculate_trajectory(srs_sim *sim, int64_t *n, double *x, double *beta) {
  SIM_GUARD(sim);
  if (!n) return fail(SRS_ERR_INVALID, "NULL argument");
  if (srs_status st = sim->ensure_particle()) return st;
  double dt;
  int64_t nf, nb;
  if (srs_status st = srs_trajectory_counts(sim->ctstart, sim->ctstop, sim->particle.t0, sim->npoints, &dt, &nf, &nb))
    return st;
  if (!x || !beta) {
    *n = nf + nb;
    return SRS_OK;
  }
  if (*n != nf + nb) return fail(SRS_ERR_INVALID, "output size does not match the trajectory");
  srs_traj_view v;
  if (srs_status st = sim->single(sim->particle, v, sim->shoot_for(SRS_PRECISION_FP64))) return st;
  std::vector<double> hx(3 * v.n), hb(3 * v.n);
  SRS_CUDA(cudaMemcpyAsync(hx.data(), v.x, sizeof(double) * 3 * v.n, cudaMemcpyDeviceToHost, sim->stream));
  SRS_CUDA(cudaMemcpyAsync(hb.data(), v.beta, sizeof(double) * 3 * v.n, cudaMemcpyDeviceToHost, sim->stream));
  SRS_CUDA(cudaStreamSynchronize(sim->stream));
  for (int64_t i = 0; i < v.n; ++i)
    for (int c = 0; c < 3; ++c) {
      x[3 * i + c] = hx[c * v.n + i];
      beta[3 * i + c] = hb[c * v.n + i];
    }
  return SRS_OK;
}

srs_status srs_sim_calculate_spectrum(srs_sim *sim, const double obs[3], const double *energies, int64_t ne,
                                      int32_t nparticles, int32_t precision, double *out, double *comp) {
  SIM_GUARD(sim);
  if (!obs || !energies || !out || ne < 1) return fail(SRS_ERR_INVALID, "bad argument");
  if (nparticles < 0) return fail(SRS_ERR_INVALID, "'nparticles' must be >= 1 (sort of)");
  DeviceBuffer de;
  SRS_CUDA(de.alloc(sizeof(double) * ne, sim->stream));
  SRS_CUDA(cudaMemcpyAsync(de.ptr, energies, sizeof(double) * ne, cudaMemcpyHostToDevice, sim->stream));
  const double *d_e = de.as<double>();
  cudaStream_t s = sim->stream;
  return sim->run(nparticles, ne, out, comp, true, precision,
                  [&](const srs_traj_view &v, const srs_beam_consts &bc, double *dv) {
    return srs_spectrum(v, bc, obs, d_e, ne, precision, dv, s);
  });
}

srs_status srs_sim_calculate_flux(srs_sim *sim, const double *points, int64_t np, const srs_grid2d *grid,
                                  double energy_ev, int32_t nparticles, int32_t precision, double *out, double *comp) {
  SIM_GUARD(sim);
  if (!out || np < 1 || (!points && !grid)) return fail(SRS_ERR_INVALID, "bad argument");
  if (nparticles < 0) return fail(SRS_ERR_INVALID, "'nparticles' must be >= 1 (sort of)");
  DeviceBuffer dp;
  const double *d_p = nullptr;
  if (points && !(precision == SRS_PRECISION_MIXED && grid)) {  // the mixed kernel walks the grid itself
    SRS_CUDA(dp.alloc(sizeof(double) * 3 * np, sim->stream));
    SRS_CUDA(cudaMemcpyAsync(dp.ptr, points, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, sim->stream));
    d_p = dp.as<double>();
  }
  cudaStream_t s = sim->stream;
  return sim->run(nparticles, np, out, comp, true, precision,
                  [&](const srs_traj_view &v, const srs_beam_consts &bc, double *dv) {
    return srs_flux(v, bc, d_p, np, grid, energy_ev, precision, dv, s);
  });
}

srs_status srs_sim_calculate_flux_plane(srs_sim *sim, const char *plane, int32_t n1, int32_t n2, double w1,
                                        double w2, const double rotations[3], const double translation[3],
                                        int32_t normal, double energy_ev, int32_t nparticles, int32_t precision,
                                        double *out, double *comp, double *xyz, double *x12, double nrm[3]) {
  SIM_GUARD(sim);
  if (!out) return fail(SRS_ERR_INVALID, "bad argument");
  if (nparticles < 0) return fail(SRS_ERR_INVALID, "'nparticles' must be >= 1 (sort of)");
  const double zero[3] = {0, 0, 0};
  if (!rotations) rotations = zero;
  if (!translation) translation = zero;
  srs_grid2d grid;
  double nv[3];
  if (srs_status st = srs_rectangle_plane(plane, n1, n2, w1, w2, rotations, translation, normal, nullptr, nullptr,
                                          nv, &grid))
    return st;
  if (nrm) std::memcpy(nrm, nv, sizeof nv);
  const int64_t np = (int64_t)n1 * n2;
  // the points: built while the GPU computes when the mixed kernel walks the grid, else first (uploaded)
  auto emit = [&](double *p, double *q) {
    srs_rectangle_plane(plane, n1, n2, w1, w2, rotations, translation, normal, p, q, nullptr, nullptr);
  };
  const bool walk = precision == SRS_PRECISION_MIXED;
  DeviceBuffer dp;
  const double *d_p = nullptr;
  std::vector<double> tmp;
  if (!walk) {
    double *p = xyz;
    if (!p) {
      tmp.resize((size_t)(3 * np));
      p = tmp.data();
    }
    emit(p, x12);
    SRS_CUDA(dp.alloc(sizeof(double) * 3 * np, sim->stream));
    SRS_CUDA(cudaMemcpyAsync(dp.ptr, p, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, sim->stream));
    d_p = dp.as<double>();
  }
  cudaStream_t s = sim->stream;
  const std::function<void()> host_work = [&]() {
    if (walk && (xyz || x12)) emit(xyz, x12);
  };
  return sim->run(
      nparticles, np, out, comp, true, precision,
      [&](const srs_traj_view &v, const srs_beam_consts &bc, double *dv) {
        return srs_flux(v, bc, d_p, np, &grid, energy_ev, precision, dv, s);
      },
      host_work);
}

srs_status srs_sim_calculate_power_density(srs_sim *sim, const double *points, const double *normals, int64_t np,
                                           const srs_grid2d *grid, int32_t directional, int32_t nparticles,
                                           int32_t weighted, int32_t precision, double *out, double *comp) {
  SIM_GUARD(sim);
  if (!points || !normals || !out || np < 1) return fail(SRS_ERR_INVALID, "bad argument");
  if (nparticles < 0) return fail(SRS_ERR_INVALID, "'nparticles' must be >= 1 (sort of)");
  DeviceBuffer dp;
  const double *d_p = nullptr, *d_n = nullptr;
  if (!(precision == SRS_PRECISION_MIXED && grid)) {  // the mixed kernel walks the grid itself
    SRS_CUDA(dp.alloc(sizeof(double) * 6 * np, sim->stream));
    SRS_CUDA(cudaMemcpyAsync(dp.ptr, points, sizeof(double) * 3 * np, cudaMemcpyHostToDevice, sim->stream));
    SRS_CUDA(cudaMemcpyAsync(dp.as<double>() + 3 * np, normals, sizeof(double) * 3 * np, cudaMemcpyHostToDevice,
                             sim->stream));
    d_p = dp.as<double>();
    d_n = d_p + 3 * np;
  }
  cudaStream_t s = sim->stream;
  return sim->run(nparticles, np, out, comp, weighted != 0, precision,
                  [&](const srs_traj_view &v, const srs_beam_consts &bc, double *dv) {
                    return srs_power_density(v, bc, d_p, d_n, np, grid, directional, precision, dv, s);
                  });
}

srs_status srs_sim_calculate_total_power(srs_sim *sim, double *out) {
  SIM_GUARD(sim);
  if (!out) return fail(SRS_ERR_INVALID, "NULL output");
  if (srs_status st = sim->ensure_particle()) return st;
  srs_traj_view v;
  if (srs_status st = sim->single(sim->particle, v, sim->shoot_for(SRS_PRECISION_FP64))) return st;
  srs_beam_consts bc{sim->particle.q, sim->particle.current};
  return srs_total_power(v, bc, &sim->particle.gamma, out, sim->stream);
}

// ---------------------------------------------------------------- geometry (host)

srs_status srs_energy_grid(int64_t n, double e0, double e1, double *out) {
  clear_error();
  if (n < 1 || !out) return fail(SRS_ERR_INVALID, "'npoints' must be > 0");
  if (n == 1) {
    out[0] = e0;
    return SRS_OK;
  }
  for (int64_t i = 0; i < n; ++i) out[i] = e0 + (e1 - e0) / (double)(size_t)(n - 1) * (double)(i + 1);
  return SRS_OK;
}

static void rect_emit(int n1, int n2, V3 start, V3 v1, V3 v2, double s1, double s2, V3 nv, double *xyz, double *x12,
                      double nrm[3], srs_grid2d *grid) {
  // the offsets of GetX1 / GetX2 (:244-259) do not depend on the point: computed once, same values
  const double off1 = mag(v1) * (n1 - 1) / 2., off2 = mag(v2) * (n2 - 1) / 2.;
  size_t i = 0;
  for (int i1 = 0; i1 < n1; ++i1) {
    const V3 row = start + v1 * (double)i1;
    const double a1 = s1 * i1 - off1;
    for (int i2 = 0; i2 < n2; ++i2, ++i) {
      const V3 p = row + v2 * (double)i2;  // TSurfacePoints_Rectangle.cc:222-230: start + v1 i1 + v2 i2
      if (xyz) put(xyz + 3 * i, p);
      if (x12) {
        x12[2 * i] = a1;
        x12[2 * i + 1] = s2 * i2 - off2;
      }
    }
  }
  if (nrm) put(nrm, unit(nv));  // TSurfacePoint normalises the normal again
  if (grid) {
    put(grid->origin, start);
    put(grid->u1, v1);
    put(grid->u2, v2);
    put(grid->normal, unit(nv));
    grid->n1 = n1;
    grid->n2 = n2;
  }
}

srs_status srs_rectangle_plane(const char *plane, int32_t n1, int32_t n2, double w1, double w2,
                               const double rotations[3], const double translation[3], int32_t normal, double *xyz,
                               double *x12, double nrm[3], srs_grid2d *grid) {
  clear_error();
  if (!plane) return fail(SRS_ERR_INVALID, "not a valid surface string: XY YX XZ ZX YZ ZY");
  if (n1 < 1 || n2 < 1) return fail(SRS_ERR_INVALID, "an entry in 'npoints' is <= 0");
  const std::string P = upper(plane);
  const double s1 = w1 / (n1 - 1), s2 = w2 / (n2 - 1);  // TSurfacePoints_Rectangle.cc:150-152
  V3 start, v1, v2;
  if (P == "XY") { start = v3(-w1 / 2., -w2 / 2., 0); v1 = v3(s1, 0, 0); v2 = v3(0, s2, 0); }
  else if (P == "YX") { start = v3(-w2 / 2., -w1 / 2., 0); v2 = v3(s2, 0, 0); v1 = v3(0, s1, 0); }
  else if (P == "XZ") { start = v3(-w1 / 2., 0, -w2 / 2.); v1 = v3(s1, 0, 0); v2 = v3(0, 0, s2); }
  else if (P == "ZX") { start = v3(-w2 / 2., 0, -w1 / 2.); v2 = v3(s2, 0, 0); v1 = v3(0, 0, s1); }
  else if (P == "YZ") { start = v3(0, -w1 / 2., -w2 / 2.); v1 = v3(0, s1, 0); v2 = v3(0, 0, s2); }
  else if (P == "ZY") { start = v3(0, -w2 / 2., -w1 / 2.); v2 = v3(0, s2, 0); v1 = v3(0, 0, s1); }
  else return fail(SRS_ERR_INVALID, "not a valid surface string: XY YX XZ ZX YZ ZY");
  start = rot(start, rotations);
  v1 = rot(v1, rotations);
  v2 = rot(v2, rotations);
  start = start + vec(translation);
  V3 nv = unit(cross(v1, v2));
  if (normal == -1) nv = nv * -1;
  else if (normal != 0 && normal != 1) return fail(SRS_ERR_INVALID, "normal must be -1, 0, or 1");
  rect_emit(n1, n2, start, v1, v2, s1, s2, nv, xyz, x12, nrm, grid);
  return SRS_OK;
}

srs_status srs_rectangle_points(int32_t n1, int32_t n2, const double x0[3], const double x1[3], const double x2[3],
                                const double rotations[3], const double translation[3], int32_t normal, double *xyz,
                                double *x12, double nrm[3], srs_grid2d *grid) {
  clear_error();
  if (n1 < 1 || n2 < 1) return fail(SRS_ERR_INVALID, "an entry in 'npoints' is <= 0");
  V3 p0 = rot(vec(x0), rotations) + vec(translation);  // OSCARSSR_Python.cc:2712-2715
  V3 p1 = rot(vec(x1), rotations) + vec(translation);
  V3 p2 = rot(vec(x2), rotations) + vec(translation);
  const double w1 = mag(p1 - p0), w2 = mag(p2 - p0);  // TSurfacePoints_Rectangle.cc:95-107
  const double s1 = w1 / (n1 - 1), s2 = w2 / (n2 - 1);
  V3 v1 = (p1 - p0) / (double)(n1 - 1), v2 = (p2 - p0) / (double)(n2 - 1);
  V3 nv = unit(cross(v1, v2));
  if (normal == -1) nv = nv * -1;
  else if (normal != 0 && normal != 1) return fail(SRS_ERR_INVALID, "normal must be -1, 0, or 1");
  rect_emit(n1, n2, p0, v1, v2, s1, s2, nv, xyz, x12, nrm, grid);
  return SRS_OK;
}

}  // extern "C"

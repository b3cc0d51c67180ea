// Heterogeneous jobs in one persistent launch: a work queue of (job, tile, trajectory chunk) items.
//
// Jobs of very different sizes (a 64-point map next to a 40401-point one, 100 energies next to 4000,
// trajectories of 5001 to 40001 points) are cut into items of the same shape as the one-shot mixed
// kernels' CTAs -- a tile of up to 128 grid points or 512 energies against one chunk of the trajectory.
// The host orders the items by decreasing cost (longest-processing-time first), and a grid of
// resident CTAs (one wave: SMs x CTAs per SM) drains them: each CTA takes the next item with one
// atomicAdd on a ticket and runs it.  No CTA waits on another (no spin), so the launch always ends.
// A second kernel adds every job's per-chunk partial sums in chunk order and writes the flux.
//
// The launch sequence (ticket reset, queue kernel, finishing kernel) is captured once into a CUDA
// graph on the queue's own stream and replayed by every srs_queue_run; the caller's stream is joined
// with events on both sides.
//
// A queue may also integrate its jobs' trajectories (srs_queue_create_shaped with particles): the jobs
// are split into groups by trajectory length, and each group is one branch of the graph: its
// trajectories integrated parallel in time (rk4_shoot.cu, ~0.3-0.6 ms each where the serial chain takes
// ~1 us per step), one after another, then a queue kernel over the group's items.  The branches run
// concurrently, so the first groups' sums start after a few milliseconds while the other branches
// are still integrating; they join before the finishing kernel.  The dependencies are graph edges
// only: no kernel waits on another.
//
// The tile shape is a parameter (srs_queue_shape): trajectory points per item, resident CTAs per SM,
// energies per thread of the spectrum items (2 or 4) and the widest strip of the flux items' tiles
// (8..16); queue.py's autotuner times candidate shapes on the jobs themselves.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <numeric>
#include <vector>

#include "mixed_tiles.cuh"
#include "srs_device.cuh"
#include "srs_internal.h"

namespace srs {
namespace {

using namespace tiles;

struct QJob {
  int kind;
  StripTiles tiles;  // flux: the map's tiles
  int64_t chunk;   // trajectory points per item
  const double *x, *beta;
  int64_t n;
  double dt;
  double omega;    // flux
  srs_grid2d g;    // flux
  V3 obs;          // spectrum
  const double *omegas;  // spectrum (device, ne)
  int64_t ne;
  double *partial;  // nchunks x 6 x nout
  int64_t nout;
  int nchunks;
  double C0, C2;
  double *out;
};

struct QItem {
  int job, tile, chunk, pad;
};

template <int K>
__global__ void __launch_bounds__(kThreads) queue_kernel(const QJob *__restrict__ jobs, const QItem *__restrict__ items,
                                                         int nitems, unsigned int *__restrict__ ticket) {
  __shared__ union {
    FluxShared f;
    SpecShared s;
  } sh;
  __shared__ int cur;
  for (;;) {
    __syncthreads();  // every thread is done with the previous item (and with `cur`)
    if (threadIdx.x == 0) cur = (int)atomicAdd(ticket, 1u);
    __syncthreads();
    const int it = cur;
    if (it >= nitems) return;  // uniform across the CTA
    const QItem w = items[it];
    const QJob &J = jobs[w.job];
    const int64_t i0 = (int64_t)w.chunk * J.chunk, i1 = imin64(J.n, i0 + J.chunk);
    double *out6 = J.partial + (int64_t)w.chunk * 6 * J.nout;
    if (J.kind == SRS_JOB_FLUX)
      flux_tile(J.x, J.beta, J.n, J.dt, J.g, J.tiles, J.omega, w.tile, i0, i1, out6, sh.f);
    else
      spectrum_tile<K>(J.x, J.beta, J.n, J.dt, J.obs, J.omegas, J.ne, w.tile, i0, i1, out6, sh.s);
  }
}

// out[o] of every job: the chunk partials added in chunk order, then the reference's final scaling.
__global__ void queue_finish(const QJob *__restrict__ jobs, int njobs, const int64_t *__restrict__ offsets,
                             int64_t total) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  int lo = 0, hi = njobs - 1;  // job with offsets[job] <= idx < offsets[job + 1]
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (offsets[mid] <= idx) lo = mid;
    else hi = mid - 1;
  }
  const QJob &J = jobs[lo];
  const int64_t o = idx - offsets[lo];
  double e[6] = {0, 0, 0, 0, 0, 0};
  for (int s = 0; s < J.nchunks; ++s) {
    const double *p = J.partial + (int64_t)s * 6 * J.nout + o;
#pragma unroll
    for (int c = 0; c < 6; ++c) e[c] += p[c * J.nout];
  }
  const double omega = J.kind == SRS_JOB_FLUX ? J.omega : J.omegas[o];
  J.out[o] = finish_flux(e, omega, J.dt, J.C0, J.C2);
}

__global__ void omegas_of(const double *__restrict__ e, int64_t ne, double *__restrict__ w) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ne) w[i] = ev_to_omega(e[i]);
}

}  // namespace
}  // namespace srs

using namespace srs;

struct srs_queue {
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  QJob *d_jobs = nullptr;
  QItem *d_items = nullptr;
  int64_t *d_offsets = nullptr;
  unsigned int *d_ticket = nullptr;  // one per group
  double *d_scratch = nullptr;       // partials, then the spectrum jobs' angular frequencies
  int njobs = 0, nitems = 0, grid = 0, K = kEnergiesPerThread, per_sm = 1, sms = 148, seg_steps = 16;
  int64_t total_out = 0;
  double evals = 0;
  size_t scratch_bytes = 0;
  // groups: items [gofs[g], gofs[g + 1]) belong to group g (one group without trajectories)
  std::vector<int> gofs;
  // the trajectories to integrate (optional): fields, and per group its particles and specs
  bool integrate = false;
  srs_field *d_fields = nullptr;
  int nfields = 0;
  int64_t stage = 0;
  bool electric = false;
  srs_particle *d_particles = nullptr;  // ordered by group
  struct Shoot {                        // one trajectory to integrate (parallel in time)
    srs_particle host;
    int index;                          // into d_particles
    double dt;
    int64_t nf, nb;
    double *x, *b, *a;
  };
  std::vector<std::vector<Shoot>> shoots;  // per group
  std::vector<void *> shoot_scratch;       // per group (its trajectories run one after another)
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> ev_join;
  cudaEvent_t ev_fork = nullptr;

  ~srs_queue() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (void *p : {(void *)d_jobs, (void *)d_items, (void *)d_offsets, (void *)d_ticket, (void *)d_scratch,
                    (void *)d_fields, (void *)d_particles})
      if (p) cudaFree(p);
    for (void *p : shoot_scratch)
      if (p) cudaFree(p);
    for (cudaEvent_t e : ev_join)
      if (e) cudaEventDestroy(e);
    for (cudaStream_t a : aux)
      if (a) cudaStreamDestroy(a);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (stream) cudaStreamDestroy(stream);
  }
};

extern "C" {

srs_status srs_queue_create_shaped(srs_queue **out, const srs_job *jobs, int32_t njobs, const srs_queue_shape *shape,
                                   const srs_field *fields, int32_t nfields, const srs_particle *particles,
                                   const double *ctstart, const double *ctstop, const double *t0,
                                   const int64_t *npoints) {
  clear_error();
  if (!out || !jobs || njobs < 1 || !shape) return fail(SRS_ERR_INVALID, "no jobs or no shape");
  int32_t chunk = shape->chunk;
  if (chunk < 128) return fail(SRS_ERR_INVALID, "chunk must be >= 128 trajectory points");
  chunk = (int32_t)aligned_chunk(chunk, 1);  // whole shared-memory sub-tiles (see aligned_chunk)
  const int K = shape->energies_per_thread == 0 ? kEnergiesPerThread : shape->energies_per_thread;
  if (K != 2 && K != 4) return fail(SRS_ERR_INVALID, "energies_per_thread must be 2 or 4 (or 0)");
  const int wmax = shape->strip_width == 0 ? 16 : shape->strip_width;
  if (wmax < 8 || wmax > 16) return fail(SRS_ERR_INVALID, "strip_width must be 8..16 (or 0)");
  const bool integrate = particles != nullptr;
  if (integrate && (!ctstart || !ctstop || !t0 || !npoints || nfields < 0 || (nfields > 0 && !fields)))
    return fail(SRS_ERR_INVALID, "trajectories: particles, ctstart, ctstop, t0, npoints and fields needed");
  constexpr int kRk4MaxFields = 16;  // the RK4 kernels copy the field list to shared memory
  if (integrate && nfields > kRk4MaxFields)
    return fail(SRS_ERR_RANGE, "trajectories: at most " + std::to_string(kRk4MaxFields) + " fields");
  int groups = integrate ? (shape->groups == 0 ? 16 : shape->groups) : 1;
  const int seg_steps = shape->steps_per_segment == 0 ? 16 : shape->steps_per_segment;
  if (seg_steps < 1) return fail(SRS_ERR_INVALID, "steps_per_segment must be >= 1 (or 0)");
  if (groups < 1) return fail(SRS_ERR_INVALID, "groups must be >= 1");
  groups = std::min(groups, (int)njobs);
  std::unique_ptr<srs_queue> q(new srs_queue());
  q->K = K;
  q->seg_steps = seg_steps;
  std::vector<QJob> hj(njobs);
  std::vector<int64_t> offsets(njobs + 1, 0);
  // group of each job: by trajectory length (shortest first), equal numbers of jobs per group
  std::vector<int> order(njobs), group_of(njobs, 0);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].traj.n < jobs[b].traj.n; });
  for (int r = 0; r < njobs; ++r) group_of[order[r]] = (int)((int64_t)r * groups / njobs);
  size_t scratch = 0, omega_doubles = 0;
  struct Cost {
    double cost;
    QItem item;
  };
  std::vector<std::vector<Cost>> items(groups);
  for (int j = 0; j < njobs; ++j) {
    const srs_job &s = jobs[j];
    if (!s.traj.x || !s.traj.beta || s.traj.n < 1 || !(s.traj.dt > 0) || !s.d_out)
      return fail(SRS_ERR_INVALID, "job " + std::to_string(j) + ": bad trajectory or output");
    QJob &J = hj[j];
    std::memset(&J, 0, sizeof J);
    J.kind = s.kind;
    J.chunk = chunk;
    J.x = s.traj.x;
    J.beta = s.traj.beta;
    J.n = s.traj.n;
    J.dt = s.traj.dt;
    J.C0 = flux_c0(s.beam.charge);
    J.C2 = flux_c2(s.beam.charge, s.beam.current);
    J.out = s.d_out;
    J.nchunks = (int)((s.traj.n + chunk - 1) / chunk);
    int ntiles;
    double per_item;
    if (s.kind == SRS_JOB_FLUX) {
      if (s.grid.n1 < 1 || s.grid.n2 < 1 || !(s.energy_ev > 0))
        return fail(SRS_ERR_INVALID, "job " + std::to_string(j) + ": bad flux grid or energy");
      J.g = s.grid;
      J.omega = ev_to_omega(s.energy_ev);
      J.tiles = strip_tiles(s.grid, wmax);
      ntiles = J.tiles.tiles;
      J.nout = (int64_t)s.grid.n1 * s.grid.n2;
      per_item = kThreads;
      q->evals += (double)J.nout * s.traj.n;
    } else if (s.kind == SRS_JOB_SPECTRUM) {
      if (s.ne < 1 || !s.d_energies) return fail(SRS_ERR_INVALID, "job " + std::to_string(j) + ": no energies");
      J.obs = v3(s.obs[0], s.obs[1], s.obs[2]);
      J.ne = s.ne;
      J.nout = s.ne;
      ntiles = (int)((s.ne + kThreads * K - 1) / (kThreads * K));
      per_item = 0.6 * kThreads * K;  // a uniform-grid energy costs ~0.6 of a map point
      omega_doubles += s.ne;
      q->evals += (double)J.nout * s.traj.n;
    } else {
      return fail(SRS_ERR_INVALID, "job " + std::to_string(j) + ": unknown kind");
    }
    scratch += (size_t)J.nchunks * 6 * J.nout;
    offsets[j + 1] = offsets[j] + J.nout;
    for (int t = 0; t < ntiles; ++t)
      for (int c = 0; c < J.nchunks; ++c) {
        const double len = (double)(std::min<int64_t>(s.traj.n, (int64_t)(c + 1) * chunk) - (int64_t)c * chunk);
        items[group_of[j]].push_back(Cost{per_item * len, QItem{j, t, c, 0}});
      }
  }
  // items: group after group, each group longest first
  std::vector<QItem> hi;
  q->gofs.assign(groups + 1, 0);
  for (int g = 0; g < groups; ++g) {
    std::stable_sort(items[g].begin(), items[g].end(), [](const Cost &a, const Cost &b) { return a.cost > b.cost; });
    for (const Cost &c : items[g]) hi.push_back(c.item);
    q->gofs[g + 1] = (int)hi.size();
  }
  if (hi.size() > (size_t)0x7fffffff) return fail(SRS_ERR_RANGE, "too many work items");
  q->njobs = njobs;
  q->nitems = (int)hi.size();
  q->total_out = offsets[njobs];
  q->scratch_bytes = sizeof(double) * (scratch + omega_doubles);
  SRS_CUDA(cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking));
  SRS_CUDA(cudaEventCreateWithFlags(&q->ev_in, cudaEventDisableTiming));
  SRS_CUDA(cudaEventCreateWithFlags(&q->ev_out, cudaEventDisableTiming));
  SRS_CUDA(cudaEventCreateWithFlags(&q->ev_fork, cudaEventDisableTiming));
  q->aux.assign(groups, nullptr);
  q->ev_join.assign(groups, nullptr);
  for (int g = 0; g < groups; ++g) {
    SRS_CUDA(cudaStreamCreateWithFlags(&q->aux[g], cudaStreamNonBlocking));
    SRS_CUDA(cudaEventCreateWithFlags(&q->ev_join[g], cudaEventDisableTiming));
  }
  SRS_CUDA(cudaMalloc(&q->d_scratch, q->scratch_bytes));
  SRS_CUDA(cudaDeviceSynchronize());  // the energies may still be being written on the caller's stream
  // carve partials and angular frequencies
  size_t off = 0;
  for (int j = 0; j < njobs; ++j) {
    hj[j].partial = q->d_scratch + off;
    off += (size_t)hj[j].nchunks * 6 * hj[j].nout;
  }
  for (int j = 0; j < njobs; ++j)
    if (hj[j].kind == SRS_JOB_SPECTRUM) {
      double *w = q->d_scratch + off;
      omegas_of<<<(unsigned)((hj[j].ne + 255) / 256), 256, 0, q->stream>>>(jobs[j].d_energies, hj[j].ne, w);
      SRS_CUDA(cudaGetLastError());
      hj[j].omegas = w;
      off += hj[j].ne;
    }
  SRS_CUDA(cudaMalloc(&q->d_jobs, sizeof(QJob) * njobs));
  SRS_CUDA(cudaMalloc(&q->d_items, sizeof(QItem) * std::max<size_t>(1, hi.size())));
  SRS_CUDA(cudaMalloc(&q->d_offsets, sizeof(int64_t) * (njobs + 1)));
  SRS_CUDA(cudaMalloc(&q->d_ticket, sizeof(unsigned int) * groups));
  SRS_CUDA(cudaMemcpyAsync(q->d_jobs, hj.data(), sizeof(QJob) * njobs, cudaMemcpyHostToDevice, q->stream));
  SRS_CUDA(cudaMemcpyAsync(q->d_items, hi.data(), sizeof(QItem) * hi.size(), cudaMemcpyHostToDevice, q->stream));
  SRS_CUDA(cudaMemcpyAsync(q->d_offsets, offsets.data(), sizeof(int64_t) * (njobs + 1), cudaMemcpyHostToDevice,
                           q->stream));
  if (integrate) {
    // the jobs' particles, ordered by group, and per group the trajectories to integrate into the jobs'
    // views with one scratch area (sized for the group's longest)
    std::vector<srs_particle> hp;
    q->shoots.assign(groups, {});
    q->shoot_scratch.assign(groups, nullptr);
    for (int g = 0; g < groups; ++g) {
      size_t need = 0;
      for (int j = 0; j < njobs; ++j) {
        if (group_of[j] != g) continue;
        double dt;
        int64_t nf, nb;
        if (srs_status st = srs_trajectory_counts(ctstart[j], ctstop[j], t0[j], npoints[j], &dt, &nf, &nb)) return st;
        if (nf + nb != jobs[j].traj.n || !jobs[j].traj.aoc)
          return fail(SRS_ERR_INVALID, "job " + std::to_string(j) + ": its trajectory view does not hold the " +
                                           std::to_string(nf + nb) + " points to integrate (or has no a/c array)");
        q->shoots[g].push_back(srs_queue::Shoot{particles[j], (int)hp.size(), dt, nf, nb,
                                                const_cast<double *>(jobs[j].traj.x),
                                                const_cast<double *>(jobs[j].traj.beta),
                                                const_cast<double *>(jobs[j].traj.aoc)});
        hp.push_back(particles[j]);
        need = std::max(need, shoot_scratch_bytes(nf, nb, seg_steps, nfields));
      }
      if (need > 0) SRS_CUDA(cudaMalloc(&q->shoot_scratch[g], need));
    }
    q->integrate = true;
    q->nfields = nfields;
    SRS_CUDA(cudaMalloc(&q->d_fields, sizeof(srs_field) * std::max(1, nfields)));
    SRS_CUDA(cudaMalloc(&q->d_particles, sizeof(srs_particle) * hp.size()));
    if (nfields > 0)
      SRS_CUDA(cudaMemcpyAsync(q->d_fields, fields, sizeof(srs_field) * nfields, cudaMemcpyHostToDevice, q->stream));
    SRS_CUDA(cudaMemcpyAsync(q->d_particles, hp.data(), sizeof(srs_particle) * hp.size(), cudaMemcpyHostToDevice,
                             q->stream));
    q->stage = nfields > 0 ? grid_stage_doubles(fields, nfields) : 0;
    q->electric = nfields > 0 && has_electric(fields, nfields);
    if (q->electric)
      return fail(SRS_ERR_INVALID, "trajectories: the queue integrates magnetic fields only (parallel in time)");
  }
  SRS_CUDA(cudaStreamSynchronize(q->stream));
  int dev = 0, sms = 0, occ = 0;
  SRS_CUDA(cudaGetDevice(&dev));
  SRS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (K == 2)
    SRS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, queue_kernel<2>, kThreads, 0));
  else
    SRS_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, queue_kernel<4>, kThreads, 0));
  q->sms = sms;
  q->per_sm = shape->ctas_per_sm > 0 ? std::min(shape->ctas_per_sm, std::max(1, occ)) : std::max(1, occ);
  q->grid = std::max(1, std::min(sms * q->per_sm, q->nitems));
  *out = q.release();
  return SRS_OK;
}

srs_status srs_queue_create(srs_queue **out, const srs_job *jobs, int32_t njobs, int32_t chunk,
                            int32_t ctas_per_sm) {
  const srs_queue_shape shape{chunk, ctas_per_sm, 0, 0, 1, 0};
  return srs_queue_create_shaped(out, jobs, njobs, &shape, nullptr, 0, nullptr, nullptr, nullptr, nullptr, nullptr);
}

srs_status srs_queue_run(srs_queue *q, void *stream) {
  clear_error();
  if (!q) return fail(SRS_ERR_INVALID, "NULL queue");
  cudaStream_t caller = static_cast<cudaStream_t>(stream);
  SRS_CUDA(cudaEventRecord(q->ev_in, caller));
  SRS_CUDA(cudaStreamWaitEvent(q->stream, q->ev_in, 0));
  if (!q->exec) {
    const int groups = (int)q->gofs.size() - 1;
    SRS_CUDA(cudaStreamBeginCapture(q->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t launch = cudaMemsetAsync(q->d_ticket, 0, sizeof(unsigned int) * groups, q->stream);
    if (launch == cudaSuccess) launch = cudaEventRecord(q->ev_fork, q->stream);
    for (int g = 0; g < groups && launch == cudaSuccess; ++g) {
      // branch g: this group's trajectories, then its items
      cudaStream_t a = q->aux[g];
      launch = cudaStreamWaitEvent(a, q->ev_fork, 0);
      if (q->integrate)
        for (const srs_queue::Shoot &t : q->shoots[g]) {
          if (launch != cudaSuccess) break;
          launch = launch_rk4_shoot(q->d_fields, q->nfields, q->d_particles + t.index, t.host, t.dt, t.nf, t.nb, t.x,
                                    t.b, t.a, a, q->stage, q->seg_steps, 0, q->shoot_scratch[g], nullptr);
        }
      const int n_g = q->gofs[g + 1] - q->gofs[g];
      if (launch == cudaSuccess && n_g > 0) {
        const int grid = std::max(1, std::min(q->sms * q->per_sm, n_g));
        if (q->K == 2)
          queue_kernel<2><<<grid, kThreads, 0, a>>>(q->d_jobs, q->d_items + q->gofs[g], n_g, q->d_ticket + g);
        else
          queue_kernel<4><<<grid, kThreads, 0, a>>>(q->d_jobs, q->d_items + q->gofs[g], n_g, q->d_ticket + g);
        launch = cudaGetLastError();
      }
      if (launch == cudaSuccess) launch = cudaEventRecord(q->ev_join[g], a);
      if (launch == cudaSuccess) launch = cudaStreamWaitEvent(q->stream, q->ev_join[g], 0);
    }
    if (launch == cudaSuccess) {
      queue_finish<<<(unsigned)((q->total_out + 255) / 256), 256, 0, q->stream>>>(q->d_jobs, q->njobs, q->d_offsets,
                                                                                   q->total_out);
      launch = cudaGetLastError();
    }
    cudaError_t end = cudaStreamEndCapture(q->stream, &q->graph);
    if (launch != cudaSuccess) return cuda_fail(launch, "capture of the queue launches");
    if (end != cudaSuccess) return cuda_fail(end, "cudaStreamEndCapture");
    SRS_CUDA(cudaGraphInstantiate(&q->exec, q->graph, 0));
  }
  SRS_CUDA(cudaGraphLaunch(q->exec, q->stream));
  SRS_CUDA(cudaEventRecord(q->ev_out, q->stream));
  SRS_CUDA(cudaStreamWaitEvent(caller, q->ev_out, 0));
  return SRS_OK;
}

srs_status srs_queue_info(srs_queue *q, int64_t *nitems, double *evals, size_t *scratch_bytes, int32_t *grid) {
  clear_error();
  if (!q) return fail(SRS_ERR_INVALID, "NULL queue");
  if (nitems) *nitems = q->nitems;
  if (evals) *evals = q->evals;
  if (scratch_bytes) *scratch_bytes = q->scratch_bytes;
  if (grid) *grid = q->grid;
  return SRS_OK;
}

void srs_queue_destroy(srs_queue *q) { delete q; }

srs_status srs_trajectory_batch(const srs_field *fields, int32_t nfields, const srs_particle *particles,
                                int32_t nparticles, const double *ctstart, const double *ctstop, const double *t0,
                                const int64_t *npoints, double *const *d_x, double *const *d_beta,
                                double *const *d_aoc, void *stream) {
  clear_error();
  if (nparticles < 1 || !particles || !ctstart || !ctstop || !t0 || !npoints || !d_x || !d_beta || !d_aoc)
    return fail(SRS_ERR_INVALID, "bad argument");
  if (nfields < 0 || (nfields > 0 && !fields)) return fail(SRS_ERR_INVALID, "bad field array");
  std::vector<TrajSpec> specs(nparticles);
  for (int p = 0; p < nparticles; ++p) {
    double dt;
    int64_t nf, nb;
    if (srs_status st = srs_trajectory_counts(ctstart[p], ctstop[p], t0[p], npoints[p], &dt, &nf, &nb)) return st;
    if (!d_x[p] || !d_beta[p] || !d_aoc[p]) return fail(SRS_ERR_INVALID, "NULL output pointer");
    specs[p] = TrajSpec{dt, nf, nb, d_x[p], d_beta[p], d_aoc[p]};
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  DeviceBuffer df, dp, ds;
  SRS_CUDA(df.alloc(sizeof(srs_field) * std::max(1, nfields), s));
  SRS_CUDA(dp.alloc(sizeof(srs_particle) * nparticles, s));
  SRS_CUDA(ds.alloc(sizeof(TrajSpec) * nparticles, s));
  if (nfields > 0) SRS_CUDA(cudaMemcpyAsync(df.ptr, fields, sizeof(srs_field) * nfields, cudaMemcpyHostToDevice, s));
  SRS_CUDA(cudaMemcpyAsync(dp.ptr, particles, sizeof(srs_particle) * nparticles, cudaMemcpyHostToDevice, s));
  SRS_CUDA(cudaMemcpyAsync(ds.ptr, specs.data(), sizeof(TrajSpec) * nparticles, cudaMemcpyHostToDevice, s));
  SRS_CUDA(launch_rk4_specs(df.as<srs_field>(), nfields, dp.as<srs_particle>(), ds.as<TrajSpec>(), nparticles, s,
                            nfields > 0 ? grid_stage_doubles(fields, nfields) : 0, has_electric(fields, nfields)));
  return SRS_OK;
}

}  // extern "C"

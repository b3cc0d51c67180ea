"""Heterogeneous job queue: many flux-map and spectrum jobs, each with its own trajectory, run as ONE
persistent launch (srs_queue_*), replayed from a CUDA graph, with an autotuner for the work-item shape.

The reference runs such a set as separate calls (``calculate_spectrum`` / ``calculate_flux_rectangle``
per job, OSCARSSR_Python.cc:2232 and :3033), each with its own launches and host synchronisation.  Here
the jobs are cut into work items of one shape -- a tile of up to 128 grid points (strips of at most
``strip_width`` points) or 128 x ``energies_per_thread`` energies against ``chunk`` trajectory points --
ordered longest first and drained by resident CTAs from an atomic ticket.  A queue can also integrate
the jobs' trajectories itself (``integrate=``, magnetic fields): the jobs are grouped by trajectory
length and each group -- its trajectories integrated parallel in time, then its work items -- forms
one branch of the queue's graph, so the sums of some groups overlap the integration of the others.  :func:`autotune` times candidate shapes (chunk,
CTAs per SM, energies per thread, strip width, and the number of groups when integrating) on the jobs
themselves and caches the winner per job-set signature and device in a JSON file.

All tensors are CUDA tensors; every call is ordered on torch's current stream.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import json
import os

import numpy as np

from . import _lib, device
from ._lib import check, lib

CHUNKS = (2048, 4096, 8192, 16384)
CTAS_PER_SM = (0,)  # 0: as many as fit
ENERGIES_PER_THREAD = (2, 4)
STRIP_WIDTHS = (8, 12, 16)
GROUPS = (8, 4, 16, 32)
SEGMENT_STEPS = (16, 32)  # steps per segment of the queue's parallel-in-time integrations


def flux_job(traj, charge, current, grid, energy_ev, out):
    """A flux map job: particle 0 of ``traj`` (device.Trajectory) on ``grid`` (srs_grid2d) at one energy;
    ``out``: CUDA float64 tensor of grid.n1 * grid.n2 values."""
    j = _lib.Job()
    j.kind = _lib.JOB_FLUX
    j.traj = traj.view()
    j.beam = _lib.BeamConsts(charge, current)
    j.grid = grid
    j.energy_ev = float(energy_ev)
    j.d_out = out.data_ptr()
    return j, (traj, out)


def spectrum_job(traj, charge, current, obs, energies, out):
    """A spectrum job: particle 0 of ``traj`` at observer ``obs``; ``energies``, ``out``: CUDA float64."""
    j = _lib.Job()
    j.kind = _lib.JOB_SPECTRUM
    j.traj = traj.view()
    j.beam = _lib.BeamConsts(charge, current)
    j.obs = _lib.v3(obs)
    j.d_energies = energies.data_ptr()
    j.ne = energies.numel()
    j.d_out = out.data_ptr()
    return j, (traj, energies, out)


class JobQueue:
    """The planned queue of a list of jobs (from :func:`flux_job` / :func:`spectrum_job`)."""

    def __init__(self, jobs, chunk=2048, ctas_per_sm=0, energies_per_thread=0, strip_width=0, integrate=None,
                 groups=0, steps_per_segment=0):
        """integrate: None (the jobs' trajectories are given), or a dict (fields, particles, ctstart,
        ctstop, t0, npoints; per-job sequences except fields) with which every run integrates them into
        the jobs' trajectory views (see :func:`trajectory_buffers`) in ``groups`` length groups."""
        self._keep = [k for _, k in jobs]  # the tensors must outlive the queue
        arr = (_lib.Job * len(jobs))(*[j for j, _ in jobs])
        self._q = C.c_void_p()
        shape = _lib.QueueShape(int(chunk), int(ctas_per_sm), int(energies_per_thread), int(strip_width), int(groups),
                                int(steps_per_segment))
        if integrate is None:
            check(lib.srs_queue_create_shaped(C.byref(self._q), arr, len(jobs), C.byref(shape), None, 0, None, None,
                                              None, None, None))
        else:
            P = len(jobs)
            fields = integrate["fields"]
            fa = (_lib.Field * max(1, len(fields)))(*fields)
            pa = (_lib.Particle * P)(*integrate["particles"])
            vals = [np.ascontiguousarray(np.broadcast_to(np.asarray(integrate[k], float), (P,)))
                    for k in ("ctstart", "ctstop", "t0")]
            npts = np.ascontiguousarray(np.broadcast_to(np.asarray(integrate["npoints"], np.int64), (P,)))
            self._keep.append((fa, pa, vals, npts))
            D = _lib._D
            check(lib.srs_queue_create_shaped(C.byref(self._q), arr, P, C.byref(shape), fa, len(fields), pa,
                                              vals[0].ctypes.data_as(D), vals[1].ctypes.data_as(D),
                                              vals[2].ctypes.data_as(D), npts.ctypes.data_as(C.POINTER(C.c_int64))))
        self.chunk, self.ctas_per_sm = int(chunk), int(ctas_per_sm)
        self.energies_per_thread, self.strip_width, self.groups = int(energies_per_thread), int(strip_width), int(groups)
        self.steps_per_segment = int(steps_per_segment)
        self.integrates = integrate is not None
        n, ev, sb, g = C.c_int64(), C.c_double(), C.c_size_t(), C.c_int32()
        check(lib.srs_queue_info(self._q, C.byref(n), C.byref(ev), C.byref(sb), C.byref(g)))
        self.nitems, self.evals, self.scratch_bytes, self.grid = n.value, ev.value, sb.value, g.value

    def run(self):
        check(lib.srs_queue_run(self._q, device._stream()))

    def close(self):
        if self._q:
            lib.srs_queue_destroy(self._q)
            self._q = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def trajectory_batch(fields, particles, ctstart, ctstop, t0, npoints):
    """RK4 trajectories of particles with per-particle ctstart/ctstop/t0/npoints (sequences) in one
    launch (srs_trajectory_batch).  Returns one device.Trajectory (nparticles = 1) per particle, all
    views into one allocation."""
    P = len(particles)
    ctstart, ctstop, t0 = (np.broadcast_to(np.asarray(v, float), (P,)).copy() for v in (ctstart, ctstop, t0))
    npoints = np.broadcast_to(np.asarray(npoints, np.int64), (P,)).copy()
    trajs = trajectory_buffers(ctstart, ctstop, t0, npoints)
    fa = (_lib.Field * max(1, len(fields)))(*fields)
    pa = (_lib.Particle * P)(*particles)
    ptrs = [(C.c_void_p * P)(*[getattr(t, a).data_ptr() for t in trajs]) for a in ("x", "beta", "aoc")]
    D = _lib._D
    check(lib.srs_trajectory_batch(fa, len(fields), pa, P, ctstart.ctypes.data_as(D), ctstop.ctypes.data_as(D),
                                   t0.ctypes.data_as(D), npoints.ctypes.data_as(C.POINTER(C.c_int64)),
                                   ptrs[0], ptrs[1], ptrs[2], device._stream()))
    return trajs


def trajectory_buffers(ctstart, ctstop, t0, npoints):
    """Device trajectories (nparticles = 1 each, all views into one allocation) sized for the given
    per-particle settings, not yet integrated: for jobs whose queue integrates them."""
    import torch
    P = len(npoints)
    shapes = [device.counts(float(ctstart[p]), float(ctstop[p]), float(t0[p]), int(npoints[p])) for p in range(P)]
    sizes = [3 * (nf + nb) for _, nf, nb in shapes]
    buf = torch.empty((3, int(sum(sizes))), dtype=torch.float64, device="cuda")
    trajs, off = [], 0
    for (dt, nf, nb), s in zip(shapes, sizes):
        v = [buf[k, off:off + s].view(1, 3, nf + nb) for k in range(3)]
        trajs.append(device.Trajectory(v[0], v[1], v[2], dt))
        off += s
    return trajs


def signature(jobs):
    """Shape signature of a job list (kinds, trajectory lengths, output sizes) and the device."""
    import torch
    h = hashlib.sha1()
    for j, _ in jobs:
        out = j.grid.n1 * j.grid.n2 if j.kind == _lib.JOB_FLUX else j.ne
        h.update(f"{j.kind}:{j.traj.n}:{out};".encode())
    h.update(torch.cuda.get_device_name().encode())
    return h.hexdigest()[:20]


def _cache_path():
    return os.environ.get("SRS_B200_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "srsoriginal_b200", "queue_tune.json"))


def time_queue(q, reps=5, warmup=2):
    """Mean device time [ms] of q.run() over reps runs (CUDA events on the current stream)."""
    import torch
    for _ in range(warmup):
        q.run()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        q.run()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def autotune(jobs, chunks=CHUNKS, ctas_per_sm=CTAS_PER_SM, energies_per_thread=ENERGIES_PER_THREAD,
             strip_widths=STRIP_WIDTHS, groups=GROUPS, integrate=None, reps=3, cache=True):
    """Pick the queue's tile shape for this job list by timing candidate queues on the jobs
    themselves: every (chunk, CTAs per SM, energies per thread, strip width), then, with integrate, the
    number of trajectory-length groups and the integrations' steps per segment for the best of those.  Returns (shape dict, table) with table
    = {shape tuple: ms}.  With cache, a previous result for the same signature is returned without
    timing, and new results are stored."""
    key = signature(jobs) + (":integrate" if integrate is not None else "")
    path = _cache_path()
    db = {}
    if cache and os.path.exists(path):
        try:
            with open(path) as f:
                db = json.load(f)
        except (OSError, ValueError):
            db = {}
        if key in db and "shape" in db[key]:
            return dict(db[key]["shape"]), {}
    table = {}

    def timed(**sh):
        q = JobQueue(jobs, integrate=integrate, **sh)
        ms = time_queue(q, reps)
        q.close()
        table[tuple(sorted(sh.items()))] = ms
        return ms

    base = {"groups": groups[0], "steps_per_segment": SEGMENT_STEPS[0]} if integrate is not None else {"groups": 0}
    best, best_ms = None, float("inf")
    for ch in chunks:
        for c in ctas_per_sm:
            for k in energies_per_thread:
                for w in strip_widths:
                    sh = dict(base, chunk=ch, ctas_per_sm=c, energies_per_thread=k, strip_width=w)
                    ms = timed(**sh)
                    if ms < best_ms:
                        best, best_ms = sh, ms
    if integrate is not None:
        start = dict(best)
        for gr in groups:
            for L in SEGMENT_STEPS:
                sh = dict(start, groups=gr, steps_per_segment=L)
                if sh == start:
                    continue
                ms = timed(**sh)
                if ms < best_ms:
                    best, best_ms = sh, ms
    if cache:
        db[key] = {"shape": best, "ms": best_ms}
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(db, f, indent=1)
        except OSError:
            pass
    return best, table

"""Benchmark: flux maps of the config-1 workload on the B200.

Workload (config 1): 3 GeV, 0.5 A electron, ideal planar undulator (1 T, 49 mm, 31 periods), RK4
trajectory of 20001 points over ct in [0, 2] m from z = -1 m; flux on a 10 mm x 10 mm XY rectangle at
z = 30 m, 101 x 101 points, at the first harmonic (E1 = 152.25 eV, the peak of the config-0
spectrum) and at 3*E1.  Synthetic inputs (no dataset).

One step = both flux maps (E1 and E3) in mixed precision from the device-resident trajectory:
2 * 20001 * 10201 = 4.08e8 integrand evaluations.  ``value`` is integrand evaluations per second of
the whole job (all ranks), device-timed with CUDA events per step; the L2 (126 MB) is flushed with a
256 MiB write before every step, outside the timed events.  ``e2e`` is the same metric through the
public API (``srsoriginal_b200.sr.sr``: RK4 trajectory on the GPU, integrated parallel in time,
host->device copies of the inputs, both maps, device->host copy of the results), host wall-clock
around synchronous calls.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NT = 20001
GRID_N = 101
WIDTH = 0.01
E1 = 152.25225225225225
ENERGIES = (E1, 3 * E1)
EVALS_PER_STEP = len(ENERGIES) * NT * GRID_N * GRID_N
METRIC = "integrand evals/s (mixed vs plain FP64 at <=1e-4 rel flux err)"
UNIT = "evals/s"

# Algorithmic work per integrand evaluation of a flux map (one trajectory point x one observation
# point) in pipe operations, a fused multiply-add counted as one (srsoriginal_b200/roofline_counts.json):
# FP32 27 (n 4, amplitude 11, three complex MACs 12), SFU 2 (sincos), FP64 0.5 (the per-tile anchor
# shared by 128 points).
_COUNTS = json.load(open(os.path.join(ROOT, "srsoriginal_b200", "roofline_counts.json")))
OPS_PER_EVAL = {k: v for k, v in _COUNTS["flux_map_mixed"].items() if isinstance(v, (int, float))}


def error_floors(a, b):
    """Relative error of a against b over the outputs >= 1e-3 and >= 1e-6 of b's maximum (max and rms),
    and normwise."""
    import numpy as np
    a, b = np.asarray(a, float), np.asarray(b, float)
    out = {}
    for floor, tag in ((1e-3, "1e-3max"), (1e-6, "1e-6max")):
        big = np.abs(b) >= floor * np.abs(b).max()
        r = np.abs(a[big] - b[big]) / np.abs(b[big])
        out[f"max_rel_over_{tag}"] = float(r.max())
        out[f"rms_rel_over_{tag}"] = float(np.sqrt(np.mean(r * r)))
        out[f"outputs_over_{tag}"] = int(big.sum())
    out["normwise"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return out


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ------------------------------------------------------------------ distributed plumbing

def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"  # gloo: the CPU tests of this plumbing
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------ clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        """Starts sampling every 100 ms and returns once the first sample is on disk."""
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100", "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            t0 = time.time()
            while time.time() - t0 < 10 and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)  # one more sample after the timed region
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ------------------------------------------------------------------ CPU baseline (the reference)

def reference_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import io
    from contextlib import redirect_stdout
    with redirect_stdout(io.StringIO()):
        import sr as ref_sr  # the reference built from its own sources by oracle/Makefile
    return ref_sr


def reference_sample(rows, threads):
    """The reference's CPU path (nthreads = host threads) on a sample of the workload: the full
    trajectory and both energies, on `rows` rows of the 101 x 101 map.  Returns (seconds, evals)."""
    from srsoriginal_b200 import workloads as W
    ref_sr = reference_module()
    o = ref_sr.sr()
    W.setup_beam(o, NT)
    W.setup_undulator(o)
    h = WIDTH * (rows - 1) / (GRID_N - 1)
    t0 = time.perf_counter()
    for e in ENERGIES:
        o.calculate_flux_rectangle(plane="XY", energy_eV=e, width=[WIDTH, h if rows > 1 else WIDTH],
                                   npoints=[GRID_N, rows], translation=[0, 0, W.SCREEN_Z], nthreads=threads)
    return time.perf_counter() - t0, len(ENERGIES) * NT * GRID_N * rows


def cpu_baseline(target_s=10.0):
    threads = os.cpu_count() or 1
    dt, ev = reference_sample(2, threads)  # calibration
    rows = max(2, min(GRID_N, int(2 * target_s / max(dt, 1e-3))))
    dt, ev = reference_sample(rows, threads)
    return {"value": ev / dt, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"reference CPU path (oracle/_ref, nthreads={threads}): full 20001-point trajectory, "
                      f"both energies, {GRID_N} x {rows} of the 101 x 101 map ({ev:.3g} evals, {dt:.1f} s)"}


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baselines_all():
    """The reference's CPU path (oracle/_ref, nthreads = all host threads) on every configuration,
    each on a bounded sample scaled to the whole configuration by its evaluation count.  For the
    record next to the GPU numbers; the bench's headline baseline is config 1 (cpu_baseline)."""
    import io
    from contextlib import redirect_stdout

    from srsoriginal_b200 import workloads as W
    ref_sr = reference_module()
    th = os.cpu_count() or 1
    out = {"cpu": _cpu_model(), "threads": th}

    def timed(fn):
        t = time.perf_counter()
        with redirect_stdout(io.StringIO()):
            fn()
        return time.perf_counter() - t

    def beam(npts, fields=W.setup_undulator, **kw):
        o = ref_sr.sr()
        W.setup_beam(o, npts, **kw)
        fields(o)
        return o

    o = beam(NT)
    s = timed(lambda: o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=1000, energy_range_eV=[100, 1000],
                                           nthreads=th))
    out["cfg0_spectrum"] = {"evals": NT * 1000, "seconds": s, "evals_per_s": NT * 1000 / s, "sample": "whole"}
    dt, ev = reference_sample(4, th)
    out["cfg1_flux_maps"] = {"evals": EVALS_PER_STEP, "evals_per_s": ev / dt,
                             "seconds_projected": EVALS_PER_STEP / (ev / dt), "sample": f"{GRID_N} x 4 rows, both maps"}
    o = beam(40001, W.setup_epu)
    rows = 4
    s = timed(lambda: o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04 * (rows - 1) / 200],
                                                          npoints=[201, rows], translation=[0, 0, W.SCREEN_Z],
                                                          nthreads=th))
    ev = 40001 * 201 * rows
    out["cfg2_power_density"] = {"evals": 40001 * 201 * 201, "evals_per_s": ev / s,
                                 "seconds_projected": 40001 * 201 * 201 / (ev / s), "sample": f"201 x {rows} rows"}
    o = beam(NT, **W.BEAM_3A)
    o.set_seed(0)
    npart = 2
    s = timed(lambda: o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=2000, energy_range_eV=[100, 1000],
                                           nparticles=npart, nthreads=th))
    ev = npart * NT * 2000
    out["cfg3a_beam_spectrum"] = {"evals": 4096 * NT * 2000, "evals_per_s": ev / s,
                                  "seconds_projected": 4096 * NT * 2000 / (ev / s),
                                  "sample": f"{npart} of the 4096 particles (the reference loops over particles)"}
    specs = W.config3b_jobs()[:16]
    tot_ev, tot_s = 0.0, 0.0
    for sp in specs:
        o = beam(sp["nt"])
        if sp["kind"] == "flux":
            n = sp["n"]
            tot_s += timed(lambda: o.calculate_flux_rectangle(plane="XY", energy_eV=W.E1_EV, width=[0.01, 0.01],
                                                              npoints=[n, n], translation=[0, 0, W.SCREEN_Z],
                                                              nthreads=th))
            tot_ev += sp["nt"] * n * n
        else:
            tot_s += timed(lambda: o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=sp["ne"],
                                                        energy_range_eV=[100, 1000], nthreads=th))
            tot_ev += sp["nt"] * sp["ne"]
    all_ev = sum(j["nt"] * (j["n"] ** 2 if j["kind"] == "flux" else j["ne"]) for j in W.config3b_jobs())
    out["cfg3b_jobs"] = {"evals": all_ev, "evals_per_s": tot_ev / tot_s, "seconds_projected": all_ev / (tot_ev / tot_s),
                         "sample": "the first 16 of the 256 jobs"}
    with tempfile.TemporaryDirectory() as td:
        z, by = W.config4_grid()
        path = os.path.join(td, "cfg4.txt")
        W.write_oscars_grid(path, z, by)
        o = ref_sr.sr()
        W.setup_beam(o, NT)
        o.add_bfield_file(ifile=path, iformat="OSCARS")
        e0, e1 = W.config4_energy_range()
        s = timed(lambda: o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=W.NE4, energy_range_eV=[e0, e1],
                                               nthreads=th))
    out["cfg4_forward"] = {"seconds": s, "note": "the reference has no gradient: central differences over the "
                           "2007 coordinates would take 4014 of these forward runs",
                           "fd_gradient_seconds_projected": 4014 * s}
    return out


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    dt, ev = reference_sample(2, threads)
    # each step: a bounded sample sized so warmup + steps stay within a few minutes
    per_step_target = max(1.0, 150.0 / max(1, args.steps + args.warmup))
    rows = max(2, min(GRID_N, int(2 * per_step_target / max(dt, 1e-3))))
    for _ in range(args.warmup):
        reference_sample(rows, threads)
    times, evals = [], 0
    for _ in range(args.steps):
        dt, ev = reference_sample(rows, threads)
        times.append(dt)
        evals = ev
    tot = sum(times)
    value = evals * args.steps / tot
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "config 1: flux maps 101x101 at E1 and 3*E1, 20001-point trajectory "
                                   f"(each step a {GRID_N} x {rows} sample of each map)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{GRID_N} x {rows} rows of each map, both energies, full trajectory"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm

def _events_ms(fn, reps, warmup=1):
    """Median device time [ms] of fn() over reps runs, CUDA events on the current stream."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    times = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def _graph_ms(fn, reps=20):
    """Device time [ms] of one fn() without the host's launch overhead: fn captured once into a CUDA
    graph, the graph replayed reps times back to back, CUDA events around the replays.  None if the
    calls cannot be captured."""
    import torch
    try:
        fn()
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fn()
        torch.cuda.current_stream().wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        g.replay()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            g.replay()
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / reps
        del g
        return ms
    except Exception as ex:  # capture of a library call that allocates or synchronises
        log(f"graph timing unavailable: {ex}")
        return None


def measure_configs(dev, peaks=None):
    """The other configurations' throughput, for the record (not the headline): each device-timed
    with CUDA events (median of a few runs) unless marked wall-clock."""
    import numpy as np
    import torch

    from srsoriginal_b200 import _lib, device as D, queue as Q, workloads as W
    from srsoriginal_b200.adjoint import backward_flux, forward_flux
    from srsoriginal_b200.sr import energy_grid, rectangle_points, sr

    out = {}
    und = [D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)]
    part, gamma = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    charge, current = -D.QE, W.CURRENT

    # config 0: plain FP64 on-axis spectrum, 1000 energies (the drop-in path)
    traj = D.trajectory(und, [part], 0.0, 2.0, 0.0, NT)
    e0 = torch.tensor(energy_grid(1000, 100.0, 1000.0), dtype=torch.float64, device=dev)
    sp = torch.empty(1000, dtype=torch.float64, device=dev)
    ms = _events_ms(lambda: D.spectrum(traj, charge, current, [0, 0, W.SCREEN_Z], e0, sp, precision=_lib.FP64), 5)
    msm = _events_ms(lambda: D.spectrum(traj, charge, current, [0, 0, W.SCREEN_Z], e0, sp, precision=_lib.MIXED), 5)
    ev = NT * 1000
    spm = torch.empty_like(sp)
    D.spectrum(traj, charge, current, [0, 0, W.SCREEN_Z], e0, spm, precision=_lib.MIXED)
    D.spectrum(traj, charge, current, [0, 0, W.SCREEN_Z], e0, sp, precision=_lib.FP64)
    # the same calls replayed from a CUDA graph: the device time without the per-call host overhead,
    # which is a large part of a 1000-energy spectrum's time
    sg = torch.empty_like(sp)  # (sp and spm hold the results compared below)
    gms = _graph_ms(lambda: D.spectrum(traj, charge, current, [0, 0, W.SCREEN_Z], e0, sg, precision=_lib.FP64))
    gmsm = _graph_ms(lambda: D.spectrum(traj, charge, current, [0, 0, W.SCREEN_Z], e0, sg, precision=_lib.MIXED))
    out["cfg0_spectrum"] = {"evals": ev, "fp64_ms": ms, "fp64_evals_per_s": ev / (ms * 1e-3), "mixed_ms": msm,
                            "mixed_evals_per_s": ev / (msm * 1e-3), "fp64_graph_ms": gms, "mixed_graph_ms": gmsm,
                            "graph_note": "one call captured in a CUDA graph and replayed back to back: device time "
                                          "without the per-call launch overhead",
                            "mixed_error_vs_fp64": error_floors(spm.cpu().numpy(), sp.cpu().numpy())}

    # the trajectory: serial RK4 chain against the parallel-in-time integration (configs 0/1 and 2)
    epu = und + [D.undulator([0.6, 0, 0], [0, 0, W.PERIOD], W.NPERIODS, phase=np.pi / 2)]
    rec = {}
    for npts, fields in ((NT, und), (40001, epu)):
        ser = D.trajectory(fields, [part], 0.0, 2.0, 0.0, npts)
        st = torch.zeros(4, dtype=torch.float64, device=dev)
        sho = D.trajectory_shoot(fields, part, 0.0, 2.0, 0.0, npts, stats=st)
        ms_ser = _events_ms(lambda: D.trajectory(fields, [part], 0.0, 2.0, 0.0, npts, out=ser), 3)
        ms_sho = _events_ms(lambda: D.trajectory_shoot(fields, part, 0.0, 2.0, 0.0, npts, out=sho, stats=st), 5)
        torch.cuda.synchronize()
        s = st.cpu().tolist()
        rec[f"{npts}_points_{len(fields)}_undulators"] = {
            "serial_ms": ms_ser, "parallel_in_time_ms": ms_sho, "speedup": ms_ser / ms_sho,
            "newton_iterations": int(s[1]), "converged": bool(s[0]),
            "max_abs_dx_m": float((sho.x - ser.x).abs().max()), "max_abs_dbeta": float((sho.beta - ser.beta).abs().max())}
    out["trajectory"] = rec

    # config 1's first map as a plain point list (no grid to anchor on): the point-list mixed kernel
    xyz1, _, _, _ = rectangle_points([GRID_N, GRID_N], "XY", [WIDTH, WIDTH], translation=[0, 0, W.SCREEN_Z])
    pts1 = torch.as_tensor(np.ascontiguousarray(xyz1.reshape(-1)), device=dev)
    fl = torch.empty(GRID_N * GRID_N, dtype=torch.float64, device=dev)
    msp = _events_ms(lambda: D.flux(traj, charge, current, E1, fl, points=pts1, precision=_lib.MIXED), 5)
    ev = NT * GRID_N * GRID_N
    out["cfg1_map_as_point_list"] = {"evals": ev, "mixed_ms": msp, "mixed_evals_per_s": ev / (msp * 1e-3),
                                     "kernel": "FP64 geometry and phase per term, FP32 amplitude (no grid anchor)"}

    # config 2: power density of the elliptical undulator, 201 x 201 on a 40 mm square, 40001 points
    epu = [D.undulator([0, 1.0, 0], [0, 0, W.PERIOD], W.NPERIODS),
           D.undulator([0.6, 0, 0], [0, 0, W.PERIOD], W.NPERIODS, phase=np.pi / 2)]
    t2 = D.trajectory(epu, [part], 0.0, 2.0, 0.0, 40001)
    xyz, _, nrm, g2 = rectangle_points([201, 201], "XY", [0.04, 0.04], translation=[0, 0, W.SCREEN_Z])
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device=dev)
    nrms = torch.as_tensor(np.ascontiguousarray(np.tile(nrm, (201 * 201, 1)).reshape(-1)), device=dev)
    pd, pd64 = (torch.empty(201 * 201, dtype=torch.float64, device=dev) for _ in range(2))
    msm = _events_ms(lambda: D.power_density(t2, charge, current, pd, grid=g2, precision=_lib.MIXED), 5)
    ms = _events_ms(lambda: D.power_density(t2, charge, current, pd64, points=pts, normals=nrms,
                                            precision=_lib.FP64), 2)
    # accuracy from fresh outputs, after the timed calls
    chk, chk64 = torch.zeros_like(pd), torch.zeros_like(pd64)
    D.power_density(t2, charge, current, chk, grid=g2, precision=_lib.MIXED)
    D.power_density(t2, charge, current, chk64, points=pts, normals=nrms, precision=_lib.FP64)
    a, b = chk.cpu().numpy(), chk64.cpu().numpy()
    ev = 40001 * 201 * 201
    out["cfg2_power_density"] = {"evals": ev, "mixed_ms": msm, "mixed_evals_per_s": ev / (msm * 1e-3),
                                 "fp64_ms": ms, "fp64_evals_per_s": ev / (ms * 1e-3),
                                 "mixed_over_fp64": ms / msm,
                                 "mixed_error_vs_fp64": error_floors(a, b),
                                 "max_fp64_W_per_mm2": float(np.abs(b).max())}
    del t2, pts, nrms

    # config 3a: 4096 Twiss-sampled electrons, 2000 energies.  Through the public API (wall clock around
    # a synchronous call: host sampling, 4096 RK4 trajectories, the mixed sums, the per-particle
    # accumulation), after one untimed call of the same size (the stream-ordered memory pool then holds
    # the 5.9 GB trajectory batch, as it does for every later call of a session); median of three.
    # Then the device phases alone, with CUDA events: the 4096-trajectory RK4 batch and the mixed
    # spectrum sums over it.
    o = sr()
    W.setup_beam(o, NT, **W.BEAM_3A)
    W.setup_undulator(o)
    kw = dict(obs=[0, 0, W.SCREEN_Z], npoints=2000, energy_range_eV=[100, 1000], nparticles=4096, precision="mixed")
    o.set_seed(0)
    o.spectrum_arrays(**kw)
    walls = []
    for _ in range(3):
        o.set_seed(0)
        torch.cuda.synchronize()
        t = time.perf_counter()
        o.spectrum_arrays(**kw)
        torch.cuda.synchronize()
        walls.append(time.perf_counter() - t)
    wall = statistics.median(walls)
    del o
    ev = 4096 * NT * 2000
    parts = [part] * 4096
    tb = D.trajectory(und, parts, 0.0, 2.0, 0.0, NT)
    rk_ms = _events_ms(lambda: D.trajectory(und, parts, 0.0, 2.0, 0.0, NT, out=tb), 2)
    e3a = torch.tensor(energy_grid(2000, 100.0, 1000.0), dtype=torch.float64, device=dev)
    s3a = torch.empty(4096 * 2000, dtype=torch.float64, device=dev)
    sum_ms = _events_ms(lambda: D.spectrum(tb, charge, current, [0, 0, W.SCREEN_Z], e3a, s3a, precision=_lib.MIXED), 3)
    # the same 4096 spectra as 4096 jobs of the persistent work queue (one graph launch over (job,
    # energy tile, trajectory chunk) items), on the same trajectories
    qjobs = [Q.spectrum_job(D.Trajectory(tb.x[p:p + 1], tb.beta[p:p + 1], tb.aoc[p:p + 1], tb.dt), charge, current,
                            [0, 0, W.SCREEN_Z], e3a, s3a[p * 2000:(p + 1) * 2000]) for p in range(4096)]
    q3a = Q.JobQueue(qjobs, chunk=8192, energies_per_thread=4)
    q3a_ms = _events_ms(q3a.run, 3)
    q3a.close()
    del qjobs, q3a, tb, s3a
    out["cfg3a_beam_spectrum"] = {"evals": ev, "wall_s": wall, "wall_s_all": walls, "evals_per_s": ev / wall,
                                  "includes": "public API call: sampling, 4096 RK4, mixed sums, accumulation",
                                  "rk4_batch_ms": rk_ms, "spectrum_sums_ms": sum_ms,
                                  "spectrum_sums_evals_per_s": ev / (sum_ms * 1e-3),
                                  "queue_sums_ms": q3a_ms,
                                  "queue_note": "the 4096 spectra as 4096 jobs of the persistent work queue (chunk "
                                                "8192, four energies per thread), one CUDA-graph launch",
                                  "spectrum_sums_fp32_frac_of_measured_peak": (
                                      _COUNTS["spectrum_uniform_mixed"]["fp32"] * ev / (sum_ms * 1e-3)
                                      / peaks["fp32"] if peaks else None),
                                  "device_phases_note": "RK4 batch of 4096 ideal particles (the same step count "
                                                        "as the sampled ones) and the mixed sums over it, CUDA events"}

    # config 3b: 256 heterogeneous jobs, trajectories included.  The queue integrates the jobs'
    # trajectories itself (grouped by length, each group's RK4 batch followed by its work items on a
    # branch of one CUDA graph) with the tile shape its autotuner picks on these jobs; against it, the
    # same work as separate calls: one batched RK4 launch for all 256 trajectories, then one one-shot
    # mixed call per job.  Also the tuned queue on trajectories integrated beforehand (sums only).
    specs = W.config3b_jobs()
    t_tune = time.perf_counter()
    q, jobs, trajs = W.build_config3b(specs, integrate=True, tune=True)
    tune_s = time.perf_counter() - t_tune
    shape = {"chunk": q.chunk, "ctas_per_sm": q.ctas_per_sm, "energies_per_thread": q.energies_per_thread,
             "strip_width": q.strip_width, "groups": q.groups, "steps_per_segment": q.steps_per_segment}
    ms = _events_ms(q.run, 5)
    qs, jobs_s, trajs_s = W.build_config3b(specs, shape=dict(shape, groups=1, steps_per_segment=0))
    ms_sums = _events_ms(qs.run, 5)

    def separate():
        Q.trajectory_batch(und, [part] * len(specs), 0.0, 2.0, 0.0, [s_["nt"] for s_ in specs])
        for (j, keep), t_, s_ in zip(jobs_s, trajs_s, specs):
            if s_["kind"] == "flux":
                D.flux(t_, charge, current, W.E1_EV, keep[-1], grid=j.grid, precision=_lib.MIXED)
            else:
                D.spectrum(t_, charge, current, [0, 0, W.SCREEN_Z], keep[1], keep[-1], precision=_lib.MIXED)
    ms_sep = _events_ms(separate, 3)
    rk = _events_ms(lambda: Q.trajectory_batch(und, [part] * len(specs), 0.0, 2.0, 0.0, [s_["nt"] for s_ in specs]), 2)
    out["cfg3b_queue"] = {"evals": q.evals, "queue_ms": ms, "evals_per_s": q.evals / (ms * 1e-3),
                          "includes": "the 256 trajectories (integrated parallel in time, grouped by length) and all sums, one CUDA graph",
                          "separate_calls_ms": ms_sep, "queue_speedup": ms_sep / ms,
                          "separate_calls_include": "one batched RK4 launch for all trajectories, then a one-shot "
                                                    "mixed call per job",
                          "queue_sums_only_ms": ms_sums, "trajectory_batch_ms": rk,
                          "work_items": q.nitems, "ctas": q.grid, "shape": shape, "autotune_s": tune_s}
    q.close()
    qs.close()
    del jobs, trajs, jobs_s, trajs_s

    # config 4: adjoint / forward time (forward = the trajectory through the 2001-sample grid, parallel in
    # time, + mixed spectrum of 200 energies; adjoint = the E_k re-formed in FP64, sum adjoint +
    # trajectory adjoint scan, FP64)
    problem, grid, ic, de = W.config4_problem(precision=_lib.MIXED)
    fw, bw = [], []
    gfl = None
    for r in range(6):
        torch.cuda.synchronize()
        a_, m_, b_ = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        a_.record()
        f, saved = forward_flux(problem, grid, None, ic, keep_efield=True)
        m_.record()
        if gfl is None:
            gfl = torch.full_like(f, -de)
        backward_flux(problem, saved, gfl)
        b_.record()
        torch.cuda.synchronize()
        if r > 0:
            fw.append(a_.elapsed_time(m_))
            bw.append(m_.elapsed_time(b_))
    out["cfg4_adjoint"] = {"forward_ms": statistics.median(fw), "adjoint_ms": statistics.median(bw),
                           "adjoint_over_forward": statistics.median(bw) / statistics.median(fw),
                           "gradient": "2001 grid samples + 6 initial conditions"}
    return out


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    from srsoriginal_b200 import _lib, device as D, workloads as W
    from srsoriginal_b200.sr import rectangle_points, sr

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream()
    fields = [D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)]
    part, gamma = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    traj = D.trajectory(fields, [part], 0.0, 2.0, 0.0, NT)
    xyz, x12, nrm, grid = rectangle_points([GRID_N, GRID_N], "XY", [WIDTH, WIDTH], translation=[0, 0, W.SCREEN_Z])
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device=dev)
    npts = GRID_N * GRID_N
    out = {e: torch.empty(npts, dtype=torch.float64, device=dev) for e in ENERGIES}
    out64 = {e: torch.empty(npts, dtype=torch.float64, device=dev) for e in ENERGIES}
    charge, current = -D.QE, W.CURRENT
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    # trajectory time (one RK4 launch, single particle), for the record
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    D.trajectory(fields, [part], 0.0, 2.0, 0.0, NT, out=traj)
    e1.record(stream)
    torch.cuda.synchronize()
    rk4_ms = e0.elapsed_time(e1)

    def step(precision, outs):
        for e in ENERGIES:
            D.flux(traj, charge, current, e, outs[e], points=pts, grid=grid, precision=precision)

    def timed(precision, outs, steps, warmup):
        for _ in range(warmup):
            step(precision, outs)
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        evs = []
        for _ in range(steps):
            flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step(precision, outs)
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs)

    # plain FP64 kernel on the same workload: the denominator of the mixed/plain ratio and the check
    # of the mixed maps' error
    fp64_ms = timed(_lib.FP64, out64, max(1, min(3, args.steps)), 1) / max(1, min(3, args.steps))
    clocks = ClockSampler(local)
    clocks.start()
    total_ms = timed(_lib.MIXED, out, args.steps, args.warmup)
    clk = clocks.stop()
    total_ms = max_over_ranks(total_ms, world)
    ms_per_step = total_ms / args.steps
    value = world * EVALS_PER_STEP / (ms_per_step * 1e-3)

    # accuracy of the mixed maps against the plain FP64 maps (the drop-in)
    err = {f"{e:.2f}eV": error_floors(out[e].cpu().numpy(), out64[e].cpu().numpy()) for e in ENERGIES}

    # roofline of the dominant kernel (mixed flux): algorithmic ops per launch / launch time
    import ctypes
    peaks = {}
    for kind, name in ((0, "fp32"), (1, "fp64"), (2, "sfu")):
        v = ctypes.c_double()
        _lib.check(_lib.lib.srs_measure_peak(kind, ctypes.byref(v), ctypes.c_void_p(stream.cuda_stream)))
        peaks[name] = v.value
    evals_per_launch = NT * npts
    launch_s = ms_per_step * 1e-3 / len(ENERGIES)
    bounds = {k: OPS_PER_EVAL[k] * evals_per_launch / peaks[k] for k in peaks}
    bound = max(bounds, key=bounds.get)
    achieved = OPS_PER_EVAL[bound] * evals_per_launch / launch_s
    roofline = {"bound": bound, "achieved": achieved / 1e12, "peak": peaks[bound] / 1e12, "unit": "Tops/s",
                "frac": achieved / peaks[bound], "traffic": None,
                "peak_source": "measured live (srs_measure_peak: FFMA / DFMA / MUFU chains, all SMs)",
                "ops_per_eval": OPS_PER_EVAL, "evals_per_launch": evals_per_launch,
                "all_peaks_Tops": {k: v / 1e12 for k, v in peaks.items()}}
    # the same kernel's ncu capture (profiles/): DRAM bytes of one launch, FMA-pipe activity and the
    # FMA-pipe operations it executes per evaluation, for comparison with the algorithmic count above
    traffic_file = os.path.join(ROOT, "profiles", "flux_mixed_cfg1_traffic.json")
    if os.path.exists(traffic_file):
        prof = json.load(open(traffic_file))
        roofline["traffic"] = prof.get("bytes_per_launch")
        for k in ("fma_pipe_active_pct", "executed_fma_pipe_ops_per_eval", "source"):
            if k in prof:
                roofline[f"ncu_{k}"] = prof[k]

    # e2e through the public API (host buffers, synchronous calls).  One step = what a user does for
    # config 1: the trajectory (RK4 on the GPU, once: the object drops its kept trajectory at the start
    # of every step; parallel in time, as the object integrates it for mixed-precision sums) and both
    # maps, with the host<->device copies of each call.
    o = sr()
    W.setup_beam(o, NT)
    W.setup_undulator(o)
    e2e_steps = max(1, min(args.steps, 10))

    def e2e_step():
        o.set_trajectory_cache(True)  # drops the kept trajectory: this step integrates it again
        for e in ENERGIES:
            o.flux_arrays(e, [GRID_N, GRID_N], "XY", [WIDTH, WIDTH], translation=[0, 0, W.SCREEN_Z],
                          precision="mixed")

    def timed_e2e(steps):
        for _ in range(min(2, args.warmup)):
            e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(steps):
            e2e_step()
        torch.cuda.synchronize()
        return max_over_ranks(time.perf_counter() - t0, world)

    # the same steps with the serial RK4 chain, for comparison (not the reported value)
    o.set_trajectory_mode("serial")
    e2e_serial_s = timed_e2e(min(3, e2e_steps))
    o.set_trajectory_mode("auto")
    # the same steps in plain FP64 (the drop-in: serial RK4 in the reference's arithmetic, FP64 maps),
    # the like-precision comparison with the reference's CPU path
    fp64_steps = max(1, min(3, e2e_steps))

    def e2e_step_fp64():
        o.set_trajectory_cache(True)
        for e in ENERGIES:
            o.flux_arrays(e, [GRID_N, GRID_N], "XY", [WIDTH, WIDTH], translation=[0, 0, W.SCREEN_Z],
                          precision="fp64")

    e2e_step_fp64()
    torch.cuda.synchronize()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(fp64_steps):
        e2e_step_fp64()
    torch.cuda.synchronize()
    e2e_fp64_s = max_over_ranks(time.perf_counter() - t0, world)
    # three timed blocks of the same steps (wall clock around synchronised steps, max over ranks); the
    # median block is reported, so that one host hiccup on a shared machine does not decide the number
    e2e_blocks = sorted(timed_e2e(e2e_steps) for _ in range(3))
    e2e_s = e2e_blocks[1]
    e2e = {"value": world * EVALS_PER_STEP * e2e_steps / e2e_s, "unit": UNIT,
           # in: the particle (RK4 once per step; each map's sums start from zero on the device);
           # out: each map's values
           "h2d_bytes_per_step": 56,
           "d2h_bytes_per_step": len(ENERGIES) * npts * 8,
           "ms_per_step": 1e3 * e2e_s / e2e_steps,
           "ms_per_step_blocks": [1e3 * t / e2e_steps for t in e2e_blocks],
           "includes": "RK4 trajectory on the GPU (once per step, parallel in time), both maps, host<->device "
                       "copies of each call",
           "ms_per_step_serial_trajectory": 1e3 * e2e_serial_s / min(3, e2e_steps)}
    e2e_fp64 = {"value": world * EVALS_PER_STEP * fp64_steps / e2e_fp64_s, "unit": UNIT,
                "h2d_bytes_per_step": 56, "d2h_bytes_per_step": len(ENERGIES) * npts * 8,
                "ms_per_step": 1e3 * e2e_fp64_s / fp64_steps,
                "includes": "plain FP64 through the same API: serial RK4 trajectory, both FP64 maps, host copies"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic",
            "config": {"workload": "config 1: flux maps 101x101 (10 mm square at 30 m) at E1=152.25 eV and "
                                   "3*E1, 20001-point trajectory, 3 GeV 0.5 A, 1 T / 49 mm / 31-period undulator",
                       "evals_per_step": EVALS_PER_STEP, "precision": "mixed",
                       "l2": "256 MiB write before every step, outside the per-step CUDA events",
                       "parallelism": f"replicas x{world} (weak)"},
            "fp64_plain": {"value": EVALS_PER_STEP / (fp64_ms * 1e-3), "unit": UNIT, "ms_per_step": fp64_ms},
            "mixed_over_fp64": (EVALS_PER_STEP / (ms_per_step * 1e-3)) / (EVALS_PER_STEP / (fp64_ms * 1e-3)),
            "mixed_error_vs_fp64": err,
            "rk4_trajectory_ms": rk4_ms,
            "roofline": roofline, "clocks": clk, "e2e": e2e, "e2e_fp64": e2e_fp64,
            "gpu_launches": args.steps * len(ENERGIES) * 2}
    if not args.no_configs:
        line["other_configs"] = measure_configs(dev, peaks)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline()
        except Exception as ex:  # the reference module is built here only when its sources exist
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                    "sample": f"unavailable: {ex}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


PROFILE_CASES = ("flux_mixed_cfg1", "flux_fp64_cfg1", "pd_fp64_51x51", "spectrum_mixed_3a256", "shoot_cfg1",
                 "spectrum_cfg0", "adjoint_cfg4")


def run_case(name):
    """One small workload, run twice, for an ncu capture of its kernel (no timing, no JSON line):
    flux_mixed_cfg1 / flux_fp64_cfg1: the config-1 map at 3*E1 (mixed / plain FP64); pd_fp64_51x51:
    config 2's power density on 51 x 51 points (40001-point trajectory, plain FP64);
    spectrum_mixed_3a256: 256 electrons of config 3a's shape (20001 points, 2000 energies, mixed);
    shoot_cfg1: the config-1 trajectory integrated parallel in time; spectrum_cfg0: config 0's
    1000-energy spectrum, mixed then plain FP64; adjoint_cfg4: config 4's forward and adjoint."""
    import numpy as np
    import torch

    from srsoriginal_b200 import _lib, device as D, workloads as W
    from srsoriginal_b200.sr import energy_grid, rectangle_points
    part, _ = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    und = [D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)]
    charge, current = -D.QE, W.CURRENT
    for _ in range(2):
        if name in ("flux_mixed_cfg1", "flux_fp64_cfg1"):
            tr = D.trajectory(und, [part], 0.0, 2.0, 0.0, NT)
            xyz, _, _, grid = rectangle_points([GRID_N, GRID_N], "XY", [WIDTH, WIDTH], translation=[0, 0, W.SCREEN_Z])
            out = torch.empty(GRID_N * GRID_N, dtype=torch.float64, device="cuda")
            if name == "flux_mixed_cfg1":
                D.flux(tr, charge, current, W.E3_EV, out, grid=grid, precision=_lib.MIXED)
            else:
                pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
                D.flux(tr, charge, current, W.E3_EV, out, points=pts, precision=_lib.FP64)
        elif name == "pd_fp64_51x51":
            epu = und + [D.undulator([0.6, 0, 0], [0, 0, W.PERIOD], W.NPERIODS, phase=np.pi / 2)]
            t2 = D.trajectory(epu, [part], 0.0, 2.0, 0.0, 40001)
            xyz, _, nrm, _ = rectangle_points([51, 51], "XY", [0.04, 0.04], translation=[0, 0, W.SCREEN_Z])
            pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
            nrms = torch.as_tensor(np.ascontiguousarray(np.tile(nrm, (51 * 51, 1)).reshape(-1)), device="cuda")
            out = torch.empty(51 * 51, dtype=torch.float64, device="cuda")
            D.power_density(t2, charge, current, out, points=pts, normals=nrms, precision=_lib.FP64)
        elif name == "spectrum_mixed_3a256":
            tb = D.trajectory(und, [part] * 256, 0.0, 2.0, 0.0, NT)
            e = torch.tensor(energy_grid(2000, 100.0, 1000.0), dtype=torch.float64, device="cuda")
            out = torch.empty(256 * 2000, dtype=torch.float64, device="cuda")
            D.spectrum(tb, charge, current, [0, 0, W.SCREEN_Z], e, out, precision=_lib.MIXED)
        elif name == "shoot_cfg1":
            D.trajectory_shoot(und, part, 0.0, 2.0, 0.0, NT)
        elif name == "adjoint_cfg4":
            from srsoriginal_b200.adjoint import backward_flux, forward_flux
            problem, grid4, ic4, de4 = W.config4_problem()
            f4, saved4 = forward_flux(problem, grid4, None, ic4, keep_efield=True)
            backward_flux(problem, saved4, torch.full_like(f4, -de4))
        elif name == "spectrum_cfg0":
            t1 = D.trajectory(und, [part], 0.0, 2.0, 0.0, NT)
            e = torch.tensor(energy_grid(1000, 100.0, 1000.0), dtype=torch.float64, device="cuda")
            out = torch.empty(1000, dtype=torch.float64, device="cuda")
            D.spectrum(t1, charge, current, [0, 0, W.SCREEN_Z], e, out, precision=_lib.MIXED)
            D.spectrum(t1, charge, current, [0, 0, W.SCREEN_Z], e, out, precision=_lib.FP64)
        torch.cuda.synchronize()
    log(f"case {name} ok")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the other configurations' measurements")
    ap.add_argument("--cpu-baselines", action="store_true",
                    help="time the reference's CPU path on every configuration and exit")
    ap.add_argument("--case", choices=PROFILE_CASES,
                    help="run one small workload twice for a profiler capture of its kernel, and exit")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case)
    if args.cpu_baselines:  # the reference on every configuration, host only
        print(json.dumps(cpu_baselines_all()), flush=True)
        return 0
    if args.impl == "reference":  # host-only: rank 0 runs the reference's CPU path, other ranks exit
        return run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
    world, rank, local = dist_init()
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        return run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())

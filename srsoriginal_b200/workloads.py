"""Synthetic workloads with the shapes of the reference's benchmark configurations.

All inputs are synthetic (there is no dataset): a 3 GeV, 0.5 A electron beam starting on axis at
z = -1 m, an ideal planar undulator (1 T, 49 mm period, 31 periods) centred at 0, observation at
z = 30 m.  ``setup_*`` functions take any object with the reference's ``oscars.sr.sr`` method
names, so the same code drives this library, the reference and the oracle.
"""
from __future__ import annotations

import math

import numpy as np

PERIOD = 0.049
NPERIODS = 31
BPEAK = 1.0
ENERGY_GEV = 3.0
CURRENT = 0.5
SCREEN_Z = 30.0

# First-harmonic on-axis peak of the config-0 spectrum (1000 points over 100-1000 eV on the
# reference's energy grid, which starts one step above 100 eV), taken from the reference's own
# output in tests/golden/spectrum_cfg0.npz; the third harmonic is 3x this energy.
E1_EV = 152.25225225225225
E3_EV = 3.0 * E1_EV


def setup_beam(osr, npoints=20001, **extra):
    """set_particle_beam + set_ctstartstop(0, 2) + set_npoints_trajectory (in that order)."""
    kw = dict(type="electron", name="beam_0", energy_GeV=ENERGY_GEV, x0=[0, 0, -1], d0=[0, 0, 1],
              current=CURRENT)
    kw.update(extra)
    osr.set_particle_beam(**kw)
    osr.set_ctstartstop(0, 2)
    osr.set_npoints_trajectory(npoints)


def setup_undulator(osr):
    osr.add_bfield_undulator(bfield=[0, BPEAK, 0], period=[0, 0, PERIOD], nperiods=NPERIODS)


def setup_epu(osr):
    """Config 2: By 1 T plus Bx 0.6 T shifted by a quarter period (phase pi/2)."""
    osr.add_bfield_undulator(bfield=[0, 1.0, 0], period=[0, 0, PERIOD], nperiods=NPERIODS)
    osr.add_bfield_undulator(bfield=[0.6, 0, 0], period=[0, 0, PERIOD], nperiods=NPERIODS,
                             phase=math.pi / 2)


BEAM_3A = dict(sigma_energy_GeV=0.003, beta=[1.5, 0.8], emittance=[1e-9, 8e-12],
               horizontal_direction=[1, 0, 0], lattice_reference=[0, 0, -1])


def undulator_by(z, period=PERIOD, nperiods=NPERIODS, bpeak=BPEAK):
    """By(z) of the ideal undulator on axis (same piecewise form as the library's field model)."""
    z = np.asarray(z, dtype=np.float64)
    L = period * (nperiods + 2)
    s = np.sin(2 * math.pi * z / period)
    out = bpeak * s
    end1 = (z < -L / 2 + period) | (z > L / 2 - period)
    end2 = (z < -L / 2 + period / 2) | (z > L / 2 - period / 2)
    out = np.where(end1, 0.75 * bpeak * s, out)
    out = np.where(end2, 0.25 * bpeak * s, out)
    out = np.where((z > L / 2) | (z < -L / 2), 0.0, out)
    return out


def config4_grid(nz=2001, z0=-1.0, z1=1.0, sigma=0.005, seed=1):
    """Config 4 field: the config-0 undulator sampled on a z grid, each pole (half period counted
    from the undulator's start) scaled by (1 + N(0, sigma^2)) drawn with numpy default_rng(seed)."""
    z = np.linspace(z0, z1, nz)
    by = undulator_by(z)
    L = PERIOD * (NPERIODS + 2)
    npoles = int(round(L / (PERIOD / 2)))
    delta = np.random.default_rng(seed).normal(0.0, sigma, npoles)
    pole = np.clip(np.floor((z + L / 2) / (PERIOD / 2)).astype(int), 0, npoles - 1)
    return z, by * (1.0 + delta[pole])


def write_oscars_grid(path, z, by, bx=None):
    """Writes a 1-D (z) field map in the reference's OSCARS text format
    (header: comment, then start/step/count for x, y and z; then 'Bx By Bz' per sample)."""
    z = np.asarray(z, dtype=np.float64)
    bx = np.zeros_like(by) if bx is None else bx
    dz = float((z[-1] - z[0]) / (len(z) - 1))
    with open(path, "w") as f:
        f.write("# OSCARS 1-D field map\n")
        f.write("0\n0\n1\n0\n0\n1\n")
        f.write(f"{float(z[0])!r}\n{dz!r}\n{len(z)}\n")
        for i in range(len(z)):
            f.write(f"{float(bx[i])!r} {float(by[i])!r} 0.0\n")


def config3b_jobs(n=256, seed=3):
    """Config 3b: n independent jobs, numpy default_rng(seed).  Each job: trajectory length
    U{5001..40001}; kind spectrum (U{100..4000} energies over 100-1000 eV, on axis at 30 m) or
    flux map (n x n, n ~ U{8..201}, 10 mm square at 30 m, at E1)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(n):
        nt = int(rng.integers(5001, 40002))
        if rng.integers(0, 2) == 0:
            jobs.append(dict(kind="spectrum", nt=nt, ne=int(rng.integers(100, 4001))))
        else:
            jobs.append(dict(kind="flux", nt=nt, n=int(rng.integers(8, 202))))
    return jobs


def build_config3b(specs, chunk=None, ctas_per_sm=0, tune=False, integrate=False, shape=None):
    """Device jobs of a config-3b style spec list (from :func:`config3b_jobs`): the ideal 3 GeV
    particle through the config-0 undulator, each job with its own trajectory length, flux maps on a
    10 mm square at 30 m at E1, spectra on axis at 30 m over the reference's 100-1000 eV energy grid.
    Returns (JobQueue, jobs, trajectories); job outputs are jobs[i][1][-1].  integrate: the queue
    integrates the trajectories itself on every run (grouped by length, overlapped with the sums);
    otherwise one srs_trajectory_batch launch computes them here.  shape: JobQueue keyword arguments
    (chunk, ctas_per_sm, energies_per_thread, strip_width, groups); tune: pick them with
    queue.autotune."""
    import torch

    from . import device as D
    from . import queue as Q
    from .sr import energy_grid, rectangle_points

    und = D.undulator([0, BPEAK, 0], [0, 0, PERIOD], NPERIODS)
    part, _ = D.ideal_particle(ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    nts = [s["nt"] for s in specs]
    if integrate:
        trajs = Q.trajectory_buffers([0.0] * len(specs), [2.0] * len(specs), [0.0] * len(specs), nts)
        how = dict(fields=[und], particles=[part] * len(specs), ctstart=0.0, ctstop=2.0, t0=0.0, npoints=nts)
    else:
        trajs = Q.trajectory_batch([und], [part] * len(specs), 0.0, 2.0, 0.0, nts)
        how = None
    charge, current = -D.QE, CURRENT
    jobs, grids, energies = [], {}, {}
    for s, t in zip(specs, trajs):
        if s["kind"] == "flux":
            n = s["n"]
            if n not in grids:
                grids[n] = rectangle_points([n, n], plane="XY", width=[0.01, 0.01], translation=[0, 0, SCREEN_Z])[3]
            out = torch.empty(n * n, dtype=torch.float64, device="cuda")
            jobs.append(Q.flux_job(t, charge, current, grids[n], E1_EV, out))
        else:
            ne = s["ne"]
            if ne not in energies:
                energies[ne] = torch.tensor(energy_grid(ne, 100.0, 1000.0), dtype=torch.float64, device="cuda")
            out = torch.empty(ne, dtype=torch.float64, device="cuda")
            jobs.append(Q.spectrum_job(t, charge, current, [0, 0, SCREEN_Z], energies[ne], out))
    sh = dict(shape or {})
    if chunk is not None:
        sh["chunk"] = chunk
    if ctas_per_sm:
        sh["ctas_per_sm"] = ctas_per_sm
    if tune:
        sh, _ = Q.autotune(jobs, integrate=how)
    sh.setdefault("chunk", 2048)
    q = Q.JobQueue(jobs, integrate=how, **sh)
    return q, jobs, trajs


NE4 = 200  # config 4: energies over +-2 % of E3 (reference energy grid)
IC_NAMES = ("x", "y", "x'", "y'", "z", "E")
IC4 = (0.0, 0.0, 0.0, 0.0, -1.0, ENERGY_GEV)
# coordinate scales for the finite-difference steps h = 1e-6 * max(|value|, scale): field samples [T],
# then x, y [m], x', y' [rad], z [m], E [GeV]
FD_SCALES = (1.0, 1e-3, 1e-3, 1e-3, 1e-3, 1.0, 1.0)


def config4_energy_range():
    return 0.98 * E3_EV, 1.02 * E3_EV


def config4_coords(n=32, seed=4, nsamples=2001):
    """The coordinates checked by finite differences, as indices into (grid samples By_0 ..
    By_{nsamples-1}, then x, y, x', y', z, E): n distinct indices drawn with numpy default_rng(seed),
    then the six initial-condition coordinates (which a random draw of 32 from 2007 rarely hits)."""
    drawn = np.random.default_rng(seed).choice(nsamples + 6, size=n, replace=False)
    extra = [k for k in range(nsamples, nsamples + 6) if k not in set(drawn.tolist())]
    return np.concatenate([drawn, np.array(extra, dtype=drawn.dtype)])


def config4_fd_step(k, by, ic=IC4, rel=1e-6):
    nz = len(by)
    if k < nz:
        return rel * max(abs(float(by[k])), FD_SCALES[0])
    j = k - nz
    return rel * max(abs(float(ic[j])), FD_SCALES[1 + j])


def config4_problem(precision=None, npoints=20001):
    """(problem, grid, ic, dE) of config 4: the perturbed-undulator 1-D grid (config4_grid) as the
    only field, the ideal 3 GeV particle from z = -1 m, on-axis flux at 30 m over NE4 energies in
    +-2 % of E3.  grid: (2001, 3) CUDA tensor (Bx, By, Bz samples); ic: the six coordinates."""
    import torch

    from . import _lib
    from . import device as D
    from .adjoint import SpectrumProblem
    from .sr import energy_grid

    z, by = config4_grid()
    dz = float((z[-1] - z[0]) / (len(z) - 1))
    f = D.grid_z(float(z[0]), dz, by, None)
    e0, e1 = config4_energy_range()
    energies = torch.tensor(energy_grid(NE4, e0, e1), dtype=torch.float64, device="cuda")
    problem = SpectrumProblem(fields=[f], obs=(0.0, 0.0, SCREEN_Z), energies=energies, npoints=npoints,
                              current=CURRENT, precision=_lib.MIXED if precision is None else precision)
    g = np.zeros((len(by), 3))
    g[:, 1] = by
    grid = torch.tensor(g, dtype=torch.float64, device="cuda")
    ic = torch.tensor(IC4, dtype=torch.float64)
    return problem, grid, ic, (e1 - e0) / (NE4 - 1)

"""Device-resident calls of the C ABI on torch CUDA tensors (inputs and outputs stay in HBM).

This is the layer for callers that keep trajectories, observation points and results on the GPU
(batched multi-particle work, benchmarks, the adjoint).  Every function launches on the caller's
current torch stream and returns without synchronising.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, lib

QE = 1.602176462e-19
ME = 9.10938356e-31
SPEED_OF_LIGHT = 2.99792458e8


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _dptr(t):
    return C.cast(t.data_ptr(), _lib._D) if t is not None else None


def _rot(v, r):
    x, y, z = (float(a) for a in v)
    s, c = math.sin(r[0]), math.cos(r[0])
    y, z = c * y - s * z, s * y + c * z
    s, c = math.sin(r[1]), math.cos(r[1])
    z, x = c * z - s * x, s * z + c * x
    s, c = math.sin(r[2]), math.cos(r[2])
    x, y = c * x - s * y, s * x + c * y
    return [x, y, z]


def undulator(bfield, period, nperiods, phase=0.0, rotations=(0, 0, 0), translation=(0, 0, 0), taper=0.0):
    """srs_field of an ideal undulator, built as add_bfield_undulator builds it (field and period
    rotated, centre = translation)."""
    f = _lib.Field()
    f.kind = _lib.UNDULATOR
    f.field = _lib.v3(_rot(bfield, rotations))
    f.period = _lib.v3(_rot(period, rotations))
    f.center = _lib.v3(translation)
    f.nperiods = int(nperiods)
    f.phase = float(phase)
    f.taper = float(taper)
    return f


def grid_z(z0, dz, values_by, device_data):
    """srs_field of a 1-D (z) field map with By samples; device_data: a CUDA float64 tensor of 3*nz
    values (Bx, By, Bz per sample) that must outlive the field."""
    f = _lib.Field()
    f.kind = _lib.GRID
    f.n[0], f.n[1], f.n[2] = 1, 1, len(values_by)
    f.start = _lib.v3([0.0, 0.0, float(z0)])
    f.step = _lib.v3([0.0, 0.0, float(dz)])
    f.data = _dptr(device_data)
    return f


def ideal_particle(energy_gev, x0, d0, charge=-QE, mass=ME):
    """(srs_particle, gamma) of the ideal particle of a beam (TParticleBeam::GetNewParticle("ideal"))."""
    g = energy_gev / (1e-9 * mass * SPEED_OF_LIGHT * SPEED_OF_LIGHT / QE)
    beta = math.sqrt(1.0 - 1.0 / (g * g))
    d = np.asarray(d0, float)
    u = d / math.sqrt(float(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]))
    b0 = [float(u[0] * beta), float(u[1] * beta), float(u[2] * beta)]
    b2 = b0[0] * b0[0] + b0[1] * b0[1] + b0[2] * b0[2]
    gamma = 1.0 / math.sqrt(1.0 - b2)
    p = _lib.Particle()
    p.x0 = _lib.v3(x0)
    p.beta0 = _lib.v3(b0)
    p.qomg = charge / mass / gamma
    return p, gamma


def counts(ctstart, ctstop, t0, npoints):
    dt, nf, nb = C.c_double(), C.c_int64(), C.c_int64()
    check(lib.srs_trajectory_counts(ctstart, ctstop, t0, npoints, C.byref(dt), C.byref(nf), C.byref(nb)))
    return dt.value, nf.value, nb.value


class Trajectory:
    """Device trajectories of nparticles particles: x, beta, a/c as (nparticles, 3, n) float64 tensors."""

    def __init__(self, x, beta, aoc, dt):
        self.x, self.beta, self.aoc, self.dt = x, beta, aoc, dt
        self.nparticles, _, self.n = x.shape

    def view(self):
        return _lib.TrajView(_dptr(self.x), _dptr(self.beta), _dptr(self.aoc), self.n, self.nparticles, self.dt)


def trajectory(fields, particles, ctstart, ctstop, t0, npoints, out=None):
    """RK4 trajectories (srs_trajectory) of a list of srs_particle through a list of srs_field."""
    import torch
    dt, nf, nb = counts(ctstart, ctstop, t0, npoints)
    n = nf + nb
    P = len(particles)
    if out is None:
        out = Trajectory(*(torch.empty((P, 3, n), dtype=torch.float64, device="cuda") for _ in range(3)), dt)
    fa = (_lib.Field * max(1, len(fields)))(*fields)
    pa = (_lib.Particle * P)(*particles)
    check(lib.srs_trajectory(fa, len(fields), pa, P, ctstart, ctstop, t0, npoints, _ptr(out.x), _ptr(out.beta),
                             _ptr(out.aoc), _stream()))
    return out


def trajectory_shoot(fields, particle, ctstart, ctstop, t0, npoints, steps_per_segment=0, max_iterations=0, out=None,
                     stats=None):
    """One particle's trajectory integrated parallel in time (srs_trajectory_shoot).  stats: optional
    CUDA float64 tensor of 4 (converged, iterations, largest segment mismatch of the last and of the
    previous iteration)."""
    import torch
    dt, nf, nb = counts(ctstart, ctstop, t0, npoints)
    n = nf + nb
    if out is None:
        out = Trajectory(*(torch.empty((1, 3, n), dtype=torch.float64, device="cuda") for _ in range(3)), dt)
    fa = (_lib.Field * max(1, len(fields)))(*fields)
    check(lib.srs_trajectory_shoot(fa, len(fields), C.byref(particle), ctstart, ctstop, t0, npoints,
                                   steps_per_segment, max_iterations, _ptr(out.x), _ptr(out.beta), _ptr(out.aoc),
                                   _ptr(stats) if stats is not None else None, _stream()))
    return out


def grid2d(grid):
    return grid


def flux(traj, charge, current, energy_ev, out, points=None, grid=None, precision=_lib.MIXED):
    """srs_flux into out (CUDA float64, nparticles*np)."""
    np_ = grid.n1 * grid.n2 if grid is not None else points.numel() // 3
    check(lib.srs_flux(traj.view(), _lib.BeamConsts(charge, current), _ptr(points), np_,
                       C.byref(grid) if grid is not None else None, energy_ev, precision, _ptr(out), _stream()))
    return out


def spectrum(traj, charge, current, obs, energies, out, precision=_lib.MIXED):
    """srs_spectrum into out (CUDA float64, nparticles*ne); energies: CUDA float64 tensor."""
    check(lib.srs_spectrum(traj.view(), _lib.BeamConsts(charge, current), _lib.v3(obs), _ptr(energies),
                           energies.numel(), precision, _ptr(out), _stream()))
    return out


def power_density(traj, charge, current, out, points=None, normals=None, grid=None, directional=0,
                  precision=_lib.MIXED):
    np_ = grid.n1 * grid.n2 if grid is not None else points.numel() // 3
    check(lib.srs_power_density(traj.view(), _lib.BeamConsts(charge, current), _ptr(points), _ptr(normals), np_,
                                C.byref(grid) if grid is not None else None, directional, precision, _ptr(out),
                                _stream()))
    return out

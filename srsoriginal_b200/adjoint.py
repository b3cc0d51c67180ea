"""Differentiable spectrum: flux at one observer as a function of the magnetic-field parameters and the
particle's initial conditions, with a hand-written adjoint behind ``torch.autograd.Function``.

Forward (all on the GPU): the RK4 trajectory through the fields (srs_trajectory_shoot, parallel in
time, for a mixed-precision forward; the serial srs_trajectory for FP64), then the spectrum with its
sums E_k kept (srs_spectrum_efield; mixed precision by default, FP64 on request).
Backward: the closed-form adjoint of the sum (srs_spectrum_adjoint) gives dL/d(x_i, beta_i) at every
trajectory point; the trajectory adjoint (srs_trajectory_adjoint) carries it back to the field
parameters and the initial state by a parallel scan over the stored RK4 states.

The reference has no derivatives; the forward calls are its calculate_trajectory /
calculate_spectrum (OSCARSSR.cc:562-874, 1154-1251).  Initial conditions are the ideal particle of a
beam (TParticleBeam::GetNewParticle("ideal")) written as six coordinates

    ic = (x, y, x', y', z, E)   with x0 = (x, y, z), d0 = (x', y', 1), energy E [GeV].
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field as dfield

import numpy as np

from . import _lib, device as D
from ._lib import check, lib

AMPLITUDE_KINDS = (_lib.UNDULATOR, _lib.GAUSSIAN, _lib.UNIFORM_BOX)


def particle_from_ic(ic, charge=-D.QE, mass=D.ME):
    """srs_particle of the ideal particle with coordinates ic = (x, y, x', y', z, E [GeV]), and the
    Jacobian d(x0[3], beta0[3], qomg) / d(ic) as a 7 x 6 array (for the chain rule)."""
    x, y, xp, yp, z, E = (float(v) for v in ic)
    c2 = D.SPEED_OF_LIGHT ** 2
    g = E / (1e-9 * mass * c2 / D.QE)
    beta = math.sqrt(1.0 - 1.0 / (g * g))
    d = np.array([xp, yp, 1.0])
    dn = float(np.sqrt(d @ d))
    u = d / dn
    b0 = u * beta
    gamma = 1.0 / math.sqrt(1.0 - float(b0 @ b0))
    p = _lib.Particle()
    p.x0 = _lib.v3([x, y, z])
    p.beta0 = _lib.v3(list(b0))
    p.qomg = charge / mass / gamma
    J = np.zeros((7, 6))
    J[0, 0] = J[1, 1] = J[2, 4] = 1.0
    du = (np.eye(3) - np.outer(u, u)) / dn  # du/dd
    J[3:6, 2] = beta * du[:, 0]
    J[3:6, 3] = beta * du[:, 1]
    dbeta_dE = (1.0 / (g ** 3 * beta)) * (g / E)
    J[3:6, 5] = u * dbeta_dE
    J[6, 5] = -p.qomg / E
    return p, J


@dataclass
class SpectrumProblem:
    """The fixed part of a differentiable spectrum.

    fields: srs_field templates in order; amplitude fields (undulator, Gaussian, uniform box) take
      their vector from the ``amps`` input, one grid field (if any) takes its samples from the
      ``grid`` input ((nsamples, 3) Bx, By, Bz), its geometry from the template.
    energies: CUDA float64 tensor of photon energies [eV].
    """
    fields: list
    obs: tuple
    energies: object
    ctstart: float = 0.0
    ctstop: float = 2.0
    t0: float = 0.0
    npoints: int = 20001
    charge: float = -D.QE
    current: float = 0.5
    mass: float = D.ME
    precision: int = _lib.MIXED
    keep: list = dfield(default_factory=list)

    def grid_index(self):
        idx = [i for i, f in enumerate(self.fields) if f.kind == _lib.GRID]
        if len(idx) > 1:
            raise ValueError("at most one differentiable grid field")
        return idx[0] if idx else None


def _build_fields(problem, grid, amps):
    import torch
    n = len(problem.fields)
    arr = (_lib.Field * max(1, n))()
    data = None
    for i, f in enumerate(problem.fields):
        C.memmove(C.byref(arr[i]), C.byref(f), C.sizeof(_lib.Field))
        if f.kind in AMPLITUDE_KINDS and amps is not None:
            arr[i].field = _lib.v3(amps[i].tolist())
        if f.kind == _lib.GRID and grid is not None:
            data = grid.detach().to(device="cuda", dtype=torch.float64).contiguous()
            arr[i].data = C.cast(data.data_ptr(), _lib._D)
    return arr, data


def forward_flux(problem, grid, amps, ic, keep_efield=False):
    """Flux per energy (CUDA float64) for the given inputs; with keep_efield also the trajectory,
    E_k and the objects the adjoint needs."""
    import torch
    arr, data = _build_fields(problem, grid, amps)
    part, J = particle_from_ic(ic.detach().cpu().numpy() if hasattr(ic, "detach") else ic, problem.charge,
                               problem.mass)
    fields = list(arr)[:len(problem.fields)]
    if problem.precision == _lib.MIXED:
        # a mixed-precision forward integrates the trajectory parallel in time, as sr does for mixed
        # single-particle calculations (within ~1e-15 m of the serial chain); the adjoint differentiates
        # the FP64 loss on whichever trajectory the forward stored
        traj = D.trajectory_shoot(fields, part, problem.ctstart, problem.ctstop, problem.t0, problem.npoints)
    else:
        traj = D.trajectory(fields, [part], problem.ctstart, problem.ctstop, problem.t0, problem.npoints)
    ne = problem.energies.numel()
    flux = torch.empty(ne, dtype=torch.float64, device="cuda")
    e6 = torch.empty(ne * 6, dtype=torch.float64, device="cuda")
    check(lib.srs_spectrum_efield(traj.view(), _lib.BeamConsts(problem.charge, problem.current),
                                  _lib.v3(problem.obs), C.c_void_p(problem.energies.data_ptr()), ne,
                                  int(problem.precision), C.c_void_p(flux.data_ptr()), C.c_void_p(e6.data_ptr()),
                                  D._stream()))
    if keep_efield:
        return flux, (traj, e6, arr, data, part, J)
    return flux


def backward_flux(problem, saved, gflux):
    """dL/d(grid samples) ((nsamples, 3) or None), dL/d(amps) ((nfields, 3)), dL/d(ic) (6,) from
    dL/dflux (CUDA float64, ne)."""
    import torch
    traj, e6, arr, data, part, J = saved
    n = traj.n
    gflux = gflux.detach().to(device="cuda", dtype=torch.float64).contiguous()
    if problem.precision != _lib.FP64:
        # The adjoint's phases must be the forward's own to the last bit (they are ~1e10 rad and the
        # per-point terms along the trajectory cancel to ~1e-10), so the sums E_k it weights with are
        # re-formed in plain FP64 (0.02 % of the forward's time): the gradient is that of the FP64
        # loss, which the mixed-precision loss approximates to ~1e-6.
        ne = problem.energies.numel()
        scratch = torch.empty(ne, dtype=torch.float64, device="cuda")
        e6 = torch.empty(ne * 6, dtype=torch.float64, device="cuda")
        check(lib.srs_spectrum_efield(traj.view(), _lib.BeamConsts(problem.charge, problem.current),
                                      _lib.v3(problem.obs), C.c_void_p(problem.energies.data_ptr()), ne, _lib.FP64,
                                      C.c_void_p(scratch.data_ptr()), C.c_void_p(e6.data_ptr()), D._stream()))
    gx = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    gb = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    beam = _lib.BeamConsts(problem.charge, problem.current)
    check(lib.srs_spectrum_adjoint(traj.view(), beam, _lib.v3(problem.obs), C.c_void_p(problem.energies.data_ptr()),
                                   problem.energies.numel(), C.c_void_p(e6.data_ptr()),
                                   C.c_void_p(gflux.data_ptr()), C.c_void_p(gx.data_ptr()), C.c_void_p(gb.data_ptr()),
                                   D._stream()))
    nf = len(problem.fields)
    gi = problem.grid_index()
    ggrid = torch.zeros_like(data) if (gi is not None and data is not None) else None
    ptrs = (C.c_void_p * max(1, nf))()
    if ggrid is not None:
        ptrs[gi] = ggrid.data_ptr()
    amp = (C.c_double * (3 * max(1, nf)))()
    icg = (C.c_double * 7)()
    check(lib.srs_trajectory_adjoint(arr, nf, C.byref(part), problem.ctstart, problem.ctstop, problem.t0,
                                     problem.npoints, C.c_void_p(traj.x.data_ptr()), C.c_void_p(traj.beta.data_ptr()),
                                     C.c_void_p(gx.data_ptr()), C.c_void_p(gb.data_ptr()), ptrs, amp, icg,
                                     D._stream()))
    g7 = np.array(list(icg))
    gic = g7 @ J
    gamps = np.array(list(amp))[:3 * nf].reshape(nf, 3) if nf else np.zeros((0, 3))
    return ggrid, gamps, gic


class SpectrumFlux:
    """``torch.autograd.Function`` wrapper: ``SpectrumFlux.apply(grid, amps, ic, problem)`` returns the
    flux per energy; gradients flow to grid ((nsamples, 3) samples of the problem's grid field),
    amps ((nfields, 3) amplitude vectors) and ic (6 coordinates)."""

    _fn = None

    @classmethod
    def apply(cls, grid, amps, ic, problem):
        if cls._fn is None:
            cls._fn = _make_function()
        return cls._fn.apply(grid, amps, ic, problem)


def _make_function():
    import torch

    class _SpectrumFlux(torch.autograd.Function):
        @staticmethod
        def forward(ctx, grid, amps, ic, problem):
            flux, saved = forward_flux(problem, grid, amps, ic, keep_efield=True)
            ctx.problem = problem
            ctx.saved = saved
            ctx.devices = (grid.device if grid is not None else None, amps.device if amps is not None else None,
                           ic.device)
            return flux

        @staticmethod
        def backward(ctx, gflux):
            ggrid, gamps, gic = backward_flux(ctx.problem, ctx.saved, gflux)
            dg, da, di = ctx.devices
            out_grid = ggrid.to(dg) if (ggrid is not None and dg is not None) else None
            out_amps = torch.tensor(gamps, dtype=torch.float64, device=da) if da is not None else None
            out_ic = torch.tensor(gic, dtype=torch.float64, device=di)
            ctx.saved = None
            return out_grid, out_amps, out_ic, None

    return _SpectrumFlux


def integrated_flux_loss(flux, de):
    """The config-4 objective: -Sum_k flux_k * dE."""
    return -(flux * de).sum()

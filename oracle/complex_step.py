"""Complex-step derivatives of the integrated on-axis flux -- test infrastructure (the checker of the
adjoint), never part of the product.

A numpy restatement of the reference's forward path for a field given as a 1-D z grid of By samples,
written so that every operation is an analytic function of its inputs:

  particle      TParticleBeam ideal particle: beta0 = d0/|d0| * sqrt(1 - 1/g^2), gamma from |beta0|,
                q/(m gamma)                                   (TParticleBeam.cc:228-265)
  field         TField3D_Grid::GetF, z-only linear interpolation, zero at or outside the ends
                                                              (TField3D_Grid.cc:124-243)
  trajectory    fixed-step RK4 in (x, v), dv/dt = q/(m gamma) v x B, stored state before each step
                                                              (OSCARSSR.cc:562-673, 826-874)
  spectrum      E_k = Sum_i [(beta_i - n_i)/D_i - i (c/w_k) n_i/D_i^2] exp(i w_k (i dt + D_i/c)),
                flux_k = C2 (C0 w_k dt)^2 |E_k|^2           (OSCARSSR.cc:1154-1251)

Every real input may carry an imaginary perturbation i*eps; Im(L)/eps is then dL/d(input) to
machine precision (the complex-step method: W. Squire and G. Trapp, SIAM Review 40 (1998) 110),
free of the subtractive cancellation that makes central differences of the FP64 loss noisy.  The
real part is the ordinary FP64 forward; it is pinned to the reference's own loss when the fixtures
are generated.  Index and branch decisions use real parts, as the reference does on real inputs.
"""
from __future__ import annotations

import numpy as np

C_LIGHT = 2.99792458e8
QE = 1.602176462e-19
ME = 9.10938356e-31
HBAR = 1.054571596e-34
H_PLANCK = 6.62606876e-34
EPS0 = 8.854187817e-12
MU0 = 1.2566370614e-6


def _div(a, b):
    """a / b to first order in the imaginary parts, with the real part computed exactly as the real
    division (numpy's complex division multiplies by a reciprocal, which moves the last bit)."""
    a = np.asarray(a, dtype=complex)
    b = np.asarray(b, dtype=complex)
    re = a.real / b.real
    return re + 1j * ((a.imag - re * b.imag) / b.real)


def _sqrt(a):
    a = np.asarray(a, dtype=complex)
    r = np.sqrt(a.real)
    return r + 1j * (a.imag / (2.0 * r))


def _particles(ic, charge=-QE, mass=ME):
    """(m, 6) complex (x, y, x', y', z, E[GeV]) -> x0 (m,3), v0 (m,3), qomg (m,), in the ideal
    particle's operation order."""
    ic = np.asarray(ic, dtype=complex)
    g = _div(ic[:, 5], 1e-9 * mass * C_LIGHT * C_LIGHT / QE)
    beta = _sqrt(1.0 - _div(1.0, g * g))
    d = [ic[:, 2], ic[:, 3], np.ones(len(ic), dtype=complex)]
    dn = _sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
    b0 = [_div(d[k], dn) * beta for k in range(3)]
    b2 = b0[0] * b0[0] + b0[1] * b0[1] + b0[2] * b0[2]
    gamma = _div(1.0, _sqrt(1.0 - b2))
    x0 = np.stack([ic[:, 0], ic[:, 1], ic[:, 4]], 1)
    v0 = np.stack([b0[k] * C_LIGHT for k in range(3)], 1)
    return x0, v0, _div(_div(charge, mass), gamma)


def grid_z_field(by, z0, dz):
    """TField3D_Grid::GetF for a z-only map (TField3D_Grid.cc:124-243): By samples per row (m, nz),
    a + ((b - a) d) / step with d = (z - start) - k step; zero at or outside the ends."""
    by = np.asarray(by, dtype=complex)

    def field(pos):
        m, nz = by.shape
        z = pos[:, 2]
        zr = z.real
        inside = (zr > z0) & (zr < z0 + (nz - 1) * dz)
        k = np.clip(((zr - z0) / dz).astype(np.int64), 0, nz - 2)
        d = (z - z0) - k * dz
        rows = np.arange(m)
        a, b = by[rows, k], by[rows, k + 1]
        B = np.zeros((m, 3), dtype=complex)
        B[:, 1] = np.where(inside, a + _div((b - a) * d, dz), 0)
        return B
    return field


def undulator_field(F, period, nperiods, phase=0.0, center=(0.0, 0.0, 0.0), taper=0.0):
    """TField3D_IdealUndulator::GetF (TField3D_IdealUndulator.cc:106-139); F: (m, 3) amplitude rows."""
    F = np.asarray(F, dtype=complex)
    per = np.asarray(period, float)
    plen = float(np.sqrt(per @ per))
    u = per / plen
    L = plen * (nperiods + 2)
    ps = phase * plen / (2.0 * np.pi)
    ctr = np.asarray(center, float)

    def field(pos):
        D = (pos[:, 0] - ctr[0]) * u[0] + (pos[:, 1] - ctr[1]) * u[1] + (pos[:, 2] - ctr[2]) * u[2]
        Dr = D.real
        s = np.sin(_div(2.0 * np.pi * (D - ps), plen))
        fac = np.where((Dr < -L / 2. + ps + plen) | (Dr > L / 2. + ps - plen),
                       np.where((Dr < -L / 2. + ps + plen / 2.) | (Dr > L / 2. + ps - plen / 2.), 0.25, 0.75), 1.0)
        fac = np.where((Dr > L / 2. + ps) | (Dr < -L / 2. + ps), 0.0, fac)
        return F * (fac * s * (1 + D * taper))[:, None]
    return field


def gaussian_field(F, center, sigma):
    """TField3D_Gaussian::GetF (TField3D_Gaussian.cc:88-113), no rotation."""
    F = np.asarray(F, dtype=complex)
    ctr, sg = np.asarray(center, float), np.asarray(sigma, float)

    def field(pos):
        frac = np.ones(len(pos), dtype=complex)
        for a in range(3):
            if sg[a] > 0:
                t = _div(pos[:, a] - ctr[a], sg[a])
                frac = frac * np.exp(-(t * t) / 2.)
        return F * frac[:, None]
    return field


def box_field(F, center, width):
    """TField3D_UniformBox::GetF (TField3D_UniformBox.cc:93-111), no rotation."""
    F = np.asarray(F, dtype=complex)
    ctr, w = np.asarray(center, float), np.asarray(width, float)

    def field(pos):
        inside = np.ones(len(pos), dtype=bool)
        for a in range(3):
            if w[a] > 0:
                inside &= np.abs((pos[:, a] - ctr[a]).real) <= abs(w[a] / 2.)
        return F * inside[:, None]
    return field


def _force(q, v, B):
    """q/(m gamma) (v x B) in the integrator's operation order."""
    return np.stack([q * (-v[:, 2] * B[:, 1] + v[:, 1] * B[:, 2]), q * (v[:, 2] * B[:, 0] - v[:, 0] * B[:, 2]),
                     q * (v[:, 0] * B[:, 1] - v[:, 1] * B[:, 0])], 1)


def _rk4(fields, q, pos, vel, h):
    def B(p):
        tot = fields[0](p)
        for f in fields[1:]:
            tot = tot + f(p)
        return tot
    hh, h6 = h * 0.5, h / 6.0
    a1 = _force(q, vel, B(pos))
    p2 = pos + hh * vel
    v2 = vel + hh * a1
    a2 = _force(q, v2, B(p2))
    p3 = pos + hh * v2
    v3 = vel + hh * a2
    p4 = pos + h * v3
    a3 = _force(q, v3, B(p3))
    v4 = vel + h * a3
    m_pos, m_vel = v3 + v2, a3 + a2
    a4 = _force(q, v4, B(p4))
    return pos + h6 * (vel + v4 + 2.0 * m_pos), vel + h6 * (a1 + a4 + 2.0 * m_vel)


def trajectory_fields(fields, ic, ctstart=0.0, ctstop=2.0, t0=0.0, npoints=20001):
    """RK4 states through a list of field callables (OSCARSSR.cc:562-673): forward from t0 stored at
    nbackward.., backward (step -dt) stored at nbackward-1 down to 0.  X, V: (m, n, 3)."""
    x0, v0, q = _particles(ic)
    dt = (ctstop - ctstart) / C_LIGHT / (npoints - 1)
    nf = int(1 + (ctstop - t0) / C_LIGHT / dt)
    nb = int((t0 - ctstart) / C_LIGHT / dt)
    m = len(ic)
    X = np.zeros((m, nf + nb, 3), dtype=complex)
    V = np.zeros((m, nf + nb, 3), dtype=complex)
    pos, vel = x0.copy(), v0.copy()
    for i in range(nf):
        X[:, nb + i], V[:, nb + i] = pos, vel
        pos, vel = _rk4(fields, q, pos, vel, dt)
    pos, vel = x0.copy(), v0.copy()
    for i in range(nb):
        pos, vel = _rk4(fields, q, pos, vel, -dt)
        X[:, nb - 1 - i], V[:, nb - 1 - i] = pos, vel
    return X, V, dt


def trajectory(by, z0, dz, ic, ctstart=0.0, ctstop=2.0, npoints=20001):
    """Forward RK4 states through a z-only grid field (t0 = ctstart): X, V of shape (m, N, 3)."""
    return trajectory_fields([grid_z_field(by, z0, dz)], ic, ctstart, ctstop, ctstart, npoints)


def flux(X, V, dt, obs, energies, charge=-QE, current=0.5):
    """(m, ne) flux of every trajectory, in the reference's CPU operation order
    (amplitude (B - N (1 + i (c/w)/D))/D, phase w (dt i + D/c)), sums in point order."""
    R = np.asarray(obs, float)[None, None, :] - X
    D = _sqrt(R[..., 0] * R[..., 0] + R[..., 1] * R[..., 1] + R[..., 2] * R[..., 2])
    n = _div(R, D[..., None])
    Bt = _div(V, C_LIGHT)
    N = X.shape[1]
    t = dt * np.arange(N)[None, :] + _div(D, C_LIGHT)
    c0 = charge / (4 * np.pi * C_LIGHT * EPS0 * np.sqrt(2 * np.pi))
    c2 = 4 * np.pi * current / (H_PLANCK * abs(charge) * MU0 * C_LIGHT) * 1e-6 * 0.001
    ar = _div(Bt - n, D[..., None])
    out = np.zeros((X.shape[0], len(energies)), dtype=complex)
    for k, e in enumerate(energies):
        w = e * QE / HBAR
        ph = w * t
        cs, sn = np.cos(ph)[..., None], np.sin(ph)[..., None]
        f = _div(C_LIGHT / w, D)[..., None]
        ai = _div(-(n * f), D[..., None])
        er = np.cumsum(ar * cs - ai * sn, axis=1)[:, -1]
        ei = np.cumsum(ar * sn + ai * cs, axis=1)[:, -1]
        g = (c0 * w) * dt
        parts = [(er[:, c] * g) * (er[:, c] * g) + (ei[:, c] * g) * (ei[:, c] * g) for c in range(3)]
        out[:, k] = c2 * ((parts[0] + parts[1]) + parts[2])
    return out


def weighted_flux(fields, ic, obs, energies, weights, ctstart=0.0, ctstop=2.0, t0=0.0, npoints=20001,
                  charge=-QE, current=0.5):
    """Sum_k weights_k flux_k for each row (fields built from per-row parameters)."""
    X, V, dt = trajectory_fields(fields, ic, ctstart, ctstop, t0, npoints)
    return (flux(X, V, dt, obs, energies, charge, current) * np.asarray(weights)[None, :]).sum(1)


def integrated_loss(by, z0, dz, ic, obs, energies, de, npoints=20001):
    """-Sum_k flux_k dE for each row of (by (m, nz), ic (m, 6))."""
    X, V, dt = trajectory(by, z0, dz, ic, npoints=npoints)
    return -(flux(X, V, dt, obs, energies) * de).sum(1)


def complex_step_gradient(by, ic, coords, z0, dz, obs, energies, de, eps=1e-30, npoints=20001):
    """dL/d(coordinate) for each index in coords (into By samples, then x, y, x', y', z, E), all
    perturbed trajectories run as one batch.  Returns (gradients, real loss)."""
    nz = len(by)
    m = len(coords)
    B = np.tile(np.asarray(by, dtype=complex), (m, 1))
    IC = np.tile(np.asarray(ic, dtype=complex), (m, 1))
    for r, k in enumerate(coords):
        if k < nz:
            B[r, k] += 1j * eps
        else:
            IC[r, k - nz] += 1j * eps
    L = integrated_loss(B, z0, dz, IC, obs, energies, de, npoints)
    return L.imag / eps, L.real

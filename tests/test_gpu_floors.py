"""Mixed-precision error at both floors the accuracy is stated on, through the C ABI.

* Outputs >= 1e-3 of their map's (or spectrum's) maximum: the mixed kernels within 1e-4 relative of
  the plain FP64 kernels, point by point, and within 1e-5 normwise.
* Outputs >= 1e-6 of the maximum.  Here the FP64 kernels stop being a yardstick at 1e-4: the retarded
  phase w (t + D/c) is 1e10-1e11 rad, FP64 keeps it to ~1e-5 rad per term in any evaluation order
  (the reference's CPU path included), and at outputs a million times below the peak that rounding
  alone moves an FP64 result by ~3e-4 (3*E1 map) to ~2e-3 (spectrum).  So the mixed and the FP64
  results are both compared with the exact sum -- the same formula on the same FP64 trajectory,
  evaluated in long double by the oracle (oracle.flux_exact / spectrum_exact, ~1e-8 rad per term) --
  at the weakest outputs above the floor and at a sample of the others, and the mixed kernel must be
  within 1e-4 of it, or no further from it than 1.5 times the FP64 kernel is.
* Power density has no phase: the mixed kernel is held to 1e-4 of the FP64 kernel at both floors.
"""
import numpy as np
import pytest

import oracle as O
from srsoriginal_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL, TOL_NORM, FP64_FACTOR = 1e-4, 1e-5, 1.5
NWEAK, NSAMPLE = 48, 48


def host_and_device_trajectory(npoints, fields="undulator"):
    import torch
    from srsoriginal_b200 import device as D
    o = O.OracleSR()
    W.setup_beam(o, npoints)
    (W.setup_undulator if fields == "undulator" else W.setup_epu)(o)
    X, B, A, dt = o.trajectory()
    t = [torch.as_tensor(np.ascontiguousarray(a).reshape(1, 3, -1), device="cuda") for a in (X, B, A)]
    return (X, B, A, dt), D.Trajectory(t[0], t[1], t[2], dt)


def floor_points(ref, floor, rng):
    """The NWEAK weakest outputs >= floor * max, and NSAMPLE others above the floor."""
    m = np.abs(ref).max()
    idx = np.where(np.abs(ref) >= floor * m)[0]
    order = idx[np.argsort(np.abs(ref[idx]))]
    weak, rest = order[:NWEAK], order[NWEAK:]
    sample = rng.choice(rest, size=min(NSAMPLE, len(rest)), replace=False) if len(rest) else rest
    return np.concatenate([weak, sample])


def check_floors(mixed, fp64, exact_at, seed=0):
    """Both floors; returns (max rel mixed vs fp64 at 1e-3, at 1e-6, mixed vs exact, fp64 vs exact)."""
    mixed, fp64 = np.asarray(mixed, float), np.asarray(fp64, float)
    m = np.abs(fp64).max()
    big = np.abs(fp64) >= 1e-3 * m
    e3 = float(np.max(np.abs(mixed[big] - fp64[big]) / np.abs(fp64[big])))
    nrm = float(np.linalg.norm(mixed - fp64) / np.linalg.norm(fp64))
    assert e3 <= TOL and nrm <= TOL_NORM, (e3, nrm)
    low = np.abs(fp64) >= 1e-6 * m
    e6 = float(np.max(np.abs(mixed[low] - fp64[low]) / np.abs(fp64[low])))
    idx = floor_points(fp64, 1e-6, np.random.default_rng(seed))
    ex = exact_at(idx)
    em = float(np.max(np.abs(mixed[idx] / ex - 1)))
    ef = float(np.max(np.abs(fp64[idx] / ex - 1)))
    assert em <= max(TOL, FP64_FACTOR * ef), (em, ef)
    return e3, e6, em, ef


@pytest.mark.parametrize("energy", [W.E1_EV, W.E3_EV])
def test_flux_cfg1_both_floors(energy):
    """Config 1 maps (101 x 101, 10 mm at 30 m) from the grid (anchored) and the point-list mixed kernels."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    (X, B, A, dt), tr = host_and_device_trajectory(20001)
    xyz, _, _, grid = rectangle_points([101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30])
    P = np.ascontiguousarray(xyz.reshape(-1, 3))
    pts = torch.as_tensor(P.reshape(-1), device="cuda")
    g, p, f = (torch.empty(101 * 101, dtype=torch.float64, device="cuda") for _ in range(3))
    D.flux(tr, -O.QE, 0.5, energy, g, grid=grid, precision=_lib.MIXED)
    D.flux(tr, -O.QE, 0.5, energy, p, points=pts, precision=_lib.MIXED)
    D.flux(tr, -O.QE, 0.5, energy, f, points=pts, precision=_lib.FP64)
    torch.cuda.synchronize()
    exact_at = lambda idx: O.flux_exact(X, B, dt, P[idx], energy, -O.QE, 0.5)
    f64 = f.cpu().numpy()
    for mixed in (g.cpu().numpy(), p.cpu().numpy()):
        check_floors(mixed, f64, exact_at)


@pytest.mark.parametrize("ne", [1000, 2000])
def test_spectrum_cfg0_both_floors(ne):
    """On-axis spectrum at 30 m over 100-1000 eV (the reference's grid), 1000 energies (config 0) and
    2000 (config 3a's grid)."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    (X, B, A, dt), tr = host_and_device_trajectory(20001)
    en = O.energy_grid(ne, 100.0, 1000.0)
    e = torch.as_tensor(en, device="cuda")
    m, f = (torch.empty(ne, dtype=torch.float64, device="cuda") for _ in range(2))
    D.spectrum(tr, -O.QE, 0.5, [0, 0, 30], e, m, precision=_lib.MIXED)
    D.spectrum(tr, -O.QE, 0.5, [0, 0, 30], e, f, precision=_lib.FP64)
    torch.cuda.synchronize()
    exact_at = lambda idx: O.spectrum_exact(X, B, dt, [0, 0, 30], en[idx], -O.QE, 0.5)
    check_floors(m.cpu().numpy(), f.cpu().numpy(), exact_at)


def test_power_density_cfg2_both_floors():
    """Config 2 (201 x 201 on 40 mm at 30 m, elliptical undulator, 40001 points): no phase, so FP64 is
    the yardstick at both floors."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    _, tr = host_and_device_trajectory(40001, "epu")
    xyz, _, nrm, grid = rectangle_points([201, 201], "XY", [0.04, 0.04], translation=[0, 0, 30])
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
    nrms = torch.as_tensor(np.ascontiguousarray(np.tile(nrm, (201 * 201, 1)).reshape(-1)), device="cuda")
    a, c = (torch.empty(201 * 201, dtype=torch.float64, device="cuda") for _ in range(2))
    D.power_density(tr, -O.QE, 0.5, a, grid=grid, precision=_lib.MIXED)
    D.power_density(tr, -O.QE, 0.5, c, points=pts, normals=nrms, precision=_lib.FP64)
    torch.cuda.synchronize()
    a, c = a.cpu().numpy(), c.cpu().numpy()
    for floor in (1e-3, 1e-6):
        big = np.abs(c) >= floor * np.abs(c).max()
        assert np.max(np.abs(a[big] - c[big]) / np.abs(c[big])) <= TOL

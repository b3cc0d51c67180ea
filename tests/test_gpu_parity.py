"""GPU parity: the CUDA path (through the C ABI) against the reference's own outputs (golden fixtures
made by running the reference) and against the oracle on seeded random inputs.

Tolerances (stated per test):
  * trajectory (FP64 RK4, reference operation order): relative 1e-12 per component scale.  It is not
    bit-identical: the device sine and glibc's differ in the last bit for some arguments (glibc's own
    sine is not correctly rounded for ~0.15% of arguments), which moves x by ~1e-18 m;
  * plain FP64 sums on the reference's trajectory (the seam the reference's GPU path uses: the host
    hands over the trajectory) vs the reference CPU path: relative 1e-10, taken as the max over outputs
    with value >= 1e-6 of the maximum (near exact nulls the relative error is ill-conditioned), plus
    the normwise error ||a-b||/||b|| <= 1e-12;
  * end to end (device trajectory + plain FP64 sums): normwise 1e-10, and 1e-6 relative over outputs
    >= 1e-6 of the maximum -- weak points of a flux map amplify the trajectory's last-bit differences;
  * mixed-precision sums vs the same reference: max relative error 1e-4 over outputs >= 1e-3 of the
    maximum, normwise 1e-5.
"""
import ctypes as C
import json
import math
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden
from srsoriginal_b200 import workloads as W

pytestmark = pytest.mark.gpu

TOL_FP64, TOL_FP64_NORM = 1e-10, 1e-12
TOL_MIXED, TOL_MIXED_NORM = 1e-4, 1e-5


def rel_err(a, b, floor):
    a, b = np.asarray(a, float), np.asarray(b, float)
    if np.abs(b).max() == 0:  # e.g. a directional power density that sees no radiation
        return float(np.abs(a).max()), float(np.abs(a).max())
    big = np.abs(b) >= floor * np.abs(b).max()
    mx = float(np.max(np.abs(a[big] - b[big]) / np.abs(b[big])))
    nrm = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return mx, nrm


def assert_fp64(a, b):
    mx, nrm = rel_err(a, b, 1e-6)
    assert mx <= TOL_FP64 and nrm <= TOL_FP64_NORM, (mx, nrm)


def assert_e2e(a, b):
    mx, nrm = rel_err(a, b, 1e-6)
    assert mx <= 1e-6 and nrm <= 1e-10, (mx, nrm)


def assert_mixed(a, b):
    mx, nrm = rel_err(a, b, 1e-3)
    assert mx <= TOL_MIXED and nrm <= TOL_MIXED_NORM, (mx, nrm)


def reference_trajectory_on_device(npoints, fields="undulator"):
    """The reference's trajectory (the oracle reproduces it bit for bit) as a device Trajectory."""
    import torch
    from srsoriginal_b200 import device as D
    o = O.OracleSR()
    W.setup_beam(o, npoints)
    (W.setup_undulator if fields == "undulator" else W.setup_epu)(o)
    X, B, A, dt = o.trajectory()
    t = [torch.as_tensor(np.ascontiguousarray(a).reshape(1, 3, -1), device="cuda") for a in (X, B, A)]
    return D.Trajectory(t[0], t[1], t[2], dt)


def test_sum_kernels_on_reference_trajectory_fp64():
    """The plain FP64 sums given the reference's own trajectory: the drop-in for the reference's GPU
    seam (OSCARSSR_Cuda_Calculate*GPU receive the host-computed trajectory)."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    g0, g1, g2 = golden("spectrum_cfg0.npz"), golden("flux_cfg1.npz"), golden("pd_cfg2.npz")
    tr = reference_trajectory_on_device(20001)
    e = torch.as_tensor(g0["energies"], device="cuda")
    out = torch.empty(1000, dtype=torch.float64, device="cuda")
    D.spectrum(tr, -O.QE, 0.5, [0, 0, 30], e, out, precision=_lib.FP64)
    torch.cuda.synchronize()
    assert_fp64(out.cpu().numpy(), g0["flux"])
    xyz, x12, nrm, grid = rectangle_points([101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30])
    pts = torch.as_tensor(xyz.reshape(-1), device="cuda")
    out = torch.empty(10201, dtype=torch.float64, device="cuda")
    for tag in ("e1", "e3"):
        D.flux(tr, -O.QE, 0.5, float(g1["energy_" + tag]), out, points=pts, grid=grid, precision=_lib.FP64)
        torch.cuda.synchronize()
        assert_fp64(out.cpu().numpy(), g1["flux_" + tag])
    tr = reference_trajectory_on_device(40001, "epu")
    xyz, x12, nrm, grid = rectangle_points([201, 201], "XY", [0.04, 0.04], translation=[0, 0, 30])
    pts = torch.as_tensor(xyz.reshape(-1), device="cuda")
    nrms = torch.as_tensor(np.tile(nrm, 201 * 201), device="cuda")
    out = torch.empty(201 * 201, dtype=torch.float64, device="cuda")
    D.power_density(tr, -O.QE, 0.5, out, points=pts, normals=nrms, precision=_lib.FP64)
    torch.cuda.synchronize()
    assert_fp64(out.cpu().numpy(), g2["pd"])


def new_sr(npoints=20001, fields="undulator", **beam):
    from srsoriginal_b200.sr import sr
    o = sr()
    W.setup_beam(o, npoints, **beam)
    if fields == "undulator":
        W.setup_undulator(o)
    elif fields == "epu":
        W.setup_epu(o)
    return o


def traj_close(X, ref, tol=1e-12):
    scale = np.maximum(np.abs(ref).max(axis=1, keepdims=True), 1e-300)
    return float(np.max(np.abs(X - ref) / scale)) <= tol


# ------------------------------------------------------------------ trajectory

def test_trajectory_cfg0_matches_reference():
    g = golden("spectrum_cfg0.npz")
    o = new_sr(2001)
    x, b = o._trajectory_arrays()
    assert traj_close(x.T, g["small_x"]) and traj_close(b.T, g["small_beta"])
    o = new_sr(20001)
    x, b = o._trajectory_arrays()
    assert x.shape[0] == int(g["n"])
    assert traj_close(x.T[:, ::50], g["x_sub"]) and traj_close(b.T[:, ::50], g["beta_sub"])
    lst = o.calculate_trajectory()
    assert len(lst) == 20001 and len(lst[0]) == 2 and len(lst[0][0]) == 3


def test_total_power_matches_reference():
    """FP64, reference order; tolerance 1e-10 (the trajectory's sine ulps reach ~1e-11 here)."""
    g = golden("spectrum_cfg0.npz")
    assert abs(new_sr(20001).calculate_total_power() / float(g["total_power"]) - 1) < 1e-10
    g2 = golden("pd_cfg2.npz")
    assert abs(new_sr(40001, "epu").calculate_total_power() / float(g2["total_power"]) - 1) < 1e-10


# ------------------------------------------------------------------ plain FP64 sums (the drop-in)

def test_spectrum_cfg0_fp64_matches_reference():
    g = golden("spectrum_cfg0.npz")
    o = new_sr(20001)
    s = np.array(o.calculate_spectrum(obs=[0, 0, 30], npoints=1000, energy_range_eV=[100, 1000]))
    assert np.array_equal(s[:, 0], g["energies"])
    assert_e2e(s[:, 1], g["flux"])


def test_flux_cfg1_fp64_matches_reference():
    g = golden("flux_cfg1.npz")
    o = new_sr(20001)
    for tag in ("e1", "e3"):
        m = o.calculate_flux_rectangle(plane="XY", energy_eV=float(g["energy_" + tag]), width=[0.01, 0.01],
                                       npoints=[101, 101], translation=[0, 0, 30])
        assert len(m) == 101 * 101  # default nthreads (threads path): one entry per point
        v = np.array([p[1] for p in m])
        assert np.array_equal(np.array([p[0][:2] for p in m]), g["x12"])
        assert_e2e(v, g["flux_" + tag])


def test_power_density_cfg2_fp64_matches_reference():
    g = golden("pd_cfg2.npz")
    o = new_sr(40001, "epu")
    m = o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04], npoints=[201, 201],
                                            translation=[0, 0, 30])
    assert len(m) == int(g["nlist"])  # threads path lists the points twice (reference quirk)
    v = np.array([p[1] for p in m])[:201 * 201]
    assert_e2e(v, g["pd"])


def test_misc_fields_surfaces_directional_fp64():
    from srsoriginal_b200.sr import sr
    g = golden("misc_fields.npz")
    o = sr()
    W.setup_beam(o, 3001)
    o.add_bfield_undulator(bfield=[0, 0.8, 0.05], period=[0, 0, 0.05], nperiods=11, phase=0.3,
                           rotations=[0.001, -0.002, 0.3], translation=[0.0001, 0, 0.05], taper=0.01)
    o.add_bfield_gaussian(bfield=[0.02, 0.3, 0], sigma=[0, 0, 0.05], translation=[0, 0, -0.5],
                          rotations=[0, 0.01, 0])
    o.add_bfield_uniform(bfield=[0.0, -0.01, 0.001], width=[0, 0, 0.2], translation=[0, 0, 0.5],
                         rotations=[0.02, 0, 0])
    bf = np.array([o.get_bfield([0.0001 * i, -0.0002 * i, -1 + 0.1 * i]) for i in range(21)])
    assert np.allclose(bf, g["bfield"], rtol=1e-15, atol=1e-300)
    x, b = o._trajectory_arrays()
    assert traj_close(x.T, g["x"]) and traj_close(b.T, g["beta"])
    s = np.array(o.calculate_spectrum(obs=[0.001, -0.0005, 20], npoints=40, energy_range_eV=[50, 2000], nthreads=1))
    assert_fp64(s[:, 1], g["flux"])
    s = np.array(o.calculate_spectrum(obs=[0, 0, 25], points_eV=[75.0, 133.3, 401.0, 999.9], nthreads=1))
    assert_fp64(s[:, 1], g["pts_flux"])
    p = o.calculate_power_density_rectangle(plane="YZ", width=[0.02, 0.03], npoints=[7, 9],
                                            rotations=[0, -math.pi / 2, 0], translation=[0.001, 0, 20], normal=1,
                                            nthreads=1)
    assert_fp64([q[1] for q in p], g["pd_dir"])
    assert np.array_equal(np.array([q[0] for q in p]), g["pd_dir_xyz"])
    p = o.calculate_power_density_rectangle(plane="YZ", width=[0.02, 0.03], npoints=[7, 9],
                                            rotations=[0, -math.pi / 2, 0], translation=[0.001, 0, 20], normal=-1,
                                            nthreads=1)
    assert_fp64([q[1] for q in p], g["pd_neg"])
    f = o.calculate_flux_rectangle(energy_eV=300.0, npoints=[6, 5], x0x1x2=[[-0.004, -0.003, 25],
                                                                           [0.004, -0.003, 25],
                                                                           [-0.004, 0.003, 25.1]],
                                   nthreads=1, dim=3)
    assert len(f) == int(g["flux_x0x1x2_len"])
    assert_fp64([q[1] for q in f][:30], g["flux_x0x1x2"])
    assert abs(o.calculate_total_power() / float(g["total_power"]) - 1) < 1e-10


def test_beam_sampling_and_multiparticle_match_reference():
    """Replays the fixture's history in one generator state: Twiss-sampled particles after set_seed(0)
    (bit-identical draws), then nparticles > 0 sums (weighted 1/N and Kahan-summed in particle order;
    the power density's CPU paths add without weight), then plain draws after set_seed(7.9).  A reseed
    keeps the normal distribution's cached value, as the reference's does."""
    from srsoriginal_b200.sr import reset_random
    g = golden("beam_3a.npz")
    o = new_sr(2001, **W.BEAM_3A)
    reset_random(0)  # a fresh process's generator after set_seed(0)
    xs = []
    for _ in range(33):
        o.set_new_particle(particle="random")
        xs.append(o.get_particle_x0() + o.get_particle_beta0())
    assert np.array_equal(np.array(xs), np.concatenate([g["x0"], g["beta0"]], axis=1))
    o.set_seed(0)
    s = np.array(o.calculate_spectrum(obs=[0, 0, 30], npoints=48, energy_range_eV=[100, 1000], nparticles=4,
                                      nthreads=1))
    assert_fp64(s[:, 1], g["flux"])
    o.set_seed(0)
    f = o.calculate_flux_rectangle(plane="XY", energy_eV=W.E1_EV, width=[0.01, 0.01], npoints=[5, 5],
                                   translation=[0, 0, 30], nparticles=3, nthreads=1)
    assert len(f) == int(g["flux_map_len"])
    assert_fp64([q[1] for q in f][:25], g["flux_map"][:25])
    o.set_seed(0)
    p = o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04], npoints=[5, 5],
                                            translation=[0, 0, 30], nparticles=3, nthreads=1)
    assert len(p) == int(g["pd_map_len"])
    assert_fp64([q[1] for q in p][:25], g["pd_map"][:25])
    o.set_seed(7.9)
    u = [o.rand() for _ in range(5)] + [o.norm() for _ in range(5)]
    assert np.array_equal(np.array(u), g["draws"])


def test_grid_field_file_cfg4():
    g = golden("grid_cfg4.npz")
    from srsoriginal_b200.sr import sr
    z, by = W.config4_grid()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "cfg4.txt")
        W.write_oscars_grid(path, z, by)
        o = sr()
        W.setup_beam(o, 20001)
        o.add_bfield_file(ifile=path, iformat="OSCARS")
    bf = np.array([o.get_bfield([0, 0, -0.9 + 0.0123 * i]) for i in range(150)])
    assert np.allclose(bf, g["bfield"], rtol=1e-15, atol=0)
    x, b = o._trajectory_arrays()
    assert traj_close(x.T[:, ::50], g["x_sub"])
    s = np.array(o.calculate_spectrum(obs=[0, 0, 30], npoints=200, energy_range_eV=[0.98 * W.E3_EV, 1.02 * W.E3_EV]))
    assert_fp64(s[:, 1], g["flux"])


def test_dispatch_list_shapes_match_reference():
    q = json.load(open(os.path.join(ROOT, "tests", "golden", "quirks.json")))
    for nthreads in (1, 2):
        o = new_sr(501)
        f = o.calculate_flux_rectangle(plane="XY", energy_eV=150.0, width=[0.01, 0.01], npoints=[3, 4],
                                       translation=[0, 0, 30], nthreads=nthreads)
        p = o.calculate_power_density_rectangle(plane="XY", width=[0.01, 0.01], npoints=[3, 4],
                                                translation=[0, 0, 30], nthreads=nthreads)
        p3 = o.calculate_power_density_rectangle(plane="XY", width=[0.01, 0.01], npoints=[3, 4],
                                                 translation=[0, 0, 30], nthreads=nthreads, dim=3)
        assert len(f) == q[f"flux_len_nthreads{nthreads}"]
        assert len(p) == q[f"pd_len_nthreads{nthreads}"]
        assert p3[0][0] == q[f"pd_dim3_first_nthreads{nthreads}"]
        assert [c[0] for c in f] == q[f"flux_coords_nthreads{nthreads}"]
    # gpu=1 path: 2N entries, the second half with x,y,z coordinates
    o = new_sr(501)
    f = o.calculate_flux_rectangle(plane="XY", energy_eV=150.0, width=[0.01, 0.01], npoints=[3, 4],
                                   translation=[0, 0, 30], gpu=1)
    assert len(f) == 24 and f[12][0][2] == 30.0
    with pytest.raises(ValueError, match="gpu is 1 and nthreads > 0"):
        o.calculate_spectrum(obs=[0, 0, 30], npoints=3, energy_range_eV=[100, 200], gpu=1, nthreads=2)
    with pytest.raises(ValueError, match="'gpu' must be 0 or 1"):
        o.calculate_spectrum(obs=[0, 0, 30], npoints=3, energy_range_eV=[100, 200], gpu=2)


# ------------------------------------------------------------------ C ABI against the oracle, random inputs

def _dev(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _vp(t):
    return C.c_void_p(t.data_ptr())


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_c_abi_random_fields_and_points_vs_oracle(seed):
    """srs_trajectory / srs_spectrum / srs_flux / srs_power_density called directly with device buffers,
    on seeded random field layouts and observation points, against the oracle."""
    import torch
    from srsoriginal_b200 import _lib
    L = _lib.lib
    rng = np.random.default_rng(seed)
    ofl = [O.undulator([0, rng.uniform(0.3, 1.2), rng.uniform(-0.1, 0.1)], [0, 0, rng.uniform(0.02, 0.08)],
                       int(rng.integers(3, 15)), phase=rng.uniform(-1, 1),
                       rotations=rng.uniform(-0.01, 0.01, 3), translation=[0, 0, rng.uniform(-0.1, 0.1)]),
           O.gaussian([rng.uniform(-0.2, 0.2), 0.1, 0], [0, 0, 0.1], translation=[0, 0, -0.4])]
    fl = (_lib.Field * 2)()
    for k, f in enumerate(ofl):
        for name, _ in _lib.Field._fields_:
            if name != "data":
                setattr(fl[k], name, getattr(f, name))
    x0 = [rng.uniform(-1e-4, 1e-4), rng.uniform(-1e-4, 1e-4), -1.0]
    bm = O.Beam(energy_GeV=rng.uniform(1.5, 3.5), x0=x0, d0=[rng.uniform(-1e-4, 1e-4), 0, 1], current=0.4)
    px0, pb0, gam, qomg = bm.particle(False)
    npts = int(rng.integers(500, 3000))
    X, Bv, A, dt = O.trajectory(ofl, px0, pb0, qomg, 0.0, 2.0, 0.0, npts)
    n = X.shape[1]
    part = _lib.Particle()
    part.x0 = _lib.v3(px0)
    part.beta0 = _lib.v3(pb0)
    part.qomg = qomg
    dx, db, da = (torch.empty(3 * n, dtype=torch.float64, device="cuda") for _ in range(3))
    _lib.check(L.srs_trajectory(fl, 2, C.byref(part), 1, 0.0, 2.0, 0.0, npts, _vp(dx), _vp(db), _vp(da), None))
    torch.cuda.synchronize()
    assert traj_close(dx.cpu().numpy().reshape(3, n), X) and traj_close(db.cpu().numpy().reshape(3, n), Bv)
    view = _lib.TrajView(C.cast(dx.data_ptr(), _lib._D), C.cast(db.data_ptr(), _lib._D),
                         C.cast(da.data_ptr(), _lib._D), n, 1, dt)
    beam = _lib.BeamConsts(bm.b.q, bm.b.current)
    # spectrum at a random observer
    obs = [rng.uniform(-1e-3, 1e-3), rng.uniform(-1e-3, 1e-3), rng.uniform(10, 40)]
    e = np.sort(rng.uniform(50, 3000, 37))
    de, out = _dev(e), torch.empty(37, dtype=torch.float64, device="cuda")
    _lib.check(L.srs_spectrum(view, beam, _lib.v3(obs), _vp(de), 37, _lib.FP64, _vp(out), None))
    assert_fp64(out.cpu().numpy(), O.spectrum(X, Bv, dt, obs, e, bm.b.q, bm.b.current))
    # flux and power density at random points
    P = np.column_stack([rng.uniform(-5e-3, 5e-3, 29), rng.uniform(-5e-3, 5e-3, 29), rng.uniform(15, 35, 29)])
    Nn = np.tile([0.0, 0.0, 1.0], (29, 1))
    dp, dn, out = _dev(P.reshape(-1)), _dev(Nn.reshape(-1)), torch.empty(29, dtype=torch.float64, device="cuda")
    _lib.check(L.srs_flux(view, beam, _vp(dp), 29, None, 411.0, _lib.FP64, _vp(out), None))
    assert_fp64(out.cpu().numpy(), O.flux(X, Bv, dt, P, 411.0, bm.b.q, bm.b.current))
    for directional in (0, 1):
        _lib.check(L.srs_power_density(view, beam, _vp(dp), _vp(dn), 29, None, directional, _lib.FP64, _vp(out),
                                       None))
        assert_fp64(out.cpu().numpy(), O.power_density(X, Bv, A, dt, P, Nn, directional, bm.b.q, bm.b.current))


def test_c_abi_rejects_bad_arguments():
    from srsoriginal_b200 import _lib
    view = _lib.TrajView(None, None, None, 0, 1, 1e-12)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib.srs_spectrum(view, _lib.BeamConsts(-1.6e-19, 0.5), _lib.v3([0, 0, 1]), None, 0,
                                         _lib.FP64, None, None))
    t = _dev(np.zeros(30))
    v = _lib.TrajView(C.cast(t.data_ptr(), _lib._D), C.cast(t.data_ptr(), _lib._D),
                      C.cast(t.data_ptr(), _lib._D), 10, 1, 1e-12)
    with pytest.raises(ValueError, match="NULL points"):  # mixed without a grid needs the point list
        _lib.check(_lib.lib.srs_flux(v, _lib.BeamConsts(-1.6e-19, 0.5), None, 3, None, 100.0, _lib.MIXED,
                                     _vp(t), None))
    g = _lib.Grid2D()
    g.n1, g.n2 = 2, 2
    with pytest.raises(ValueError, match="grid size"):
        _lib.check(_lib.lib.srs_flux(v, _lib.BeamConsts(-1.6e-19, 0.5), None, 3, C.byref(g), 100.0, _lib.MIXED,
                                     _vp(t), None))


def test_sim_sums_fresh_and_accumulated_outputs():
    """srs_sim_calculate_*: with comp the sums are Kahan-added into the caller's out/comp; without it
    they start from zero on the device and overwrite out.  Both give the same first result, bit for bit,
    and a second call with comp adds to the first."""
    from srsoriginal_b200 import _lib
    from srsoriginal_b200.sr import rectangle_points
    o = new_sr(2001)
    xyz, _, _, grid = rectangle_points([9, 7], "XY", [0.01, 0.01], translation=[0, 0, 30])
    pts = np.ascontiguousarray(xyz.reshape(-1))
    n = len(xyz)
    for prec in (_lib.FP64, _lib.MIXED):
        fresh = np.full(n, 123.0)  # not read without comp
        _lib.check(_lib.lib.srs_sim_calculate_flux(o._h, _lib.dptr(pts), n, C.byref(grid), 150.0, 0, prec,
                                                   _lib.dptr(fresh), None))
        acc, comp = np.zeros(n), np.zeros(n)
        for _ in range(2):
            _lib.check(_lib.lib.srs_sim_calculate_flux(o._h, _lib.dptr(pts), n, C.byref(grid), 150.0, 0, prec,
                                                       _lib.dptr(acc), _lib.dptr(comp)))
        assert np.all(fresh > 0)
        assert np.array_equal(acc, fresh + fresh)  # x + x is exact, and its compensation is 0
        assert np.all(comp == 0)
    e, obs = np.linspace(100.0, 300.0, 17), np.array([0.0, 0.0, 30.0])
    s1, s2, c2 = np.full(len(e), -1.0), np.zeros(len(e)), np.zeros(len(e))
    _lib.check(_lib.lib.srs_sim_calculate_spectrum(o._h, _lib.dptr(obs), _lib.dptr(e), len(e), 0, _lib.FP64,
                                                   _lib.dptr(s1), None))
    _lib.check(_lib.lib.srs_sim_calculate_spectrum(o._h, _lib.dptr(obs), _lib.dptr(e), len(e), 0, _lib.FP64,
                                                   _lib.dptr(s2), _lib.dptr(c2)))
    assert np.array_equal(s1, s2)


def test_flux_plane_one_call_matches_points_call():
    """srs_sim_calculate_flux_plane (rectangle built on the host while the GPU computes) gives the same
    surface and the same values, bit for bit, as building the rectangle first and calling
    srs_sim_calculate_flux with its points and grid."""
    from srsoriginal_b200 import _lib
    from srsoriginal_b200.sr import rectangle_points
    o = new_sr(2001)
    for plane, npts, rot, prec in (("XY", [9, 7], [0, 0, 0], _lib.MIXED), ("ZY", [6, 11], [0.1, -0.2, 0.3], _lib.MIXED),
                                   ("XY", [9, 7], [0, 0, 0], _lib.FP64), ("YX", [5, 4], [0, 0.2, 0], _lib.FP64)):
        xyz0, x120, nrm0, grid = rectangle_points(npts, plane, [0.01, 0.008], rotations=rot,
                                                  translation=[0.001, 0, 30])
        n = len(xyz0)
        pts = np.ascontiguousarray(xyz0.reshape(-1))
        ref = np.zeros(n)
        _lib.check(_lib.lib.srs_sim_calculate_flux(o._h, _lib.dptr(pts), n, C.byref(grid), 150.0, 0, prec,
                                                   _lib.dptr(ref), None))
        out, xyz, x12, nrm = np.zeros(n), np.empty(3 * n), np.empty(2 * n), np.empty(3)
        _lib.check(_lib.lib.srs_sim_calculate_flux_plane(o._h, plane.encode(), npts[0], npts[1], 0.01, 0.008,
                                                         _lib.v3(rot), _lib.v3([0.001, 0, 30]), 0, 150.0, 0, prec,
                                                         _lib.dptr(out), None, _lib.dptr(xyz), _lib.dptr(x12),
                                                         _lib.dptr(nrm)))
        assert np.array_equal(out, ref)
        assert np.array_equal(xyz, xyz0.reshape(-1)) and np.array_equal(x12, x120.reshape(-1))
        assert np.array_equal(nrm, nrm0)
        p2, v2 = o.flux_arrays(150.0, npts, plane, [0.01, 0.008], rotations=rot, translation=[0.001, 0, 30],
                               precision="mixed" if prec == _lib.MIXED else "fp64")
        assert np.array_equal(v2, ref) and np.array_equal(p2, xyz0)
    with pytest.raises(ValueError, match="surface string"):
        _lib.check(_lib.lib.srs_sim_calculate_flux_plane(o._h, b"QQ", 3, 3, 0.01, 0.01, None, None, 0, 150.0, 0,
                                                         _lib.MIXED, _lib.dptr(np.zeros(9)), None, None, None, None))


def test_edge_cases_small_sizes():
    o = new_sr(2)  # two trajectory points
    s = o.calculate_spectrum(obs=[0, 0, 30], npoints=1, energy_range_eV=[150, 150])
    assert len(s) == 1 and np.isfinite(s[0][1])
    o = new_sr(201)
    for prec in ("mixed", "fp64"):
        m = o.calculate_flux_rectangle(plane="XY", energy_eV=150.0, width=[0.01, 0.01], npoints=[2, 3],
                                       translation=[0, 0, 30], precision=prec)
        assert len(m) == 6 and all(np.isfinite(q[1]) for q in m)
        p = o.power_density_arrays([3, 2], "XY", [0.01, 0.01], translation=[0, 0, 30], precision=prec)[1]
        assert np.all(np.isfinite(p)) and np.all(p > 0)
    # a 1-point side has step width/0: the reference's coordinates are NaN (inf*0), and so are ours
    m = o.calculate_flux_rectangle(plane="XY", energy_eV=150.0, width=[0.01, 0.01], npoints=[1, 1],
                                   translation=[0, 0, 30])
    assert len(m) == 1 and np.isnan(m[0][0][0])


# ------------------------------------------------------------------ mixed precision vs the reference

def test_flux_cfg1_mixed_within_tolerance():
    g = golden("flux_cfg1.npz")
    o = new_sr(20001)
    for tag in ("e1", "e3"):
        pts, v = o.flux_arrays(float(g["energy_" + tag]), [101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30],
                               precision="mixed")
        assert_mixed(v, g["flux_" + tag])


def test_power_density_cfg2_mixed_within_tolerance():
    g = golden("pd_cfg2.npz")
    o = new_sr(40001, "epu")
    pts, v = o.power_density_arrays([201, 201], "XY", [0.04, 0.04], translation=[0, 0, 30], precision="mixed")
    assert_mixed(v, g["pd"])


def test_spectrum_mixed_within_tolerance():
    g = golden("spectrum_cfg0.npz")
    o = new_sr(20001)
    e, f = o.spectrum_arrays([0, 0, 30], 1000, [100, 1000], precision="mixed")
    assert_mixed(f, g["flux"])
    # non-uniform grid: one sincos per term
    gm = golden("misc_fields.npz")
    e, f = o.spectrum_arrays([0, 0, 30], points_eV=[151.0, 152.25225225225225, 455.0, 460.1], precision="mixed")
    e2, f2 = o.spectrum_arrays([0, 0, 30], points_eV=[151.0, 152.25225225225225, 455.0, 460.1])
    assert_mixed(f, f2)


@pytest.mark.parametrize("obs, lo, hi, ne", [([0, 0, 30], 100.0, 1000.0, 700),   # x, y near field left out
                                               ([0.002, -0.001, 3], 10.0, 60.0, 500),  # kept in the drifts
                                               ([0, 0, 1], 5.0, 20.0, 300)])           # kept nearly everywhere
def test_spectrum_mixed_near_field_paths(obs, lo, hi, ne):
    """The mixed spectrum tile leaves out a sub-tile's x, y near-field terms only when they can reach at
    most 1e-10 of its sum of |a|: observers at 30 m (left out everywhere), 3 m at 10-60 eV (kept in the
    drifts) and 1 m at 5-20 eV (kept nearly everywhere) all agree with the plain FP64 kernel; so does a
    non-uniform grid of the same size (one sincos per term, every near-field term kept)."""
    o = new_sr(20001)
    _, f = o.spectrum_arrays(obs, ne, [lo, hi], precision="mixed")
    _, f64 = o.spectrum_arrays(obs, ne, [lo, hi], precision="fp64")
    assert_mixed(f, f64)
    pts = np.sort(np.random.default_rng(7).uniform(lo, hi, ne)).tolist()
    _, f = o.spectrum_arrays(obs, points_eV=pts, precision="mixed")
    _, f64 = o.spectrum_arrays(obs, points_eV=pts, precision="fp64")
    assert_mixed(f, f64)


def test_spectrum_mixed_batched_near_observer_and_nonuniform():
    """Four energies per thread (the batched launch: 8 particles, 4096 energies) on the paths the
    30-m tests do not take: an observer 3 m away at 10-60 eV (sub-tiles that keep the x, y near-field
    terms) and a non-uniform grid (one sincos per term); against the plain FP64 kernel, per particle."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import energy_grid
    part, _ = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    und = [D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)]
    tb = D.trajectory(und, [part] * 8, 0.0, 2.0, 0.0, 20001)
    uniform = energy_grid(4096, 10.0, 60.0)
    ragged = np.sort(np.random.default_rng(11).uniform(10.0, 60.0, 4096))
    for ev in (uniform, ragged):
        e = torch.tensor(ev, dtype=torch.float64, device="cuda")
        fm = torch.empty(8 * 4096, dtype=torch.float64, device="cuda")
        f64 = torch.empty_like(fm)
        D.spectrum(tb, -D.QE, W.CURRENT, [0.002, -0.001, 3.0], e, fm, precision=_lib.MIXED)
        D.spectrum(tb, -D.QE, W.CURRENT, [0.002, -0.001, 3.0], e, f64, precision=_lib.FP64)
        a, b = fm.cpu().numpy().reshape(8, -1), f64.cpu().numpy().reshape(8, -1)
        for p in range(8):
            assert_mixed(a[p], b[p])


def test_beam_spectrum_cfg3a_subsample():
    """Config 3a at its shape (20001-point trajectories, 2000 energies over 100-1000 eV, weight
    1/nparticles) on the reference's own 32-particle subsample from set_seed(0): plain FP64 end to end,
    and the mixed-precision batched path against it."""
    from srsoriginal_b200.sr import reset_random
    g = golden("beam32_cfg3a.npz")
    o = new_sr(20001, **W.BEAM_3A)
    kw = dict(obs=[0, 0, W.SCREEN_Z], npoints=2000, energy_range_eV=[100, 1000], nparticles=32)
    reset_random(0)
    o.set_seed(0)
    e, f64 = o.spectrum_arrays(**kw, precision="fp64")
    assert np.array_equal(e, g["energies"])
    assert_e2e(f64, g["flux"])
    reset_random(0)
    o.set_seed(0)
    _, fm = o.spectrum_arrays(**kw, precision="mixed")
    assert_mixed(fm, f64)


def test_point_surfaces_fp64_and_mixed():
    """calculate_flux / calculate_power_density on a list of points with their own normals
    (OSCARSSR_Python.cc:2403-2577, 2829-3008): coordinates after rotation and translation, list
    lengths per dispatch path and values against the reference; the mixed-precision point-list
    kernels against the plain FP64 ones."""
    g = golden("points_surface.npz")
    pts = g["points"].tolist()
    o = new_sr(2001)
    kw = dict(rotations=[2e-5, -3e-5, 0.3], translation=[0.0005, -0.0002, 0.1])
    n = len(pts)
    f1 = o.calculate_flux(energy_eV=W.E1_EV, points=pts, nthreads=1, **kw)
    assert len(f1) == int(g["flux_len_t1"])
    assert np.array_equal(np.array([c for c, _ in f1]), g["flux_coords"])
    v1 = np.array([v for _, v in f1])
    assert_e2e(v1[:n], g["flux"][:n])
    assert np.all(v1[n:] == 0)
    assert len(o.calculate_flux(energy_eV=W.E1_EV, points=pts, nthreads=2, **kw)) == int(g["flux_len_t2"])
    assert len(o.calculate_flux(energy_eV=W.E1_EV, points=pts, gpu=1, **kw)) == 2 * n
    fm = o.calculate_flux(energy_eV=W.E1_EV, points=pts, nthreads=1, precision="mixed", **kw)
    assert_mixed([v for _, v in fm][:n], v1[:n])
    for nrm, key in ((0, "pd0"), (1, "pd1"), (-1, "pdm1")):
        p = o.calculate_power_density(points=pts, normal=nrm, nthreads=1, **kw)
        assert len(p) == int(g["pd_len_t1"])
        vals = np.array([v for _, v in p])
        assert_e2e(vals, g[key])
        if nrm == 0:
            assert np.array_equal(np.array([c for c, _ in p]), g["pd0_coords"])
        pm = o.calculate_power_density(points=pts, normal=nrm, nthreads=1, precision="mixed", **kw)
        assert_mixed([v for _, v in pm], vals)
    assert len(o.calculate_power_density(points=pts, normal=0, nthreads=2, **kw)) == int(g["pd_len_t2"])


def test_mixed_point_list_kernels_match_grid_kernels():
    """The point-list mixed kernels on the config-1 and config-2 grids given as plain point lists,
    against the grid (anchored) mixed kernels and the plain FP64 kernels."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    tr = reference_trajectory_on_device(20001)
    xyz, _, nrm, grid = rectangle_points([101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30])
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
    for e in (W.E1_EV, W.E3_EV):
        a, b, c = (torch.empty(101 * 101, dtype=torch.float64, device="cuda") for _ in range(3))
        D.flux(tr, -O.QE, 0.5, e, a, points=pts, precision=_lib.MIXED)
        D.flux(tr, -O.QE, 0.5, e, b, grid=grid, precision=_lib.MIXED)
        D.flux(tr, -O.QE, 0.5, e, c, points=pts, precision=_lib.FP64)
        torch.cuda.synchronize()
        assert_mixed(a.cpu().numpy(), c.cpu().numpy())
        assert_mixed(a.cpu().numpy(), b.cpu().numpy())
    t2 = reference_trajectory_on_device(40001, "epu")
    xyz, _, nrm, grid = rectangle_points([51, 51], "XY", [0.04, 0.04], translation=[0, 0, 30])
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
    nrms = torch.as_tensor(np.ascontiguousarray(np.tile(nrm, (51 * 51, 1)).reshape(-1)), device="cuda")
    a, c = (torch.empty(51 * 51, dtype=torch.float64, device="cuda") for _ in range(2))
    D.power_density(t2, -O.QE, 0.5, a, points=pts, normals=nrms, precision=_lib.MIXED)
    D.power_density(t2, -O.QE, 0.5, c, points=pts, normals=nrms, precision=_lib.FP64)
    torch.cuda.synchronize()
    assert_mixed(a.cpu().numpy(), c.cpu().numpy())


@pytest.mark.parametrize("n1,n2", [(2, 17), (17, 2), (3, 5), (5, 200), (200, 5), (13, 13), (129, 7), (37, 101)])
def test_mixed_grid_tiles_ragged_shapes(n1, n2):
    """The grid mixed kernels tile the map into strips of 8-16 points (narrower strips for n2 < 8) and
    take 128 consecutive points of a strip per CTA: every shape gives every point once, within the
    mixed tolerance of the plain FP64 kernels on the same points."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    tr = reference_trajectory_on_device(2001)
    xyz, _, nrm, grid = rectangle_points([n1, n2], "XY", [0.004, 0.006], translation=[0, 0, 30])
    n = n1 * n2
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
    nrms = torch.as_tensor(np.ascontiguousarray(np.tile(nrm, (n, 1)).reshape(-1)), device="cuda")
    a, c = (torch.full((n,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2))
    D.flux(tr, -O.QE, 0.5, W.E1_EV, a, grid=grid, precision=_lib.MIXED)
    D.flux(tr, -O.QE, 0.5, W.E1_EV, c, points=pts, precision=_lib.FP64)
    torch.cuda.synchronize()
    assert np.all(np.isfinite(a.cpu().numpy()))
    assert_mixed(a.cpu().numpy(), c.cpu().numpy())
    a.fill_(float("nan"))
    D.power_density(tr, -O.QE, 0.5, a, grid=grid, precision=_lib.MIXED)
    D.power_density(tr, -O.QE, 0.5, c, points=pts, normals=nrms, precision=_lib.FP64)
    torch.cuda.synchronize()
    assert np.all(np.isfinite(a.cpu().numpy()))
    assert_mixed(a.cpu().numpy(), c.cpu().numpy())


@pytest.mark.parametrize("n,width,z,energy", [(41, 0.05, 30.0, 1000.0), (41, 0.05, 10.0, 1000.0), (21, 0.05, 10.0, 1000.0),
                                              (51, 0.02, 5.0, 500.0), (31, 0.1, 30.0, 456.0), (21, 0.1, 3.0, 456.0)])
def test_mixed_grid_coarse_and_near_maps(n, width, z, energy):
    """Coarse grids and near screens, where the tiles' anchor expansion would leave phase errors of
    1e-3 rad and more: every anchor bounds what the expansion leaves out, and those sub-tiles are
    summed with exact FP64 geometry per term.  The flux is held to the point-list mixed kernel (FP64
    geometry for every term) and to normwise 1e-5 of FP64.  At 1 keV the retarded phase w (t + D/c) is
    ~1e11 rad, whose FP64 rounding (~1e-5 rad per term, in the FP64 kernel as in any other evaluation)
    moves the weakest points of such a map by up to ~1e-3 between two correct evaluations: there the
    max relative error at 1e-3 of the maximum may exceed 1e-4, but not 1.5 x the point-list kernel's
    nor 1e-3."""
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    tr = reference_trajectory_on_device(20001)
    xyz, _, nrm, grid = rectangle_points([n, n], "XY", [width, width], translation=[0, 0, z])
    m = n * n
    pts = torch.as_tensor(np.ascontiguousarray(xyz.reshape(-1)), device="cuda")
    nrms = torch.as_tensor(np.ascontiguousarray(np.tile(nrm, (m, 1)).reshape(-1)), device="cuda")
    a, c, q = (torch.empty(m, dtype=torch.float64, device="cuda") for _ in range(3))
    D.flux(tr, -O.QE, 0.5, energy, a, grid=grid, precision=_lib.MIXED)
    D.flux(tr, -O.QE, 0.5, energy, q, points=pts, precision=_lib.MIXED)
    D.flux(tr, -O.QE, 0.5, energy, c, points=pts, precision=_lib.FP64)
    torch.cuda.synchronize()
    mx, nrm = rel_err(a.cpu().numpy(), c.cpu().numpy(), 1e-3)
    mq, _ = rel_err(q.cpu().numpy(), c.cpu().numpy(), 1e-3)
    # relative to the point-list kernel, and never above 1e-3 whatever that kernel does
    assert nrm <= TOL_MIXED_NORM and mx <= min(1e-3, max(TOL_MIXED, 1.5 * mq)), (mx, mq, nrm)
    D.power_density(tr, -O.QE, 0.5, a, grid=grid, precision=_lib.MIXED)
    D.power_density(tr, -O.QE, 0.5, c, points=pts, normals=nrms, precision=_lib.FP64)
    torch.cuda.synchronize()
    assert_mixed(a.cpu().numpy(), c.cpu().numpy())

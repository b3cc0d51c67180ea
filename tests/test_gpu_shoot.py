"""Parallel-in-time trajectory (srs_trajectory_shoot) against the serial RK4 kernel.

The shooting trajectory is built from segments that step with the serial kernel's arithmetic from
start states found by Newton iterations; it equals the serial trajectory up to the ulps by which a
start state a few ulps away rounds differently.  Bars: positions within 2e-14 m, beta within 2e-14,
a/c within 1e-12 of its largest value; the mixed-precision sums on it within 1e-6 of the same sums on
the serial trajectory (their own bar against FP64 is 1e-4)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _fields_cfg2():
    from srsoriginal_b200 import device as D, workloads as W
    return [D.undulator([0, 1.0, 0], [0, 0, W.PERIOD], W.NPERIODS),
            D.undulator([0.6, 0, 0], [0, 0, W.PERIOD], W.NPERIODS, phase=np.pi / 2)]


def _mixed_fields():
    from srsoriginal_b200 import _lib, device as D, workloads as W
    und = D.undulator([0, 1.0, 0], [0, 0, W.PERIOD], W.NPERIODS)
    gau = _lib.Field()
    gau.kind = _lib.GAUSSIAN
    gau.field = _lib.v3([0.0, 0.05, 0.0])
    gau.center = _lib.v3([0.0, 0.0, 0.9])
    gau.sigma_or_width = _lib.v3([0.0, 0.0, 0.03])
    gau.rotations = _lib.v3([0.01, 0.02, 0.03])
    box = _lib.Field()
    box.kind = _lib.UNIFORM_BOX
    box.field = _lib.v3([0.002, 0.0, 0.0])
    box.center = _lib.v3([0.0, 0.0, -0.9])
    box.sigma_or_width = _lib.v3([0.0, 0.0, 0.05])
    return [und, gau, box]


def _grid_field(keep):
    from srsoriginal_b200 import device as D, workloads as W
    z = np.linspace(-1.0, 1.0, 2001)
    by = np.sin(2 * np.pi * z / W.PERIOD) * (np.abs(z) < 0.75) * 0.8
    data = np.zeros((2001, 3))
    data[:, 1] = by
    t = torch.tensor(data.reshape(-1), dtype=torch.float64, device="cuda")
    keep.append(t)
    return D.grid_z(-1.0, 0.001, by, t)


def _compare(fields, t0=0.0, npts=20001, steps=0, iters=0, ctstart=0.0, ctstop=2.0):
    from srsoriginal_b200 import device as D, workloads as W
    part, _ = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1 + t0], [0, 0, 1])
    ser = D.trajectory(fields, [part], ctstart, ctstop, t0, npts)
    stats = torch.zeros(4, dtype=torch.float64, device="cuda")
    sho = D.trajectory_shoot(fields, part, ctstart, ctstop, t0, npts, steps_per_segment=steps, max_iterations=iters,
                             stats=stats)
    torch.cuda.synchronize()
    dx = float((sho.x - ser.x).abs().max())
    db = float((sho.beta - ser.beta).abs().max())
    da = float((sho.aoc - ser.aoc).abs().max() / ser.aoc.abs().max().clamp_min(1e-300))
    return ser, sho, stats.cpu().numpy(), (dx, db, da)


@pytest.mark.parametrize("steps", [0, 16, 61])
def test_shoot_matches_serial_undulator(steps):
    from srsoriginal_b200 import device as D, workloads as W
    und = D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)
    _, _, st, (dx, db, da) = _compare([und], steps=steps)
    assert st[0] == 1 and 1 <= st[1] <= 8, st
    assert st[2] <= 2.0 ** -51, st  # the stored trajectory's largest segment mismatch
    assert dx <= 2e-14 and db <= 2e-14 and da <= 1e-12, (dx, db, da, st)


def test_shoot_two_chains_and_all_field_kinds():
    """t0 inside the trajectory (a backward chain too), two undulators with a phase, then an
    undulator + rotated Gaussian + uniform box, then a grid map staged in shared memory."""
    keep = []
    for fields, t0 in ((_fields_cfg2(), 0.0), (_mixed_fields(), 0.7), ([_grid_field(keep)], 1.3)):
        _, _, st, (dx, db, da) = _compare(fields, t0=t0, npts=12001)
        assert st[0] == 1, st
        assert dx <= 2e-14 and db <= 2e-14 and da <= 1e-12, (dx, db, da, st)


def test_shoot_falls_back_to_serial_when_not_converged():
    """One Newton iteration cannot converge from straight flight: the serial kernel writes the
    trajectory (bit for bit) and the statistics say so."""
    from srsoriginal_b200 import device as D, workloads as W
    und = D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)
    ser, sho, st, _ = _compare([und], iters=1)
    assert st[0] == 0 and st[1] == 1 and st[2] > 1e-10, st
    for a in ("x", "beta", "aoc"):
        assert torch.equal(getattr(sho, a), getattr(ser, a)), a


def test_shoot_short_and_degenerate_trajectories():
    from srsoriginal_b200 import device as D, workloads as W
    und = D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)
    for npts, t0 in ((2, 0.0), (3, 0.0), (101, 2.0), (257, 1.0)):
        ser, sho, st, (dx, db, da) = _compare([und], t0=t0, npts=npts)
        assert sho.n == ser.n
        assert dx <= 2e-14 and db <= 2e-14 and da <= 1e-12, (npts, t0, dx, db, da, st)


def test_mixed_flux_on_shooting_trajectory():
    from srsoriginal_b200 import _lib, device as D, workloads as W
    from srsoriginal_b200.sr import rectangle_points
    und = D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)
    ser, sho, st, _ = _compare([und])
    xyz, _, _, grid = rectangle_points([101, 101], "XY", [0.01, 0.01], translation=[0, 0, W.SCREEN_Z])
    pts = torch.tensor(np.asarray(xyz, float).reshape(-1), dtype=torch.float64, device="cuda")
    outs = []
    for t, prec in ((ser, _lib.FP64), (ser, _lib.MIXED), (sho, _lib.MIXED)):
        o = torch.empty(101 * 101, dtype=torch.float64, device="cuda")
        if prec == _lib.FP64:
            D.flux(t, -D.QE, W.CURRENT, W.E1_EV, o, points=pts, precision=prec)
        else:
            D.flux(t, -D.QE, W.CURRENT, W.E1_EV, o, grid=grid, precision=prec)
        outs.append(o)
    torch.cuda.synchronize()
    f64, mser, msho = (o.cpu().numpy() for o in outs)
    assert np.linalg.norm(msho - mser) <= 1e-6 * np.linalg.norm(mser)
    assert np.abs(msho - f64).max() <= 1e-4 * np.abs(f64).max()


def test_shoot_rejects_bad_arguments():
    from srsoriginal_b200 import _lib, device as D, workloads as W
    und = D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)
    part, _ = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    buf = torch.zeros(3 * 101, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    fa = (_lib.Field * 1)(und)
    lib = _lib.lib
    assert lib.srs_trajectory_shoot(fa, 1, C.byref(part), 0.0, 2.0, 0.0, 101, 0, 33, p, p, p, None,
                                    None) == _lib.SRS_ERR_INVALID
    assert lib.srs_trajectory_shoot(fa, 1, C.byref(part), 0.0, 2.0, 0.0, 101, -1, 0, p, p, p, None,
                                    None) == _lib.SRS_ERR_INVALID
    assert lib.srs_trajectory_shoot(fa, 1, None, 0.0, 2.0, 0.0, 101, 0, 0, p, p, p, None, None) == _lib.SRS_ERR_INVALID
    assert lib.srs_trajectory_shoot(fa, 1, C.byref(part), 0.0, 2.0, 0.0, 101, 0, 0, None, p, p, None,
                                    None) == _lib.SRS_ERR_INVALID
    assert lib.srs_trajectory_shoot(fa, 1, C.byref(part), 2.0, 0.0, 0.0, 101, 0, 0, p, p, p, None,
                                    None) == _lib.SRS_ERR_RANGE


def test_sr_trajectory_modes():
    """The sr object integrates parallel in time for mixed-precision maps ('auto'), serially for FP64;
    both modes give the same mixed map to 1e-6; calculate_trajectory is serial unless 'parallel'."""
    from srsoriginal_b200 import workloads as W
    from srsoriginal_b200.sr import sr
    o = sr()
    W.setup_beam(o, 20001)
    W.setup_undulator(o)
    kw = dict(translation=[0, 0, W.SCREEN_Z], precision="mixed")
    maps = {}
    for mode in ("serial", "auto", "parallel"):
        o.set_trajectory_mode(mode)
        maps[mode] = np.asarray(o.flux_arrays(W.E1_EV, [41, 41], "XY", [0.01, 0.01], **kw)[-1])
    ref = maps["serial"]
    for mode in ("auto", "parallel"):
        assert np.linalg.norm(maps[mode] - ref) <= 1e-6 * np.linalg.norm(ref), mode
    o.set_trajectory_mode("parallel")
    tp = np.asarray(o.calculate_trajectory(), dtype=object)
    o.set_trajectory_mode("serial")
    ts = np.asarray(o.calculate_trajectory(), dtype=object)
    xp = np.array([p[0] for p in tp], float)
    xs = np.array([p[0] for p in ts], float)
    assert np.abs(xp - xs).max() <= 2e-14
    with pytest.raises(ValueError):
        o.set_trajectory_mode("fast")

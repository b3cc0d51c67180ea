"""Electric fields against the reference (tests/golden/efield.npz, made by running it): trajectories
with E only and with E and B (DerivativesE / DerivativesEB, OSCARSSR.cc:690-793), the fields at
points, the time-domain field (OSCARSSR.cc:2646-2690), the FP64 spectrum through an E+B trajectory,
and the reference's disabled magnetic add_field_gaussian."""
import json
import os

import numpy as np
import pytest

from conftest import golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _traj(o):
    t = np.asarray(o.calculate_trajectory(), dtype=np.float64)
    return t[:, 0, :].T, t[:, 1, :].T


def _rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def _e_only():
    from srsoriginal_b200 import workloads as W
    from srsoriginal_b200.sr import sr
    o = sr()
    W.setup_beam(o, 4001)
    o.add_efield_uniform(efield=[3e6, 0, 0], width=[0, 0, 0.5])
    o.add_efield_gaussian(efield=[0, 5e6, 1e5], sigma=[0.02, 0.0, 0.1], translation=[0, 0, 0.5],
                          rotations=[0.0, 0.01, 0.0])
    return o


def test_electric_only_trajectory_fields_and_time_domain():
    g = golden("efield.npz")
    o = _e_only()
    X, B = _traj(o)
    assert _rel(X, g["e_only_x"]) <= 1e-12 and _rel(B, g["e_only_beta"]) <= 1e-12
    pts = g["points"]
    ef = np.array([o.get_efield(list(map(float, p))) for p in pts])
    bf = np.array([o.get_bfield(list(map(float, p))) for p in pts])
    np.testing.assert_allclose(ef, g["e_only_efield"], rtol=1e-14, atol=0)
    assert np.array_equal(bf, g["e_only_bfield"])  # no magnetic field: zeros
    r = o.calculate_efield_vs_time(obs=[0, 0, 30])
    t = np.array([q[0] for q in r])
    e = np.array([q[1] for q in r])
    np.testing.assert_allclose(t, g["e_only_t"], rtol=1e-14, atol=0)
    assert np.linalg.norm(e - g["e_only_e"]) <= 1e-10 * np.linalg.norm(g["e_only_e"])


def test_electric_and_magnetic_trajectory_and_spectrum():
    from srsoriginal_b200 import workloads as W
    from srsoriginal_b200.sr import sr
    g = golden("efield.npz")
    o = sr()
    W.setup_beam(o, 8001)
    W.setup_undulator(o)
    o.add_efield_undulator(efield=[0, 2e7, 0], period=[0, 0, W.PERIOD], nperiods=W.NPERIODS, phase=0.3)
    X, B = _traj(o)
    assert _rel(X, g["eb_x"]) <= 1e-12 and _rel(B, g["eb_beta"]) <= 1e-12
    pts = g["points"]
    ef = np.array([o.get_efield(list(map(float, p))) for p in pts])
    np.testing.assert_allclose(ef, g["eb_efield"], rtol=1e-14, atol=1e-300)
    sp = np.array(o.calculate_spectrum(obs=[0, 0, 30], npoints=20, energy_range_eV=[140, 160], gpu=1))
    ref = g["eb_spectrum"]
    assert np.array_equal(sp[:, 0], ref[:, 0])
    assert np.linalg.norm(sp[:, 1] - ref[:, 1]) <= 1e-10 * np.linalg.norm(ref[:, 1])
    r = o.calculate_efield_vs_time(obs=[0.001, 0, 30])
    e = np.array([q[1] for q in r])
    assert np.linalg.norm(e - g["eb_e"]) <= 1e-10 * np.linalg.norm(g["eb_e"])
    o.clear_bfields()  # the electric container stays
    ef = np.array([o.get_efield(list(map(float, p))) for p in pts[:5]])
    np.testing.assert_allclose(ef, g["eb_cleared_b_efield"], rtol=1e-14, atol=1e-300)
    o.clear_efields()
    assert o.get_efield(list(map(float, pts[0]))) == [0.0, 0.0, 0.0]


def test_add_field_gaussian_and_errors(tmp_path):
    from srsoriginal_b200 import workloads as W
    from srsoriginal_b200.sr import sr
    g = golden("efield.npz")
    errs = json.load(open(os.path.join(HERE, "golden", "efield_errors.json")))
    o = sr()
    W.setup_beam(o, 2001)
    o.add_field_gaussian(sigma=[0, 0, 0.1], bfield=[0, 1.0, 0])  # disabled in the reference: no field
    X, _ = _traj(o)
    assert np.array_equal(X, g["fg_b_x"])
    o.add_field_gaussian(sigma=[0, 0, 0.1], efield=[1e6, 0, 0])
    ef = np.array([o.get_efield(list(map(float, p))) for p in g["points"][:5]])
    np.testing.assert_allclose(ef, g["fg_e_efield"], rtol=1e-14, atol=1e-300)
    for key, call in (("fg_both", lambda: o.add_field_gaussian(sigma=[0, 0, 1], bfield=[0, 1, 0], efield=[1, 0, 0])),
                      ("fg_none", lambda: o.add_field_gaussian(sigma=[0, 0, 1])),
                      ("efield_format", lambda: o.add_efield_uniform(efield=[1, 0]))):
        with pytest.raises(ValueError) as e:
            call()
        assert str(e.value) == errs[key]
    with pytest.raises(ValueError, match="Could not import electric field"):
        o.add_efield_file(ifile=str(tmp_path / "missing.txt"), iformat="OSCARS")


def test_electric_trajectory_c_abi_paths_agree():
    """srs_trajectory for one particle (the warp kernel with a whole block), for 200 copies (narrow lane
    groups) and srs_trajectory_shoot (which integrates fields with E serially) agree bit for bit."""
    import ctypes as C
    from srsoriginal_b200 import _lib, device as D, workloads as W
    f = _lib.Field()
    f.kind = _lib.UNIFORM_BOX | _lib.ELECTRIC
    f.field = _lib.v3([3e6, 0, 0])
    f.sigma_or_width = _lib.v3([0, 0, 0.5])
    und = D.undulator([0, W.BPEAK, 0], [0, 0, W.PERIOD], W.NPERIODS)
    part, _ = D.ideal_particle(W.ENERGY_GEV, [0, 0, -1], [0, 0, 1])
    one = D.trajectory([und, f], [part], 0.0, 2.0, 0.0, 4001)
    many = D.trajectory([und, f], [part] * 200, 0.0, 2.0, 0.0, 4001)
    st = torch.zeros(4, dtype=torch.float64, device="cuda")
    sh = D.trajectory_shoot([und, f], part, 0.0, 2.0, 0.0, 4001, stats=st)
    torch.cuda.synchronize()
    assert torch.equal(many.x[17], one.x[0]) and torch.equal(sh.x[0], one.x[0])
    assert float(st[0]) == 0.0  # integrated serially
    assert float((one.x[0, 0] - D.trajectory([und], [part], 0.0, 2.0, 0.0, 4001).x[0, 0]).abs().max()) > 1e-9

"""CPU-only checks: the C-ABI library loads and exports every declared entry point, and the host-side
logic (surfaces, energy grid, argument validation) matches the reference/oracle.  No GPU needed."""
import math
import os
import re

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden

HEADER = os.path.join(ROOT, "include", "srs_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(srs_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import ctypes
    from srsoriginal_b200 import _lib
    names = declared_functions()
    assert len(names) >= 40
    so = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in names if not hasattr(so, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.EXPORTED) | set(names)


def test_library_loads_without_a_gpu():
    from srsoriginal_b200 import _lib
    assert _lib.lib.srs_version().startswith(b"srs_b200")
    assert _lib.lib.srs_device_count() >= 0


@pytest.mark.parametrize("plane,rot,normal", [
    ("XY", (0, 0, 0), 0), ("yx", (0, 0, 0), 1), ("XZ", (0.1, 0.2, 0.3), -1), ("ZX", (0, 0, 0), 0),
    ("YZ", (0, -math.pi / 2, 0), 1), ("ZY", (0.01, 0, -0.2), 0)])
def test_rectangle_plane_matches_oracle(plane, rot, normal):
    from srsoriginal_b200.sr import rectangle_points
    xyz, x12, nrm, grid = rectangle_points([7, 5], plane, [0.02, 0.03], rotations=rot, translation=[0.001, 0, 20],
                                           normal=normal)
    a, b, c = O.rectangle([7, 5], plane, [0.02, 0.03], rotations=rot, translation=[0.001, 0, 20], normal=normal)
    assert np.array_equal(xyz, a) and np.array_equal(x12, b) and np.array_equal(nrm, c)
    # the grid description reproduces the points to rounding
    o, u1, u2 = np.array(grid.origin), np.array(grid.u1), np.array(grid.u2)
    i = np.arange(35)
    pts = o + np.outer(i // 5, u1) + np.outer(i % 5, u2)
    assert np.allclose(pts, xyz, rtol=0, atol=1e-12)


def test_rectangle_x0x1x2_matches_reference_fixture():
    from srsoriginal_b200.sr import rectangle_points
    g = golden("misc_fields.npz")
    xyz, x12, nrm, grid = rectangle_points([6, 5], x0x1x2=[[-0.004, -0.003, 25], [0.004, -0.003, 25],
                                                           [-0.004, 0.003, 25.1]])
    assert np.array_equal(xyz, g["flux_x0x1x2_xyz"])


def test_rectangle_coordinates_match_reference_fixture():
    from srsoriginal_b200.sr import rectangle_points
    g = golden("flux_cfg1.npz")
    xyz, x12, nrm, grid = rectangle_points([101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30])
    assert np.array_equal(x12, g["x12"])


def test_energy_grid_matches_reference():
    from srsoriginal_b200.sr import energy_grid
    g = golden("spectrum_cfg0.npz")
    assert np.array_equal(energy_grid(1000, 100, 1000), g["energies"])
    assert np.array_equal(energy_grid(1, 123.0, 1000), [123.0])


def test_bad_arguments_raise_valueerror():
    from srsoriginal_b200.sr import rectangle_points
    with pytest.raises(ValueError, match="not a valid surface string"):
        rectangle_points([3, 3], "XQ", [0.01, 0.01])
    with pytest.raises(ValueError, match="npoints"):
        rectangle_points([0, 3], "XY", [0.01, 0.01])
    with pytest.raises(ValueError, match="normal must be"):
        rectangle_points([3, 3], "XY", [0.01, 0.01], normal=2)


def test_trajectory_counts_match_oracle():
    import ctypes as C
    from srsoriginal_b200 import _lib
    for (a, b, t0, n) in [(0, 2, 0, 20001), (0, 2, 0, 40001), (-1, 1, 0, 20001), (0, 2, 0.7, 3001), (0, 1, 0, 2)]:
        dt, nf, nb = C.c_double(), C.c_int64(), C.c_int64()
        _lib.check(_lib.lib.srs_trajectory_counts(a, b, t0, n, C.byref(dt), C.byref(nf), C.byref(nb)))
        assert (dt.value, nf.value, nb.value) == O.trajectory_counts(a, b, t0, n)
    with pytest.raises(ValueError, match="start time is greater than T0"):
        _lib.check(_lib.lib.srs_trajectory_counts(1, 2, 0, 100, None, None, None))


def test_sim_without_device_reports_the_reference_message():
    from srsoriginal_b200 import _lib
    if _lib.lib.srs_device_count() > 0:
        pytest.skip("a GPU is present")
    from srsoriginal_b200.sr import sr
    with pytest.raises(ValueError, match="You are requesting the GPU, but none were found"):
        sr()


def test_quirk_fixture_shapes_documented():
    """The reference's list lengths that the drop-in reproduces (checked on the GPU in test_gpu_*)."""
    import json
    q = json.load(open(os.path.join(ROOT, "tests", "golden", "quirks.json")))
    assert q["flux_len_nthreads1"] == 24 and q["flux_len_nthreads2"] == 12
    assert q["pd_len_nthreads1"] == 12 and q["pd_len_nthreads2"] == 24


def test_particle_from_ic_jacobian():
    """The chain-rule Jacobian d(x0, beta0, q/(m gamma))/d(x, y, x', y', z, E) of the adjoint's
    initial conditions against central differences (no GPU)."""
    from srsoriginal_b200.adjoint import particle_from_ic

    def vec(ic):
        p, _ = particle_from_ic(ic)
        return np.array(list(p.x0) + list(p.beta0) + [p.qomg])

    ic = np.array([1e-4, -2e-4, 3e-4, -1e-4, -1.0, 3.0])
    _, J = particle_from_ic(ic)
    for j in range(6):
        h = 1e-7 * max(abs(ic[j]), 1e-3)
        a, b = ic.copy(), ic.copy()
        a[j] += h
        b[j] -= h
        fd = (vec(a) - vec(b)) / (2 * h)
        scale = np.abs(J).max(axis=1) + 1e-300
        tol = 1e-6 * scale + 4e-16 * np.abs(vec(ic)) / h  # relative accuracy, plus rounding over 2h
        # q/(m gamma) takes gamma from |beta0|^2 (as the reference does), 1 - |beta0|^2 ~ 3e-8, so its
        # rounding is ~1e-16 / 3e-8 relative: the differences carry that noise over 2h
        tol[6] += 1e-8 * abs(vec(ic)[6]) / h
        assert np.all(np.abs(fd - J[:, j]) <= tol), (j, fd, J[:, j])


def test_point_surface_coordinates_match_reference():
    """The point-list surface (rotation about X, Y, Z, normal inversion, translation) gives the
    reference's coordinates bit for bit (no GPU)."""
    from conftest import golden
    from srsoriginal_b200.sr import sr
    g = golden("points_surface.npz")
    xyz, nrm = sr._surface_3d(g["points"].tolist(), [2e-5, -3e-5, 0.3], [0.0005, -0.0002, 0.1], False)
    assert np.array_equal(xyz, g["pd0_coords"])
    with pytest.raises(ValueError, match="Incorrect format in 'points'"):
        sr._surface_3d([[[0, 0, 1]]], None, None, False)
    with pytest.raises(ValueError, match="Point or Normal does not have 3 elements"):
        sr._surface_3d([[[0, 0], [0, 0, 1]]], None, None, False)

"""srs_flux_mixed_noalloc: the mixed-precision flux on a grid for callers that cannot allocate device
memory while they run (device memory reserved up front by their own allocator, or loops that may not
call cudaMalloc).  Its scratch is a fixed array inside the library instead of a stream-ordered
allocation.  Checked through the C ABI against srs_flux on two calls in a row, and for its size limit.

This file is collected last on purpose (pytest runs files in name order), so a failure here comes
after every other test has run.  It also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

E1 = 152.25225225225225


def _setup():
    import torch
    from srsoriginal_b200 import _lib, device as D
    from srsoriginal_b200.sr import rectangle_points
    fields = [D.undulator([0, 1.0, 0], [0, 0, 0.049], 31)]
    part, gamma = D.ideal_particle(3.0, [0, 0, -1], [0, 0, 1])
    traj = D.trajectory(fields, [part], 0.0, 2.0, 0.0, 20001)
    xyz, x12, nrm, grid = rectangle_points([101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30])
    torch.cuda.synchronize()
    return torch, _lib, D, traj, grid


def test_noalloc_flux_matches_srs_flux_on_two_calls_in_a_row():
    torch, _lib, D, traj, grid = _setup()
    L = _lib.lib
    beam = _lib.BeamConsts(-1.602176462e-19, 0.5)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    n = grid.n1 * grid.n2
    for energy in (E1, 3 * E1, E1):  # consecutive calls share (and overwrite) the library's scratch
        ref = torch.empty(n, dtype=torch.float64, device="cuda")
        got = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        _lib.check(L.srs_flux(traj.view(), beam, None, n, C.byref(grid), energy, _lib.MIXED,
                              C.c_void_p(ref.data_ptr()), stream))
        _lib.check(L.srs_flux_mixed_noalloc(traj.view(), beam, C.byref(grid), energy, C.c_void_p(got.data_ptr()),
                                            stream))
        torch.cuda.synchronize()
        r, g = ref.cpu().numpy(), got.cpu().numpy()
        assert np.all(np.isfinite(g))
        # same kernels and, at this size, the same trajectory chunking: equal to rounding of the chunk sums
        assert np.max(np.abs(g - r)) <= 1e-12 * np.abs(r).max()


def test_noalloc_flux_rejects_sizes_beyond_its_scratch():
    torch, _lib, D, traj, grid = _setup()
    big = _lib.Grid2D()
    big.origin, big.u1, big.u2, big.normal = grid.origin, grid.u1, grid.u2, grid.normal
    big.n1, big.n2 = 500, 500  # 250000 points > 174762
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    st = _lib.lib.srs_flux_mixed_noalloc(traj.view(), _lib.BeamConsts(-1.602176462e-19, 0.5), C.byref(big), E1,
                                         C.c_void_p(out.data_ptr()), None)
    assert st == _lib.SRS_ERR_RANGE
    assert b"exceeds its fixed scratch" in _lib.lib.srs_last_error()

"""Adjoint of the spectrum through the RK4 trajectory (config 4).

The exact derivative of the reference's FP64 loss is taken by the complex-step method on the
oracle's analytic restatement of the same forward path (oracle/complex_step.py, whose real part
reproduces the reference's loss bit for bit; fixture tests/golden/adjoint_cfg4.npz).  Central
differences of the FP64 loss at h = 1e-6 relative are also stored (the reference run through
perturbed grid files and beam arguments), but they are not a usable truth at 1e-5: the phases
w (t + D/c) are ~7e10 rad, one ulp of a retarded time moves a term's phase by ~1e-5 rad, and the loss
jumps by ~3e-7 of itself when the rounding pattern of the trajectory changes -- a noise of the order
of the gradient itself over 2h.  The library's FP64 forward reproduces the reference's losses at
the perturbed inputs, noise included."""
import numpy as np
import pytest

from conftest import golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _problem(precision):
    from srsoriginal_b200 import workloads as W
    return W.config4_problem(precision=precision)


def _loss_and_grad(problem, grid, ic, de):
    from srsoriginal_b200.adjoint import SpectrumFlux, integrated_flux_loss
    g = grid.clone().requires_grad_(True)
    c = ic.clone().requires_grad_(True)
    loss = integrated_flux_loss(SpectrumFlux.apply(g, None, c, problem), de)
    loss.backward()
    return float(loss), g.grad[:, 1].cpu().numpy(), c.grad.numpy()


def _loss_only(problem, grid, ic, de):
    from srsoriginal_b200.adjoint import forward_flux
    f = forward_flux(problem, grid, None, ic)
    return float(-(f * de).sum())


def _close(g, ref, h, L, rtol):
    """|g - ref| h <= rtol |ref| h + 1e-12 |L|: the loss change each gradient predicts over a step h
    agrees to rtol, down to the loss's own rounding level (for coordinates whose derivative is 0)."""
    return np.abs(g - ref) * h <= rtol * np.abs(ref) * h + 1e-12 * abs(L)


@pytest.fixture(scope="module")
def fp64_grad():
    from srsoriginal_b200 import _lib
    problem, grid, ic, de = _problem(_lib.FP64)
    L, gby, gic = _loss_and_grad(problem, grid, ic, de)
    return problem, grid, ic, de, L, np.concatenate([gby, gic])


def test_adjoint_matches_complex_step(fp64_grad):
    problem, grid, ic, de, L, g = fp64_grad
    ref = golden("adjoint_cfg4.npz")
    assert abs(L - float(ref["loss"])) <= 1e-9 * abs(float(ref["loss"]))
    coords = ref["coords"]
    h = 0.5 * (ref["theta_plus"] - ref["theta_minus"])
    ok = _close(g[coords], ref["grad_cs"], h, L, 1e-5)
    assert ok.all(), list(zip(coords[~ok], g[coords][~ok], ref["grad_cs"][~ok]))


def test_adjoint_within_reference_difference_noise(fp64_grad):
    """Against the reference's central differences the adjoint is off by no more than the exact
    derivative is (the differences' own noise)."""
    _, _, _, _, L, g = fp64_grad
    ref = golden("adjoint_cfg4.npz")
    coords = ref["coords"]
    fd, cs = ref["grad_fd"], ref["grad_cs"]
    h = 0.5 * (ref["theta_plus"] - ref["theta_minus"])
    assert np.all(np.abs(g[coords] - fd) <= np.abs(cs - fd) + 1e-5 * np.abs(cs) + 1e-12 * abs(L) / h)


def test_fp64_forward_reproduces_reference_losses_at_perturbed_inputs(fp64_grad):
    """The library's FP64 loss at each perturbed input of the reference's central differences equals
    the reference's loss there, so the library's own differences carry the same values."""
    problem, grid, ic, de, L, _ = fp64_grad
    ref = golden("adjoint_cfg4.npz")
    nz = grid.shape[0]
    worst = 0.0
    for k, tp, tm, lp, lm in zip(ref["coords"], ref["theta_plus"], ref["theta_minus"], ref["loss_plus"],
                                 ref["loss_minus"]):
        vals = []
        for t in (tp, tm):
            g2, c2 = grid.clone(), ic.clone()
            if k < nz:
                g2[k, 1] = float(t)
            else:
                c2[k - nz] = float(t)
            vals.append(_loss_only(problem, g2, c2, de))
        worst = max(worst, abs(vals[0] - lp) / abs(lp), abs(vals[1] - lm) / abs(lm))
    assert worst <= 1e-10, worst


def test_adjoint_mixed_forward_close_to_fp64(fp64_grad):
    from srsoriginal_b200 import _lib
    _, _, _, _, L64, g64 = fp64_grad
    problem, grid, ic, de = _problem(_lib.MIXED)
    L, gby, gic = _loss_and_grad(problem, grid, ic, de)
    g = np.concatenate([gby, gic])
    assert abs(L - L64) <= 1e-5 * abs(L64)
    nz = len(gby)
    assert np.linalg.norm(g[:nz] - g64[:nz]) <= 1e-4 * np.linalg.norm(g64[:nz])
    big = np.abs(g64[nz:]) > 1e-6 * np.abs(g64[nz:]).max()
    assert np.all(np.abs(g[nz:] - g64[nz:])[big] <= 1e-4 * np.abs(g64[nz:])[big])


def test_adjoint_backward_chain_and_amplitude_fields():
    """t0 inside the trajectory (points before t0 come from the backward RK4 chain), undulator,
    Gaussian and uniform-field amplitudes: the adjoint kernels against complex-step derivatives of
    the oracle's restatement.

    The gradient of this loss moves by ~2e-5 of itself when the trajectory moves by one ulp (the
    phases are ~1e10 rad), and the library's RK4 evaluates sin with CUDA's libm, not glibc's, so its
    trajectory differs from the restatement's by ulps.  The adjoint is therefore run on the
    restatement's own trajectory (uploaded), which isolates the derivative arithmetic."""
    import ctypes as C
    import complex_step as CS
    from srsoriginal_b200 import _lib, device as D, workloads as W
    from srsoriginal_b200.adjoint import SpectrumProblem, backward_flux, particle_from_ic
    from srsoriginal_b200.sr import energy_grid
    und = D.undulator([0, 1.0, 0], [0, 0, W.PERIOD], W.NPERIODS)
    gau = _lib.Field()
    gau.kind = _lib.GAUSSIAN
    gau.field = _lib.v3([0.0, 0.05, 0.0])
    gau.center = _lib.v3([0.0, 0.0, 0.9])
    gau.sigma_or_width = _lib.v3([0.0, 0.0, 0.03])
    box = _lib.Field()
    box.kind = _lib.UNIFORM_BOX
    box.field = _lib.v3([0.002, 0.0, 0.0])
    box.center = _lib.v3([0.0, 0.0, -0.9])
    box.sigma_or_width = _lib.v3([0.0, 0.0, 0.05])
    e_np = energy_grid(40, 0.98 * W.E1_EV, 1.02 * W.E1_EV)
    e = torch.tensor(e_np, dtype=torch.float64, device="cuda")
    npts, t0 = 4001, 0.6
    problem = SpectrumProblem(fields=[und, gau, box], obs=(0.0, 0.0, 30.0), energies=e, ctstart=0.0, ctstop=2.0,
                              t0=t0, npoints=npts, precision=_lib.FP64)
    amps0 = np.array([[0.0, 1.0, 0.0], [0.0, 0.05, 0.0], [0.002, 0.0, 0.0]])
    ic0 = np.array([1e-5, -2e-5, 3e-5, 1e-5, -0.4, 3.0])
    weights_np = np.linspace(0.5, 1.5, len(e_np))

    # complex-step: one row per checked coordinate (row 0 also gives the trajectory)
    checks = [("amp", 0, 1), ("amp", 1, 1), ("amp", 2, 0), ("amp", 0, 0)] + [("ic", j, None) for j in range(6)]
    m = len(checks)
    eps = 1e-30
    A = np.tile(amps0.astype(complex), (m, 1, 1))
    IC = np.tile(ic0.astype(complex), (m, 1))
    for r, (kind, i, j) in enumerate(checks):
        if kind == "amp":
            A[r, i, j] += 1j * eps
        else:
            IC[r, i] += 1j * eps
    fields = [CS.undulator_field(A[:, 0], [0, 0, W.PERIOD], W.NPERIODS),
              CS.gaussian_field(A[:, 1], [0, 0, 0.9], [0, 0, 0.03]),
              CS.box_field(A[:, 2], [0, 0, -0.9], [0, 0, 0.05])]
    X, V, dt = CS.trajectory_fields(fields, IC, 0.0, 2.0, t0, npts)
    val = (CS.flux(X, V, dt, [0, 0, 30.0], e_np) * weights_np[None, :]).sum(1)
    cs = val.imag / eps

    # the adjoint kernels on the restatement's (real) trajectory
    x = torch.tensor(X[0].real.T.copy(), dtype=torch.float64, device="cuda").reshape(1, 3, -1).contiguous()
    beta = torch.tensor((V[0].real / CS.C_LIGHT).T.copy(), dtype=torch.float64, device="cuda").reshape(1, 3, -1)
    traj = D.Trajectory(x, beta.contiguous(), torch.zeros_like(x), dt)
    ne = e.numel()
    flux = torch.empty(ne, dtype=torch.float64, device="cuda")
    e6 = torch.empty(6 * ne, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib.srs_spectrum_efield(traj.view(), _lib.BeamConsts(problem.charge, problem.current),
                                            _lib.v3(problem.obs), C.c_void_p(e.data_ptr()), ne, _lib.FP64,
                                            C.c_void_p(flux.data_ptr()), C.c_void_p(e6.data_ptr()), None))
    L = float((flux.cpu().numpy() * weights_np).sum())
    assert abs(L - val.real[0]) <= 1e-12 * abs(L)
    arr = (_lib.Field * 3)(und, gau, box)
    part, J = particle_from_ic(ic0)
    _, gamps, gic = backward_flux(problem, (traj, e6, arr, None, part, J),
                                  torch.tensor(weights_np, dtype=torch.float64, device="cuda"))
    got = np.array([gamps[i, j] if kind == "amp" else gic[i] for kind, i, j in checks])
    scale = np.abs(cs).max()
    rel = np.abs(got - cs) / (np.abs(cs) + 1e-10 * scale)
    assert np.all(rel <= 1e-6), "\n".join(f"{checks[r]} adjoint {got[r]!r} complex-step {cs[r]!r} rel {rel[r]:.2e}"
                                          for r in range(m))


def test_adjoint_rejects_bad_arguments():
    import ctypes as C
    from srsoriginal_b200 import _lib
    part = _lib.Particle()
    st = _lib.lib.srs_trajectory_adjoint(None, 0, C.byref(part), 0.0, 2.0, 0.0, 101, None, None, None, None, None,
                                         None, None, None)
    assert st == _lib.SRS_ERR_INVALID
    too_many = (_lib.Field * 17)()
    icg = (C.c_double * 7)()
    dummy = torch.zeros(3 * 101, dtype=torch.float64, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    st = _lib.lib.srs_trajectory_adjoint(too_many, 17, C.byref(part), 0.0, 2.0, 0.0, 101, p, p, p, p, None, None,
                                         icg, None)
    assert st == _lib.SRS_ERR_INVALID

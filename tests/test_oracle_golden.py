"""Pins the oracle (plain-C restatement of the reference's CPU algorithm) to the reference's own
outputs, stored as fixtures by tests/golden/make_golden.py.  Bit-exact: the restatement runs the same
IEEE-double operations in the same order as the reference."""
import json
import math
import os
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN, golden
from srsoriginal_b200 import workloads as W


def cfg_sr(npoints, fields="undulator", **beam):
    o = O.OracleSR()
    W.setup_beam(o, npoints, **beam)
    if fields == "undulator":
        W.setup_undulator(o)
    elif fields == "epu":
        W.setup_epu(o)
    return o


def test_energy_grid_is_shifted_one_step():
    g = golden("spectrum_cfg0.npz")
    e = O.energy_grid(1000, 100.0, 1000.0)
    assert np.array_equal(e, g["energies"])
    assert e[0] > 100.0 and e[-1] > 1000.0  # the reference's grid starts one step above EFirst


def test_cfg0_small_trajectory_spectrum_power_bitexact():
    g = golden("spectrum_cfg0.npz")
    o = cfg_sr(2001)
    X, B, A, dt = o.trajectory()
    assert np.array_equal(X, g["small_x"]) and np.array_equal(B, g["small_beta"])
    e, f = o.calculate_spectrum(obs=[0, 0, 30], npoints=64, energy_range_eV=[100, 1000])
    assert np.array_equal(e, g["small_energies"]) and np.array_equal(f, g["small_flux"])
    assert o.calculate_total_power() == float(g["small_total_power"])


def test_cfg0_full_trajectory_and_spectrum_subset_bitexact():
    g = golden("spectrum_cfg0.npz")
    o = cfg_sr(20001)
    X, B, A, dt = o.trajectory()
    assert X.shape[1] == int(g["n"])
    assert np.array_equal(X[:, ::50], g["x_sub"]) and np.array_equal(B[:, ::50], g["beta_sub"])
    assert np.array_equal(X[:, -1], g["x_last"]) and np.array_equal(B[:, -1], g["beta_last"])
    idx = np.arange(0, 1000, 37)
    f = O.spectrum(X, B, dt, [0, 0, 30], g["energies"][idx], -O.QE, 0.5)
    assert np.array_equal(f, g["flux"][idx])
    assert o.calculate_total_power() == float(g["total_power"])


def test_cfg1_flux_subset_bitexact():
    g = golden("flux_cfg1.npz")
    o = cfg_sr(20001)
    X, B, A, dt = o.trajectory()
    xyz, x12, nrm = O.rectangle([101, 101], "XY", [0.01, 0.01], translation=[0, 0, 30])
    assert np.array_equal(x12, g["x12"])
    idx = np.random.default_rng(0).choice(101 * 101, 24, replace=False)
    for tag in ("e1", "e3"):
        f = O.flux(X, B, dt, xyz[idx], float(g["energy_" + tag]), -O.QE, 0.5)
        assert np.array_equal(f, g["flux_" + tag][idx])


def test_cfg2_power_density_subset_and_total_power_bitexact():
    g = golden("pd_cfg2.npz")
    o = cfg_sr(40001, fields="epu")
    X, B, A, dt = o.trajectory()
    xyz, x12, nrm = O.rectangle([201, 201], "XY", [0.04, 0.04], translation=[0, 0, 30])
    assert np.array_equal(x12, g["x12"])
    idx = np.random.default_rng(1).choice(201 * 201, 16, replace=False)
    p = O.power_density(X, B, A, dt, xyz[idx], np.tile(nrm, (16, 1)), False, -O.QE, 0.5)
    assert np.array_equal(p, g["pd"][idx])
    assert o.calculate_total_power() == float(g["total_power"])
    # the analytic total power of this field is within 1e-3 (config 2's check)
    gamma = o.particle[2]
    int_b2 = (1 + 0.36) * W.PERIOD * (W.NPERIODS / 2 + 0.3125)  # both undulators, end poles included
    p_an = W.CURRENT * O.QE ** 3 * gamma ** 2 * int_b2 \
        / (6 * math.pi * 8.854187817e-12 * O.ME ** 2 * O.SPEED_OF_LIGHT ** 2)
    assert abs(o.calculate_total_power() / p_an - 1) < 1e-3


def misc_sr():
    o = O.OracleSR()
    W.setup_beam(o, 3001)
    o.add_bfield_undulator(bfield=[0, 0.8, 0.05], period=[0, 0, 0.05], nperiods=11, phase=0.3,
                           rotations=[0.001, -0.002, 0.3], translation=[0.0001, 0, 0.05], taper=0.01)
    o.add_bfield_gaussian(bfield=[0.02, 0.3, 0], sigma=[0, 0, 0.05], translation=[0, 0, -0.5],
                          rotations=[0, 0.01, 0])
    o.add_bfield_uniform(bfield=[0.0, -0.01, 0.001], width=[0, 0, 0.2], translation=[0, 0, 0.5],
                         rotations=[0.02, 0, 0])
    return o


def test_misc_fields_surfaces_directional_bitexact():
    g = golden("misc_fields.npz")
    o = misc_sr()
    bf = np.array([O.field_eval(o.fields, [0.0001 * i, -0.0002 * i, -1 + 0.1 * i]) for i in range(21)])
    assert np.array_equal(bf, g["bfield"])
    X, B, A, dt = o.trajectory()
    assert np.array_equal(X, g["x"]) and np.array_equal(B, g["beta"])
    e, f = o.calculate_spectrum(obs=[0.001, -0.0005, 20], npoints=40, energy_range_eV=[50, 2000])
    assert np.array_equal(e, g["energies"]) and np.array_equal(f, g["flux"])
    e, f = o.calculate_spectrum(obs=[0, 0, 25], points_eV=[75.0, 133.3, 401.0, 999.9])
    assert np.array_equal(f, g["pts_flux"])
    xyz, x12, nrm = O.rectangle([7, 9], "YZ", [0.02, 0.03], rotations=[0, -math.pi / 2, 0],
                                translation=[0.001, 0, 20], normal=1)
    assert np.array_equal(x12, g["pd_dir_xyz"][:, :2])
    assert np.array_equal(o.calculate_power_density(xyz, nrm, True), g["pd_dir"])
    xyz, x12, nrm = O.rectangle([7, 9], "YZ", [0.02, 0.03], rotations=[0, -math.pi / 2, 0],
                                translation=[0.001, 0, 20], normal=-1)
    assert np.array_equal(o.calculate_power_density(xyz, nrm, True), g["pd_neg"])
    xyz, x12, nrm = O.rectangle([6, 5], x0x1x2=[[-0.004, -0.003, 25], [0.004, -0.003, 25],
                                                [-0.004, 0.003, 25.1]])
    assert np.array_equal(xyz, g["flux_x0x1x2_xyz"])
    assert np.array_equal(o.calculate_flux(xyz, 300.0), g["flux_x0x1x2"])
    assert o.calculate_total_power() == float(g["total_power"])


def test_beam_sampling_rng_and_multiparticle_bitexact():
    g = golden("beam_3a.npz")
    o = cfg_sr(2001, **W.BEAM_3A)
    O.rng_clear_cache()
    O.rng_seed(0)
    xs, bs = [], []
    for _ in range(33):
        o.set_new_particle("random")
        xs.append(o.particle[0])
        bs.append(o.particle[1])
    assert np.array_equal(np.array(xs), g["x0"]) and np.array_equal(np.array(bs), g["beta0"])
    O.rng_seed(0)
    e, f = o.calculate_spectrum(obs=[0, 0, 30], npoints=48, energy_range_eV=[100, 1000], nparticles=4)
    assert np.array_equal(f, g["flux"])
    O.rng_seed(0)
    xyz, x12, nrm = O.rectangle([5, 5], "XY", [0.01, 0.01], translation=[0, 0, 30])
    assert np.array_equal(o.calculate_flux(xyz, W.E1_EV, nparticles=3), g["flux_map"][:25])
    O.rng_seed(0)
    xyz, x12, nrm = O.rectangle([5, 5], "XY", [0.04, 0.04], translation=[0, 0, 30])
    assert np.array_equal(o.calculate_power_density(xyz, nrm, False, nparticles=3), g["pd_map"][:25])


def test_rng_uniform_and_normal_draws_bitexact():
    """rand()/norm() after set_seed(7.9) (the seed is truncated to 7).  The fixture's history before
    that reseed drew 33*5 + 4*5 + 3*5 + 3*5 = 215 normals: an odd count, so one value was cached, and
    a reseed replaces the engine but not the normal distribution's cached value."""
    g = golden("beam_3a.npz")
    O.rng_clear_cache()  # the fixture started from a fresh process
    for count in (33 * 5, 4 * 5, 3 * 5, 3 * 5):  # replay the fixture's draws, each after set_seed(0)
        O.rng_seed(0)
        for _ in range(count):
            O.rng_normal()
    O.rng_seed(int(7.9))
    u = [O.rng_uniform() for _ in range(5)] + [O.rng_normal() for _ in range(5)]
    assert np.array_equal(np.array(u), g["draws"])


def test_grid_field_file_bitexact():
    g = golden("grid_cfg4.npz")
    z, by = W.config4_grid()
    assert np.array_equal(by, g["by"])
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "cfg4.txt")
        W.write_oscars_grid(path, z, by)
        o = O.OracleSR()
        W.setup_beam(o, 20001)
        o.add_bfield_file(path)
        bf = np.array([O.field_eval(o.fields, [0, 0, -0.9 + 0.0123 * i]) for i in range(150)])
        assert np.array_equal(bf, g["bfield"])
        X, B, A, dt = o.trajectory()
        assert np.array_equal(X[:, ::50], g["x_sub"]) and np.array_equal(X[:, -1], g["x_last"])
        idx = np.arange(0, 200, 23)
        f = O.spectrum(X, B, dt, [0, 0, 30], g["energies"][idx], -O.QE, 0.5)
        assert np.array_equal(f, g["flux"][idx])


def test_exact_sums_pinned_to_reference_and_its_rounding_at_weak_outputs():
    """The long-double sums (oracle.flux_exact / spectrum_exact) are the reference's formula: at the
    strongest outputs of the reference's own config-0 spectrum and config-1 maps, where FP64 keeps the
    retarded phase accurately enough, they agree with it to 1e-5.  At the weakest outputs above 1e-6 of
    the maximum the reference's FP64 result is itself off the exact sum by more than 1e-4 (3*E1 map,
    spectrum): the FP64 rounding of a retarded phase of 1e10-1e11 rad, ~1e-5 rad per term.  That is the
    yardstick the GPU floor tests (test_gpu_floors.py) use below 1e-3 of the maximum."""
    g, g0 = golden("flux_cfg1.npz"), golden("spectrum_cfg0.npz")
    o = O.OracleSR()
    W.setup_beam(o, 20001)
    W.setup_undulator(o)
    X, B, A, dt = o.trajectory()
    xs = np.linspace(-0.005, 0.005, 101)
    weakest = {}
    for tag in ("e1", "e3"):
        ref = g["flux_" + tag]
        strong = np.argsort(ref)[::-1][:12]
        idx = np.where(ref >= 1e-6 * ref.max())[0]
        weak = idx[np.argsort(ref[idx])][:12]
        for sel, name in ((strong, "strong"), (weak, "weak")):
            P = np.array([[xs[j // 101], xs[j % 101], 30.0] for j in sel])
            ex = O.flux_exact(X, B, dt, P, float(g["energy_" + tag]), -O.QE, 0.5)
            err = float(np.max(np.abs(ref[sel] / ex - 1)))
            if name == "strong":
                assert err <= 1e-5, (tag, err)
            else:
                weakest[tag] = err
    e, ref = g0["energies"], g0["flux"]
    strong = np.argsort(ref)[::-1][:12]
    idx = np.where(ref >= 1e-6 * ref.max())[0]
    weak = idx[np.argsort(ref[idx])][:12]
    assert np.max(np.abs(ref[strong] / O.spectrum_exact(X, B, dt, [0, 0, 30], e[strong], -O.QE, 0.5) - 1)) <= 1e-5
    weakest["spectrum"] = float(np.max(np.abs(ref[weak] / O.spectrum_exact(X, B, dt, [0, 0, 30], e[weak], -O.QE, 0.5) - 1)))
    assert weakest["e3"] > 1e-4 and weakest["spectrum"] > 1e-4, weakest

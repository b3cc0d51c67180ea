"""Generates the golden fixtures in this directory by running the reference itself.

The reference (dhidas/SRSOriginal, OSCARS SR 1.31.05) is built from its own sources by
``make -C oracle reference`` into ``oracle/_ref/`` (module ``sr``); this script imports it, runs the
hot-path calls on seeded synthetic inputs and stores the outputs as compressed ``.npz`` files.  It
needs the reference sources, so it runs only where they are mounted; the fixtures it writes are
committed and are all the tests need.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import io
import json
import math
import os
import sys
import tempfile
from contextlib import redirect_stdout

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))

from srsoriginal_b200 import workloads as W  # noqa: E402

NT = os.cpu_count() or 2


def new_sr():
    with redirect_stdout(io.StringIO()):
        import sr  # the reference, built by oracle/Makefile
    return sr.sr()


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})
    print("wrote", path, os.path.getsize(path), "bytes")


def traj_arrays(tr):
    t = np.asarray(tr, dtype=np.float64)  # (n, 2, 3)
    return t[:, 0, :].T.copy(), t[:, 1, :].T.copy()


def values(lst):
    return np.array([p[1] for p in lst], dtype=np.float64)


def coords(lst):
    return np.array([p[0] for p in lst], dtype=np.float64)


def cfg0():
    o = new_sr()
    W.setup_beam(o, 20001)
    W.setup_undulator(o)
    X, B = traj_arrays(o.calculate_trajectory())
    s = np.array(o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=1000,
                                      energy_range_eV=[100, 1000], nthreads=NT))
    power = o.calculate_total_power()
    # small companion case (full trajectory stored)
    o2 = new_sr()
    W.setup_beam(o2, 2001)
    W.setup_undulator(o2)
    Xs, Bs = traj_arrays(o2.calculate_trajectory())
    ss = np.array(o2.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=64,
                                        energy_range_eV=[100, 1000], nthreads=1))
    save("spectrum_cfg0.npz", energies=s[:, 0], flux=s[:, 1], x_sub=X[:, ::50], beta_sub=B[:, ::50],
         x_last=X[:, -1], beta_last=B[:, -1], n=X.shape[1], total_power=power,
         small_x=Xs, small_beta=Bs, small_energies=ss[:, 0], small_flux=ss[:, 1],
         small_total_power=o2.calculate_total_power())
    k = int(np.argmax(np.where(s[:, 0] < 300, s[:, 1], 0)))
    return float(s[k, 0])


def cfg1(e1):
    out = {}
    for tag, e in (("e1", e1), ("e3", 3 * e1)):
        o = new_sr()
        W.setup_beam(o, 20001)
        W.setup_undulator(o)
        m = o.calculate_flux_rectangle(plane="XY", energy_eV=e, width=[0.01, 0.01],
                                       npoints=[101, 101], translation=[0, 0, W.SCREEN_Z], nthreads=NT)
        out["flux_" + tag] = values(m)
        out["x12"] = coords(m)[:, :2]
        out["energy_" + tag] = e
    save("flux_cfg1.npz", **out)


def cfg2():
    o = new_sr()
    W.setup_beam(o, 40001)
    W.setup_epu(o)
    m = o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04], npoints=[201, 201],
                                            translation=[0, 0, W.SCREEN_Z], nthreads=NT)
    n = 201 * 201
    save("pd_cfg2.npz", pd=values(m)[:n], x12=coords(m)[:n, :2], total_power=o.calculate_total_power(),
         nlist=len(m))


def misc():
    """Other field kinds, rotations, surfaces and the directional power density."""
    o = new_sr()
    W.setup_beam(o, 3001)
    o.add_bfield_undulator(bfield=[0, 0.8, 0.05], period=[0, 0, 0.05], nperiods=11, phase=0.3,
                           rotations=[0.001, -0.002, 0.3], translation=[0.0001, 0, 0.05], taper=0.01)
    o.add_bfield_gaussian(bfield=[0.02, 0.3, 0], sigma=[0, 0, 0.05], translation=[0, 0, -0.5],
                          rotations=[0, 0.01, 0])
    o.add_bfield_uniform(bfield=[0.0, -0.01, 0.001], width=[0, 0, 0.2], translation=[0, 0, 0.5],
                         rotations=[0.02, 0, 0])
    X, B = traj_arrays(o.calculate_trajectory())
    s = np.array(o.calculate_spectrum(obs=[0.001, -0.0005, 20], npoints=40,
                                      energy_range_eV=[50, 2000], nthreads=1))
    sp = np.array(o.calculate_spectrum(obs=[0.0, 0.0, 25], points_eV=[75.0, 133.3, 401.0, 999.9],
                                       nthreads=1))
    bf = np.array([o.get_bfield([0.0001 * i, -0.0002 * i, -1 + 0.1 * i]) for i in range(21)])
    pd1 = o.calculate_power_density_rectangle(plane="YZ", width=[0.02, 0.03], npoints=[7, 9],
                                              rotations=[0, -math.pi / 2, 0],
                                              translation=[0.001, 0, 20], normal=1, nthreads=1)
    pdm = o.calculate_power_density_rectangle(plane="YZ", width=[0.02, 0.03], npoints=[7, 9],
                                              rotations=[0, -math.pi / 2, 0],
                                              translation=[0.001, 0, 20], normal=-1, nthreads=1)
    fx = o.calculate_flux_rectangle(energy_eV=300.0, npoints=[6, 5],
                                    x0x1x2=[[-0.004, -0.003, 25], [0.004, -0.003, 25], [-0.004, 0.003, 25.1]],
                                    nthreads=1, dim=3)
    save("misc_fields.npz", x=X, beta=B, energies=s[:, 0], flux=s[:, 1], pts_energies=sp[:, 0],
         pts_flux=sp[:, 1], bfield=bf, pd_dir=values(pd1), pd_dir_xyz=coords(pd1), pd_neg=values(pdm),
         flux_x0x1x2=values(fx)[:30], flux_x0x1x2_xyz=coords(fx)[:30], flux_x0x1x2_len=len(fx),
         total_power=o.calculate_total_power())


def beam():
    """Twiss-sampled particles (config 3a beam) from set_seed(0), and a 4-particle spectrum."""
    o = new_sr()
    W.setup_beam(o, 2001, **W.BEAM_3A)
    W.setup_undulator(o)
    o.set_seed(0)
    x0, b0 = [], []
    for _ in range(33):
        o.set_new_particle(particle="random")
        x0.append(o.get_particle_x0())
        b0.append(o.get_particle_beta0())
    o.set_seed(0)
    s = np.array(o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=48, energy_range_eV=[100, 1000],
                                      nparticles=4, nthreads=1))
    o.set_seed(0)
    f = o.calculate_flux_rectangle(plane="XY", energy_eV=W.E1_EV, width=[0.01, 0.01], npoints=[5, 5],
                                   translation=[0, 0, W.SCREEN_Z], nparticles=3, nthreads=1)
    o.set_seed(0)
    p = o.calculate_power_density_rectangle(plane="XY", width=[0.04, 0.04], npoints=[5, 5],
                                            translation=[0, 0, W.SCREEN_Z], nparticles=3, nthreads=1)
    o.set_seed(7.9)
    u = [o.rand() for _ in range(5)] + [o.norm() for _ in range(5)]
    save("beam_3a.npz", x0=np.array(x0), beta0=np.array(b0), energies=s[:, 0], flux=s[:, 1],
         flux_map=values(f), flux_map_len=len(f), pd_map=values(p), pd_map_len=len(p), draws=np.array(u))


def points_surface():
    """Config-0 beam on a 2001-point trajectory; 40 scattered points on a tilted patch near the axis at
    30 m, with their own normals, through calculate_flux and calculate_power_density with rotations,
    translation and each normal option, on the one-thread and the threaded paths."""
    rng = np.random.default_rng(5)
    pts = []
    for _ in range(40):
        x, y = rng.uniform(-0.004, 0.004, 2)
        n = [rng.uniform(-0.2, 0.2), rng.uniform(-0.2, 0.2), 1.0]
        pts.append([[float(x), float(y), float(30.0 + 0.2 * x)], [float(v) for v in n]])
    o = new_sr()
    W.setup_beam(o, 2001)
    W.setup_undulator(o)
    kw = dict(rotations=[2e-5, -3e-5, 0.3], translation=[0.0005, -0.0002, 0.1])
    with redirect_stdout(io.StringIO()):
        f1 = o.calculate_flux(energy_eV=W.E1_EV, points=pts, nthreads=1, **kw)
        f2 = o.calculate_flux(energy_eV=W.E1_EV, points=pts, nthreads=2, **kw)
        pd = {}
        for nrm in (0, 1, -1):
            pd[nrm] = o.calculate_power_density(points=pts, normal=nrm, nthreads=1, **kw)
        pd2 = o.calculate_power_density(points=pts, normal=0, nthreads=2, **kw)
    save("points_surface.npz", points=np.array(pts, dtype=np.float64),
         flux_coords=coords(f1), flux=values(f1), flux_len_t1=len(f1), flux_len_t2=len(f2),
         pd0_coords=coords(pd[0]), pd0=values(pd[0]), pd1=values(pd[1]), pdm1=values(pd[-1]),
         pd_len_t1=len(pd[0]), pd_len_t2=len(pd2))


def beam32():
    """Config 3a on a 32-particle subsample: 20001-point trajectories, 2000 energies over 100-1000 eV on
    axis at 30 m, summed with weight 1/32, after set_seed(0) in a fresh process."""
    o = new_sr()
    W.setup_beam(o, 20001, **W.BEAM_3A)
    W.setup_undulator(o)
    o.set_seed(0)
    with redirect_stdout(io.StringIO()):
        s = np.array(o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=2000, energy_range_eV=[100, 1000],
                                          nparticles=32, nthreads=NT))
    save("beam32_cfg3a.npz", energies=s[:, 0], flux=s[:, 1])


def grid():
    """Config 4 field from an OSCARS-format grid file."""
    z, by = W.config4_grid()
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "cfg4.txt")
        W.write_oscars_grid(path, z, by)
        o = new_sr()
        W.setup_beam(o, 20001)
        o.add_bfield_file(ifile=path, iformat="OSCARS")
        X, B = traj_arrays(o.calculate_trajectory())
        e3 = W.E3_EV
        s = np.array(o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], npoints=200,
                                          energy_range_eV=[0.98 * e3, 1.02 * e3], nthreads=NT))
        bf = np.array([o.get_bfield([0, 0, -0.9 + 0.0123 * i]) for i in range(150)])
    save("grid_cfg4.npz", by=by, x_sub=X[:, ::50], beta_sub=B[:, ::50], x_last=X[:, -1], n=X.shape[1],
         energies=s[:, 0], flux=s[:, 1], bfield=bf)


def adjoint():
    """Config 4 reference gradient: central differences of the reference's own integrated flux
    -Sum_k flux_k dE through perturbed grid files and beam arguments, on the coordinates the
    adjoint tests check."""
    z, by = W.config4_grid()
    e0, e1 = W.config4_energy_range()
    de = (e1 - e0) / (W.NE4 - 1)

    def loss(by_, ic):
        o = new_sr()
        W.setup_beam(o, 20001, x0=[ic[0], ic[1], ic[4]], d0=[ic[2], ic[3], 1.0], energy_GeV=ic[5])
        with tempfile.TemporaryDirectory() as td:
            path = os.path.join(td, "cfg4.txt")
            W.write_oscars_grid(path, z, by_)
            o.add_bfield_file(ifile=path, iformat="OSCARS")
            with redirect_stdout(io.StringIO()):
                s = o.calculate_spectrum(obs=[0, 0, W.SCREEN_Z], energy_range_eV=[e0, e1], npoints=W.NE4,
                                         nthreads=NT)
        f = values(s)
        return -float(np.sum(f * de)), f

    base, flux = loss(by, list(W.IC4))
    coords = W.config4_coords()
    tp, tm, lp, lm = [], [], [], []
    for k in coords:
        h = W.config4_fd_step(int(k), by)
        vals = []
        for sgn in (+1, -1):
            b2, ic2 = by.copy(), list(W.IC4)
            if k < len(by):
                b2[k] = by[k] + sgn * h
                t = float(b2[k])
            else:
                ic2[k - len(by)] = W.IC4[k - len(by)] + sgn * h
                t = ic2[k - len(by)]
            vals.append((t, loss(b2, ic2)[0]))
        (a, la), (b, lb) = vals
        tp.append(a); lp.append(la); tm.append(b); lm.append(lb)
    tp, tm, lp, lm = map(np.array, (tp, tm, lp, lm))
    # complex-step derivatives of the oracle's analytic restatement of the same forward path, whose
    # real part must reproduce the reference's loss
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import complex_step as CS
    from srsoriginal_b200.sr import energy_grid
    energies = energy_grid(W.NE4, e0, e1)
    dz = float((z[-1] - z[0]) / (len(z) - 1))
    g_cs, l_re = CS.complex_step_gradient(by, list(W.IC4), [int(k) for k in coords], float(z[0]), dz,
                                          [0, 0, W.SCREEN_Z], energies, de)
    rel = np.abs(l_re - base).max() / abs(base)
    print("complex-step restatement: loss vs reference", rel)
    assert rel < 1e-9, rel
    save("adjoint_cfg4.npz", coords=coords, theta_plus=tp, theta_minus=tm, loss_plus=lp, loss_minus=lm,
         loss=base, flux=flux, de=de, grad_fd=(lp - lm) / (tp - tm), grad_cs=g_cs, loss_cs=l_re)


def quirks():
    """Output-list lengths of the dispatch paths (reference behaviour, kept by the drop-in)."""
    res = {}
    for nthreads in (1, 2):
        o = new_sr()
        W.setup_beam(o, 501)
        W.setup_undulator(o)
        f = o.calculate_flux_rectangle(plane="XY", energy_eV=150.0, width=[0.01, 0.01], npoints=[3, 4],
                                       translation=[0, 0, 30], nthreads=nthreads)
        p = o.calculate_power_density_rectangle(plane="XY", width=[0.01, 0.01], npoints=[3, 4],
                                                translation=[0, 0, 30], nthreads=nthreads)
        p3 = o.calculate_power_density_rectangle(plane="XY", width=[0.01, 0.01], npoints=[3, 4],
                                                 translation=[0, 0, 30], nthreads=nthreads, dim=3)
        res[f"flux_len_nthreads{nthreads}"] = len(f)
        res[f"pd_len_nthreads{nthreads}"] = len(p)
        res[f"pd_dim3_first_nthreads{nthreads}"] = p3[0][0]
        res[f"flux_coords_nthreads{nthreads}"] = [q[0] for q in f]
    with open(os.path.join(HERE, "quirks.json"), "w") as fh:
        json.dump(res, fh, indent=1)


def aggregate():
    """Running sums (add_to_* / get_*) and file averages (average_*) of the reference's containers
    (OSCARSSR_Python.cc:3252-3572, TSpectrumContainer.cc:159-175, 318-395, T3DScalarContainer.cc:31-320)
    on seeded synthetic spectra and maps: values spanning many magnitudes so the compensated sums
    matter, weights, dim 2 and 3, text and binary files."""
    rng = np.random.default_rng(5)
    out = {}
    o = new_sr()
    ne = 37
    e = np.linspace(100.0, 1000.0, ne)
    spectra = [(rng.lognormal(0.0, 6.0, ne) * rng.choice([1.0, 1e-9, 1e9], ne)).tolist() for _ in range(4)]
    weights = [0.25, 1.0 / 3.0, 0.7, 1e-3]
    for k, (sp, w) in enumerate(zip(spectra, weights)):
        o.add_to_spectrum(spectrum=[[float(a), float(b)] for a, b in zip(e, sp)], weight=w)
    got = o.get_spectrum()
    out["spec_in"] = np.array(spectra)
    out["spec_e"] = e
    out["spec_w"] = np.array(weights)
    out["spec_sum"] = np.array(got)
    npt = 23
    xyz = rng.normal(0.0, 0.01, (npt, 3))
    maps = [(rng.lognormal(0.0, 5.0, npt) * rng.choice([1.0, 1e-8, 1e8], npt)).tolist() for _ in range(3)]
    mw = [0.5, 1.0 / 7.0, 2.0]
    for fn, getter, tag in ((o.add_to_flux, o.get_flux, "flux"), (o.add_to_power_density, o.get_power_density, "pd")):
        for m, w in zip(maps, mw):
            kw = {"flux" if tag == "flux" else "power_density": [[list(map(float, x)), float(v)] for x, v in zip(xyz, m)],
                  "weight": w}
            fn(**kw)
        r = getter()
        out[f"{tag}_xyz"] = np.array([q[0] for q in r])
        out[f"{tag}_sum"] = np.array([q[1] for q in r])
    out["map_in"] = np.array(maps)
    out["map_xyz"] = xyz
    out["map_w"] = np.array(mw)
    # file averages: text spectra (the reference's own %e format, and full precision), dim-2 and
    # dim-3 text maps, dim-2 and dim-3 binary maps, the outputs the reference writes
    with tempfile.TemporaryDirectory() as td:
        files = []
        for k in range(3):
            path = os.path.join(td, f"s{k}.txt")
            with open(path, "w") as fh:
                for a, b in zip(e, spectra[k]):
                    fh.write(f"{a:.6e} {b:.6e}\n" if k != 1 else f"{float(a)!r} {float(b)!r}\n")
            files.append(path)
        # the first file without a trailing newline: the reference drops its last point
        path = os.path.join(td, "s_nonl.txt")
        with open(path, "w") as fh:
            fh.write("\n".join(f"{a:.6e} {b:.6e}" for a, b in zip(e, spectra[3])))
        files_nonl = [path, files[0]]
        oav = new_sr()
        ofile = os.path.join(td, "avg.txt")
        r = oav.average_spectra(ifiles=[f.encode() for f in files], ofile=ofile)
        out["avg_spec"] = np.array(r)
        out["avg_spec_ofile"] = np.frombuffer(open(ofile, "rb").read(), dtype=np.uint8)
        r = oav.average_spectra(ifiles=[f.encode() for f in files_nonl])
        out["avg_spec_nonl"] = np.array(r)
        out["avg_spec_binary_len"] = len(oav.average_spectra(bifiles=[f.encode() for f in files]))
        for k in range(3):
            with open(files[k]) as fh:
                out[f"spec_file{k}"] = np.frombuffer(fh.read().encode(), dtype=np.uint8)
        with open(files_nonl[0]) as fh:
            out["spec_file_nonl"] = np.frombuffer(fh.read().encode(), dtype=np.uint8)
        for dim in (2, 3):
            tf, bf = [], []
            for k in range(3):
                tp, bp = os.path.join(td, f"m{dim}_{k}.txt"), os.path.join(td, f"m{dim}_{k}.bin")
                with open(tp, "w") as fh:
                    for x, v in zip(xyz, maps[k]):
                        cols = list(x[:dim]) + [v]
                        fh.write(" ".join(f"{c:.6e}" for c in cols) + "\n")
                rows = np.column_stack([xyz[:, :dim], maps[k]]).astype(np.float64)
                rows.tofile(bp)
                tf.append(tp)
                bf.append(bp)
                out[f"map{dim}_text{k}"] = np.frombuffer(open(tp, "rb").read(), dtype=np.uint8)
                out[f"map{dim}_bin{k}"] = np.frombuffer(open(bp, "rb").read(), dtype=np.uint8)
            of_t, of_b = os.path.join(td, "avgm.txt"), os.path.join(td, "avgm.bin")
            r = oav.average_flux(ifiles=[f.encode() for f in tf], dim=dim, ofile=of_t, bofile=of_b)
            out[f"avg_flux{dim}_text"] = np.array([[*q[0], q[1]] for q in r])
            out[f"avg_flux{dim}_ofile"] = np.frombuffer(open(of_t, "rb").read(), dtype=np.uint8)
            out[f"avg_flux{dim}_bofile"] = np.frombuffer(open(of_b, "rb").read(), dtype=np.uint8)
            r = oav.average_power_density(bifiles=[f.encode() for f in bf], dim=dim)
            out[f"avg_pd{dim}_binary"] = np.array([[*q[0], q[1]] for q in r])
    errs = {}
    for name, call in (("both_kinds", lambda: oav.average_spectra(ifiles=[b"a"], bifiles=[b"b"])),
                       ("no_files", lambda: oav.average_spectra()),
                       ("no_files_flux", lambda: oav.average_flux()),
                       ("empty_spectrum", lambda: o.add_to_spectrum(spectrum=[])),
                       ("empty_flux", lambda: o.add_to_flux(flux=[])),
                       ("empty_pd", lambda: o.add_to_power_density(power_density=[]))):
        try:
            call()
            errs[name] = None
        except ValueError as exc:
            errs[name] = str(exc)
    with open(os.path.join(HERE, "aggregate_errors.json"), "w") as fh:
        json.dump(errs, fh, indent=1)
    save("aggregate.npz", **out)


def field_file_cases(td):
    """Synthetic field files in each of the reference's formats (seeded) and the add_bfield_* calls that
    read them: (name, kind, arguments, evaluation points).  Written by make_golden.py into the
    fixture, so the tests rebuild the same files without the generator."""
    rng = np.random.default_rng(11)
    cases = []
    # OSCARS1D: irregular z samples, unsorted, a comment line, blank and '#' lines, three columns in the
    # order Z By Bx with scale factors
    z = np.sort(rng.uniform(-0.8, 0.8, 400))
    z[0], z[-1] = -0.8, 0.8
    rng.shuffle(z)
    by = np.sin(2 * np.pi * z / 0.049) * 0.9
    bx = 0.1 * np.cos(2 * np.pi * z / 0.07)
    lines = ["# OSCARS1D test map"]
    for k, (a, b, c) in enumerate(zip(z, by, bx)):
        if k % 97 == 5:
            lines.append("")
        if k % 131 == 7:
            lines.append("# a comment")
        lines.append(f"{float(a)!r} {float(b)!r} {float(c)!r}")
    p1 = os.path.join(td, "map1d.txt")
    with open(p1, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    pts1 = np.column_stack([rng.uniform(-1e-3, 1e-3, 300), rng.uniform(-1e-3, 1e-3, 300), rng.uniform(-0.85, 0.85, 300)])
    cases.append(("oscars1d", "file", dict(ifile=p1, iformat="OSCARS1D Z By Bx", scale=[1.0, 0.95, 1.2]), pts1))
    cases.append(("oscars1d_rot", "file", dict(ifile=p1, iformat="oscars1d Z By Bx", rotations=[0.0, 0.01, 0.02],
                                               translation=[0.0, 0.0, 0.05]), pts1))
    # SRW: a 2-D (x, z) grid with '#' header values
    nx, nz = 5, 161
    xs, dx, zs, dz = -0.002, 0.001, -0.4, 0.005
    lines = ["# SRW test map", f"#{xs!r}", f"#{dx!r}", f"#{nx}", "#0.0", "#0.0", "#1", f"#{zs!r}", f"#{dz!r}", f"#{nz}"]
    for ix in range(nx):
        for iz in range(nz):
            zz = zs + iz * dz
            lines.append(f"{0.01 * ix!r} {float(np.sin(zz * 40.0))!r} {float(0.001 * zz)!r}")
    p2 = os.path.join(td, "srw.txt")
    with open(p2, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    pts2 = np.column_stack([rng.uniform(-0.0025, 0.0025, 300), rng.uniform(-1e-3, 1e-3, 300), rng.uniform(-0.45, 0.45, 300)])
    cases.append(("srw", "file", dict(ifile=p2, iformat="SRW"), pts2))
    # SPECTRA: a 3-D grid, steps in mm, centred on 0
    sx, sy, sz, mx, my, mz = 1.0, 2.0, 5.0, 3, 3, 81
    lines = ["SPECTRA test map", f"{sx!r} {sy!r} {sz!r} {mx} {my} {mz}"]
    for ix in range(mx):
        for iy in range(my):
            for iz in range(mz):
                lines.append(f"{0.001 * (ix + iy)!r} {float(np.cos(iz * 0.3)) * (1 + 0.1 * ix)!r} {0.002 * iy!r}")
    p3 = os.path.join(td, "spectra.txt")
    with open(p3, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    pts3 = np.column_stack([rng.uniform(-0.0012, 0.0012, 300), rng.uniform(-0.0025, 0.0025, 300), rng.uniform(-0.22, 0.22, 300)])
    cases.append(("spectra", "file", dict(ifile=p3, iformat="SPECTRA", rotations=[0.003, 0.0, 0.0]), pts3))
    # interpolated OSCARS maps (gap scan): three files, mapping unsorted
    paths = []
    for gap, amp in ((15.0, 1.2), (25.0, 0.6), (20.0, 0.85)):
        n = 201
        lines = [f"# gap {gap}", "0", "0", "1", "0", "0", "1", "-0.5", "0.005", f"{n}"]
        for iz in range(n):
            zz = -0.5 + iz * 0.005
            lines.append(f"0 {amp * float(np.sin(2 * np.pi * zz / 0.05))!r} {0.01 * amp!r}")
        pth = os.path.join(td, f"gap{int(gap)}.txt")
        with open(pth, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        paths.append((gap, pth))
    pts4 = np.column_stack([np.zeros(300), np.zeros(300), rng.uniform(-0.55, 0.55, 300)])
    mapping = [[g, p] for g, p in paths]
    cases.append(("interp", "interpolated", dict(mapping=mapping, iformat="OSCARS", parameter=18.3,
                                                  scale=[1.0, 1.0, 1.1, 1.0, 0.9]), pts4))
    cases.append(("interp_top", "interpolated", dict(mapping=mapping, iformat="OSCARS", parameter=25.0), pts4))
    cases.append(("interp_first", "interpolated", dict(mapping=mapping, iformat="OSCARS", parameter=15.0), pts4))
    return cases


def field_files():
    """add_bfield_file / add_bfield_interpolated on files of every format: the reference's field at
    seeded points (src/TField3D_Grid.cc:25-45, 533-1446, OSCARSSR_Python.cc:337-510)."""
    out, meta = {}, {}
    with tempfile.TemporaryDirectory() as td:
        for name, kind, kw, pts in field_file_cases(td):
            o = new_sr()
            args = dict(kw)
            if kind == "file":
                args["ifile"] = args["ifile"]
                o.add_bfield_file(**args)
                files = [args["ifile"]]
            else:
                args["mapping"] = [[g, p.encode()] for g, p in args["mapping"]]
                o.add_bfield_interpolated(**args)
                files = [p for _, p in kw["mapping"]]
            out[f"{name}_points"] = pts
            out[f"{name}_b"] = np.array([o.get_bfield(list(map(float, p))) for p in pts])
            for k, fpath in enumerate(files):
                out[f"{name}_file{k}"] = np.frombuffer(open(fpath, "rb").read(), dtype=np.uint8)
            m = {kk: vv for kk, vv in kw.items() if kk not in ("ifile", "mapping")}
            if kind == "interpolated":
                m["mapping_params"] = [g for g, _ in kw["mapping"]]
            meta[name] = dict(kind=kind, nfiles=len(files), **m)
        # errors: lower-case column names, an unknown format, a parameter outside the mapping
        errs = {}
        o = new_sr()
        p1 = os.path.join(td, "x.txt")
        with open(p1, "w") as fh:
            fh.write("# c\n0 1\n0.1 2\n")
        for key, call in (("oscars1d_lowercase_columns", lambda: o.add_bfield_file(ifile=p1, iformat="OSCARS1D z by")),
                          ("unknown_format", lambda: o.add_bfield_file(ifile=p1, iformat="FOO"))):
            try:
                call()
                errs[key] = None
            except ValueError as exc:
                errs[key] = str(exc)
        meta["errors"] = errs
    with open(os.path.join(HERE, "field_files.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    save("field_files.npz", **out)


def efield():
    """Electric fields (OSCARSSR_Python.cc:876-1390, OSCARSSR.cc:690-793) in the RK4, their evaluation,
    the time-domain field (OSCARSSR.cc:2646-2690), and the disabled magnetic add_field_gaussian."""
    out = {}
    rng = np.random.default_rng(13)
    pts = np.column_stack([rng.uniform(-0.01, 0.01, 50), rng.uniform(-0.01, 0.01, 50), rng.uniform(-1.0, 1.0, 50)])
    out["points"] = pts

    def setup(o, n):
        W.setup_beam(o, n)

    # E only: a uniform box and a rotated Gaussian
    o = new_sr()
    setup(o, 4001)
    o.add_efield_uniform(efield=[3e6, 0, 0], width=[0, 0, 0.5])
    o.add_efield_gaussian(efield=[0, 5e6, 1e5], sigma=[0.02, 0.0, 0.1], translation=[0, 0, 0.5],
                          rotations=[0.0, 0.01, 0.0])
    X, B = traj_arrays(o.calculate_trajectory())
    out["e_only_x"], out["e_only_beta"] = X, B
    out["e_only_efield"] = np.array([o.get_efield(list(map(float, p))) for p in pts])
    out["e_only_bfield"] = np.array([o.get_bfield(list(map(float, p))) for p in pts])
    r = o.calculate_efield_vs_time(obs=[0, 0, 30])
    out["e_only_t"] = np.array([q[0] for q in r])
    out["e_only_e"] = np.array([q[1] for q in r])
    # E and B: an undulator and an electric undulator with a phase
    o = new_sr()
    setup(o, 8001)
    W.setup_undulator(o)
    o.add_efield_undulator(efield=[0, 2e7, 0], period=[0, 0, W.PERIOD], nperiods=W.NPERIODS, phase=0.3)
    X, B = traj_arrays(o.calculate_trajectory())
    out["eb_x"], out["eb_beta"] = X, B
    out["eb_efield"] = np.array([o.get_efield(list(map(float, p))) for p in pts])
    sp = o.calculate_spectrum(obs=[0, 0, 30], npoints=20, energy_range_eV=[140, 160], nthreads=NT)
    out["eb_spectrum"] = np.array(sp)
    r = o.calculate_efield_vs_time(obs=[0.001, 0, 30])
    out["eb_t"] = np.array([q[0] for q in r])
    out["eb_e"] = np.array([q[1] for q in r])
    # clearing one container keeps the other
    o.clear_bfields()
    out["eb_cleared_b_efield"] = np.array([o.get_efield(list(map(float, p))) for p in pts[:5]])
    # the magnetic add_field_gaussian adds nothing; the electric one adds a Gaussian
    o = new_sr()
    setup(o, 2001)
    o.add_field_gaussian(sigma=[0, 0, 0.1], bfield=[0, 1.0, 0])
    X, _ = traj_arrays(o.calculate_trajectory())
    out["fg_b_x"] = X
    o.add_field_gaussian(sigma=[0, 0, 0.1], efield=[1e6, 0, 0])
    out["fg_e_efield"] = np.array([o.get_efield(list(map(float, p))) for p in pts[:5]])
    errs = {}
    for key, call in (("fg_both", lambda: o.add_field_gaussian(sigma=[0, 0, 1], bfield=[0, 1, 0], efield=[1, 0, 0])),
                      ("fg_none", lambda: o.add_field_gaussian(sigma=[0, 0, 1])),
                      ("efield_format", lambda: o.add_efield_uniform(efield=[1, 0]))):
        try:
            call()
            errs[key] = None
        except ValueError as exc:
            errs[key] = str(exc)
    with open(os.path.join(HERE, "efield_errors.json"), "w") as fh:
        json.dump(errs, fh, indent=1)
    save("efield.npz", **out)


if __name__ == "__main__":
    parts = sys.argv[1:] or ["cfg0", "cfg1", "cfg2", "misc", "beam", "beam32", "points", "grid", "adjoint",
                             "quirks", "aggregate", "fieldfiles", "efield"]
    if "cfg0" in parts:
        e1 = cfg0()
        print("E1 (first-harmonic peak of the config-0 spectrum):", repr(e1))
        if abs(e1 - W.E1_EV) > 1e-9:
            print("NOTE: update workloads.E1_EV to", repr(e1))
    if "cfg1" in parts:
        cfg1(W.E1_EV)
    for name, fn in (("cfg2", cfg2), ("misc", misc), ("beam", beam), ("beam32", beam32), ("points", points_surface),
                     ("grid", grid),
                     ("adjoint", adjoint),
                     ("quirks", quirks), ("aggregate", aggregate), ("fieldfiles", field_files),
                     ("efield", efield)):
        if name in parts:
            fn()

"""The aggregation methods of the sr object (add_to_* / get_* / average_*) against the reference's
results (tests/golden/aggregate.npz), and a multi-particle spectrum built the way the reference's MPI
examples build it: per-batch spectra added with add_to_spectrum."""
import json
import os

import numpy as np
import pytest

from conftest import golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def test_sr_running_sums_and_averages(tmp_path):
    from srsoriginal_b200.sr import sr
    g = golden("aggregate.npz")
    o = sr()
    for sp, w in zip(g["spec_in"], g["spec_w"]):
        o.add_to_spectrum(spectrum=[[float(a), float(b)] for a, b in zip(g["spec_e"], sp)], weight=float(w))
    assert np.array_equal(np.array(o.get_spectrum()), g["spec_sum"])
    for m, w in zip(g["map_in"], g["map_w"]):
        pts = [[list(map(float, x)), float(v)] for x, v in zip(g["map_xyz"], m)]
        o.add_to_flux(flux=pts, weight=float(w))
        o.add_to_power_density(power_density=pts, weight=float(w))
    for tag, got in (("flux", o.get_flux()), ("pd", o.get_power_density())):
        assert np.array_equal(np.array([p[0] for p in got]), g[f"{tag}_xyz"])
        assert np.array_equal(np.array([p[1] for p in got]), g[f"{tag}_sum"])
    files = []
    for k in range(3):
        p = tmp_path / f"s{k}.txt"
        p.write_bytes(bytes(g[f"spec_file{k}"]))
        files.append(str(p).encode())
    assert np.array_equal(np.array(o.average_spectra(ifiles=files)), g["avg_spec"])
    for dim in (2, 3):
        bf = []
        for k in range(3):
            p = tmp_path / f"m{dim}_{k}.bin"
            p.write_bytes(bytes(g[f"map{dim}_bin{k}"]))
            bf.append(str(p))
        got = o.average_power_density(bifiles=bf, dim=dim)
        assert np.array_equal(np.array([[*p[0], p[1]] for p in got]), g[f"avg_pd{dim}_binary"])
    errs = json.load(open(os.path.join(HERE, "golden", "aggregate_errors.json")))
    for call, key in ((lambda: o.add_to_spectrum(spectrum=[]), "empty_spectrum"),
                      (lambda: o.add_to_flux(flux=[]), "empty_flux"),
                      (lambda: o.add_to_power_density(power_density=[]), "empty_pd")):
        with pytest.raises(ValueError) as e:
            call()
        assert str(e.value) == errs[key]
    with pytest.raises(ValueError, match="number of elements not 3"):
        o.add_to_flux(flux=[[[0.0, 0.0], 1.0]])


def test_multiparticle_spectrum_from_batches():
    """Four batches of 8 particles added with weight 1/4 equal, to 1e-12, one 32-particle call on the
    same particle sequence (the particles come from one seeded generator either way)."""
    from srsoriginal_b200 import workloads as W
    from srsoriginal_b200.sr import sr
    def setup():
        o = sr()
        W.setup_beam(o, 5001, **W.BEAM_3A)
        W.setup_undulator(o)
        return o
    kw = dict(obs=[0, 0, 30], npoints=200, energy_range_eV=[100, 1000])
    o = setup()
    sr.set_seed(7)
    whole = np.array(o.calculate_spectrum(nparticles=32, **kw))
    o2 = setup()
    sr.set_seed(7)
    acc = sr()
    for _ in range(4):
        acc.add_to_spectrum(spectrum=o2.calculate_spectrum(nparticles=8, **kw), weight=0.25)
    got = np.array(acc.get_spectrum())
    assert np.array_equal(got[:, 0], whole[:, 0])
    assert np.linalg.norm(got[:, 1] - whole[:, 1]) <= 1e-12 * np.linalg.norm(whole[:, 1])

"""Running sums and file averages of spectra and maps against the reference's own results
(tests/golden/aggregate.npz, made by running the reference: OSCARSSR_Python.cc:3252-3572), bit for
bit, and the sum over ranks on gloo (world size 2)."""
import json
import os

import numpy as np
import pytest

from conftest import golden

from srsoriginal_b200 import aggregate as A

HERE = os.path.dirname(os.path.abspath(__file__))


def _write(tmp_path, name, arr):
    p = tmp_path / name
    p.write_bytes(bytes(np.asarray(arr, dtype=np.uint8)))
    return str(p)


def test_running_spectrum_sum_matches_reference():
    g = golden("aggregate.npz")
    s = A.SpectrumSum()
    for sp, w in zip(g["spec_in"], g["spec_w"]):
        s.add(g["spec_e"], sp, w)
    got = np.array(s.as_list())
    assert np.array_equal(got, g["spec_sum"])


@pytest.mark.parametrize("tag", ["flux", "pd"])
def test_running_map_sums_match_reference(tag):
    g = golden("aggregate.npz")
    s = A.ScalarSum()
    for m, w in zip(g["map_in"], g["map_w"]):
        s.add(g["map_xyz"], m, w)
    assert np.array_equal(s.xyz, g[f"{tag}_xyz"])
    assert np.array_equal(s.value, g[f"{tag}_sum"])


def test_kahan_sum_is_compensated():
    # 1 + 1e-16 added a million times: the plain sum stays 1, the compensated one reaches 1 + 1e-10
    s = A.SpectrumSum()
    s.add([0.0], [1.0])
    for _ in range(1000):
        s.add([0.0], [1e-16 * 1000])
    assert abs(s.flux[0] - (1.0 + 1e-10)) < 1e-15


def test_average_spectra_text_files(tmp_path):
    g = golden("aggregate.npz")
    files = [_write(tmp_path, f"s{k}.txt", g[f"spec_file{k}"]) for k in range(3)]
    out = str(tmp_path / "avg.txt")
    got = np.array(A.average_spectra(ifiles=[f.encode() for f in files], ofile=out))
    assert np.array_equal(got, g["avg_spec"])
    assert open(out, "rb").read() == bytes(g["avg_spec_ofile"])
    # str paths work too
    assert np.array_equal(np.array(A.average_spectra(ifiles=files)), g["avg_spec"])


def test_average_spectra_quirks(tmp_path):
    """The first file without a trailing newline loses its last point; binary spectrum input is not
    read (empty result), both as in the reference."""
    g = golden("aggregate.npz")
    nonl = _write(tmp_path, "nonl.txt", g["spec_file_nonl"])
    f0 = _write(tmp_path, "s0.txt", g["spec_file0"])
    got = np.array(A.average_spectra(ifiles=[nonl, f0]))
    assert got.shape == g["avg_spec_nonl"].shape and np.array_equal(got, g["avg_spec_nonl"])
    assert len(A.average_spectra(bifiles=[f0])) == int(g["avg_spec_binary_len"]) == 0


@pytest.mark.parametrize("dim", [2, 3])
def test_average_maps_text_and_binary(tmp_path, dim):
    g = golden("aggregate.npz")
    tf = [_write(tmp_path, f"m{k}.txt", g[f"map{dim}_text{k}"]) for k in range(3)]
    bf = [_write(tmp_path, f"m{k}.bin", g[f"map{dim}_bin{k}"]) for k in range(3)]
    ot, ob = str(tmp_path / "o.txt"), str(tmp_path / "o.bin")
    got = A.average_scalars(ifiles=tf, dim=dim, ofile=ot, bofile=ob)
    assert np.array_equal(np.array([[*p[0], p[1]] for p in got]), g[f"avg_flux{dim}_text"])
    assert open(ot, "rb").read() == bytes(g[f"avg_flux{dim}_ofile"])
    assert open(ob, "rb").read() == bytes(g[f"avg_flux{dim}_bofile"])
    got = A.average_scalars(bifiles=bf, dim=dim)
    assert np.array_equal(np.array([[*p[0], p[1]] for p in got]), g[f"avg_pd{dim}_binary"])


def test_aggregation_errors(tmp_path):
    errs = json.load(open(os.path.join(HERE, "golden", "aggregate_errors.json")))
    with pytest.raises(ValueError, match="^" + errs["both_kinds"].replace(".", r"\.") + "$"):
        A.average_spectra(ifiles=["a"], bifiles=["b"])
    with pytest.raises(ValueError) as e:
        A.average_spectra()
    assert str(e.value) == errs["no_files"]
    with pytest.raises(ValueError) as e:
        A.average_scalars()
    assert str(e.value) == errs["no_files_flux"]
    s = A.SpectrumSum()
    s.add([1.0, 2.0], [1.0, 1.0])
    with pytest.raises(ValueError, match="dimensions do not match"):
        s.add([1.0], [1.0])
    g = golden("aggregate.npz")
    f0 = _write(tmp_path, "s0.txt", g["spec_file0"])
    short = tmp_path / "short.txt"
    short.write_text("1.0 2.0\n")
    with pytest.raises(ValueError):  # a later file with fewer points (the reference aborts)
        A.average_spectra(ifiles=[f0, str(short)])
    with pytest.raises(ValueError):
        A.average_scalars(ifiles=[f0], dim=4)

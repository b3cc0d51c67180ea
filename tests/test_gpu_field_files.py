"""sr.add_bfield_file / add_bfield_interpolated with every file format, the field evaluated on the
device (sr.get_bfield), against the reference's values (tests/golden/field_files.npz); and a
trajectory through an OSCARS1D map against the serial kernel through the same map as a grid."""
import json
import os

import numpy as np
import pytest

from conftest import golden

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "field_files.json")))
CASES = [k for k in META if k != "errors"]


@pytest.mark.parametrize("name", CASES)
def test_sr_field_files_match_reference(tmp_path, name):
    from srsoriginal_b200.sr import sr
    g = golden("field_files.npz")
    m = META[name]
    files = []
    for k in range(m["nfiles"]):
        p = tmp_path / f"{name}_{k}.txt"
        p.write_bytes(bytes(g[f"{name}_file{k}"]))
        files.append(str(p))
    kw = {k: m[k] for k in ("rotations", "translation", "scale") if k in m}
    o = sr()
    if m["kind"] == "file":
        o.add_bfield_file(ifile=files[0], iformat=m["iformat"], **kw)
    else:
        o.add_bfield_interpolated(mapping=[[p, f.encode()] for p, f in zip(m["mapping_params"], files)],
                                  iformat=m["iformat"], parameter=m["parameter"], **kw)
    got = np.array([o.get_bfield(list(map(float, p))) for p in g[f"{name}_points"]])
    assert np.array_equal(got, g[f"{name}_b"], equal_nan=True), np.nanmax(np.abs(got - g[f"{name}_b"]))


def test_sr_field_file_errors(tmp_path):
    from srsoriginal_b200.sr import sr
    bad = tmp_path / "x.txt"
    bad.write_text("# c\n0 1\n0.1 2\n")
    o = sr()
    errs = META["errors"]
    with pytest.raises(ValueError) as e:
        o.add_bfield_file(ifile=str(bad), iformat="OSCARS1D z by")
    assert str(e.value) == errs["oscars1d_lowercase_columns"]
    with pytest.raises(ValueError) as e:
        o.add_bfield_file(ifile=str(bad), iformat="FOO")
    assert str(e.value) == errs["unknown_format"]
    with pytest.raises(ValueError, match="Incorrect format in 'mapping'"):
        o.add_bfield_interpolated(mapping=[[1.0]], iformat="OSCARS", parameter=1.0)
    with pytest.raises(ValueError, match="'iformat' is blank"):
        o.add_bfield_interpolated(mapping=[], iformat="", parameter=1.0)


def test_trajectory_through_oscars1d_map(tmp_path):
    from srsoriginal_b200 import workloads as W
    from srsoriginal_b200.sr import sr
    g = golden("field_files.npz")
    p = tmp_path / "map1d.txt"
    p.write_bytes(bytes(g["oscars1d_file0"]))
    o = sr()
    W.setup_beam(o, 4001)
    o.add_bfield_file(ifile=str(p), iformat="OSCARS1D Z By Bx")
    t = np.array(o.calculate_trajectory(), dtype=object)
    x = np.array([q[0] for q in t], float)
    assert np.isfinite(x).all() and np.abs(x[:, 0]).max() > 1e-7  # deflected by the map's By

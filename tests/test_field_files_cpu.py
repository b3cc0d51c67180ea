"""Field-map files of every format the reference reads (OSCARS1D, SRW, SPECTRA, interpolated OSCARS
maps) through the library's host readers, evaluated by the oracle's grid field, against the
reference's own field values at seeded points (tests/golden/field_files.npz, made by running the
reference: src/TField3D_Grid.cc:25-45, 533-1446)."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from conftest import golden

import oracle as O
from srsoriginal_b200 import fieldmaps

HERE = os.path.dirname(os.path.abspath(__file__))
META = json.load(open(os.path.join(HERE, "golden", "field_files.json")))
CASES = [k for k in META if k != "errors"]


def _files(tmp_path, g, name, n):
    out = []
    for k in range(n):
        p = tmp_path / f"{name}_{k}.txt"
        p.write_bytes(bytes(g[f"{name}_file{k}"]))
        out.append(str(p))
    return out


def _read(tmp_path, name):
    g = golden("field_files.npz")
    m = META[name]
    files = _files(tmp_path, g, name, m["nfiles"])
    kw = {k: m[k] for k in ("rotations", "translation", "scale") if k in m}
    if m["kind"] == "file":
        f, data = fieldmaps.read_field_file(files[0], m["iformat"], **kw)
    else:
        mapping = [[p, path] for p, path in zip(m["mapping_params"], files)]
        f, data = fieldmaps.read_field_interpolated(mapping, m["iformat"], m["parameter"], **kw)
    return g, f, data


def _oracle_field(f, data):
    of = O.OrcField()
    of.kind = O.GRID
    for k in range(3):
        of.rotations[k] = f.rotations[k]
        of.translation[k] = f.translation[k]
        of.start[k] = f.start[k]
        of.step[k] = f.step[k]
        of.n[k] = f.n[k]
    buf = np.ascontiguousarray(data.reshape(-1))
    of.data = buf.ctypes.data_as(C.POINTER(C.c_double))
    return of, buf


@pytest.mark.parametrize("name", CASES)
def test_field_file_matches_reference(tmp_path, name):
    g, f, data = _read(tmp_path, name)
    of, keep = _oracle_field(f, data)
    got = np.array([O.field_eval([of], p) for p in g[f"{name}_points"]])
    ref = g[f"{name}_b"]
    assert np.array_equal(got, ref, equal_nan=True), np.abs(got - ref).max()


def test_interpolated_at_first_parameter_is_nan(tmp_path):
    """The reference's interpolation leaves its 'before' index unset at exactly the first mapping
    parameter: 0/0 slope, NaN field (reproduced)."""
    g, f, data = _read(tmp_path, "interp_first")
    assert np.isnan(data).all()
    assert np.isnan(g["interp_first_b"][np.abs(g["interp_first_points"][:, 2]) < 0.49]).all()


def test_field_file_errors(tmp_path):
    bad = tmp_path / "x.txt"
    bad.write_text("# c\n0 1\n0.1 2\n")
    for fmt in ("OSCARS1D z by", "FOO", "OSCARS1D Z By Bx Bz Y"):
        with pytest.raises(ValueError):
            fieldmaps.read_field_file(str(bad), fmt)
    with pytest.raises(ValueError):  # more scale factors than columns (the reference writes out of bounds)
        fieldmaps.read_field_file(str(bad), "OSCARS1D Z By", scale=[1, 1, 1])
    g = golden("field_files.npz")
    files = _files(tmp_path, g, "interp", 3)
    mapping = [[p, path] for p, path in zip(META["interp"]["mapping_params"], files)]
    for par in (14.0, 25.5, float("nan")):
        with pytest.raises(ValueError):
            fieldmaps.read_field_interpolated(mapping, "OSCARS", par)
    with pytest.raises(ValueError):
        fieldmaps.read_field_interpolated(mapping[:1], "OSCARS", 15.0)

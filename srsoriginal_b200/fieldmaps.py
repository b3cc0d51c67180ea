"""Field maps read from files on the host (srs_read_field_file / srs_read_field_interpolated): the
grid descriptor and its rotated samples as numpy, in the reference's formats (OSCARS, OSCARS1D, SRW,
SPECTRA, and maps interpolated between OSCARS files; src/TField3D_Grid.cc).  ``sr.add_bfield_file``
and ``sr.add_bfield_interpolated`` use the same readers and keep the samples on the device."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


def _v3(v):
    return _lib.v3(list(v) if v is not None and len(v) else [0.0, 0.0, 0.0])


def _read(call):
    f = _lib.Field()
    n = C.c_int64(0)
    check(call(f, None, n))
    data = np.zeros(max(1, n.value), dtype=np.float64)
    check(call(f, data.ctypes.data_as(_lib._D), n))
    return f, data[:n.value].reshape(-1, 3)


def read_field_file(path, iformat, rotations=None, translation=None, scale=None):
    """(srs_field descriptor with data NULL, samples (n, 3)) of a field-map file."""
    sc = [float(s) for s in (scale or [])]
    arr = (C.c_double * max(1, len(sc)))(*sc)
    p = path if isinstance(path, bytes) else str(path).encode()
    return _read(lambda f, d, n: lib.srs_read_field_file(p, str(iformat).encode(), _v3(rotations), _v3(translation),
                                                         arr, len(sc), C.byref(f), d, C.byref(n)))


def read_field_interpolated(mapping, iformat, parameter, rotations=None, translation=None, scale=None):
    """The same for a map interpolated between files: mapping = [[parameter, path], ...]."""
    params = [float(m[0]) for m in mapping]
    paths = [m[1] if isinstance(m[1], bytes) else str(m[1]).encode() for m in mapping]
    parr = (C.c_double * max(1, len(params)))(*params)
    farr = (C.c_char_p * max(1, len(paths)))(*paths)
    sc = [float(s) for s in (scale or [])]
    arr = (C.c_double * max(1, len(sc)))(*sc)
    return _read(lambda f, d, n: lib.srs_read_field_interpolated(parr, farr, len(params), str(iformat).encode(),
                                                                 float(parameter), _v3(rotations), _v3(translation),
                                                                 arr, len(sc), C.byref(f), d, C.byref(n)))

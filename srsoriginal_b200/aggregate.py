"""Multi-particle aggregation: running sums of spectra, flux maps and power-density maps, averages of
result files, and the sum over ranks of a multi-process run.

The reference keeps one spectrum and two 3-D scalar containers per ``sr`` object and adds weighted
results into them with compensated (Kahan) sums (``add_to_spectrum`` / ``add_to_flux`` /
``add_to_power_density`` and ``get_*``, src/OSCARSSR_Python.cc:3329-3470, src/OSCARSSR.cc:1331-1400);
it averages result files point by point (``average_spectra``, ``average_flux``,
``average_power_density``, src/OSCARSSR_Python.cc:3252-3320, 3472-3572, src/TSpectrumContainer.cc:
318-395, src/T3DScalarContainer.cc:66-320); and its multi-process examples send every worker's
spectrum to rank 0, which adds them with ``add_to_spectrum`` (Examples/Example_122_*_MPI.py).

Here the containers are numpy arrays with the same IEEE-double operations in the same order (numpy
does not contract multiply-adds), so sums and averages equal the reference's bit for bit; the rank
sum runs over ``torch.distributed`` (gloo or NCCL) instead of MPI, in rank order.
"""
from __future__ import annotations

import os

import numpy as np


def _kahan_add(total, comp, v):
    """total, comp += v elementwise, the reference's compensated sum (TSpectrumContainer.cc:159-175,
    T3DScalarContainer.cc:31-46): y = v - c; t = s + y; c = (t - s) - y; s = t."""
    y = v - comp
    t = total + y
    comp[:] = (t - total) - y
    total[:] = t


class SpectrumSum:
    """A spectrum container: energies, summed flux and the compensation of each point."""

    def __init__(self):
        self.energy = np.zeros(0)
        self.flux = np.zeros(0)
        self.comp = np.zeros(0)

    def __len__(self):
        return len(self.energy)

    def add(self, energy, flux, weight=1.0):
        """OSCARSSR::AddToSpectrum (OSCARSSR.cc:1331-1348): the first spectrum sets the points
        (flux * weight), later ones add flux * weight to each point with the compensated sum."""
        energy = np.asarray(energy, dtype=np.float64).reshape(-1)
        flux = np.asarray(flux, dtype=np.float64).reshape(-1) * float(weight)
        if len(self) == 0:
            self.energy, self.flux, self.comp = energy.copy(), flux.copy(), np.zeros(len(energy))
        elif len(energy) == len(self):
            _kahan_add(self.flux, self.comp, flux)
        else:
            raise ValueError("spectra dimensions do not match")

    def as_list(self):
        return [[float(a), float(b)] for a, b in zip(self.energy, self.flux)]

    def write_text(self, path):
        """TSpectrumContainer::WriteToFileText (TSpectrumContainer.cc:224-258): "E flux" in %e."""
        with open(path, "w") as f:
            for a, b in zip(self.energy, self.flux):
                f.write(f"{a:.6e} {b:.6e}\n")


class ScalarSum:
    """A 3-D scalar container (flux or power-density map): points, summed values, compensations."""

    def __init__(self):
        self.xyz = np.zeros((0, 3))
        self.value = np.zeros(0)
        self.comp = np.zeros(0)

    def __len__(self):
        return len(self.value)

    def add(self, xyz, value, weight=1.0):
        """OSCARSSR::AddToFlux / AddToPowerDensity (OSCARSSR.cc:1355-1400): the first map sets the
        points, later ones add value * weight to each point (their positions are not compared)."""
        xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
        value = np.asarray(value, dtype=np.float64).reshape(-1) * float(weight)
        if len(self) == 0:
            self.xyz, self.value, self.comp = xyz.copy(), value.copy(), np.zeros(len(value))
        elif len(value) == len(self):
            _kahan_add(self.value, self.comp, value)
        else:
            raise ValueError("spectra dimensions do not match")

    def as_list(self):
        return [[[float(c) for c in x], float(v)] for x, v in zip(self.xyz, self.value)]

    def write_text(self, path, dim):
        """T3DScalarContainer::WriteToFileText (T3DScalarContainer.cc:322-348)."""
        if dim not in (2, 3):
            raise ValueError("incorrect dimensions")
        with open(path, "w") as f:
            for x, v in zip(self.xyz, self.value):
                cols = list(x[:dim]) + [v]
                f.write(" ".join(f"{c:.6e}" for c in cols) + "\n")

    def write_binary(self, path, dim):
        """T3DScalarContainer::WriteToFileBinary (T3DScalarContainer.cc:351-395): native doubles,
        (x, y, v) or (x, y, z, v) per point."""
        if dim not in (2, 3):
            raise ValueError("incorrect dimensions")
        np.column_stack([self.xyz[:, :dim], self.value]).astype(np.float64).tofile(path)


# ---------------------------------------------------------------- reading result files

def _path(p):
    return os.fsdecode(p) if isinstance(p, (bytes, bytearray)) else str(p)


def _read_text(path, k):
    """The records an ``ifstream >> x`` loop reads from a text file, k numbers each: every complete
    group of k tokens, except that a read which reaches the end of the file ends the loop before its
    record is added -- so the last record is dropped when the file does not end in whitespace
    (TSpectrumContainer.cc:342-380)."""
    with open(_path(path), "rb") as f:
        text = f.read().decode()
    tokens = text.split()
    try:
        vals = np.array([float(t) for t in tokens], dtype=np.float64)
    except ValueError as exc:
        raise ValueError(f"cannot read {path}: {exc}") from None
    n = len(vals) // k
    if n > 0 and len(vals) % k == 0 and text and not text[-1].isspace():
        n -= 1
    return vals[:n * k].reshape(n, k)


def _read_binary(path, k):
    """Native doubles, k per record; a partial last record ends the loop (TSpectrumContainer.cc:
    397-460)."""
    raw = np.fromfile(_path(path), dtype=np.float64)
    n = len(raw) // k
    return raw[:n * k].reshape(n, k)


def _average(tables, k):
    """The point-by-point average of several files: the first file's positions, value_0 / N, then
    value_i / N added with the compensated sum for i = 1..N-1 in file order; the first file's length
    decides, and a later file that ends earlier is an error (T3DScalarContainer.cc:66-188)."""
    n0 = len(tables[0])
    for t in tables[1:]:
        if len(t) < n0:
            raise ValueError("a file has fewer points than the first")
    N = float(len(tables))
    total = tables[0][:, k - 1] / N
    comp = np.zeros(n0)
    for t in tables[1:]:
        _kahan_add(total, comp, t[:n0, k - 1] / N)
    return tables[0][:, :k - 1], total


def _file_lists(ifiles, bifiles):
    ifiles, bifiles = list(ifiles or []), list(bifiles or [])
    if ifiles and bifiles:
        raise ValueError("either text or binary files may be added, but not both.")
    if not ifiles and not bifiles:
        raise ValueError("No files given.  You need at least one file as input in a list.")
    return ifiles, bifiles


def average_spectra(ifiles=None, bifiles=None, ofile="", bofile=""):
    """``sr.average_spectra`` (OSCARSSR_Python.cc:3252-3320): the average of text spectrum files.  As
    in the reference, binary input is not read (its reader is disabled there): the result is then
    empty.  A binary output file is not written (the reference's writer aborts)."""
    ifiles, bifiles = _file_lists(ifiles, bifiles)
    s = SpectrumSum()
    if ifiles:
        pos, val = _average([_read_text(f, 2) for f in ifiles], 2)
        s.energy, s.flux, s.comp = pos[:, 0].copy(), val, np.zeros(len(val))
    if ofile:
        s.write_text(_path(ofile))
    if bofile:
        raise ValueError("binary spectrum output is not available (the reference aborts on it)")
    return s.as_list()


def average_scalars(ifiles=None, bifiles=None, ofile="", bofile="", dim=2):
    """``sr.average_flux`` / ``sr.average_power_density`` (OSCARSSR_Python.cc:3472-3572): the average
    of text or binary map files with dim = 2 (x, y, v) or 3 (x, y, z, v) columns; the result's points
    are 3-D (z = 0 for dim 2)."""
    ifiles, bifiles = _file_lists(ifiles, bifiles)
    if dim not in (2, 3):
        raise ValueError("incorrect dimensions")
    k = dim + 1
    tables = [_read_text(f, k) for f in ifiles] if ifiles else [_read_binary(f, k) for f in bifiles]
    pos, val = _average(tables, k)
    s = ScalarSum()
    s.xyz = np.column_stack([pos, np.zeros(len(val))]) if dim == 2 else pos.copy()
    s.value, s.comp = val, np.zeros(len(val))
    if ofile:
        s.write_text(_path(ofile), dim)
    if bofile:
        s.write_binary(_path(bofile), dim)
    return s.as_list()


# ---------------------------------------------------------------- ranks

def sum_over_ranks(values, weight=1.0, dst=0, group=None):
    """The multi-process pattern of the reference's MPI examples on ``torch.distributed``: every rank
    contributes its result array (a spectrum's or a map's values), rank ``dst`` receives all of them
    and returns their compensated, weighted sum in rank order (deterministic, where the examples add
    in arrival order); other ranks return None.  Device tensors are used with the NCCL backend, host
    tensors with gloo."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    mine = torch.as_tensor(np.ascontiguousarray(values, dtype=np.float64), device=dev)
    parts = [torch.empty_like(mine) for _ in range(world)] if rank == dst else None
    dist.gather(mine, parts, dst=dst, group=group)
    if rank != dst:
        return None
    total = SpectrumSum()
    for p in parts:
        v = p.cpu().numpy()
        total.add(np.zeros(len(v)), v, weight)
    return total.flux

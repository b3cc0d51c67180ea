"""ORACLE -- test infrastructure only.

ctypes front end to ``liboracle.so`` (the plain-C restatement in ``srs_oracle.c`` of the reference's
CPU algorithm) plus ``OracleSR``, a small restatement of the reference's Python-facing dispatch
(``src/OSCARSSR_Python.cc`` / ``src/OSCARSSR.cc``) built on it.  Only the tests, the smoke check and
the CPU-baseline leg of ``bench.py`` use this module, always as the checker; the shipped library
never imports it.  It is pinned against the reference's own outputs by ``tests/test_oracle_golden.py``.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

UNDULATOR, GAUSSIAN, UNIFORM_BOX, GRID = 1, 2, 3, 4
SPEED_OF_LIGHT = 2.99792458e8
QE = 1.602176462e-19
ME = 9.10938356e-31


class OrcField(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("field", C.c_double * 3),
        ("period", C.c_double * 3),
        ("center", C.c_double * 3),
        ("nperiods", C.c_int),
        ("phase", C.c_double),
        ("taper", C.c_double),
        ("sigma_or_width", C.c_double * 3),
        ("rotations", C.c_double * 3),
        ("translation", C.c_double * 3),
        ("start", C.c_double * 3),
        ("step", C.c_double * 3),
        ("n", C.c_int64 * 3),
        ("data", C.POINTER(C.c_double)),
    ]


class OrcBeam(C.Structure):
    _fields_ = [
        ("q", C.c_double), ("m", C.c_double), ("current", C.c_double),
        ("x0", C.c_double * 3), ("u0", C.c_double * 3),
        ("e0", C.c_double), ("t0", C.c_double),
        ("hdir", C.c_double * 3), ("vdir", C.c_double * 3),
        ("sigma_u", C.c_double * 2), ("sigma_up", C.c_double * 2),
        ("sigma_at", C.c_double * 3), ("sigma_e", C.c_double),
    ]


_D = C.POINTER(C.c_double)


def lib():
    """Load (building it first if needed) the restatement library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "srs_oracle.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        import subprocess
        subprocess.check_call(["make", "-s", "-C", _HERE, "restatement"])
    L = C.CDLL(path)
    L.orc_field_eval.argtypes = [C.POINTER(OrcField), C.c_int, _D, _D]
    L.orc_grid_read_oscars.argtypes = [C.c_char_p, _D, _D, _D, C.c_int, C.POINTER(OrcField)]
    L.orc_grid_read_oscars.restype = C.c_int
    L.orc_free.argtypes = [C.c_void_p]
    L.orc_trajectory_counts.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int64, _D,
                                        C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    L.orc_trajectory.argtypes = [C.POINTER(OrcField), C.c_int, _D, _D, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_int64, _D, _D, _D, _D]
    L.orc_trajectory.restype = C.c_int64
    L.orc_spectrum.argtypes = [_D, _D, C.c_int64, C.c_double, _D, _D, C.c_int64, C.c_double,
                               C.c_double, C.c_double, _D, _D]
    L.orc_flux.argtypes = [_D, _D, C.c_int64, C.c_double, _D, C.c_int64, C.c_double, C.c_double,
                           C.c_double, C.c_double, _D, _D]
    L.orc_flux_exact.argtypes = [_D, _D, C.c_int64, C.c_double, _D, C.c_int64, C.c_double, C.c_double,
                                 C.c_double, _D]
    L.orc_spectrum_exact.argtypes = [_D, _D, C.c_int64, C.c_double, _D, _D, C.c_int64, C.c_double,
                                     C.c_double, _D]
    L.orc_power_density.argtypes = [_D, _D, _D, C.c_int64, C.c_double, _D, _D, C.c_int64, C.c_int,
                                    C.c_double, C.c_double, _D, _D]
    L.orc_total_power.argtypes = [_D, _D, C.c_int64, C.c_double, C.c_double, C.c_double, C.c_double]
    L.orc_total_power.restype = C.c_double
    L.orc_energy_grid.argtypes = [C.c_int64, C.c_double, C.c_double, _D]
    L.orc_rectangle_plane.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_double, C.c_double, _D, _D,
                                      C.c_int, _D, _D, _D]
    L.orc_rectangle_plane.restype = C.c_int
    L.orc_rectangle_points.argtypes = [C.c_int, C.c_int, _D, _D, _D, _D, _D, C.c_int, _D, _D, _D]
    L.orc_rectangle_points.restype = C.c_int
    L.orc_rng_seed.argtypes = [C.c_uint32]
    L.orc_rng_normal.restype = C.c_double
    L.orc_rng_uniform.restype = C.c_double
    L.orc_beam_init.argtypes = [C.POINTER(OrcBeam), C.c_char_p, C.c_double, _D, _D, C.c_double,
                                C.c_double, C.c_double, _D, _D, _D, _D, _D, _D, C.c_double, C.c_double]
    L.orc_beam_init.restype = C.c_int
    L.orc_beam_particle.argtypes = [C.POINTER(OrcBeam), C.c_int, _D, _D, _D, _D]
    _LIB = L
    return L


def _p(a):
    return a.ctypes.data_as(_D)


def _v3(v):
    a = (C.c_double * 3)()
    a[0], a[1], a[2] = float(v[0]), float(v[1]), float(v[2])
    return a


def _arr(v, n):
    a = np.ascontiguousarray(np.asarray(v, dtype=np.float64).reshape(n))
    return a


# ---------------------------------------------------------------- vector helpers (TVector3D.cc)

def rotate_xyz(v, rot):
    """TVector3D::RotateSelfXYZ (src/TVector3D.cc:196-205), in Python floats (IEEE double)."""
    x, y, z = (float(t) for t in v)
    s, c = math.sin(rot[0]), math.cos(rot[0])
    y, z = c * y - s * z, s * y + c * z
    s, c = math.sin(rot[1]), math.cos(rot[1])
    z, x = c * z - s * x, s * z + c * x
    s, c = math.sin(rot[2]), math.cos(rot[2])
    x, y = c * x - s * y, s * x + c * y
    return [x, y, z]


# ---------------------------------------------------------------- field builders

def undulator(bfield, period, nperiods, phase=0.0, rotations=(0, 0, 0), translation=(0, 0, 0),
              taper=0.0):
    """add_bfield_undulator (src/OSCARSSR_Python.cc:736-818): field and period rotated, centre = translation."""
    f = OrcField()
    f.kind = UNDULATOR
    f.field = _v3(rotate_xyz(bfield, rotations))
    f.period = _v3(rotate_xyz(period, rotations))
    f.center = _v3(translation)
    f.nperiods = int(nperiods)
    f.phase = float(phase)
    f.taper = float(taper)
    return f


def gaussian(bfield, sigma, rotations=(0, 0, 0), translation=(0, 0, 0)):
    """add_bfield_gaussian (src/OSCARSSR_Python.cc:561-632) -> TField3D_Gaussian.cc:22-46."""
    f = OrcField()
    f.kind = GAUSSIAN
    f.field = _v3(rotate_xyz(bfield, rotations))
    f.center = _v3(translation)
    f.sigma_or_width = _v3(sigma)
    f.rotations = _v3(rotations)
    return f


def uniform(bfield, width=(0, 0, 0), rotations=(0, 0, 0), translation=(0, 0, 0)):
    """add_bfield_uniform (src/OSCARSSR_Python.cc:640-716) -> TField3D_UniformBox.cc:32-58."""
    f = OrcField()
    f.kind = UNIFORM_BOX
    f.field = _v3(rotate_xyz(bfield, rotations))
    f.center = _v3(translation)
    f.sigma_or_width = _v3(width)
    f.rotations = _v3(rotations)
    return f


class GridField:
    """An OSCARS-format field file (TField3D_Grid::ReadFile), read by the C restatement."""

    def __init__(self, path, rotations=(0, 0, 0), translation=(0, 0, 0), scale=()):
        self.f = OrcField()
        sc = (C.c_double * max(1, len(scale)))(*[float(s) for s in scale]) if scale else None
        rc = lib().orc_grid_read_oscars(path.encode(), _v3(rotations), _v3(translation),
                                        sc if sc is not None else None, len(scale), C.byref(self.f))
        if rc != 0:
            raise ValueError(f"cannot read grid file {path} ({rc})")

    def __del__(self):
        try:
            if self.f.data:
                lib().orc_free(C.cast(self.f.data, C.c_void_p))
                self.f.data = None
        except Exception:
            pass


def _field_array(fields):
    structs = [f.f if isinstance(f, GridField) else f for f in fields]
    arr = (OrcField * max(1, len(structs)))(*structs)
    return arr, len(structs)


def field_eval(fields, x):
    arr, n = _field_array(fields)
    out = (C.c_double * 3)()
    lib().orc_field_eval(arr, n, _v3(x), out)
    return [out[0], out[1], out[2]]


# ---------------------------------------------------------------- trajectory and sums

def trajectory_counts(ctstart, ctstop, t0, npoints):
    dt = C.c_double()
    nf, nb = C.c_int64(), C.c_int64()
    lib().orc_trajectory_counts(ctstart, ctstop, t0, npoints, C.byref(dt), C.byref(nf), C.byref(nb))
    return dt.value, nf.value, nb.value


def trajectory(fields, x0, b0, qomg, ctstart, ctstop, t0, npoints):
    """RK4 trajectory: returns (x, beta, a_over_c) as (3, n) arrays and dt."""
    dt, nf, nb = trajectory_counts(ctstart, ctstop, t0, npoints)
    n = nf + nb
    X = np.zeros(3 * n)
    B = np.zeros(3 * n)
    A = np.zeros(3 * n)
    arr, nfld = _field_array(fields)
    dto = C.c_double()
    lib().orc_trajectory(arr, nfld, _v3(x0), _v3(b0), qomg, ctstart, ctstop, t0, npoints,
                         _p(X), _p(B), _p(A), C.byref(dto))
    return X.reshape(3, n), B.reshape(3, n), A.reshape(3, n), dto.value


def spectrum(X, B, dt, obs, energies, charge, current, weight=1.0, out=None, comp=None):
    X = np.ascontiguousarray(X, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    e = np.ascontiguousarray(energies, dtype=np.float64)
    out = np.zeros(len(e)) if out is None else out
    comp = np.zeros(len(e)) if comp is None else comp
    lib().orc_spectrum(_p(X), _p(B), X.shape[1], dt, _v3(obs), _p(e), len(e), charge, current, weight,
                       _p(out), _p(comp))
    return out


def flux(X, B, dt, points, energy_ev, charge, current, weight=1.0, out=None, comp=None):
    X = np.ascontiguousarray(X, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    P = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(P)) if out is None else out
    comp = np.zeros(len(P)) if comp is None else comp
    lib().orc_flux(_p(X), _p(B), X.shape[1], dt, _p(P), len(P), energy_ev, charge, current, weight,
                   _p(out), _p(comp))
    return out


def flux_exact(X, B, dt, points, energy_ev, charge, current):
    """The flux sum of flux() evaluated in long double (the exact value FP64 evaluations approximate)."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    P = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(P))
    lib().orc_flux_exact(_p(X), _p(B), X.shape[1], dt, _p(P), len(P), energy_ev, charge, current, _p(out))
    return out


def spectrum_exact(X, B, dt, obs, energies, charge, current):
    """The spectrum sum of spectrum() evaluated in long double."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    e = np.ascontiguousarray(energies, dtype=np.float64)
    out = np.zeros(len(e))
    lib().orc_spectrum_exact(_p(X), _p(B), X.shape[1], dt, _v3(obs), _p(e), len(e), charge, current, _p(out))
    return out


def power_density(X, B, A, dt, points, normals, directional, charge, current, out=None, comp=None):
    X = np.ascontiguousarray(X, dtype=np.float64)
    B = np.ascontiguousarray(B, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    P = np.ascontiguousarray(points, dtype=np.float64).reshape(-1, 3)
    Nn = np.ascontiguousarray(normals, dtype=np.float64).reshape(-1, 3)
    out = np.zeros(len(P)) if out is None else out
    comp = np.zeros(len(P)) if comp is None else comp
    lib().orc_power_density(_p(X), _p(B), _p(A), X.shape[1], dt, _p(P), _p(Nn), len(P),
                            int(bool(directional)), charge, current, _p(out), _p(comp))
    return out


def total_power(B, A, dt, charge, current, gamma):
    B = np.ascontiguousarray(B, dtype=np.float64)
    A = np.ascontiguousarray(A, dtype=np.float64)
    return lib().orc_total_power(_p(B), _p(A), B.shape[1], dt, charge, current, gamma)


def energy_grid(n, e0, e1):
    out = np.zeros(n)
    lib().orc_energy_grid(n, e0, e1, _p(out))
    return out


def rectangle(npoints, plane="", width=(0, 0), x0x1x2=None, rotations=(0, 0, 0),
              translation=(0, 0, 0), normal=0):
    """Rectangle points as the reference builds them (OSCARSSR_Python.cc:2636-2717)."""
    nx1, nx2 = int(npoints[0]), int(npoints[1])
    np_ = nx1 * nx2
    xyz = np.zeros(3 * np_)
    x12 = np.zeros(2 * np_)
    nrm = (C.c_double * 3)()
    rc = -1
    if x0x1x2 is not None:
        rc = lib().orc_rectangle_points(nx1, nx2, _v3(x0x1x2[0]), _v3(x0x1x2[1]), _v3(x0x1x2[2]),
                                        _v3(rotations), _v3(translation), int(normal), _p(xyz),
                                        _p(x12), nrm)
    elif plane and width[0] > 0 and width[1] > 0:
        rc = lib().orc_rectangle_plane(plane.encode(), nx1, nx2, float(width[0]), float(width[1]),
                                       _v3(rotations), _v3(translation), int(normal), _p(xyz),
                                       _p(x12), nrm)
    if rc != 0:
        raise ValueError("bad rectangle")
    return xyz.reshape(np_, 3), x12.reshape(np_, 2), np.array([nrm[0], nrm[1], nrm[2]])


def rng_seed(seed):
    lib().orc_rng_seed(int(seed) & 0xFFFFFFFF)


def rng_clear_cache():
    lib().orc_rng_clear_cache()


def rng_normal():
    return lib().orc_rng_normal()


def rng_uniform():
    return lib().orc_rng_uniform()


class Beam:
    """set_particle_beam arguments -> TParticleBeam state (restated in C)."""

    def __init__(self, type="electron", energy_GeV=3.0, d0=(0, 0, 1), x0=(0, 0, 0),
                 sigma_energy_GeV=0.0, t0=0.0, current=0.0, rotations=(0, 0, 0),
                 translation=(0, 0, 0), horizontal_direction=None, beta=None, emittance=None,
                 lattice_reference=(0, 0, 0), mass=0.0, charge=0.0):
        self.b = OrcBeam()
        hd = _v3(horizontal_direction) if horizontal_direction is not None else None
        be = (C.c_double * 2)(*beta) if beta is not None else None
        em = (C.c_double * 2)(*emittance) if emittance is not None else None
        rc = lib().orc_beam_init(C.byref(self.b), type.encode(), energy_GeV, _v3(d0), _v3(x0),
                                 sigma_energy_GeV, t0, current, _v3(rotations), _v3(translation),
                                 hd, be, em, _v3(lattice_reference), mass, charge)
        if rc != 0:
            raise ValueError("bad beam")

    def particle(self, random=False):
        x0 = (C.c_double * 3)()
        b0 = (C.c_double * 3)()
        g = C.c_double()
        q = C.c_double()
        lib().orc_beam_particle(C.byref(self.b), int(bool(random)), x0, b0, C.byref(g), C.byref(q))
        return list(x0), list(b0), g.value, q.value


class OracleSR:
    """A restatement of the reference's single-beam dispatch (OSCARSSR.cc:933-984, :1603-1677,
    :2418-2489) for the calls on the hot path; results are the CPU path's (nthreads=1) values."""

    def __init__(self):
        self.fields = []
        self.beam = None
        self.particle = None
        self.ctstart = 0.0
        self.ctstop = 0.0
        self.npoints = 0

    def set_ctstartstop(self, start, stop):
        self.npoints = int(10000 * (stop - start))
        self.ctstart, self.ctstop = float(start), float(stop)

    def set_npoints_trajectory(self, n):
        self.npoints = int(n)

    def add_bfield_undulator(self, **kw):
        self.fields.append(undulator(**kw))

    def add_bfield_gaussian(self, **kw):
        self.fields.append(gaussian(**kw))

    def add_bfield_uniform(self, **kw):
        self.fields.append(uniform(**kw))

    def add_bfield_file(self, ifile, iformat="OSCARS", rotations=(0, 0, 0), translation=(0, 0, 0),
                        scale=()):
        self.fields.append(GridField(ifile, rotations, translation, scale))

    def set_particle_beam(self, **kw):
        kw.pop("name", None)
        kw.pop("weight", None)
        self.beam = Beam(**kw)
        self.particle = self.beam.particle(False)

    def set_new_particle(self, particle="random"):
        self.particle = self.beam.particle(particle == "random")

    def trajectory(self):
        x0, b0, g, qomg = self.particle
        return trajectory(self.fields, x0, b0, qomg, self.ctstart, self.ctstop, self.beam.b.t0,
                          self.npoints)

    def calculate_spectrum(self, obs, npoints=0, energy_range_eV=None, points_eV=None, nparticles=0):
        e = np.asarray(points_eV, float) if points_eV else energy_grid(npoints, *energy_range_eV)
        out, comp = np.zeros(len(e)), np.zeros(len(e))
        runs = [1.0] if nparticles == 0 else [1.0 / nparticles] * nparticles
        for w in runs:
            if nparticles:
                self.set_new_particle("random")
            X, B, A, dt = self.trajectory()
            spectrum(X, B, dt, obs, e, self.beam.b.q, self.beam.b.current, w, out, comp)
        return e, out

    def calculate_flux(self, points, energy_eV, nparticles=0):
        P = np.asarray(points, float).reshape(-1, 3)
        out, comp = np.zeros(len(P)), np.zeros(len(P))
        runs = [1.0] if nparticles == 0 else [1.0 / nparticles] * nparticles
        for w in runs:
            if nparticles:
                self.set_new_particle("random")
            X, B, A, dt = self.trajectory()
            flux(X, B, dt, P, energy_eV, self.beam.b.q, self.beam.b.current, w, out, comp)
        return out

    def calculate_power_density(self, points, normal_vec, directional, nparticles=0):
        P = np.asarray(points, float).reshape(-1, 3)
        Nn = np.tile(np.asarray(normal_vec, float), (len(P), 1))
        out, comp = np.zeros(len(P)), np.zeros(len(P))
        for _ in range(max(1, nparticles)):
            if nparticles:
                self.set_new_particle("random")
            X, B, A, dt = self.trajectory()
            power_density(X, B, A, dt, P, Nn, directional, self.beam.b.q, self.beam.b.current,
                          out, comp)
        return out

    def calculate_total_power(self):
        X, B, A, dt = self.trajectory()
        return total_power(B, A, dt, self.beam.b.q, self.beam.b.current, self.particle[2])

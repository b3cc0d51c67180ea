"""``sr``: the reference's Python type (``oscars.sr.sr``, src/OSCARSSR_Python.cc) for the radiation
hot path, on the B200.

Same method names, keyword names, positional order, defaults, return shapes and ValueError messages
as the reference for the calls on the hot path; every calculation runs on the GPU through the C ABI
of ``libsrs_b200.so`` (include/srs_b200.h).  The ``nthreads``/``gpu`` switch is kept: it selects the
reference dispatch path whose observable behaviour is reproduced (output-list length, particle
weighting), while the arithmetic always runs on the device.

One addition: ``precision`` ('fp64' -- the default, the plain IEEE-double drop-in -- or 'mixed'),
as a keyword of the calculate_* calls and through ``set_precision_global``.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from . import aggregate as _agg
from ._lib import check, dptr, lib, v3

_ZERO3 = (0.0, 0.0, 0.0)
_PRECISIONS = {"fp64": _lib.FP64, "mixed": _lib.MIXED}


def _list3(v, what):
    """OSCARSSR_ListAsTVector3D: exactly three numbers, else ValueError("Incorrect format in 'what'")."""
    try:
        if len(v) != 3:
            raise ValueError
        return [float(v[0]), float(v[1]), float(v[2])]
    except (TypeError, ValueError):
        raise ValueError(f"Incorrect format in '{what}'") from None


def _list2(v, what):
    try:
        if len(v) != 2:
            raise ValueError
        return [float(v[0]), float(v[1])]
    except (TypeError, ValueError):
        raise ValueError(f"Incorrect format in '{what}'") from None


def _opt3(v, what):
    return _ZERO3 if v is None or len(v) == 0 else _list3(v, what)


class sr:  # noqa: N801  (the reference's type name)
    """Simulation object: fields, particle beams, trajectory settings and the radiation calculations."""

    def __init__(self):
        h = C.c_void_p()
        check(lib.srs_sim_create(C.byref(h)))
        self._h = h
        self._nthreads_global = 2
        self._precision = _lib.FP64
        self._spectrum_sum = _agg.SpectrumSum()
        self._flux_sum = _agg.ScalarSum()
        self._pd_sum = _agg.ScalarSum()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib.srs_sim_destroy(h)
            self._h = None

    # ------------------------------------------------------------ constants and globals
    @staticmethod
    def pi():
        return 3.14159265358979323846

    @staticmethod
    def qe():
        return 1.602176462e-19

    @staticmethod
    def me():
        return 9.10938356e-31

    @staticmethod
    def rand():
        return lib.srs_random_uniform()

    @staticmethod
    def norm():
        return lib.srs_random_normal()

    @staticmethod
    def set_seed(seed):
        """TRandomA::SetSeed: the value is truncated to int (OSCARSSR_Python.cc:184-194)."""
        lib.srs_set_seed(float(seed))

    def set_gpu_global(self, gpu):
        check(lib.srs_sim_set_gpu_global(self._h, int(gpu)))

    @staticmethod
    def check_gpu():
        """Number of CUDA devices (the reference returns -1 when built without CUDA)."""
        return lib.srs_device_count()

    def set_nthreads_global(self, nthreads):
        self._nthreads_global = int(nthreads)
        check(lib.srs_sim_set_nthreads_global(self._h, int(nthreads)))

    def set_precision_global(self, precision):
        """Default arithmetic of the sums: 'fp64' (plain, the drop-in) or 'mixed'."""
        self._precision = self._prec(precision)

    def _prec(self, precision):
        if precision is None:
            return self._precision
        try:
            return _PRECISIONS[str(precision).lower()]
        except KeyError:
            raise ValueError("'precision' must be 'fp64' or 'mixed'") from None

    # ------------------------------------------------------------ trajectory settings
    def get_ctstart(self):
        a, b = C.c_double(), C.c_double()
        check(lib.srs_sim_get_ctstartstop(self._h, C.byref(a), C.byref(b)))
        return a.value

    def get_ctstop(self):
        a, b = C.c_double(), C.c_double()
        check(lib.srs_sim_get_ctstartstop(self._h, C.byref(a), C.byref(b)))
        return b.value

    def set_ctstartstop(self, start, stop):
        try:
            start, stop = float(start), float(stop)
        except (TypeError, ValueError):
            raise ValueError("Incorrect format") from None
        check(lib.srs_sim_set_ctstartstop(self._h, start, stop))

    def set_npoints_trajectory(self, npoints):
        check(lib.srs_sim_set_npoints_trajectory(self._h, int(npoints)))

    def get_npoints_trajectory(self):
        return int(lib.srs_sim_get_npoints_trajectory(self._h))

    # ------------------------------------------------------------ fields
    def add_bfield_file(self, ifile, iformat, rotations=None, translation=None, scale=None):
        if not ifile or not iformat:
            raise ValueError("'ifile' or 'iformat' is blank")
        rot = _opt3(rotations, "rotations")
        tr = _opt3(translation, "translation")
        sc = [float(s) for s in (scale or [])]
        arr = (C.c_double * max(1, len(sc)))(*sc)
        st = lib.srs_sim_add_bfield_file(self._h, str(ifile).encode(), str(iformat).encode(), v3(rot),
                                         v3(tr), arr, len(sc))
        if st != _lib.SRS_OK:
            msg = lib.srs_last_error().decode()
            if msg == "'ifile' or 'iformat' is blank":
                raise ValueError(msg)
            raise ValueError("Could not import magnetic field.  Check 'ifile' and 'iformat' are correct")

    def add_bfield_interpolated(self, mapping, iformat, parameter, rotations=None, translation=None, scale=None):
        """A field map interpolated between files by a parameter (e.g. an undulator gap):
        mapping = [[parameter value, file name], ...] of OSCARS-format files with the same grid
        (OSCARSSR_Python.cc:419-510)."""
        params, paths = [], []
        for pair in mapping or []:
            if len(pair) != 2:
                raise ValueError("Incorrect format in 'mapping'")
            params.append(float(pair[0]))
            f = pair[1]
            paths.append(f if isinstance(f, bytes) else str(f).encode())
        if not iformat:
            raise ValueError("'iformat' is blank")
        rot = _opt3(rotations, "rotations")
        tr = _opt3(translation, "translation")
        sc = [float(s) for s in (scale or [])]
        parr = (C.c_double * max(1, len(params)))(*params)
        farr = (C.c_char_p * max(1, len(paths)))(*paths)
        scarr = (C.c_double * max(1, len(sc)))(*sc)
        st = lib.srs_sim_add_bfield_interpolated(self._h, parr, farr, len(params), str(iformat).encode(),
                                                 float(parameter), v3(rot), v3(tr), scarr, len(sc))
        if st != _lib.SRS_OK:
            raise ValueError("Could not import magnetic field.  Check filenames and 'iformat' are correct")

    def add_bfield_gaussian(self, bfield, sigma, rotations=None, translation=None):
        b = _list3(bfield, "bfield")
        s = _list3(sigma, "sigma")
        check(lib.srs_sim_add_bfield_gaussian(self._h, v3(b), v3(s), v3(_opt3(rotations, "rotations")),
                                              v3(_opt3(translation, "translation"))))

    def add_bfield_uniform(self, bfield, width=None, rotations=None, translation=None):
        b = _list3(bfield, "bfield")
        w = _opt3(width, "width")
        check(lib.srs_sim_add_bfield_uniform(self._h, v3(b), v3(w), v3(_opt3(rotations, "rotations")),
                                             v3(_opt3(translation, "translation"))))

    def add_bfield_undulator(self, bfield, period, nperiods, phase=0.0, rotations=None, translation=None,
                             taper=0.0):
        b = _list3(bfield, "bfield")
        p = _list3(period, "period")
        check(lib.srs_sim_add_bfield_undulator(self._h, v3(b), v3(p), int(nperiods), float(phase),
                                               v3(_opt3(rotations, "rotations")),
                                               v3(_opt3(translation, "translation")), float(taper)))

    def add_bfield_grid(self, start, step, n, data, rotations=None, translation=None):
        """A field map given as arrays: start/step/n per axis (x, y, z) and data[nx*ny*nz][3] in the
        OSCARS file order (index ix*ny*nz + iy*nz + iz).  Same field as add_bfield_file."""
        d = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(-1))
        nn = (C.c_int64 * 3)(*[int(x) for x in n])
        check(lib.srs_sim_add_bfield_grid(self._h, v3(start), v3(step), nn, dptr(d),
                                          v3(_opt3(rotations, "rotations")),
                                          v3(_opt3(translation, "translation"))))

    def get_bfield(self, x):
        if not isinstance(x, list) or len(x) != 3:
            raise ValueError("Incorrect format in 'rotations'")
        pts = np.ascontiguousarray(np.array(x, dtype=np.float64))
        out = np.zeros(3)
        check(lib.srs_sim_get_bfield(self._h, dptr(pts), 1, dptr(out)))
        return [float(out[0]), float(out[1]), float(out[2])]

    # ------------------------------------------------------------ electric fields
    def add_efield_file(self, ifile, iformat, rotations=None, translation=None, scale=None):
        """An electric field map file (OSCARSSR_Python.cc:876-935); like the reference, scale is accepted
        and not applied."""
        if not ifile or not iformat:
            raise ValueError("'ifile' or 'iformat' is blank")
        rot = _opt3(rotations, "rotations")
        tr = _opt3(translation, "translation")
        st = lib.srs_sim_add_efield_file(self._h, str(ifile).encode(), str(iformat).encode(), v3(rot), v3(tr))
        if st != _lib.SRS_OK:
            raise ValueError("Could not import electric field.  Check 'ifile' and 'iformat' are correct")

    def add_efield_gaussian(self, efield, sigma, rotations=None, translation=None):
        e = _list3(efield, "efield")
        s = _list3(sigma, "sigma")
        check(lib.srs_sim_add_efield_gaussian(self._h, v3(e), v3(s), v3(_opt3(rotations, "rotations")),
                                              v3(_opt3(translation, "translation"))))

    def add_efield_uniform(self, efield, width=None, rotations=None, translation=None):
        e = _list3(efield, "efield")
        w = _opt3(width, "width")
        check(lib.srs_sim_add_efield_uniform(self._h, v3(e), v3(w), v3(_opt3(rotations, "rotations")),
                                             v3(_opt3(translation, "translation"))))

    def add_efield_undulator(self, efield, period, nperiods, phase=0.0, rotations=None, translation=None):
        e = _list3(efield, "efield")
        p = _list3(period, "period")
        check(lib.srs_sim_add_efield_undulator(self._h, v3(e), v3(p), int(nperiods), float(phase),
                                               v3(_opt3(rotations, "rotations")),
                                               v3(_opt3(translation, "translation"))))

    def add_field_gaussian(self, sigma, bfield=None, efield=None, rotations=None, translation=None):
        """A Gaussian electric field (OSCARSSR_Python.cc:1306-1390); as in the reference, a 'bfield' here
        adds nothing (its call is disabled there)."""
        has_b, has_e = bool(bfield) and len(bfield) > 0, bool(efield) and len(efield) > 0
        if has_b and has_e:
            raise ValueError("You cannot define both 'bfield' and 'efield'")
        if has_b:
            _list3(bfield, "bfield")
        elif has_e:
            e = _list3(efield, "efield")
        else:
            raise ValueError("You must define either 'bfield' or 'efield'")
        s = _list3(sigma, "sigma")
        rot = _opt3(rotations, "rotations")
        tr = _opt3(translation, "translation")
        if has_e:
            check(lib.srs_sim_add_efield_gaussian(self._h, v3(e), v3(s), v3(rot), v3(tr)))

    def get_efield(self, x):
        if not isinstance(x, list) or len(x) != 3:
            raise ValueError("Incorrect format in 'rotations'")
        pts = np.ascontiguousarray(np.array(x, dtype=np.float64))
        out = np.zeros(3)
        check(lib.srs_sim_get_efield(self._h, dptr(pts), 1, dptr(out)))
        return [float(out[0]), float(out[1]), float(out[2])]

    def clear_efields(self):
        check(lib.srs_sim_clear_efields(self._h))

    def clear_bfields(self):
        check(lib.srs_sim_clear_bfields(self._h))

    def set_trajectory_cache(self, enabled=True):
        """Keep (True, the default) or not the device trajectory of the last single-particle call for
        reuse while the particle, fields and trajectory settings are unchanged; any call drops the
        kept trajectory."""
        check(lib.srs_sim_set_trajectory_cache(self._h, 1 if enabled else 0))

    _TRAJ_MODES = {"auto": 0, "serial": 1, "parallel": 2}

    def set_trajectory_mode(self, mode="auto"):
        """How single-particle trajectories are integrated: 'auto' (default) parallel in time for the
        mixed-precision sums and serially, with the reference's roundings, for everything else;
        'serial' always serially; 'parallel' always parallel in time (multiple shooting: equal to the
        serial trajectory to ~1e-16 m).  Not in the reference."""
        if mode not in self._TRAJ_MODES:
            raise ValueError("'mode' must be one of 'auto', 'serial', 'parallel'")
        check(lib.srs_sim_set_trajectory_mode(self._h, self._TRAJ_MODES[mode]))

    # ------------------------------------------------------------ particle beams
    def add_particle_beam(self, type, name, energy_GeV, d0, x0, sigma_energy_GeV=0.0, t0=0.0, current=0.0,
                          weight=1.0, rotations=None, translation=None, horizontal_direction=None, beta=None,
                          emittance=None, lattice_reference=None, mass=0.0, charge=0.0):
        if not type or not name:
            raise ValueError("'type' or 'name' is blank")
        a = _lib.BeamArgs()
        a.type = str(type).encode()
        a.name = str(name).encode()
        a.energy_gev = float(energy_GeV)
        pos = _opt3(x0, "x0")
        a.x0 = v3(pos)
        if d0 is None or len(d0) == 0:
            raise ValueError("Incorrect format in 'd0'")
        a.d0 = v3(_list3(d0, "d0"))
        if sigma_energy_GeV < 0:
            raise ValueError("'sigma_energy_GeV' cannot be less than zero")
        a.sigma_energy_gev = float(sigma_energy_GeV)
        a.t0 = float(t0)
        a.current = float(current)
        a.weight = float(weight)
        a.rotations = v3(_opt3(rotations, "rotations"))
        a.translation = v3(_opt3(translation, "translation"))
        keep = []
        if horizontal_direction is not None and len(horizontal_direction) != 0:
            hd = v3(_list3(horizontal_direction, "horizontal_direction"))
            keep.append(hd)
            a.horizontal_direction = C.cast(hd, _lib._D)
        has_beta = beta is not None and len(beta) != 0
        has_em = emittance is not None and len(emittance) != 0
        if has_beta:
            bt = (C.c_double * 2)(*_list2(beta, "beta"))
        if has_em:
            em = (C.c_double * 2)(*_list2(emittance, "emittance"))
        if has_beta and has_em:
            keep += [bt, em]
            a.beta = C.cast(bt, _lib._D)
            a.emittance = C.cast(em, _lib._D)
        a.lattice_reference = v3(_opt3(lattice_reference, "lattice_reference"))
        a.mass = float(mass)
        a.charge = float(charge)
        check(lib.srs_sim_add_particle_beam(self._h, C.byref(a)))

    def set_particle_beam(self, *args, **kwargs):
        """clear_particle_beams + add_particle_beam + the ideal particle (OSCARSSR_Python.cc:1641-1655)."""
        self.clear_particle_beams()
        self.add_particle_beam(*args, **kwargs)
        check(lib.srs_sim_set_new_particle(self._h, b"", b"ideal"))

    def clear_particle_beams(self):
        check(lib.srs_sim_clear_particle_beams(self._h))

    def set_new_particle(self, beam="", particle=""):
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        b, p = str(beam).lower(), str(particle).lower()
        if p != "" and p not in ("ideal", "random"):
            raise ValueError("'particle' must be 'ideal' or 'random'")
        st = lib.srs_sim_set_new_particle(self._h, b.encode(), p.encode())
        if st != _lib.SRS_OK:
            raise ValueError("'beam' name not found")

    def _particle(self):
        x0, b0 = _lib._V3(), _lib._V3()
        e0, g = C.c_double(), C.c_double()
        check(lib.srs_sim_get_particle(self._h, x0, b0, C.byref(e0), C.byref(g)))
        return list(x0), list(b0), e0.value

    def get_particle_x0(self):
        return self._particle()[0]

    def get_particle_beta0(self):
        return self._particle()[1]

    def get_particle_e0(self):
        return self._particle()[2]

    # ------------------------------------------------------------ trajectory
    def _trajectory_arrays(self):
        n = C.c_int64()
        check(lib.srs_sim_calculate_trajectory(self._h, C.byref(n), None, None))
        x = np.zeros(3 * n.value)
        b = np.zeros(3 * n.value)
        check(lib.srs_sim_calculate_trajectory(self._h, C.byref(n), dptr(x), dptr(b)))
        return x.reshape(-1, 3), b.reshape(-1, 3)

    def calculate_trajectory(self):
        """[[[x, y, z], [bx, by, bz]], ...] of the current particle (OSCARSSR_Python.cc:1988-2037)."""
        x, b = self._trajectory_arrays()
        self._last_trajectory = (x, b)
        return [[xi, bi] for xi, bi in zip(x.tolist(), b.tolist())]

    def get_trajectory(self):
        x, b = getattr(self, "_last_trajectory", (np.zeros((0, 3)), np.zeros((0, 3))))
        return [[xi, bi] for xi, bi in zip(x.tolist(), b.tolist())]

    # ------------------------------------------------------------ spectrum
    def calculate_spectrum(self, obs, npoints=0, energy_range_eV=None, points_eV=None, nparticles=0, nthreads=0,
                           gpu=0, ofile="", bofile="", precision=None):
        """[[E, flux], ...] in photons/s/0.1%bw/mm^2 (OSCARSSR_Python.cc:2215-2349)."""
        e, flux = self.spectrum_arrays(obs, npoints, energy_range_eV, points_eV, nparticles, nthreads, gpu,
                                       precision)
        if ofile:
            with open(ofile, "w") as f:
                for a, b in zip(e, flux):
                    f.write(f"{a:.6e} {b:.6e}\n")
        if bofile:
            np.column_stack([e, flux]).astype(np.float64).tofile(bofile)
        return [[float(a), float(b)] for a, b in zip(e, flux)]

    def spectrum_arrays(self, obs, npoints=0, energy_range_eV=None, points_eV=None, nparticles=0, nthreads=0,
                        gpu=0, precision=None):
        """calculate_spectrum returning (energies, flux) numpy arrays."""
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        pts = [float(p) for p in (points_eV or [])]
        if energy_range_eV is not None and len(energy_range_eV) != 0 and len(energy_range_eV) != 2:
            raise ValueError("'energy_range_eV' must be a list of length 2")
        o = _list3(obs, "obs")
        self._check_gpu_threads(gpu, nthreads)
        prec = self._prec(precision)
        if not pts:
            if npoints < 1:
                raise ValueError("'npoints' must be > 0")
            if energy_range_eV is None or len(energy_range_eV) != 2:
                raise ValueError("'energy_range_eV' must be a list of length 2")
            e = np.zeros(int(npoints))
            check(lib.srs_energy_grid(int(npoints), float(energy_range_eV[0]), float(energy_range_eV[1]), dptr(e)))
        else:
            e = np.ascontiguousarray(np.array(pts, dtype=np.float64))
        out = np.zeros(len(e))
        check(lib.srs_sim_calculate_spectrum(self._h, v3(o), dptr(e), len(e), int(nparticles), prec, dptr(out),
                                             None))
        return e, out

    # ------------------------------------------------------------ surfaces
    @staticmethod
    def _rect_spec(npoints, width, rotations, translation):
        if not isinstance(npoints, (list, tuple)) or len(npoints) != 2:
            raise ValueError("'npoints' must be [int, int]")
        n1, n2 = int(npoints[0]), int(npoints[1])
        if n1 <= 0 or n2 <= 0:
            raise ValueError("an entry in 'npoints' is <= 0")
        rot = _opt3(rotations, "rotations")
        tr = _opt3(translation, "translation")
        w1 = w2 = 0.0
        if width is not None and len(width) == 2:
            w1, w2 = float(width[0]), float(width[1])
        return n1, n2, w1, w2, rot, tr

    def _rectangle(self, npoints, plane, width, x0x1x2, rotations, translation, normal):
        n1, n2, w1, w2, rot, tr = sr._rect_spec(npoints, width, rotations, translation)
        np_ = n1 * n2
        xyz, x12 = np.zeros(3 * np_), np.zeros(2 * np_)
        nrm = _lib._V3()
        grid = _lib.Grid2D()
        ok = False
        if plane and w1 > 0 and w2 > 0:
            check(lib.srs_rectangle_plane(str(plane).encode(), n1, n2, w1, w2, v3(rot), v3(tr), int(normal),
                                          dptr(xyz), dptr(x12), nrm, C.byref(grid)))
            ok = True
        if x0x1x2 is not None and len(x0x1x2) != 0:
            if len(x0x1x2) != 3:
                raise ValueError("'x0x1x2' must have 3 XYZ points defined correctly")
            p = [_list3(q, "x0x1x2") for q in x0x1x2]
            check(lib.srs_rectangle_points(n1, n2, v3(p[0]), v3(p[1]), v3(p[2]), v3(rot), v3(tr), int(normal),
                                           dptr(xyz), dptr(x12), nrm, C.byref(grid)))
            ok = True
        if not ok:
            raise ValueError("no surface defined: give 'plane' and 'width', or 'x0x1x2'")
        return xyz.reshape(np_, 3), x12.reshape(np_, 2), np.array(list(nrm)), grid

    def _check_gpu_threads(self, gpu, nthreads):
        if gpu not in (0, 1):
            raise ValueError("'gpu' must be 0 or 1")
        if nthreads < 0:
            raise ValueError("'nthreads' must be > 0")
        if nthreads > 0 and gpu == 1:
            raise ValueError("gpu is 1 and nthreads > 0.  Both are not currently allowed.")

    @staticmethod
    def _coords(xyz, x12, dim):
        if dim == 2:
            return np.column_stack([x12, np.zeros(len(x12))])
        return xyz

    @staticmethod
    def _write_points(ofile, coords, vals, dim):
        with open(ofile, "w") as f:
            for c, v in zip(coords, vals):
                if dim == 2:
                    f.write(f"{c[0]:.6e} {c[1]:.6e} {v:.6e}\n")
                else:
                    f.write(f"{c[0]:.6e} {c[1]:.6e} {c[2]:.6e} {v:.6e}\n")

    # ------------------------------------------------------------ arbitrary point surfaces
    @staticmethod
    def _rotate_xyz(v, r):
        """TVector3D::RotateSelfXYZ (TVector3D.cc:150-205): about X, then Y, then Z."""
        x, y, z = v
        s, c = math.sin(r[0]), math.cos(r[0])
        y, z = c * y - s * z, s * y + c * z
        s, c = math.sin(r[1]), math.cos(r[1])
        z, x = c * z - s * x, s * z + c * x
        s, c = math.sin(r[2]), math.cos(r[2])
        x, y = c * x - s * y, s * x + c * y
        return [x, y, z]

    @staticmethod
    def _surface_3d(points, rotations, translation, invert_normal):
        """TSurfacePoints_3D from [[x, y, z], [nx, ny, nz]] pairs as the reference's point-list calls
        build it (OSCARSSR_Python.cc:2449-2502, 2875-2920): point and normal rotated, the normal
        optionally inverted and made a unit vector (TSurfacePoint.cc:12-16), the point translated.
        Returns (points (N,3), unit normals (N,3))."""
        rot = _list3(rotations, "rotations") if rotations is not None and len(rotations) != 0 else [0.0, 0.0, 0.0]
        tr = _list3(translation, "translation") if translation is not None and len(translation) != 0 \
            else [0.0, 0.0, 0.0]
        xs, ns = [], []
        for item in points:
            if not hasattr(item, "__len__") or len(item) != 2:
                raise ValueError("Incorrect format in 'points'")
            try:
                X = _list3(item[0], "points")
                N = _list3(item[1], "points")
            except ValueError:
                raise ValueError("Incorrect format in 'points': Point or Normal does not have 3 elements") from None
            X = sr._rotate_xyz(X, rot)
            N = sr._rotate_xyz(N, rot)
            if invert_normal:
                N = [-N[0], -N[1], -N[2]]
            m = math.sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2])  # TSurfacePoint keeps the unit normal
            xs.append([X[0] + tr[0], X[1] + tr[1], X[2] + tr[2]])
            ns.append([N[0] / m, N[1] / m, N[2] / m])
        return np.array(xs, dtype=np.float64).reshape(-1, 3), np.array(ns, dtype=np.float64).reshape(-1, 3)

    def _point_list(self, xyz, out, nparticles, nthreads, gpu, pd):
        """The reference's list for a point surface (dim = 3): the points, then the zero entries its
        dispatch path appends (see calculate_flux_rectangle / calculate_power_density_rectangle)."""
        nth = nthreads if nthreads >= 1 else self._nthreads_global
        calls = max(1, int(nparticles))
        extra = gpu == 1 or (nth != 1 if pd else nth == 1)
        coords = np.concatenate([xyz] + ([xyz] * calls if extra else []))
        vals = np.concatenate([out] + ([np.zeros(len(xyz))] * calls if extra else []))
        return coords, vals

    def calculate_flux(self, energy_eV, points, normal=0, rotations=None, translation=None, nparticles=0,
                       nthreads=0, gpu=0, ofile="", precision=None):
        """[[[x, y, z], flux], ...] at any list of points [[x, y, z], [nx, ny, nz]]
        (OSCARSSR_Python.cc:2829-3008; the normals are carried but unused by the flux)."""
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        xyz, _ = self._surface_3d(points, rotations, translation, False)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu_threads(gpu, nthreads)
        npts = len(xyz)
        out = np.zeros(npts)
        if npts:
            pts = np.ascontiguousarray(xyz.reshape(-1))
            check(lib.srs_sim_calculate_flux(self._h, dptr(pts), npts, None, float(energy_eV), int(nparticles),
                                             self._prec(precision), dptr(out), None))
        C_, V = self._point_list(xyz, out, nparticles, nthreads, gpu, pd=False)
        if ofile:
            self._write_points(ofile, C_, V, 3)
        return [[c, float(v)] for c, v in zip(C_.tolist(), V)]

    def calculate_power_density(self, points, normal=0, rotations=None, translation=None, nparticles=0, gpu=0,
                                nthreads=0, ofile="", precision=None):
        """[[[x, y, z], W/mm^2], ...] at any list of points with their normals [[x, y, z], [nx, ny, nz]]
        (OSCARSSR_Python.cc:2403-2577): normal = -1 inverts the normals, normal != 0 makes the
        calculation directional."""
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        xyz, nrm = self._surface_3d(points, rotations, translation, normal == -1)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu_threads(gpu, nthreads)
        npts = len(xyz)
        out = np.zeros(npts)
        if npts:
            pts = np.ascontiguousarray(xyz.reshape(-1))
            nrms = np.ascontiguousarray(nrm.reshape(-1))
            check(lib.srs_sim_calculate_power_density(self._h, dptr(pts), dptr(nrms), npts, None,
                                                      0 if normal == 0 else 1, int(nparticles), 1 if gpu == 1 else 0,
                                                      self._prec(precision), dptr(out), None))
        C_, V = self._point_list(xyz, out, nparticles, nthreads, gpu, pd=True)
        if ofile:
            self._write_points(ofile, C_, V, 3)
        return [[c, float(v)] for c, v in zip(C_.tolist(), V)]

    # ------------------------------------------------------------ flux
    def calculate_flux_rectangle(self, energy_eV, npoints, plane="", normal=0, dim=2, width=None, rotations=None,
                                 translation=None, x0x1x2=None, nparticles=0, polarization="", nthreads=0, gpu=0,
                                 ofile="", precision=None):
        """[[[x1, x2, 0] or [x, y, z], flux], ...] (OSCARSSR_Python.cc:3009-3233).

        List length follows the reference's dispatch (OSCARSSR.cc:2418-2489): every path first lists the
        N surface points; nthreads == 1 appends N zero entries per calculation (OSCARSSR.cc:2352-2363),
        gpu == 1 appends N zero entries with x,y,z coordinates per calculation (:2570-2572), other
        nthreads append nothing."""
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        if dim != 2 and dim != 3:
            raise ValueError("'dim' must be 2 or 3")
        xyz, x12, nrm, grid = self._rectangle(npoints, plane, width, x0x1x2, rotations, translation, normal)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu_threads(gpu, nthreads)
        prec = self._prec(precision)
        npts = len(xyz)
        out = np.zeros(npts)
        pts = np.ascontiguousarray(xyz.reshape(-1))
        check(lib.srs_sim_calculate_flux(self._h, dptr(pts), npts, C.byref(grid), float(energy_eV),
                                         int(nparticles), prec, dptr(out), None))
        nth = nthreads if nthreads >= 1 else self._nthreads_global
        calls = max(1, int(nparticles))
        coords = [self._coords(xyz, x12, dim)]
        vals = [out]
        if gpu == 1:
            coords += [xyz] * calls
            vals += [np.zeros(npts)] * calls
        elif nth == 1:
            coords += [self._coords(xyz, x12, dim)] * calls
            vals += [np.zeros(npts)] * calls
        C_ = np.concatenate(coords)
        V = np.concatenate(vals)
        if ofile:
            self._write_points(ofile, C_, V, dim)
        return [[c, float(v)] for c, v in zip(C_.tolist(), V)]

    def flux_arrays(self, energy_eV, npoints, plane="", width=None, rotations=None, translation=None, x0x1x2=None,
                    nparticles=0, precision=None, normal=0):
        """The flux on a rectangle as numpy arrays (points (N,3), values (N,)), without list building.
        A plane and width (and no x0x1x2) go to the device in one call that builds the points while
        the GPU computes."""
        if plane and (x0x1x2 is None or len(x0x1x2) == 0):
            n1, n2, w1, w2, rot, tr = sr._rect_spec(npoints, width, rotations, translation)
            if w1 > 0 and w2 > 0:
                npts = n1 * n2
                xyz, out = np.empty(3 * npts), np.zeros(npts)
                check(lib.srs_sim_calculate_flux_plane(self._h, str(plane).encode(), n1, n2, w1, w2, v3(rot), v3(tr),
                                                       int(normal), float(energy_eV), int(nparticles),
                                                       self._prec(precision), dptr(out), None, dptr(xyz), None,
                                                       None))
                return xyz.reshape(npts, 3), out
        xyz, x12, nrm, grid = self._rectangle(npoints, plane, width, x0x1x2, rotations, translation, normal)
        npts = len(xyz)
        out = np.zeros(npts)
        pts = np.ascontiguousarray(xyz.reshape(-1))
        check(lib.srs_sim_calculate_flux(self._h, dptr(pts), npts, C.byref(grid), float(energy_eV),
                                         int(nparticles), self._prec(precision), dptr(out), None))
        return xyz, out

    # ------------------------------------------------------------ power density
    def calculate_power_density_rectangle(self, npoints, plane="", width=None, x0x1x2=None, rotations=None,
                                          translation=None, ofile="", normal=0, nparticles=0, gpu=0, nthreads=0,
                                          dim=2, precision=None):
        """[[[x1, x2, 0] or [x, y, z], W/mm^2], ...] (OSCARSSR_Python.cc:2587-2807).

        List length and weighting follow the reference's dispatch (OSCARSSR.cc:1603-1677): nthreads == 1
        lists the N points once and sums particles without weight; other nthreads append N zero entries
        per calculation (OSCARSSR.cc:1804-1815), also without weight; gpu == 1 appends N zero entries
        with x,y,z coordinates per calculation and applies the 1/nparticles weight
        (src/OSCARSSR_Cuda.cu:1486-1489)."""
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        if dim != 2 and dim != 3:
            raise ValueError("'dim' must be 2 or 3")
        xyz, x12, nrm, grid = self._rectangle(npoints, plane, width, x0x1x2, rotations, translation, normal)
        if nparticles < 0:
            raise ValueError("'nparticles' must be >= 1 (sort of)")
        self._check_gpu_threads(gpu, nthreads)
        prec = self._prec(precision)
        directional = 0 if normal == 0 else 1
        npts = len(xyz)
        out = np.zeros(npts)
        pts = np.ascontiguousarray(xyz.reshape(-1))
        nrms = np.ascontiguousarray(np.tile(nrm, npts))
        check(lib.srs_sim_calculate_power_density(self._h, dptr(pts), dptr(nrms), npts, C.byref(grid), directional,
                                                  int(nparticles), 1 if gpu == 1 else 0, prec, dptr(out),
                                                  None))
        nth = nthreads if nthreads >= 1 else self._nthreads_global
        calls = max(1, int(nparticles))
        coords = [self._coords(xyz, x12, dim)]
        vals = [out]
        if gpu == 1:
            coords += [xyz] * calls
            vals += [np.zeros(npts)] * calls
        elif nth != 1:
            coords += [self._coords(xyz, x12, dim)] * calls
            vals += [np.zeros(npts)] * calls
        C_ = np.concatenate(coords)
        V = np.concatenate(vals)
        if ofile:
            self._write_points(ofile, C_, V, dim)
        return [[c, float(v)] for c, v in zip(C_.tolist(), V)]

    def power_density_arrays(self, npoints, plane="", width=None, rotations=None, translation=None, x0x1x2=None,
                             normal=0, nparticles=0, precision=None, weighted=False):
        """Power density on a rectangle as numpy arrays (points (N,3), W/mm^2 (N,))."""
        xyz, x12, nrm, grid = self._rectangle(npoints, plane, width, x0x1x2, rotations, translation, normal)
        npts = len(xyz)
        out = np.zeros(npts)
        pts = np.ascontiguousarray(xyz.reshape(-1))
        nrms = np.ascontiguousarray(np.tile(nrm, npts))
        check(lib.srs_sim_calculate_power_density(self._h, dptr(pts), dptr(nrms), npts, C.byref(grid),
                                                  0 if normal == 0 else 1, int(nparticles), int(bool(weighted)),
                                                  self._prec(precision), dptr(out), None))
        return xyz, out

    # ------------------------------------------------------------ total power
    def calculate_efield_vs_time(self, obs, ofile=""):
        """The electric field at obs in the time domain (OSCARSSR_Python.cc:3573-3640,
        OSCARSSR.cc:2646-2690): [[t, [Ex, Ey, Ez]], ...] for every trajectory point in time order; the
        arrival times are not evenly spaced.  ofile gets "Ex Ey Ez t" lines, the reference's dim-3 scalar
        format."""
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        o = _list3(obs, "obs")
        n = C.c_int64(0)
        check(lib.srs_sim_calculate_efield_time(self._h, dptr(np.array(o)), None, None, C.byref(n)))
        t, e = np.zeros(n.value), np.zeros(3 * n.value)
        check(lib.srs_sim_calculate_efield_time(self._h, dptr(np.array(o)), dptr(t), dptr(e), C.byref(n)))
        e = e.reshape(-1, 3)
        if ofile:
            with open(ofile, "w") as f:
                for ee, tt in zip(e, t):
                    f.write(f"{ee[0]:.6e} {ee[1]:.6e} {ee[2]:.6e} {tt:.6e}\n")
        return [[float(tt), [float(ee[0]), float(ee[1]), float(ee[2])]] for tt, ee in zip(t, e)]

    def calculate_total_power(self):
        """Total radiated power [W] of the current particle (OSCARSSR.cc:1939-1978)."""
        if lib.srs_sim_get_nparticle_beams(self._h) < 1:
            raise ValueError("No particle beam defined")
        out = C.c_double()
        check(lib.srs_sim_calculate_total_power(self._h, C.byref(out)))
        return out.value


def _spectrum_from_list(spectrum):
    """OSCARSSR_GetSpectrumFromList (OSCARSSR_Python.cc:2113-2143): [[E, flux], ...]."""
    rows = []
    for p in spectrum:
        if len(p) != 2:
            _bad_entry()
        rows.append((float(p[0]), float(p[1])))
    a = np.array(rows, dtype=np.float64).reshape(-1, 2)
    return a[:, 0], a[:, 1]


def _scalars_from_list(points):
    """OSCARSSR_GetT3DScalarContainerFromList (OSCARSSR_Python.cc:2151-2180): [[[x, y, z], v], ...];
    a position that is not three numbers is a length error ("number of elements not 3")."""
    xyz, vals = [], []
    for p in points:
        if len(p) != 2:
            _bad_entry()
        if len(p[0]) != 3:
            raise ValueError("number of elements not 3")
        xyz.append([float(c) for c in p[0]])
        vals.append(float(p[1]))
    return np.array(xyz, dtype=np.float64).reshape(-1, 3), np.array(vals, dtype=np.float64)


def _bad_entry():
    raise ValueError("each entry must be a list of 2 elements")


def _aggregation_methods():
    """The reference's running sums and file averages (OSCARSSR_Python.cc:3252-3572), attached to sr."""

    def add_to_spectrum(self, spectrum, weight=1):
        """Add weight * spectrum to the object's running spectrum (compensated sum)."""
        if len(spectrum) < 1:
            raise ValueError("No points in spectrum.")
        e, f = _spectrum_from_list(spectrum)
        self._spectrum_sum.add(e, f, float(weight))

    def get_spectrum(self):
        return self._spectrum_sum.as_list()

    def add_to_flux(self, flux, weight=1):
        """Add weight * flux (a map [[[x, y, z], v], ...]) to the object's running flux."""
        if len(flux) < 1:
            raise ValueError("No points in flux.")
        xyz, v = _scalars_from_list(flux)
        self._flux_sum.add(xyz, v, float(weight))

    def get_flux(self):
        return self._flux_sum.as_list()

    def add_to_power_density(self, power_density, weight=1):
        """Add weight * power_density to the object's running power density."""
        if len(power_density) < 1:
            raise ValueError("No points in flux.")  # the reference's message
        xyz, v = _scalars_from_list(power_density)
        self._pd_sum.add(xyz, v, float(weight))

    def get_power_density(self):
        return self._pd_sum.as_list()

    def average_spectra(self, ifiles=None, bifiles=None, ofile="", bofile=""):
        """The point-by-point average of spectrum files (text; binary input gives an empty result,
        as in the reference)."""
        return _agg.average_spectra(ifiles, bifiles, ofile, bofile)

    def average_flux(self, ifiles=None, bifiles=None, ofile="", bofile="", dim=2):
        """The point-by-point average of flux-map files (text or binary, dim 2 or 3)."""
        return _agg.average_scalars(ifiles, bifiles, ofile, bofile, dim)

    def average_power_density(self, ifiles=None, bifiles=None, ofile="", bofile="", dim=2):
        """The point-by-point average of power-density files (text or binary, dim 2 or 3)."""
        return _agg.average_scalars(ifiles, bifiles, ofile, bofile, dim)

    for fn in (add_to_spectrum, get_spectrum, add_to_flux, get_flux, add_to_power_density, get_power_density,
               average_spectra, average_flux, average_power_density):
        setattr(sr, fn.__name__, fn)


_aggregation_methods()


def rectangle_points(npoints, plane="", width=None, x0x1x2=None, rotations=None, translation=None, normal=0):
    """Points (N,3), in-plane coordinates (N,2), unit normal (3,) and the Grid2D of a rectangle,
    as the reference builds them (TSurfacePoints_Rectangle)."""
    return sr._rectangle(None, npoints, plane, width, x0x1x2, rotations, translation, normal)


def reset_random(seed):
    """The process-wide generator as a freshly started process has it after set_seed(seed): reseeded,
    with no cached normal value (set_seed alone keeps the cached value, as the reference's does)."""
    lib.srs_random_reset(float(seed))


def energy_grid(npoints, e0, e1):
    """The reference's spectrum energies e0 + (e1-e0)/(n-1)*(i+1) (TSpectrumContainer.cc:55-86)."""
    e = np.zeros(int(npoints))
    check(lib.srs_energy_grid(int(npoints), float(e0), float(e1), dptr(e)))
    return e


__all__ = ["sr", "rectangle_points", "energy_grid"]

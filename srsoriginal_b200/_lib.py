"""ctypes binding of libsrs_b200.so (include/srs_b200.h).

The library is built in-tree (``python -m srsoriginal_b200.build``).  There is no fallback: if the
library is missing or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsrs_b200.so")

SRS_OK, SRS_ERR_INVALID, SRS_ERR_RANGE, SRS_ERR_CUDA, SRS_ERR_NO_DEVICE, SRS_ERR_TIMEOUT, SRS_ERR_IO = range(7)
UNDULATOR, GAUSSIAN, UNIFORM_BOX, GRID = 1, 2, 3, 4
ELECTRIC = 0x100  # kind flag of an electric field
FP64, MIXED = 0, 1

_D = C.POINTER(C.c_double)
_V3 = C.c_double * 3


class Field(C.Structure):
    _fields_ = [("kind", C.c_int32), ("nperiods", C.c_int32), ("field", _V3), ("period", _V3),
                ("center", _V3), ("phase", C.c_double), ("taper", C.c_double),
                ("sigma_or_width", _V3), ("rotations", _V3), ("translation", _V3), ("start", _V3),
                ("step", _V3), ("n", C.c_int64 * 3), ("data", _D)]


class Particle(C.Structure):
    _fields_ = [("x0", _V3), ("beta0", _V3), ("qomg", C.c_double)]


class TrajView(C.Structure):
    _fields_ = [("x", _D), ("beta", _D), ("aoc", _D), ("n", C.c_int64), ("nparticles", C.c_int32),
                ("dt", C.c_double)]


class BeamConsts(C.Structure):
    _fields_ = [("charge", C.c_double), ("current", C.c_double)]


class Grid2D(C.Structure):
    _fields_ = [("origin", _V3), ("u1", _V3), ("u2", _V3), ("normal", _V3), ("n1", C.c_int32),
                ("n2", C.c_int32)]


class Job(C.Structure):
    _fields_ = [("kind", C.c_int32), ("traj", TrajView), ("beam", BeamConsts), ("grid", Grid2D),
                ("energy_ev", C.c_double), ("obs", _V3), ("d_energies", C.c_void_p), ("ne", C.c_int64),
                ("d_out", C.c_void_p)]


JOB_FLUX, JOB_SPECTRUM = 0, 1


class QueueShape(C.Structure):
    _fields_ = [("chunk", C.c_int32), ("ctas_per_sm", C.c_int32), ("energies_per_thread", C.c_int32),
                ("strip_width", C.c_int32), ("groups", C.c_int32), ("steps_per_segment", C.c_int32)]


class BeamArgs(C.Structure):
    _fields_ = [("type", C.c_char_p), ("name", C.c_char_p), ("energy_gev", C.c_double), ("d0", _V3),
                ("x0", _V3), ("sigma_energy_gev", C.c_double), ("t0", C.c_double),
                ("current", C.c_double), ("weight", C.c_double), ("rotations", _V3),
                ("translation", _V3), ("horizontal_direction", _D), ("beta", _D), ("emittance", _D),
                ("lattice_reference", _V3), ("mass", C.c_double), ("charge", C.c_double)]


class SrsError(RuntimeError):
    """A CUDA-level failure inside the library (status SRS_ERR_CUDA / SRS_ERR_TIMEOUT)."""


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build the CUDA library first (python -m srsoriginal_b200.build)")
    L = C.CDLL(LIB_PATH)
    S = C.c_int
    P = C.c_void_p
    sig = {
        "srs_last_error": (C.c_char_p, []),
        "srs_version": (C.c_char_p, []),
        "srs_device_count": (C.c_int, []),
        "srs_trim_memory": (S, []),
        "srs_trajectory_counts": (S, [C.c_double, C.c_double, C.c_double, C.c_int64, _D,
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
        "srs_trajectory": (S, [C.POINTER(Field), C.c_int32, C.POINTER(Particle), C.c_int32, C.c_double,
                               C.c_double, C.c_double, C.c_int64, P, P, P, P]),
        "srs_trajectory_shoot": (S, [C.POINTER(Field), C.c_int32, C.POINTER(Particle), C.c_double, C.c_double,
                                     C.c_double, C.c_int64, C.c_int32, C.c_int32, P, P, P, P, P]),
        "srs_spectrum": (S, [TrajView, BeamConsts, _D, P, C.c_int64, C.c_int32, P, P]),
        "srs_flux": (S, [TrajView, BeamConsts, P, C.c_int64, C.POINTER(Grid2D), C.c_double, C.c_int32,
                         P, P]),
        "srs_power_density": (S, [TrajView, BeamConsts, P, P, C.c_int64, C.POINTER(Grid2D), C.c_int32,
                                  C.c_int32, P, P]),
        "srs_total_power": (S, [TrajView, BeamConsts, _D, _D, P]),
        "srs_accumulate": (S, [P, C.c_int32, C.c_int64, C.c_double, _D, _D, P]),
        "srs_sim_create": (S, [C.POINTER(P)]),
        "srs_sim_destroy": (None, [P]),
        "srs_sim_set_ctstartstop": (S, [P, C.c_double, C.c_double]),
        "srs_sim_set_npoints_trajectory": (S, [P, C.c_int64]),
        "srs_sim_get_ctstartstop": (S, [P, _D, _D]),
        "srs_sim_get_npoints_trajectory": (C.c_int64, [P]),
        "srs_sim_set_nthreads_global": (S, [P, C.c_int32]),
        "srs_sim_set_gpu_global": (S, [P, C.c_int32]),
        "srs_sim_add_bfield_undulator": (S, [P, _D, _D, C.c_int32, C.c_double, _D, _D, C.c_double]),
        "srs_sim_add_bfield_gaussian": (S, [P, _D, _D, _D, _D]),
        "srs_sim_add_bfield_uniform": (S, [P, _D, _D, _D, _D]),
        "srs_sim_add_bfield_file": (S, [P, C.c_char_p, C.c_char_p, _D, _D, _D, C.c_int32]),
        "srs_sim_add_bfield_interpolated": (S, [P, _D, C.POINTER(C.c_char_p), C.c_int32, C.c_char_p, C.c_double,
                                                _D, _D, _D, C.c_int32]),
        "srs_read_field_file": (S, [C.c_char_p, C.c_char_p, _D, _D, _D, C.c_int32, C.POINTER(Field), _D,
                                    C.POINTER(C.c_int64)]),
        "srs_read_field_interpolated": (S, [_D, C.POINTER(C.c_char_p), C.c_int32, C.c_char_p, C.c_double, _D, _D,
                                            _D, C.c_int32, C.POINTER(Field), _D, C.POINTER(C.c_int64)]),
        "srs_sim_add_bfield_grid": (S, [P, _D, _D, C.POINTER(C.c_int64), _D, _D, _D]),
        "srs_sim_clear_bfields": (S, [P]),
        "srs_sim_clear_efields": (S, [P]),
        "srs_sim_add_efield_undulator": (S, [P, _D, _D, C.c_int32, C.c_double, _D, _D]),
        "srs_sim_add_efield_gaussian": (S, [P, _D, _D, _D, _D]),
        "srs_sim_add_efield_uniform": (S, [P, _D, _D, _D, _D]),
        "srs_sim_add_efield_file": (S, [P, C.c_char_p, C.c_char_p, _D, _D]),
        "srs_sim_get_efield": (S, [P, _D, C.c_int64, _D]),
        "srs_sim_calculate_efield_time": (S, [P, _D, _D, _D, C.POINTER(C.c_int64)]),
        "srs_sim_set_trajectory_cache": (S, [P, C.c_int32]),
        "srs_sim_set_trajectory_mode": (S, [P, C.c_int32]),
        "srs_sim_get_nfields": (C.c_int32, [P]),
        "srs_sim_get_bfield": (S, [P, _D, C.c_int64, _D]),
        "srs_sim_set_field_grid_data": (S, [P, C.c_int32, P, C.c_int32]),
        "srs_sim_add_particle_beam": (S, [P, C.POINTER(BeamArgs)]),
        "srs_sim_clear_particle_beams": (S, [P]),
        "srs_sim_get_nparticle_beams": (C.c_int32, [P]),
        "srs_sim_set_new_particle": (S, [P, C.c_char_p, C.c_char_p]),
        "srs_sim_get_particle": (S, [P, _D, _D, _D, _D]),
        "srs_set_seed": (None, [C.c_double]),
        "srs_random_uniform": (C.c_double, []),
        "srs_random_normal": (C.c_double, []),
        "srs_random_reset": (None, [C.c_double]),
        "srs_sim_calculate_trajectory": (S, [P, C.POINTER(C.c_int64), _D, _D]),
        "srs_sim_calculate_spectrum": (S, [P, _D, _D, C.c_int64, C.c_int32, C.c_int32, _D, _D]),
        "srs_sim_calculate_flux": (S, [P, _D, C.c_int64, C.POINTER(Grid2D), C.c_double, C.c_int32,
                                       C.c_int32, _D, _D]),
        "srs_sim_calculate_flux_plane": (S, [P, C.c_char_p, C.c_int32, C.c_int32, C.c_double, C.c_double, _D, _D,
                                             C.c_int32, C.c_double, C.c_int32, C.c_int32, _D, _D, _D, _D, _D]),
        "srs_sim_calculate_power_density": (S, [P, _D, _D, C.c_int64, C.POINTER(Grid2D), C.c_int32,
                                                C.c_int32, C.c_int32, C.c_int32, _D, _D]),
        "srs_sim_calculate_total_power": (S, [P, _D]),
        "srs_measure_peak": (S, [C.c_int32, _D, P]),
        "srs_flux_mixed_noalloc": (S, [TrajView, BeamConsts, C.POINTER(Grid2D), C.c_double, P, P]),
        "srs_queue_create": (S, [C.POINTER(P), C.POINTER(Job), C.c_int32, C.c_int32, C.c_int32]),
        "srs_queue_create_shaped": (S, [C.POINTER(P), C.POINTER(Job), C.c_int32, C.POINTER(QueueShape),
                                        C.POINTER(Field), C.c_int32, C.POINTER(Particle), _D, _D, _D,
                                        C.POINTER(C.c_int64)]),
        "srs_queue_run": (S, [P, P]),
        "srs_queue_info": (S, [P, C.POINTER(C.c_int64), _D, C.POINTER(C.c_size_t), C.POINTER(C.c_int32)]),
        "srs_queue_destroy": (None, [P]),
        "srs_trajectory_batch": (S, [C.POINTER(Field), C.c_int32, C.POINTER(Particle), C.c_int32, _D, _D, _D,
                                     C.POINTER(C.c_int64), C.POINTER(P), C.POINTER(P), C.POINTER(P), P]),
        "srs_spectrum_efield": (S, [TrajView, BeamConsts, _D, P, C.c_int64, C.c_int32, P, P, P]),
        "srs_spectrum_adjoint": (S, [TrajView, BeamConsts, _D, P, C.c_int64, P, P, P, P, P]),
        "srs_trajectory_adjoint": (S, [C.POINTER(Field), C.c_int32, C.POINTER(Particle), C.c_double, C.c_double,
                                       C.c_double, C.c_int64, P, P, P, P, C.POINTER(P), _D, _D, P]),
        "srs_spectrum_host": (S, [_D, _D, C.c_int64, C.c_double, BeamConsts, _D, _D, C.c_int64, C.c_int32, _D]),
        "srs_flux_host": (S, [_D, _D, C.c_int64, C.c_double, BeamConsts, _D, C.c_int64, C.c_double, _D]),
        "srs_power_density_host": (S, [_D, _D, _D, C.c_int64, C.c_double, BeamConsts, _D, _D, C.c_int64, C.c_int32,
                                       _D]),
        "srs_energy_grid": (S, [C.c_int64, C.c_double, C.c_double, _D]),
        "srs_rectangle_plane": (S, [C.c_char_p, C.c_int32, C.c_int32, C.c_double, C.c_double, _D, _D,
                                    C.c_int32, _D, _D, _D, C.POINTER(Grid2D)]),
        "srs_rectangle_points": (S, [C.c_int32, C.c_int32, _D, _D, _D, _D, _D, C.c_int32, _D, _D, _D,
                                     C.POINTER(Grid2D)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


lib = _load()
EXPORTED = (
    "srs_last_error srs_version srs_device_count srs_trim_memory srs_trajectory_counts srs_trajectory srs_trajectory_shoot srs_spectrum "
    "srs_flux srs_power_density srs_total_power srs_accumulate srs_sim_create srs_sim_destroy "
    "srs_sim_set_ctstartstop srs_sim_set_npoints_trajectory srs_sim_get_ctstartstop "
    "srs_sim_get_npoints_trajectory srs_sim_set_nthreads_global srs_sim_set_gpu_global "
    "srs_sim_add_bfield_undulator srs_sim_add_bfield_gaussian srs_sim_add_bfield_uniform "
    "srs_read_field_file srs_read_field_interpolated srs_sim_add_bfield_interpolated srs_sim_add_bfield_file srs_sim_add_bfield_grid srs_sim_clear_efields srs_sim_add_efield_undulator srs_sim_add_efield_gaussian srs_sim_add_efield_uniform srs_sim_add_efield_file srs_sim_get_efield srs_sim_calculate_efield_time srs_sim_clear_bfields srs_sim_get_nfields "
    "srs_sim_set_trajectory_cache srs_sim_set_trajectory_mode "
    "srs_sim_get_bfield srs_sim_set_field_grid_data srs_sim_add_particle_beam "
    "srs_sim_clear_particle_beams srs_sim_get_nparticle_beams srs_sim_set_new_particle "
    "srs_sim_get_particle srs_set_seed srs_random_uniform srs_random_normal srs_random_reset "
    "srs_sim_calculate_trajectory srs_sim_calculate_spectrum srs_sim_calculate_flux srs_sim_calculate_flux_plane "
    "srs_sim_calculate_power_density srs_sim_calculate_total_power srs_energy_grid "
    "srs_rectangle_plane srs_rectangle_points srs_measure_peak srs_flux_mixed_noalloc "
    "srs_queue_create srs_queue_create_shaped srs_queue_run srs_queue_info srs_queue_destroy srs_trajectory_batch "
    "srs_spectrum_efield srs_spectrum_adjoint srs_trajectory_adjoint srs_spectrum_host srs_flux_host "
    "srs_power_density_host"
).split()


def check(status):
    """Raise for a non-zero status: argument/range/IO errors as ValueError (as the reference's Python
    layer maps std::invalid_argument/out_of_range/length_error), CUDA failures as SrsError."""
    if status == SRS_OK:
        return
    msg = (lib.srs_last_error() or b"").decode(errors="replace")
    if status in (SRS_ERR_CUDA, SRS_ERR_TIMEOUT):
        raise SrsError(msg)
    raise ValueError(msg)


def v3(v):
    a = _V3()
    a[0], a[1], a[2] = float(v[0]), float(v[1]), float(v[2])
    return a


def dptr(a):
    """double* of a contiguous float64 numpy array."""
    return a.ctypes.data_as(_D)

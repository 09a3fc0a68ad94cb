"""ctypes mirror of ``include/dem_b200.h`` (the engine's C ABI).

This module only loads the shared library and declares its structures and
signatures. It never falls back to another implementation: if the library is
missing or cannot be loaded, importing :mod:`mercurydpm_fork_b200` raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdem_b200.so")

DEM_OK = 0
DEM_ERR_CAPACITY = 1
DEM_ERR_TIMEOUT = 2
DEM_ERR_NAN = 3
DEM_ERR_BAD_INPUT = 4
DEM_ERR_CUDA = 5
DEM_ERR_STATE = 6
DEM_ERR_DOMAIN = 7
STATUS_NAMES = {0: "OK", 1: "CAPACITY", 2: "TIMEOUT", 3: "NAN", 4: "BAD_INPUT", 5: "CUDA", 6: "STATE",
                7: "DOMAIN"}

DEM_NORMAL_LINEAR_VISCOELASTIC = 0
DEM_NORMAL_HERTZIAN_VISCOELASTIC = 1
DEM_FRICTION_NONE = 0
DEM_FRICTION_SLIDING = 1
DEM_FRICTION_ROLLING_TORSION = 2
DEM_FRICTION_MINDLIN = 3
DEM_FRICTION_MINDLIN_ROLLING_TORSION = 4

DEM_WALL_INFINITE = 0
DEM_WALL_AXISYMMETRIC = 1
DEM_WALL_INTERSECTION = 2
DEM_WALL_TRIANGLE = 3
DEM_MAX_TRIANGLE_CONTACTS = 8
DEM_MAX_LEVELS = 4
DEM_MAX_WALL_FACES = 8
DEM_MAX_DELETION_PER_INSTANCE = 2
DEM_MAX_INSERTION_PER_INSTANCE = 4
DEM_MAX_PSD_POINTS = 64
DEM_INSERTION_CUBE = 0
DEM_INSERTION_CHUTE = 1

DEM_CG_NFIELDS = 29
DEM_CG_O = 0
DEM_CG_XZ = 1
DEM_CG_XYZ = 2

_d = C.c_double
_i32 = C.c_int32
_i64 = C.c_int64
_u32 = C.c_uint32
_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)


class SpeciesPair(C.Structure):
    _fields_ = [
        ("normal_law", _i32), ("friction_law", _i32), ("constant_restitution", _i32), ("reserved", _i32),
        ("stiffness", _d), ("dissipation", _d), ("elastic_modulus", _d), ("shear_modulus", _d),
        ("sliding_stiffness", _d), ("sliding_dissipation", _d), ("sliding_mu", _d), ("sliding_mu_static", _d),
        ("rolling_stiffness", _d), ("rolling_dissipation", _d), ("rolling_mu", _d), ("rolling_mu_static", _d),
        ("torsion_stiffness", _d), ("torsion_dissipation", _d), ("torsion_mu", _d), ("torsion_mu_static", _d),
        ("interaction_distance", _d),
    ]


class Wall(C.Structure):
    _fields_ = [
        ("type", _i32), ("species", _i32), ("instance", _i32), ("n_faces", _i32), ("group", _i32),
        ("reserved", _i32), ("position", _d * 3), ("orientation", _d * 4), ("velocity", _d * 3), ("angular_velocity", _d * 3),
        ("faces", (_d * 6) * DEM_MAX_WALL_FACES),
    ]


class ParticlesSoA(C.Structure):
    _fields_ = [
        ("n", _i64), ("position", _pd), ("velocity", _pd), ("angular_velocity", _pd), ("orientation", _pd),
        ("radius", _pd), ("inv_mass", _pd), ("inv_inertia", _pd), ("species", _pi), ("id", _pi),
        ("instance", _pi),
    ]


class ContactsSoA(C.Structure):
    _fields_ = [
        ("n", _i64), ("id_p", _pi), ("id_i", _pi), ("is_wall", _pi), ("periodic", _pi), ("springs", _pd),
        ("force", _pd), ("overlap", _pd),
    ]


class DeletionBoundary(C.Structure):
    _fields_ = [("instance", _i32), ("reserved", _i32), ("normal", _d * 3), ("distance", _d)]


class InsertionBoundary(C.Structure):
    _fields_ = [
        ("kind", _i32), ("reserved", _i32), ("instance", _i32), ("species", _i32), ("max_failed", _i32),
        ("n_psd", _i32), ("pos_min", _d * 3), ("pos_max", _d * 3), ("vel_min", _d * 3), ("vel_max", _d * 3),
        ("density", _d), ("volume_flow_rate", _d), ("initial_volume", _d), ("fixed_particle_radius", _d),
        ("inflow_velocity", _d), ("inflow_velocity_variance", _d),
        ("psd_radius", _d * DEM_MAX_PSD_POINTS), ("psd_probability", _d * DEM_MAX_PSD_POINTS),
        ("psd_seed", C.c_uint64),
    ]


class ChuteFill(C.Structure):
    _fields_ = [
        ("instance", _i32), ("species", _i32), ("density", _d), ("x_min", _d), ("x_max", _d), ("y_min", _d),
        ("y_max", _d), ("z_min", _d), ("inflow_height", _d), ("min_radius", _d), ("max_radius", _d),
        ("fixed_particle_radius", _d),
    ]


class InstanceDesc(C.Structure):
    _fields_ = [
        ("domain_min", _d * 3), ("domain_max", _d * 3), ("gravity", _d * 3), ("periodic_mask", _u32),
        ("species_offset", _i32), ("n_species", _i32), ("reserved", _i32), ("periodic_min", _d * 3),
        ("periodic_max", _d * 3),
    ]


class Config(C.Structure):
    _fields_ = [
        ("time_step", _d), ("background_drag", _d), ("rotation", _i32), ("device", _i32),
        ("max_neighbors", _i32), ("use_graphs", _i32), ("skin", _d), ("n_instances", _i32), ("max_contacts", _i32),
    ]


class Globals(C.Structure):
    _fields_ = [
        ("kinetic_energy", _d), ("rotational_energy", _d), ("gravitational_energy", _d), ("elastic_energy", _d),
        ("momentum", _d * 3), ("angular_momentum", _d * 3), ("mass", _d), ("centre_of_mass", _d * 3),
        ("n_contacts", _i64), ("n_wall_contacts", _i64), ("time", _d), ("n_steps", _i64),
    ]


class CGGrid(C.Structure):
    _fields_ = [
        ("coordinates", _i32), ("instance", _i32), ("n", _i32 * 3), ("reserved", _i32), ("min", _d * 3),
        ("max", _d * 3), ("width", _d), ("cutoff_factor", _d),
    ]


class Tuning(C.Structure):
    _fields_ = [
        ("detect_block", _i32), ("contacts_blocks_per_sm", _i32), ("sum_block", _i32), ("reserved", _i32),
        ("ms_before", _d), ("ms_after", _d),
    ]


_SIGNATURES = {
    "dem_create": (C.c_int, [C.POINTER(Config), C.POINTER(InstanceDesc), C.POINTER(C.c_void_p)]),
    "dem_set_species": (C.c_int, [C.c_void_p, C.POINTER(SpeciesPair), C.c_int]),
    "dem_set_walls": (C.c_int, [C.c_void_p, C.POINTER(Wall), C.c_int]),
    "dem_set_periodic": (C.c_int, [C.c_void_p, C.c_int, _pd, _pd, C.c_uint32]),
    "dem_upload_particles": (C.c_int, [C.c_void_p, C.POINTER(ParticlesSoA)]),
    "dem_upload_contacts": (C.c_int, [C.c_void_p, C.POINTER(ContactsSoA)]),
    "dem_step": (C.c_int, [C.c_void_p, C.c_int]),
    "dem_download_particles": (C.c_int, [C.c_void_p, C.POINTER(ParticlesSoA)]),
    "dem_download_forces": (C.c_int, [C.c_void_p, _pd, _pd]),
    "dem_download_walls": (C.c_int, [C.c_void_p, C.POINTER(Wall), C.c_int]),
    "dem_download_contacts": (C.c_int, [C.c_void_p, C.POINTER(ContactsSoA), _i64, C.POINTER(_i64)]),
    "dem_reduce": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Globals)]),
    "dem_reduce_batch": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(Globals)]),
    "dem_batch_create": (C.c_int, [C.POINTER(Config), C.c_int, C.POINTER(InstanceDesc), C.POINTER(C.c_void_p)]),
    "dem_batch_run": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Globals)]),
    "dem_set_deletion_boundaries": (C.c_int, [C.c_void_p, C.POINTER(DeletionBoundary), C.c_int]),
    "dem_reduce_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Globals)]),
    "dem_cg_eval": (C.c_int, [C.c_void_p, C.POINTER(CGGrid), _pd]),
    "dem_last_step_stats": (C.c_int, [C.c_void_p, _pd, C.POINTER(_i64), C.POINTER(_i64)]),
    "dem_get_info": (C.c_int, [C.c_void_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "dem_get_memory": (C.c_int, [C.c_void_p, C.POINTER(_i64), C.POINTER(_i64)]),
    "dem_remove_wall": (C.c_int, [C.c_void_p, C.c_int]),
    "dem_set_insertion_boundaries": (C.c_int, [C.c_void_p, C.POINTER(InsertionBoundary), C.c_int,
                                               C.POINTER(C.c_uint64)]),
    "dem_get_insertion_counts": (C.c_int, [C.c_void_p, C.POINTER(_i64), _pd, C.c_int]),
    "dem_set_chute_fills": (C.c_int, [C.c_void_p, C.POINTER(ChuteFill), C.c_int]),
    "dem_get_chute_fill_results": (C.c_int, [C.c_void_p, _pd, C.POINTER(_i64), C.c_int]),
    "dem_rng_draws": (C.c_int, [C.c_uint64, C.c_int, _pd]),
    "dem_psd_draws": (C.c_int, [C.POINTER(InsertionBoundary), C.c_int, _pd]),
    "dem_get_counts": (C.c_int, [C.c_void_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "dem_time_force_kernel": (C.c_int, [C.c_void_p, C.c_int, _pd]),
    "dem_selftest_wait_expiry": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(C.c_uint32)]),
    "dem_download_contact_geometry": (C.c_int, [C.c_void_p, _pd, _pd, _pd, C.c_int64, C.POINTER(C.c_int64)]),
    "dem_autotune": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Tuning)]),
    "dem_set_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "dem_get_tuning": (C.c_int, [C.c_void_p, C.POINTER(Tuning)]),
    "dem_last_error": (C.c_char_p, [C.c_void_p]),
    "dem_destroy": (None, [C.c_void_p]),
}

EXPORTED = tuple(_SIGNATURES)


def load(path: str = LIB_PATH) -> C.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"libdem_b200.so not found at {path}; build it with `python -m mercurydpm_fork_b200.build` "
            "(the engine has no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib

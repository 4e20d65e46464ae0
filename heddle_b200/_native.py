"""ctypes binding of libheddle_b200.so (the C ABI of include/heddle_b200.h).

The library is the product: there is no Python or CPU fallback.  Importing
this module without a built library raises immediately; calls that need a
GPU fail with the library's own error status when none is present.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libheddle_b200.so"

HB_OK = 0
ERROR_NAMES = {
    1: "HB_ERR_INVALID_ARGUMENT",
    2: "HB_ERR_CUDA",
    3: "HB_ERR_NL_OVERFLOW",
    4: "HB_ERR_BOX_TOO_SMALL",
    5: "HB_ERR_INVALID_GRID",
    6: "HB_ERR_CONSTRAINT_SHAPE",
    7: "HB_ERR_DEVICE_TIMEOUT",
    8: "HB_ERR_UNSUPPORTED",
    9: "HB_ERR_NOT_FINITE",
}

HB_FORCES_ONLY, HB_FORCES_AND_SCALARS = 0, 1
HB_INTEGRATOR_VV, HB_INTEGRATOR_VV_LOSSLESS, HB_INTEGRATOR_LANGEVIN = 0, 1, 2
HB_CONSTRAINT_SETTLE, HB_CONSTRAINT_SHAKE = 0, 1
HB_PAIRS_FAST, HB_PAIRS_EXACT = 0, 1
HB_LAUNCH_PAIR_BLOCKS_PER_SM = 0
HB_LAUNCH_NL_SLAB = 1
HB_LAUNCH_PAIR_CHUNK = 2
HB_LAUNCH_FFT_PLANE = 3
HB_LAUNCH_GATHER_FORM = 4
HB_LAUNCH_PAIR_QUOTA = 5
HB_LAUNCH_NL_WAIT_TEST = 6

PD = C.POINTER(C.c_double)
PU32 = C.POINTER(C.c_uint32)
PI32 = C.POINTER(C.c_int32)
PU64 = C.POINTER(C.c_uint64)
PF32 = C.POINTER(C.c_float)


class SystemDesc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_uint32),
        ("positions", PD),
        ("velocities", PD),
        ("masses", PD),
        ("charges", PD),
        ("types", PU32),
        ("images", PI32),
        ("box", C.c_double * 6),
    ]


class BarostatDesc(C.Structure):
    _fields_ = [
        ("pressure", C.c_double),
        ("temperature", C.c_double),
        ("frequency", C.c_uint32),
        ("volume_step", C.c_double),
        ("seed", C.c_uint64),
        ("n_molecules", C.c_uint32),
        ("mol_offsets", PU32),
        ("mol_atoms", PU32),
    ]


class ThermostatDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("temperature", C.c_double),
        ("tau", C.c_double),
        ("collision_rate", C.c_double),
        ("seed", C.c_uint64),
        ("n_constraints", C.c_uint32),
    ]


class PcoupleDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("pressure", C.c_double),
        ("temperature", C.c_double),
        ("tau", C.c_double),
        ("compressibility", C.c_double),
        ("seed", C.c_uint64),
    ]


class MinimizerDesc(C.Structure):
    _fields_ = [
        ("initial_step", C.c_double),
        ("max_step", C.c_double),
        ("step_increase", C.c_double),
        ("step_decrease", C.c_double),
        ("force_tolerance", C.c_double),
        ("energy_tolerance", C.c_double),
        ("max_iterations", C.c_uint64),
    ]


class MinReport(C.Structure):
    _fields_ = [
        ("iteration", C.c_uint64),
        ("energy", C.c_double),
        ("max_force", C.c_double),
        ("step", C.c_double),
        ("accepted", C.c_int),
        ("converged", C.c_int),
    ]


class ForceFieldDesc(C.Structure):
    _fields_ = [
        ("lj_enabled", C.c_int),
        ("n_types", C.c_uint32),
        ("lj_sigma", PD),
        ("lj_epsilon", PD),
        ("lj_cutoff", PD),
        ("lj_switch", PD),
        ("coulomb_enabled", C.c_int),
        ("alpha", C.c_double),
        ("r_cut_coulomb", C.c_double),
        ("recip_enabled", C.c_int),
        ("grid", C.c_uint32 * 3),
        ("spline_order", C.c_uint32),
        ("excl_offsets", PU32),
        ("excl_partners", PU32),
        ("excl_lj_scale", PD),
        ("excl_coulomb_scale", PD),
        ("r_skin", C.c_double),
        ("pair_mode", C.c_int),
        ("n_bonds", C.c_uint32),
        ("bond_atoms", PU32),
        ("bond_k", PD),
        ("bond_r0", PD),
        ("n_angles", C.c_uint32),
        ("angle_atoms", PU32),
        ("angle_k", PD),
        ("angle_theta0", PD),
        ("n_dihedrals", C.c_uint32),
        ("dihedral_atoms", PU32),
        ("dihedral_k", PD),
        ("dihedral_phi0", PD),
        ("dihedral_n", PU32),
    ]


class ConstraintsDesc(C.Structure):
    _fields_ = [
        ("n_groups", C.c_uint32),
        ("group_offsets", PU32),
        ("group_atoms", PU32),
        ("group_kind", PU32),
        ("settle_ra", PD),
        ("settle_rb", PD),
        ("settle_rc", PD),
        ("con_offsets", PU32),
        ("con_i", PU32),
        ("con_j", PU32),
        ("con_dist", PD),
        ("shake_tol", C.c_double),
        ("shake_max_iter", C.c_uint32),
        ("shake_tol_relative", C.c_int),
    ]


class IntegratorDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int),
        ("dt", C.c_double),
        ("friction", C.c_double),
        ("temperature", C.c_double),
        ("seed", C.c_uint64),
        ("step0", C.c_uint64),
    ]


VP = C.c_void_p
PVP = C.POINTER(C.c_void_p)

# name -> (restype, argtypes); every entry point declared in include/heddle_b200.h
SIGNATURES = {
    "hb_last_error": (C.c_char_p, []),
    "hb_version": (C.c_char_p, []),
    "hb_context_create": (C.c_int, [C.c_int, PVP]),
    "hb_context_destroy": (C.c_int, [VP]),
    "hb_context_synchronize": (C.c_int, [VP]),
    "hb_system_create": (C.c_int, [VP, C.POINTER(SystemDesc), PVP]),
    "hb_system_destroy": (C.c_int, [VP]),
    "hb_system_set_state": (C.c_int, [VP, PD, PD]),
    "hb_system_get_state": (C.c_int, [VP, PD, PD, PI32, PD]),
    "hb_system_set_state_f32": (C.c_int, [VP, PF32, PF32]),
    "hb_system_get_state_f32": (C.c_int, [VP, PF32, PF32, PI32, PF32]),
    "hb_system_set_box": (C.c_int, [VP, PD]),
    "hb_system_get_box": (C.c_int, [VP, PD]),
    "hb_system_flip_velocities": (C.c_int, [VP]),
    "hb_forcefield_create": (C.c_int, [VP, C.POINTER(ForceFieldDesc), PVP]),
    "hb_forcefield_destroy": (C.c_int, [VP]),
    "hb_forcefield_step": (C.c_int, [VP, C.c_int]),
    "hb_forcefield_pre_step": (C.c_int, [VP, C.c_int, C.POINTER(C.c_int)]),
    "hb_forcefield_scalars": (C.c_int, [VP, PD]),
    "hb_forcefield_set_launch": (C.c_int, [VP, C.c_int, C.c_int]),
    "hb_forcefield_get_per_atom": (C.c_int, [VP, PD, PD]),
    "hb_neighbor_pairs": (C.c_int, [VP, PU32, C.c_uint64, PU64, PU64]),
    "hb_neighbor_stats": (C.c_int, [VP, PU64]),
    "hb_neighbor_capacity": (C.c_int, [VP, PU64]),
    "hb_constraints_create": (C.c_int, [VP, C.POINTER(ConstraintsDesc), PVP]),
    "hb_constraints_destroy": (C.c_int, [VP]),
    "hb_constraints_before_drift": (C.c_int, [VP]),
    "hb_constraints_after_drift": (C.c_int, [VP, C.c_double]),
    "hb_constraints_after_kick": (C.c_int, [VP, C.c_double]),
    "hb_constraints_get_virial": (C.c_int, [VP, PD]),
    "hb_constraints_shake_stats": (C.c_int, [VP, PD, C.c_int]),
    "hb_constraints_record": (C.c_int, [VP, C.c_int]),
    "hb_constraints_fuse_head": (C.c_int, [VP, C.c_int]),
    "hb_constraints_get_record": (C.c_int, [VP, PF32, PD, PD, PD, PU32]),
    "hb_constraints_set_warm_start": (C.c_int, [VP, VP]),
    "hb_shake_mlp_create": (C.c_int, [VP, C.c_uint64, PVP]),
    "hb_shake_mlp_destroy": (C.c_int, [VP]),
    "hb_shake_mlp_param_count": (C.c_uint32, []),
    "hb_shake_mlp_get_params": (C.c_int, [VP, PF32, C.c_uint32]),
    "hb_shake_mlp_set_params": (C.c_int, [VP, PF32, C.c_uint32]),
    "hb_shake_mlp_set_normalization": (C.c_int, [VP, PF32, PF32, C.c_float]),
    "hb_shake_mlp_predict": (C.c_int, [VP, PF32, C.c_uint64, PF32]),
    "hb_shake_mlp_set_wait_limit": (C.c_int, [VP, C.c_uint32, C.c_int]),
    "hb_shake_mlp_gradients": (C.c_int, [VP, PF32, PF32, C.c_uint32, PF32, PD]),
    "hb_shake_mlp_train": (C.c_int, [VP, PF32, PF32, C.c_uint64, C.c_uint32, C.c_uint32,
                                     C.c_double, C.c_uint64, PD]),
    "hb_integrator_create": (C.c_int, [VP, C.POINTER(IntegratorDesc), PVP]),
    "hb_integrator_destroy": (C.c_int, [VP]),
    "hb_integrator_step": (C.c_int, [VP, VP, VP, C.c_uint32, C.c_uint32]),
    "hb_integrator_step_graph": (C.c_int, [VP, VP, VP, C.c_uint32]),
    "hb_integrator_step_exchange_f32": (C.c_int, [VP, VP, VP, C.c_uint32, PF32, PF32, PF32, PF32,
                                                   PI32, PF32]),
    "hb_integrator_count_launches": (C.c_int, [VP, VP, VP, PU64]),
    "hb_barostat_create": (C.c_int, [VP, C.POINTER(BarostatDesc), PVP]),
    "hb_barostat_destroy": (C.c_int, [VP]),
    "hb_barostat_mc_move": (C.c_int, [VP, VP]),
    "hb_barostat_stats": (C.c_int, [VP, PD]),
    "hb_integrator_set_barostat": (C.c_int, [VP, VP]),
    "hb_thermostat_create": (C.c_int, [VP, C.POINTER(ThermostatDesc), PVP]),
    "hb_thermostat_destroy": (C.c_int, [VP]),
    "hb_thermostat_stats": (C.c_int, [VP, PD]),
    "hb_integrator_set_thermostat": (C.c_int, [VP, VP]),
    "hb_pcouple_create": (C.c_int, [VP, C.POINTER(PcoupleDesc), PVP]),
    "hb_pcouple_destroy": (C.c_int, [VP]),
    "hb_pcouple_stats": (C.c_int, [VP, PD]),
    "hb_integrator_set_pcouple": (C.c_int, [VP, VP]),
    "hb_minimizer_create": (C.c_int, [VP, VP, C.POINTER(MinimizerDesc), PVP]),
    "hb_minimizer_destroy": (C.c_int, [VP]),
    "hb_minimizer_begin": (C.c_int, [VP, C.POINTER(MinReport)]),
    "hb_minimizer_iterate": (C.c_int, [VP, C.c_uint32, C.POINTER(MinReport), C.POINTER(C.c_uint32)]),
    "hb_batch_create": (C.c_int, [VP, C.c_uint32, PVP, PVP, PVP, PVP]),
    "hb_batch_destroy": (C.c_int, [VP]),
    "hb_batch_step": (C.c_int, [VP, C.c_uint32]),
    "hb_batch_count_launches": (C.c_int, [VP, PU64]),
    "hb_batch_set_pair_form": (C.c_int, [VP, C.c_int]),
    "hb_batch_pair_form": (C.c_int, [VP, C.POINTER(C.c_int)]),
    "hb_reduce_kinetic": (C.c_int, [VP, PD]),
    "hb_spme_recip_noalloc": (C.c_int, [C.c_void_p, C.c_uint32, PD, PU32, C.c_uint32, C.c_double,
                                        C.c_void_p, PD, C.c_void_p]),
    "hb_timing_enable": (C.c_int, [VP, C.c_int]),
    "hb_timing_get": (C.c_int, [VP, PD]),
}


class HeddleError(RuntimeError):
    """A failing C-ABI call: .code is the HB_ERR_* status, .name its name."""

    def __init__(self, code: int, message: str):
        self.code = code
        self.name = ERROR_NAMES.get(code, f"HB_ERR_{code}")
        super().__init__(f"{self.name}: {message}")


_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (built by heddle_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m heddle_b200.build` "
            "(the force path has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != HB_OK:
        msg = load().hb_last_error().decode(errors="replace")
        raise HeddleError(rc, msg)


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(PD)


def u32ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(PU32)


def f32ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(PF32)


def i32ptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(PI32)

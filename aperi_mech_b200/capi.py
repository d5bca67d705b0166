"""ctypes binding of the C ABI in include/aperi_b200.h (libaperi_b200.so).

The shared library is the product: there is no Python or CPU fallback. Loading
fails loudly when the library is missing or a CUDA device is unavailable.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import build as _build

AM_OK, AM_EINVAL, AM_ENOMEM, AM_ECUDA, AM_ENONPOS_J, AM_ENAN, AM_ESTATE, AM_ERANGE = range(8)
AM_FP64, AM_MIXED = 0, 1
AM_HOST, AM_DEVICE = 0, 1
AM_TET4_GAUSS, AM_HEX8_GAUSS, AM_SMOOTHED_CELLS = 0, 1, 2
AM_LINEAR_ELASTIC, AM_NEO_HOOKEAN, AM_ELASTIC_SVK = 0, 1, 2
AM_BC_DISPLACEMENT, AM_BC_VELOCITY = 0, 1
AM_TF_RAMP, AM_TF_SMOOTH_STEP = 0, 1
AM_MAX_BCS = 10

EXPORTED = [
    "am_create", "am_destroy", "am_set_stream", "am_add_block", "am_set_boundary_conditions",
    "am_set_body_acceleration", "am_set_mass", "am_finalize", "am_set_state", "am_get_state", "am_get_mass",
    "am_internal_force", "am_init_acceleration", "am_run", "am_run_schedule", "am_solve", "am_vjp_force",
    "am_adjoint", "am_stress", "am_quadrature", "am_last_error", "am_status_string", "am_launch_count",
    "am_profile_enable", "am_profile_read", "am_complete_properties", "am_set_block_fields",
    "am_tet4_internal_force_noalloc", "am_rkpm_nodal_cells", "am_cells_sizes", "am_cells_get",
    "am_cells_get_points", "am_cells_destroy", "am_get_layout", "am_rkpm_element_cells", "am_set_power_method",
    "am_stable_time_increment", "am_solve_power_method", "am_set_interface", "am_nccl_unique_id",
    "am_set_nccl", "am_set_rk_functions", "am_set_cell_groups", "am_rkpm_nodal_subcells", "am_cells_groups",
    "am_set_formulation", "am_rkpm_hex8_element_cells", "am_noalloc_status",
    "am_measure_fma_peak", "am_element_order", "am_smoothed_element_cells", "am_set_neighbors",
    "am_rkpm_nodal_cells_two_pass", "am_set_rk_points",
]

# Tets per call of am_tet4_internal_force_noalloc (AM_NOALLOC_MAX_TETS in include/aperi_b200.h).
AM_NOALLOC_MAX_TETS = 174762

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class BlockDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("material", C.c_int32),
        ("lam", C.c_double), ("mu", C.c_double), ("density", C.c_double),
        ("mu_field", _dp), ("kappa_field", _dp), ("num_elems", C.c_int64),
        ("conn", _ip), ("cell_ptr", _lp), ("cell_nodes", _ip), ("cell_grads", _dp), ("cell_volumes", _dp),
    ]


class BCDesc(C.Structure):
    _fields_ = [
        ("num_nodes", C.c_int64), ("nodes", _ip), ("component_mask", C.c_int32), ("kind", C.c_int32),
        ("time_function", C.c_int32), ("num_points", C.c_int32), ("values", C.c_double * 3),
        ("abscissa", _dp), ("ordinate", _dp), ("active_start", C.c_double), ("active_end", C.c_double),
    ]


class AmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_LIB = None


def library_path() -> Path:
    return _build.LIB


def load(build_if_missing: bool = False) -> C.CDLL:
    """Load libaperi_b200.so (building it first only when asked)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not path.exists():
        if not build_if_missing:
            raise FileNotFoundError(f"{path} is missing: run `python -m aperi_mech_b200.build`")
        _build.build()
    lib = C.CDLL(str(path))
    vp = C.c_void_p
    sig = {
        "am_create": (C.c_int, [C.c_int64, _dp, C.POINTER(vp)]),
        "am_destroy": (None, [vp]),
        "am_set_stream": (C.c_int, [vp, vp]),
        "am_add_block": (C.c_int, [vp, C.POINTER(BlockDesc), _ip]),
        "am_set_boundary_conditions": (C.c_int, [vp, C.c_int32, C.POINTER(BCDesc)]),
        "am_set_body_acceleration": (C.c_int, [vp, _dp]),
        "am_set_mass": (C.c_int, [vp, _dp]),
        "am_finalize": (C.c_int, [vp]),
        "am_set_state": (C.c_int, [vp, C.c_int, vp, vp, vp]),
        "am_get_state": (C.c_int, [vp, C.c_int, vp, vp, vp]),
        "am_get_mass": (C.c_int, [vp, _dp]),
        "am_internal_force": (C.c_int, [vp, C.c_int, C.c_int, vp, vp, C.c_int]),
        "am_init_acceleration": (C.c_int, [vp, C.c_int]),
        "am_run": (C.c_int, [vp, C.c_int, C.c_int64, C.c_double, C.c_double]),
        "am_run_schedule": (C.c_int, [vp, C.c_int, C.c_int64, _dp, C.c_double]),
        "am_solve": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_int64, _lp]),
        "am_vjp_force": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp]),
        "am_adjoint": (C.c_int, [vp, C.c_int64, C.c_double, C.c_int32, C.c_int32, _ip, _dp, _dp, _dp]),
        "am_stress": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_int64, C.c_int, vp, vp]),
        "am_quadrature": (C.c_int, [C.c_int32, C.c_int32, C.c_int64, C.c_int, vp, vp, vp]),
        "am_last_error": (C.c_char_p, [vp]),
        "am_status_string": (C.c_char_p, [C.c_int]),
        "am_launch_count": (C.c_int64, [vp]),
        "am_profile_enable": (C.c_int, [vp, C.c_int]),
        "am_profile_read": (C.c_int, [vp, _dp, _lp]),
        "am_complete_properties": (C.c_int, [_dp, C.c_char_p, C.c_int]),
        "am_set_block_fields": (C.c_int, [vp, C.c_int32, _dp, _dp]),
        "am_tet4_internal_force_noalloc": (C.c_int, [C.c_int32, C.c_double, C.c_double, C.c_int64, C.c_int64, vp, vp,
                                                    vp, vp, vp, vp, vp]),
        "am_rkpm_nodal_cells": (C.c_int, [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, C.POINTER(vp)]),
        "am_rkpm_element_cells": (C.c_int, [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double, C.POINTER(vp)]),
        "am_cells_sizes": (C.c_int, [vp, _lp, _lp, _lp, _lp]),
        "am_cells_get": (C.c_int, [vp, _lp, _ip, _dp, _dp, _dp]),
        "am_cells_get_points": (C.c_int, [vp, _dp, _lp, _ip, _dp]),
        "am_cells_destroy": (None, [vp]),
        "am_get_layout": (C.c_int, [vp, _lp, _ip]),
        "am_set_interface": (C.c_int, [vp, C.c_int64, _ip, _ip, C.c_int64]),
        "am_set_power_method": (C.c_int, [vp, _dp, _dp]),
        "am_stable_time_increment": (C.c_int, [vp, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double, _dp, _ip,
                                               _ip]),
        "am_solve_power_method": (C.c_int, [vp, C.c_int, C.c_double, C.c_int64, C.c_double, C.c_int64, _lp, _dp]),
        "am_nccl_unique_id": (C.c_int, [C.c_char_p]),
        "am_set_nccl": (C.c_int, [vp, C.c_char_p, C.c_int32, C.c_int32]),
        "am_set_rk_functions": (C.c_int, [vp, _lp, _ip, _dp]),
        "am_set_cell_groups": (C.c_int, [vp, C.c_int32, C.c_int64, _lp]),
        "am_rkpm_nodal_subcells": (C.c_int, [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double,
                                             C.POINTER(vp)]),
        "am_cells_groups": (C.c_int, [vp, _lp, _lp]),
        "am_set_formulation": (C.c_int, [vp, C.c_int32, C.c_int32]),
        "am_rkpm_hex8_element_cells": (C.c_int, [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double,
                                                 C.POINTER(vp)]),
        "am_noalloc_status": (C.c_int, [vp, _ip, _lp]),
        "am_measure_fma_peak": (C.c_int, [C.c_int32, vp, _dp]),
        "am_element_order": (C.c_int, [C.c_int64, _dp, C.c_int64, C.c_int32, _ip, C.c_int32, _ip, _ip]),
        "am_smoothed_element_cells": (C.c_int, [C.c_int64, _dp, C.c_int64, C.c_int32, _ip, C.c_double,
                                                C.POINTER(vp)]),
        "am_set_neighbors": (C.c_int, [vp, C.c_int32, C.c_int32, _ip, _lp, _ip]),
        "am_rkpm_nodal_cells_two_pass": (C.c_int, [C.c_int64, _dp, C.c_int64, _ip, _dp, C.c_int32, C.c_double,
                                                   C.POINTER(vp)]),
        "am_set_rk_points": (C.c_int, [vp, C.c_int64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _ptr(a: np.ndarray | None, ctype=C.c_double):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))


def _vp(a) -> int | None:
    """Host numpy array or torch tensor -> raw address."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


def check(rc: int, ctx=None) -> None:
    if rc != AM_OK:
        lib = load()
        msg = lib.am_last_error(ctx).decode() if lib.am_last_error(ctx) else ""
        raise AmError(rc, f"{lib.am_status_string(rc).decode()}: {msg}")


def stress(material: int, lam: float, mu: float, H: np.ndarray) -> np.ndarray:
    """Material::StressFunctor::GetStress on a batch of displacement gradients (GPU)."""
    lib = load()
    H = np.ascontiguousarray(H, dtype=np.float64).reshape(-1, 9)
    P = np.empty_like(H)
    check(lib.am_stress(material, lam, mu, H.shape[0], AM_HOST, H.ctypes.data, P.ctypes.data))
    return P.reshape(-1, 3, 3)


def quadrature(kind: int, X: np.ndarray, smoothed: bool = False):
    """Quadrature::ComputeBMatrixAndWeight (or the smoothed quadrature) on a batch of elements (GPU)."""
    lib = load()
    nn = 8 if kind == AM_HEX8_GAUSS else 4
    npnt = 1 if (smoothed or kind == AM_TET4_GAUSS) else 8
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, nn, 3)
    n = X.shape[0]
    B = np.empty((n, npnt, nn, 3))
    w = np.empty((n, npnt))
    check(lib.am_quadrature(kind, int(smoothed), n, AM_HOST, X.ctypes.data, B.ctypes.data, w.ctypes.data))
    return B, w

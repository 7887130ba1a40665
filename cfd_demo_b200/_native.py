"""ctypes binding of ``libcfd_b200.so`` (the C ABI declared in include/cfd_b200.h).

The library is built in-tree by ``cfd_demo_b200.build``. Loading fails loudly
when it is missing: the package has no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os

from . import build as _build

LIB_PATH = _build.LIB

CFD_FP64 = 0
CFD_FP32_MIXED = 1
FACE_INTERIOR, FACE_SLIP_WALL, FACE_FIXED_STATE = 0, 1, 2
RUN_ACTIVE, RUN_DONE, RUN_BAD_DT, RUN_REJECTED = 0, 1, -1, -2
NOALLOC_MAX_ELEMENTS = 16384  # CFD_NOALLOC_MAX_ELEMENTS of include/cfd_b200.h
ADJ_HOLD_THETA = 1  # CFD_ADJ_HOLD_THETA
LIMIT_LIST_HEADER = 16  # CFD_LIMIT_LIST_HEADER
ABI_VERSION = 2  # CFD_ABI_VERSION

_p = C.c_void_p
_i32 = C.c_int32
_f64 = C.c_double


class CfdMesh(C.Structure):
    _fields_ = [
        ("num_elements", _i32), ("ld", _i32), ("num_instances", _i32), ("flags", _i32),
        ("metric", _p), ("face_geo", _p), ("face_hlen", _p), ("dt_geo", _p), ("jacobian", _p), ("cs_coef", _p),
        ("neighbor", _p), ("face_info", _p), ("instance", _p), ("bc_states", _p),
        ("metric32", _p), ("face_geo32", _p), ("cs_coef32", _p),
    ]


class CfdMeshBuild(C.Structure):
    _fields_ = [
        ("num_vertices", _i32), ("num_elements", _i32), ("ld", _i32), ("num_boundary_edges", _i32),
        ("num_tags", _i32), ("reserved", _i32), ("vertices", _p), ("elements", _p), ("boundary_edges", _p),
        ("boundary_tag", _p), ("tag_kind", _p), ("tag_row", _p),
    ]


class CfdStageAcc(C.Structure):
    _fields_ = [("boundary_flux", _f64 * 4), ("min_rho_key", C.c_uint64), ("min_p_key", C.c_uint64),
                ("dt_key", C.c_uint64), ("troubled", _i32), ("flags", _i32)]


class CfdStepReport(C.Structure):
    _fields_ = [("boundary_flux", _f64 * 4), ("min_density", _f64), ("min_pressure", _f64), ("dt", _f64),
                ("dt_next", _f64), ("admissible", _i32), ("troubled_cells", _i32), ("reserved", _i32 * 2)]


class CfdControl(C.Structure):
    _fields_ = [("time", _f64), ("final_time", _f64), ("dt", _f64), ("flux_integral", _f64 * 4),
                ("min_density", _f64), ("min_pressure", _f64), ("steps", _i32), ("rejected", _i32),
                ("attempts", _i32), ("max_troubled", _i32), ("parity", _i32), ("status", _i32),
                ("reaches_end", _i32), ("reserved", _i32)]


class CfdSolver(C.Structure):
    _fields_ = [("mesh", CfdMesh), ("flux", _i32), ("limiter", _i32), ("precision", _i32), ("max_rejections", _i32),
                ("gamma", _f64), ("cfl", _f64), ("averages", _p), ("element_aux", _p), ("acc", _p),
                ("report", _p), ("control", _p), ("block_size", _i32), ("variant", _i32), ("limit_list", _p),
                ("troubled_flags", _p)]


SIZES = {"CfdMesh": C.sizeof(CfdMesh), "CfdStageAcc": C.sizeof(CfdStageAcc),
         "CfdStepReport": C.sizeof(CfdStepReport), "CfdControl": C.sizeof(CfdControl), "CfdSolver": C.sizeof(CfdSolver)}

_SP = C.POINTER(CfdSolver)
_PROTOS = {
    "cfd_abi_version": (C.c_int, []),
    "cfd_last_error": (C.c_char_p, []),
    "cfd_struct_sizes": (C.c_int, [_p, _i32]),
    "cfd_pack_state": (C.c_int, [_p, _p, _i32, _i32, _i32, _p]),
    "cfd_unpack_state": (C.c_int, [_p, _p, _i32, _i32, _i32, _p]),
    "cfd_rhs": (C.c_int, [_SP, _p, _p, _p, _p]),
    "cfd_limit": (C.c_int, [_SP, _p, _p, _p, _p]),
    "cfd_time_step": (C.c_int, [_SP, _p, _p, _p]),
    "cfd_cell_averages": (C.c_int, [_SP, _p, _p, _p]),
    "cfd_integrate": (C.c_int, [_SP, _p, _p, _p]),
    "cfd_check_state": (C.c_int, [_SP, _p, _p, _p]),
    "cfd_rk3_attempt": (C.c_int, [_SP, _p, _p, _p, _p]),
    "cfd_rk3_begin": (C.c_int, [_SP, _p]),
    "cfd_rk3_stage": (C.c_int, [_SP, _p, _p, _p, _i32, _p]),
    "cfd_rk3_finish": (C.c_int, [_SP, _p]),
    "cfd_run_control": (C.c_int, [_SP, _p]),
    "cfd_run_init": (C.c_int, [_SP, _p, _p, _p]),
    "cfd_batch_advance": (C.c_int, [_SP, _p, _p, _p, _i32, _p]),
    "cfd_rk3_step_noalloc": (C.c_int, [C.POINTER(CfdMesh), _i32, _i32, _i32, _f64, _f64, _p, _p, _f64, _p, _p]),
    "cfd_tape_bytes": (C.c_int64, [_i32, _i32]),
    "cfd_adjoint_work_bytes": (C.c_int64, [_i32, _i32]),
    "cfd_rk3_step_fixed": (C.c_int, [_SP, _p, _p, _p, _p, _p, _p]),
    "cfd_rk3_step_adjoint": (C.c_int, [_SP, _p, _p, _p, _p, _p, _p, _i32, _p, _p]),
    "cfd_mesh_build_work_bytes": (C.c_int64, [_i32, _i32]),
    "cfd_mesh_build": (C.c_int, [C.POINTER(CfdMeshBuild), C.POINTER(CfdMesh), _p, _f64, _p, C.c_int64, _p, _p]),
    "cfd_interface_flux": (C.c_int, [_i32, _i32, _p, _p, _p, _p, _f64, _p, _p]),
    "cfd_limiter_phi": (C.c_int, [_i32, _i32, _p, _p, _p]),
}

_lib = None


def exported_symbols() -> list[str]:
    return list(_PROTOS)


def load(path: str | None = None):
    """Load (once) and return the library with prototypes attached."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} is missing: build the CUDA library first (python -m cfd_demo_b200.build). "
            "cfd_demo_b200 has no CPU fallback.")
    lib = C.CDLL(path)
    for name, (res, args) in _PROTOS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.cfd_abi_version() != ABI_VERSION:
        raise RuntimeError("libcfd_b200.so ABI version mismatch; rebuild it.")
    if path == LIB_PATH:
        _lib = lib
    return lib


class NativeError(RuntimeError):
    pass


def check(rc: int) -> None:
    if rc != 0:
        msg = load().cfd_last_error().decode(errors="replace")
        raise NativeError(f"libcfd_b200 error {rc}: {msg}")

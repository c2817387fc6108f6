"""ctypes binding of libtmb.so (declarations of include/tmb.h).

The library must have been built (``python -m tetmag_b200.build``); loading
fails loudly otherwise -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libtmb.so"

TMB_OK, TMB_ERR_ARG, TMB_ERR_CUDA, TMB_ERR_NOCONVERGE, TMB_ERR_STATE, TMB_ERR_NAN, TMB_ERR_STEP, TMB_ERR_INTERNAL = range(8)
TMB_FP64, TMB_MIXED = 0, 1
TMB_PTR_HOST, TMB_PTR_DEVICE = 0, 1

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_L = C.POINTER(C.c_longlong)
_int, _dbl = C.c_int, C.c_double

# name -> argument types (all return int except tmb_last_error)
SIGNATURES = {
    "tmb_version": [],
    "tmb_kernel_launches": [_L],
    "tmb_mesh_create": [_int, _int, _D, _I, C.POINTER(_P)],
    "tmb_mesh_destroy": [_P],
    "tmb_mesh_info": [_P, _L],
    "tmb_mesh_get_operators": [_P, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D],
    "tmb_mesh_get_boundary": [_P, _I, _I, _D, _D, _D, _D, _D],
    "tmb_ctx_create": [_int, C.POINTER(_P)],
    "tmb_ctx_destroy": [_P],
    "tmb_ctx_set_stream": [_P, _P],
    "tmb_set_precision": [_P, _int],
    "tmb_set_mesh": [_P, _P],
    "tmb_set_operators": [_P, _int, _int, _I, _I, _D, _D, _D, _D, _D, _D, _D, _D, _int, _I, _D, _D],
    "tmb_bem_assemble": [_P, _P],
    "tmb_bem_assemble_ex": [_P, _P, _int],
    "tmb_set_bem_dense": [_P, _int, _D],
    "tmb_set_components": [_P, _int, _I, _int],
    "tmb_set_replicas": [_P, _int],
    "tmb_set_bem_gemm_kind": [_P, _int],
    "tmb_bem_gemm_info": [_P, _D],
    "tmb_get_bem_dense": [_P, _D],
    "tmb_bem_compress": [_P, _D, _D, _int, _dbl, _dbl, _dbl, _int, _int],
    "tmb_bem_build_h": [_P, _P, _int, _dbl, _dbl, _dbl, _int],
    "tmb_set_bem_accuracy": [_P, _dbl],
    "tmb_set_bem_mode": [_P, _int],
    "tmb_bem_h2": [_P, _dbl, _dbl, _int],
    "tmb_bem_h2_info": [_P, _D],
    "tmb_bem_info": [_P, _D],
    "tmb_bem_verify": [_P, _D, _D],
    "tmb_bem_apply": [_P, _P, _P, _int, _int],
    "tmb_set_material": [_P, _D, _D, _D, _D, _D, _dbl],
    "tmb_set_dmi_kind": [_P, _int],
    "tmb_set_applied_field": [_P, _P, _int],
    "tmb_set_llg_options": [_P, _int],
    "tmb_set_solver_params": [_P, _dbl, _int],
    "tmb_demag_field": [_P, _P, _P, _int],
    "tmb_set_demag_frozen": [_P, _P, _int],
    "tmb_field_eval": [_P, _P, _P, _P, _int],
    "tmb_effective_field": [_P, _P, _P, _int],
    "tmb_llg_rhs": [_P, _dbl, _P, _P, _int],
    "tmb_llg_rhs_noalloc": [_P, _dbl, _D, _D],
    "tmb_max_torque": [_P, _P, _D, _int],
    "tmb_normalize": [_P, _P, _int],
    "tmb_relax": [_P, _P, _dbl, _dbl, _dbl, _dbl, _D, _int],
    "tmb_energies": [_P, _P, _D, _int],
    "tmb_write_vtu": [C.c_char_p, _int, _D, _int, _I, _D, _I, _dbl, _D, C.c_char_p, _int],
    "tmb_read_magnetization": [C.c_char_p, _int, _D, _D],
    "tmb_log_header": [C.c_char_p, C.c_char_p, C.c_char_p, C.c_char_p, _int],
    "tmb_log_row": [_P, _P, _int, _dbl, _dbl, C.c_char_p, _int],
    "tmb_log_format": [_dbl, _D, _dbl, _D, _D, C.c_char_p, _int],
    "tmb_set_cubic_anisotropy": [_P, _D, _D, _D],
    "tmb_set_surface_anisotropy": [_P, _D],
    "tmb_set_stt": [_P, _D, _dbl, _dbl],
    "tmb_set_bz_pulse": [_P, _int, _D, _dbl, _dbl],
    "tmb_step_rk4": [_P, _P, _int, _dbl, _int, _dbl, _int, _D, _int],
    "tmb_adjoint_rk4": [_P, _P, _int, _dbl, _int, _int, _dbl, _int, _P, _P, _P, _P, _D, _D, _D, _int],
    "tmb_get_stats": [_P, _D],
    "tmb_profile_enable": [_P, _int],
    "tmb_profile_read": [_P, _D],
    "tmb_solver_create": [_P, C.POINTER(_P)],
    "tmb_solver_destroy": [_P],
    "tmb_solver_set_matrix": [_P, _int, _int, _I, _I, _D],
    "tmb_solver_set_tolerance": [_P, _dbl, _int],
    "tmb_solver_compute": [_P],
    "tmb_solver_solve": [_P, _P, _P, _int],
    "tmb_solver_info": [_P, _D],
}

_lib = None


class TmbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[tmb error {code}] {msg}")
        self.code = code


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m tetmag_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, argtypes in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = argtypes
            f.restype = C.c_int
        L.tmb_last_error.argtypes = []
        L.tmb_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(code: int) -> int:
    if code != TMB_OK:
        raise TmbError(code, lib().tmb_last_error().decode(errors="replace"))
    return code

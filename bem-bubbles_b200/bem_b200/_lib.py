"""ctypes binding of libbem_b200.so (the C ABI declared in include/bem_b200.h).

The library is built in-tree (``make -C bem-bubbles_b200``); loading fails loudly when it is
missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_ROOT, "libbem_b200.so")

BEM_OK = 0
BEM_ERR_ARG = 1
BEM_ERR_CUDA = 2
BEM_ERR_NEGATIVE_X = 3
BEM_ERR_SINGULAR = 4
BEM_ERR_NOT_CONVERGED = 5
BEM_ERR_NOMEM = 6
BEM_ERR_STATE = 7

SOLVER_BICGSTAB = 0
SOLVER_LU = 1
SOLVER_MIXED = 2
FLAG_BICGSTAB_MULTIKERNEL = 1
FLAG_NO_STAGE_PREDICTOR = 2
FLAG_STEP_ASSEMBLE_H = 4
FLAG_REFINE_PERSISTENT = 8
FLAG_INVERSE_GJ = 16
FLAG_INVERSE_NS = 32
FLAG_NO_IR_GATE = 64

_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)


class Params(C.Structure):
    """bem_params (include/bem_b200.h)."""
    _fields_ = [("p_inf", C.c_double), ("epsilon", C.c_double), ("sigma", C.c_double), ("gamma", C.c_double),
                ("field_amp", C.c_double), ("field_kx", C.c_double), ("field_omega", C.c_double),
                ("field_phase", C.c_double), ("min_dt", C.c_double), ("dp_balance", C.c_double),
                ("nopen_eps", C.c_double), ("mirror", C.c_int32), ("solver", C.c_int32),
                ("mixed_tol", C.c_double), ("max_iters", C.c_int32), ("flags", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("solves", C.c_int64), ("last_iters", C.c_int32), ("precond_refresh", C.c_int32),
                ("last_rel_residual", C.c_double), ("ns_steps", C.c_int64), ("gmres_fallbacks", C.c_int64),
                ("fp64_fallbacks", C.c_int64),
                ("total_iters", C.c_int64), ("wait_expired", C.c_int64), ("gj_inverses", C.c_int64),
                ("ir_rounds", C.c_int64)]


class Profile(C.Structure):
    _fields_ = [("assemble_ms", C.c_double), ("assemble_launches", C.c_int64), ("solve_ms", C.c_double),
                ("solve_calls", C.c_int64), ("kernel_launches", C.c_int64)]


FIELD_FN = C.CFUNCTYPE(C.c_double, C.POINTER(C.c_double), C.c_double, C.c_void_p)

# name -> (restype, argtypes)
SIGNATURES = {
    "bem_default_params": (None, [C.POINTER(Params)]),
    "bem_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(Params)]),
    "bem_destroy": (C.c_int, [C.c_void_p]),
    "bem_last_error": (C.c_char_p, [C.c_void_p]),
    "bem_set_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "bem_get_params": (C.c_int, [C.c_void_p, C.POINTER(Params)]),
    "bem_set_mesh": (C.c_int, [C.c_void_p, C.c_int64, _D, C.c_int64, _I64]),
    "bem_num_verts": (C.c_int, [C.c_void_p, _I64]),
    "bem_set_vertices": (C.c_int, [C.c_void_p, _D]),
    "bem_get_vertices": (C.c_int, [C.c_void_p, _D]),
    "bem_set_phi": (C.c_int, [C.c_void_p, _D]),
    "bem_get_phi": (C.c_int, [C.c_void_p, _D]),
    "bem_set_psi": (C.c_int, [C.c_void_p, _D]),
    "bem_get_psi": (C.c_int, [C.c_void_p, _D]),
    "bem_set_time": (C.c_int, [C.c_void_p, C.c_double]),
    "bem_get_time": (C.c_int, [C.c_void_p, _D]),
    "bem_set_V0": (C.c_int, [C.c_void_p, C.c_double]),
    "bem_get_V0": (C.c_int, [C.c_void_p, _D]),
    "bem_get_volume": (C.c_int, [C.c_void_p, _D]),
    "bem_set_field_callback": (C.c_int, [C.c_void_p, FIELD_FN, C.c_void_p]),
    "bem_assemble": (C.c_int, [C.c_void_p, _D, _D, _D]),
    "bem_assemble_rhs": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "bem_solve_system": (C.c_int, [C.c_void_p, _D, _D, _D]),
    "bem_position_t": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "bem_position_t_inout": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "bem_set_state": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "bem_get_state": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "bem_set_pinned": (C.c_int, [C.c_void_p, C.c_int64, C.c_double, C.c_double, C.c_double]),
    "bem_get_pinned": (C.c_int, [C.c_void_p, _I64]),
    "bem_trace_mesh": (C.c_int, [C.c_void_p, C.c_int64, _D, C.c_int64, _I64, C.c_int64, _D, _D, _D, _I64,
                                 C.POINTER(C.c_int32)]),
    "bem_pot_t_multi": (C.c_int, [C.c_void_p, _D, _D, C.c_double, _D]),
    "bem_evolve_rk4": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, _D]),
    "bem_evolve_euler": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, _D]),
    "bem_evolve_rk4_n": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "bem_get_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "bem_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int64]),
    "bem_sync": (C.c_int, [C.c_void_p]),
    "bem_set_profiling": (C.c_int, [C.c_void_p, C.c_int32]),
    "bem_get_profile": (C.c_int, [C.c_void_p, C.POINTER(Profile)]),
    "bem_reset_profile": (C.c_int, [C.c_void_p]),
    "bem_measure_fma_peaks": (C.c_int, [C.c_int, _D, _D]),
    "bem_get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "bem_gemm_bf16x3": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "bem_gemm_bf16x3_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "bem_set_mesh_blocks": (C.c_int, [C.c_void_p, C.c_int64, _D, C.c_int64, _I64, C.c_int32, _I64]),
    "bem_num_blocks": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "bem_set_block_params": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D]),
    "bem_get_block_params": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D]),
    "bem_get_block_stats": (C.c_int, [C.c_void_p, _D, _D, C.POINTER(C.c_int32)]),
    "bem_evolve_rk4_graph": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "bem_autotune_assembly": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), _D]),
    "bem_export_ply_async": (C.c_int, [C.c_void_p, C.c_char_p]),
    "bem_export_wait": (C.c_int, [C.c_void_p]),
    "bem_exterior_potential": (C.c_int, [C.c_void_p, C.c_int64, _D, _D, _D, _D]),
    "bem_adjoint_record": (C.c_int, [C.c_void_p, C.c_double, C.c_int32]),
    "bem_adjoint_backward": (C.c_int, [C.c_void_p, _D, _D, _D, _D]),
    "bem_adjoint_backward_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "bem_volume_gradient": (C.c_int, [C.c_void_p, _D]),
    "bem_set_state_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "bem_get_state_device": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
}

_lib = None


def load():
    """Load libbem_b200.so and declare every entry point; raises if the library is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libbem_b200.so not built at {LIB_PATH}: run `make -C {PKG_ROOT}`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class BemError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code

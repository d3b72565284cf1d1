"""ctypes binding of libhlld_b200.so (the C ABI declared in include/hlld_b200.h).

Loading fails loudly: there is no CPU or PyTorch fallback for any kernel.
"""
from __future__ import annotations

import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
# HLLD_B200_LIB overrides the library path (e.g. an alternative build)
LIB_PATH = os.environ.get("HLLD_B200_LIB") or os.path.join(HERE, "libhlld_b200.so")

HLLD_OK = 0
FP64, FP64_EXACT, MIXED, FP32 = 0, 1, 2, 3
PRECISIONS = {"fp64": FP64, "fp64_exact": FP64_EXACT, "mixed": MIXED, "fp32": FP32}
SOLVERS = {"hlle": 0, "hlld": 1, "hllc": 2}
EMF_MODES = {"solver": 0, "hll": 1}
LIMITERS = {"pcm": 0, "mc": 1, "minmod": 2, "weno5z": 3, "mp5": 4, "mp7": 5}
BCS = {"outflow": 0, "periodic": 1}

ST_BRACKET_OK, ST_CONVERGED, ST_V_CLAMPED, ST_ATMO, ST_BISECTED = 1, 2, 4, 8, 16
RF_WAVE_ORDER_BAD, RF_BN_ZERO, RF_FAILED = 1, 2, 4

_u64 = ctypes.c_ulonglong


class FluxDiag(ctypes.Structure):
    _fields_ = [("n_faces", _u64), ("n_not_converged", _u64), ("n_wave_order_bad", _u64),
                ("n_bn_zero", _u64), ("n_failed", _u64), ("iters_sum_conv", _u64),
                ("n_conv", _u64), ("max_iters", _u64), ("fd_max_bits", _u64)]


class StepDiag(ctypes.Structure):
    _fields_ = [("sweep", FluxDiag * 2), ("c2p_not_converged", _u64), ("c2p_bisected", _u64),
                ("c2p_atmo", _u64), ("c2p_bad_bracket", _u64), ("speed_max_bits", _u64 * 2)]


class Grid2DC(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("ng", ctypes.c_int32),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double),
                ("bc_x", ctypes.c_int32), ("bc_y", ctypes.c_int32),
                ("limiter", ctypes.c_int32), ("solver", ctypes.c_int32),
                ("gamma", ctypes.c_double), ("atmo_rho", ctypes.c_double),
                ("upwind", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("emf_mode", ctypes.c_int32)]


class State2DC(ctypes.Structure):
    _fields_ = [("cons", ctypes.c_void_p * 6), ("Bxf", ctypes.c_void_p), ("Byf", ctypes.c_void_p),
                ("prims", ctypes.c_void_p * 9)]


class TubesC(ctypes.Structure):
    _fields_ = [("ntubes", ctypes.c_int32), ("ng", ctypes.c_int32),
                ("ncells", ctypes.c_void_p), ("cell_off", ctypes.c_void_p),
                ("dx", ctypes.c_void_p), ("order", ctypes.c_void_p),
                ("cfl", ctypes.c_double), ("tend", ctypes.c_double),
                ("max_steps", ctypes.c_int32), ("limiter", ctypes.c_int32),
                ("solver", ctypes.c_int32), ("scheme", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("gamma", ctypes.c_double),
                ("atmo_rho", ctypes.c_double), ("flavor", ctypes.c_int32),
                ("resume", ctypes.c_int32)]


TUBE_RK_STEP, TUBE_DRIVER1D_LIGHT, TUBE_DRIVER1D_CFL = 0, 1, 2


# exported symbol -> (restype, argtypes)
_VP = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)
SIGNATURES = {
    "hlld_version": (ctypes.c_int, []),
    "hlld_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "hlld_last_error_detail": (ctypes.c_char_p, []),
    "hlld_prim_to_cons": (ctypes.c_int, [ctypes.c_int64, _PP, ctypes.c_int, _PP, _VP]),
    "hlld_cons_to_prim": (ctypes.c_int, [ctypes.c_int64, _PP, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, _PP, _VP, _VP]),
    "hlld_riemann_faces": (ctypes.c_int, [ctypes.c_int64, _PP, _PP, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_int, _PP, _PP, _VP, _VP, _VP,
                                          _VP, _VP, _VP]),
    "hlld_step2d_scratch_bytes": (ctypes.c_int, [ctypes.POINTER(Grid2DC),
                                                 ctypes.POINTER(ctypes.c_size_t)]),
    "hlld_rk_step_ct": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC), _VP,
                                       ctypes.c_size_t, ctypes.c_double, _VP, ctypes.c_int, _VP,
                                       _VP]),
    "hlld_rk_step_ct_events": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                              _VP, ctypes.c_size_t, ctypes.c_double, _VP,
                                              ctypes.c_int, _VP, _VP, _VP, _VP]),
    "hlld_rk_step_ct_static": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                              ctypes.c_double, _VP, ctypes.c_int, _VP, _VP]),
    "hlld_sync_state": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC), _VP,
                                       _VP, _VP]),
    "hlld_sync_state_roots": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                             _VP, _VP, _VP, _VP, _VP]),
    "hlld_sync_state_from_prims": (ctypes.c_int, [ctypes.POINTER(Grid2DC),
                                                  ctypes.POINTER(State2DC), _VP, _VP, _VP, _VP]),
    "hlld_sweep2d": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                    ctypes.c_int, _PP, _VP, _VP]),
    "hlld_ct_update2d": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC), _PP,
                                        _PP, _VP, _PP, _VP, _VP, _VP, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, _VP, _VP]),
    "hlld_tubes_run": (ctypes.c_int, [ctypes.POINTER(TubesC), _PP, _PP, _PP, _PP, _VP, _VP, _VP,
                                      ctypes.c_int, ctypes.c_int, _VP]),
    "hlld_compute_dt_2d": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                          ctypes.c_double, _VP, _VP, _VP]),
    "hlld_prim_to_cons_vjp": (ctypes.c_int, [ctypes.c_int64, _PP, _PP, _PP, _VP]),
    "hlld_adjoint_scratch_bytes": (ctypes.c_int, [ctypes.POINTER(Grid2DC),
                                                  ctypes.POINTER(ctypes.c_size_t)]),
    "hlld_adjoint_tape_bytes": (ctypes.c_int, [ctypes.POINTER(Grid2DC),
                                               ctypes.POINTER(ctypes.c_size_t),
                                               ctypes.POINTER(ctypes.c_size_t)]),
    "hlld_adjoint_record_step": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                                ctypes.c_double, ctypes.c_int, _VP, ctypes.c_size_t,
                                                _VP, ctypes.c_size_t, _VP]),
    "hlld_adjoint_reverse_step": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                                 ctypes.POINTER(State2DC), ctypes.c_double,
                                                 ctypes.c_int, _VP, ctypes.c_size_t,
                                                 ctypes.POINTER(State2DC), _VP, ctypes.c_size_t,
                                                 _VP]),
    "hlld_adjoint_rk_step_ct": (ctypes.c_int, [ctypes.POINTER(Grid2DC), ctypes.POINTER(State2DC),
                                               ctypes.POINTER(State2DC), ctypes.c_double,
                                               ctypes.c_int, ctypes.POINTER(State2DC), _VP,
                                               ctypes.c_size_t, _VP]),
}

_lib = None


class HlldError(RuntimeError):
    """A C-ABI call returned an error code."""


def lib() -> ctypes.CDLL:
    """The loaded library; raises if it is missing (build it with
    ``python -m hlld_ai_b200.build``)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: the CUDA kernels are not built "
                              "(python -m hlld_ai_b200.build); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != HLLD_OK:
        L = lib()
        raise HlldError(f"{what}: {L.hlld_error_string(rc).decode()} "
                        f"({L.hlld_last_error_detail().decode()})")


def stream_handle(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def ptr_array(tensors) -> ctypes.Array:
    return (ctypes.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


def require_cuda(t: torch.Tensor, name: str, dtype=torch.float64) -> torch.Tensor:
    """Kernels run on the GPU only: CPU tensors are an error, not a fallback."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA tensor (hlld_ai_b200 has no CPU path)")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    return t.contiguous()

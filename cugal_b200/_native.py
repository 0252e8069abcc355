"""ctypes binding of the C ABI in ``include/fugal_b200.h`` (``lib/libfugal_b200.so``).

This is the thin host layer between the Python mirror of cuGAL and the sm_100a
kernels: it loads the in-tree library, declares every entry point's signature,
validates tensors (device, dtype, row stride, alignment) before handing raw
pointers over, passes torch's current CUDA stream, and turns a non-OK status
into ``NativeError`` with the library's message.  There is no fallback: if the
library is missing or a tensor is not on a CUDA device, the call raises.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_double, c_float, c_int, c_int64, c_size_t, c_void_p, c_char_p
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libfugal_b200.so"

FUGAL_F32, FUGAL_BF16, FUGAL_F16 = 0, 1, 2
LAP_GREEDY, LAP_DOUBLE_GREEDY, LAP_PARALLEL_GREEDY, LAP_ORDERED = 0, 1, 2, 3
(KERNEL_SWEEP, KERNEL_SWEEP_F32, KERNEL_ABSORB, KERNEL_FINALIZE, KERNEL_COLUMN_PASS, KERNEL_GRADIENT,
 KERNEL_UPDATE, KERNEL_OTHER) = range(8)
KERNEL_FAMILY_NAMES = ["sweep16", "sweep32", "absorb", "finalize", "column_pass", "gradient", "update", "other"]
MAX_RECORDED_ERRORS = 256

STREAM_DTYPES = {None: FUGAL_F32, torch.float32: FUGAL_F32, torch.bfloat16: FUGAL_BF16, torch.float16: FUGAL_F16}


class NativeError(RuntimeError):
    """A kernel entry point returned a non-OK fugal_status."""


class SolveParams(ctypes.Structure):
    _fields_ = [
        ("n", c_int64), ("cost32", c_void_p), ("ld32", c_int64), ("cost16", c_void_p), ("ld16", c_int64),
        ("stream_dtype", c_int), ("max_iterations", c_int), ("threshold", c_double), ("eval_freq", c_int),
        ("momentum_start", c_int), ("fp32_warmup_sweeps", c_int), ("reabsorb_every", c_int),
        ("polish_sweeps", c_int), ("u_out", c_void_p), ("v_out", c_void_p), ("record", c_void_p),
        ("column_partials", c_void_p), ("column_partial_chunks", ctypes.c_int32), ("column_partial_ld", c_int64),
    ]


class SolveRecord(ctypes.Structure):
    _fields_ = [
        ("iteration_count", ctypes.c_int32), ("n_errors", ctypes.c_int32), ("status", ctypes.c_int32),
        ("polish_count", ctypes.c_int32), ("last_error", c_double), ("polish_error", c_double),
        ("errors", c_double * MAX_RECORDED_ERRORS),
    ]


RECORD_BYTES = ctypes.sizeof(SolveRecord)

_P, _I64, _F, _D, _INT, _SZ = c_void_p, c_int64, c_float, c_double, c_int, c_size_t

SIGNATURES = {
    "fugal_status_string": (c_char_p, [_INT]),
    "fugal_last_error": (c_char_p, []),
    "fugal_version": (_INT, []),
    "fugal_adjacency_matmul": (_INT, [_P, _P, _I64, _P, _I64, _INT, _P, _I64, _INT, _P]),
    "fugal_create_adjacency_workspace_size": (_INT, [_I64, _I64, POINTER(c_size_t)]),
    "fugal_create_adjacency": (_INT, [_P, _I64, _I64, _P, _P, _P, _SZ, _P]),
    "fugal_graph_features": (_INT, [_P, _P, _I64, _P, _P, _P, _P, _P]),
    "fugal_average_neighbor_features": (_INT, [_P, _P, _I64, _P, _P, _P]),
    "fugal_sinkhorn_log_step": (_INT, [_P, _I64, _I64, _I64, _P, _P, _F, _P]),
    "fugal_sinkhorn_log_marginal": (_INT, [_P, _I64, _I64, _P, _P, _INT, _P, _P]),
    "fugal_add_distance": (_INT, [_P, _P, _I64, _P, _I64, _P]),
    "fugal_regularize": (_INT, [_P, _I64, _P, _I64, _I64, _INT, _P]),
    "fugal_update_quasi_permutation_log": (_INT, [_P, _I64, _P, _I64, _P, _P, _I64, _F, _F, _P, _P]),
    "fugal_greedy_lap_workspace_size": (_INT, [_I64, _INT, POINTER(c_size_t)]),
    "fugal_greedy_lap": (_INT, [_P, _I64, _I64, _INT, _P, _INT, _INT, _P, _P, _SZ, _P]),
    "fugal_sampled_lap": (_INT, [_P, _I64, _I64, _P, _P, _INT, _P, _P]),
    "fugal_exact_lap_workspace_size": (_INT, [_I64, POINTER(c_size_t)]),
    "fugal_exact_lap": (_INT, [_P, _I64, _I64, _INT, _I64, _P, _P, _P, _P, _SZ, _P]),
    "fugal_count_le": (_INT, [_P, _I64, _I64, _F, _P, _P]),
    "fugal_alignment_overlap_workspace_size": (_INT, [_I64, POINTER(c_size_t)]),
    "fugal_alignment_overlap": (_INT, [_P, _P, _P, _P, _I64, _P, _P, _P, _P, _P, _SZ, _P]),
    "fugal_gradient_workspace_size": (_INT, [_I64, POINTER(c_size_t)]),
    "fugal_fw_gradient": (_INT, [_I64, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _I64, _D, _D, _D, _P, _P, _P, _I64,
                                 _P, _SZ, _P]),
    "fugal_fw_gradient_fixed_scratch": (_INT, [_I64, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _I64, _D, _D, _D, _P, _P,
                                               _P, _I64, _P]),
    "fugal_sinkhorn_standard_workspace_size": (_INT, [_I64, POINTER(c_size_t)]),
    "fugal_sinkhorn_standard_solve": (_INT, [_P, _I64, _I64, _P, _P, _INT, _D, _INT, _INT, _P, _P, _SZ, _P]),
    "fugal_exp_scale": (_INT, [_P, _I64, _I64, _D, _P, _I64, _P]),
    "fugal_fw_update_standard": (_INT, [_I64, _P, _I64, _P, _I64, _P, _P, _P, _I64, _D, _P, _P]),
    "fugal_sinkhorn_plan": (_INT, [_P, _I64, _I64, _P, _P, _P, _I64, _P]),
    "fugal_plan_matvec_workspace_size": (_INT, [_I64, POINTER(c_size_t)]),
    "fugal_plan_matvec": (_INT, [_P, _I64, _P, _I64, _I64, _P, _P, _P, _P, _P, _SZ, _P]),
    "fugal_sinkhorn_adjoint": (_INT, [_P, _I64, _P, _I64, _I64, _P, _P, _D, _P, _I64, _P]),
    "fugal_sinkhorn_unrolled_step_backward": (_INT, [_P, _I64, _I64, _P, _P, _P, _INT, _P, _I64, _P, _P, _SZ, _P]),
    "fugal_sinkhorn_workspace_size": (_INT, [_I64, _INT, POINTER(c_size_t)]),
    "fugal_sinkhorn_plan_info": (_INT, [_I64, _INT, _P]),
    "fugal_sinkhorn_solve": (_INT, [POINTER(SolveParams), _P, _SZ, _P]),
    "fugal_gradient_column_chunks": (_INT, [_I64, POINTER(ctypes.c_int32)]),
    "fugal_fw_gradient_column_stats": (_INT, [_I64, _P, _P, _P, _P, _P, _I64, _P, _P, _P, _I64, _D, _D, _D, _P, _P,
                                              _P, _I64, _P, _SZ, _P, _I64, _P]),
    "fugal_fw_update": (_INT, [_I64, _P, _I64, _P, _I64, _P, _P, _P, _P, _D, _D, _P, _INT, _P]),
    "fugal_fw_update_collect": (_INT, [_I64, _P, _I64, _P, _I64, _P, _P, _P, _P, _D, _D, _P, _INT, _P, _P, _INT,
                                       _P]),
    "fugal_csr_edge_rows": (_INT, [_P, _I64, _I64, _P, _P]),
    "fugal_structural_refresh": (_INT, [_I64, _P, _P, _P, _P, _P, _I64, _P, _I64, _INT, _P, _SZ, _P, _P]),
    "fugal_structural_scatter": (_INT, [_I64, _P, _P, _I64, _P, _P, _P, _P, _INT, _D, _P, _I64, _P, _P]),
    "fugal_fw_gradient_structural": (_INT, [_I64, _P, _I64, _D, _INT, _P, _I64, _P, _P, _P, _I64, _D, _D, _D, _P,
                                            _P, _P, _I64, _P, _I64, _P]),
    "fugal_fw_direction": (_INT, [_I64, _P, _I64, _P, _I64, _P, _I64, _P, _P, _P, _P, _D, _P, _I64, _P, _INT,
                                  _P]),
    "fugal_fw_line_search_update": (_INT, [_I64, _P, _I64, _P, _I64, _P, _I64, _D, _P, _P, _P, _P]),
    "fugal_timing_enable": (None, [_INT]),
    "fugal_timing_reset": (None, []),
    "fugal_timing_query": (_INT, [_INT, POINTER(c_int64), POINTER(c_double)]),
    "fugal_launch_count": (c_int64, []),
}

_lib = None


def lib() -> ctypes.CDLL:
    """The loaded kernel library (raises ImportError if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing; build it with `python -m cugal_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def check(status: int, what: str) -> None:
    if status != 0:
        L = lib()
        raise NativeError(f"{what}: {L.fugal_status_string(status).decode()} "
                          f"({L.fugal_last_error().decode()})")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)


def stream_handle(device: torch.device | None = None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def require_cuda(t: torch.Tensor, name: str, dtype: torch.dtype | None = None) -> None:
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise ValueError(f"{name} must be a CUDA tensor (this library has no CPU path)")
    if dtype is not None and t.dtype != dtype:
        raise ValueError(f"{name} must have dtype {dtype}, got {t.dtype}")


def matrix_ld(t: torch.Tensor, name: str) -> int:
    """Leading dimension of a row-major 2-D tensor (unit column stride)."""
    if t.dim() != 2 or t.stride(1) != 1:
        raise ValueError(f"{name} must be a row-major 2-D tensor with unit column stride")
    return t.stride(0)


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def workspace_size(fn: str, *args) -> int:
    out = c_size_t(0)
    call(fn, *args, ctypes.byref(out))
    return out.value


def timing_enable(on: bool) -> None:
    lib().fugal_timing_enable(1 if on else 0)


def timing_reset() -> None:
    lib().fugal_timing_reset()


def timing_query(family: int) -> tuple[int, float]:
    n, ms = c_int64(0), c_double(0.0)
    call("fugal_timing_query", family, ctypes.byref(n), ctypes.byref(ms))
    return n.value, ms.value


def sinkhorn_plan(n: int, stream_dtype: int) -> dict:
    """Launch shape the solve uses for size n on the current device."""
    info = (ctypes.c_int32 * 6)()
    call("fugal_sinkhorn_plan_info", n, stream_dtype, ctypes.cast(info, c_void_p))
    keys = ["threads", "cluster", "clusters", "stages", "smem_bytes", "rows_per_batch"]
    return dict(zip(keys, list(info)))


def launch_count() -> int:
    return int(lib().fugal_launch_count())


def exported_symbols() -> list[str]:
    return list(SIGNATURES)

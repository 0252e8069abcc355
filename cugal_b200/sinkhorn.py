"""Log-domain Sinkhorn (reference ``cugal/sinkhorn.py:51-156``).

``SinkhornSolver`` drives ``fugal_sinkhorn_solve`` for one problem size: it owns
the solve workspace and runs a whole solve -- first column update, fused sweeps with
on-device convergence decisions, optional reduced-precision streaming and FP32
polish -- as one call on the current stream.

``SinkhornState`` mirrors the reference class: it keeps the warm-started dual
potentials u, v across solves and ``solve(C, config, profile)`` returns
``(K, u, v)`` with K = -C/reg.  Internally the duals are held in FP64 and folded
into the kernel input (the solver works on K + u_i + v_j, whose entries near the
optimal plan are O(1) instead of O(1/reg)).  Only ``SinkhornMethod.LOG`` runs
on the GPU path.
"""

from __future__ import annotations

import ctypes

import torch

from . import _native as N
from .config import Config, SinkhornMethod
from .profile import SinkhornProfile, TimeStamp


def padded_ld(n: int) -> int:
    """Row stride used for every n x n buffer: a multiple of 8 elements (16 bytes
    for both FP32 and 16-bit rows)."""
    return (n + 7) // 8 * 8


class SinkhornSolver:
    """Workspace + launch parameters of the fused log-domain solve for size n."""

    def __init__(self, n: int, config: Config, device):
        self.n = n
        self.device = torch.device(device)
        self.config = config
        self.stream_dtype = N.STREAM_DTYPES.get(config.stream_dtype)
        if self.stream_dtype is None:
            raise ValueError(f"unsupported stream_dtype {config.stream_dtype}")
        ws = N.workspace_size("fugal_sinkhorn_workspace_size", n, self.stream_dtype)
        self.workspace = torch.empty(ws, dtype=torch.uint8, device=self.device)
        self.ld16 = padded_ld(n)
        self.cost16 = None
        if self.stream_dtype != N.FUGAL_F32:
            self.cost16 = torch.zeros((n, self.ld16), dtype=config.stream_dtype, device=self.device)

    def params(self, cost32: torch.Tensor, u_out: torch.Tensor, v_out: torch.Tensor, record_ptr: int | None,
               column_partials: torch.Tensor | None = None):
        c = self.config
        p = N.SolveParams()
        p.n = self.n
        p.cost32 = cost32.data_ptr()
        p.ld32 = N.matrix_ld(cost32, "cost32")
        p.cost16 = None if self.cost16 is None else self.cost16.data_ptr()
        p.ld16 = self.ld16
        p.stream_dtype = self.stream_dtype
        p.max_iterations = c.sinkhorn_iterations
        p.threshold = c.sinkhorn_threshold
        p.eval_freq = c.sinkhorn_eval_freq
        p.momentum_start = -1 if c.sinkhorn_momentum_start is None else int(c.sinkhorn_momentum_start)
        p.fp32_warmup_sweeps = c.fp32_warmup_sweeps
        p.reabsorb_every = c.reabsorb_every
        p.polish_sweeps = c.polish_sweeps
        p.u_out = u_out.data_ptr()
        p.v_out = v_out.data_ptr()
        p.record = record_ptr
        if column_partials is not None:
            # (chunks, 2 ld) float32 = chunks x ld (max, sum) pairs
            p.column_partials = column_partials.data_ptr()
            p.column_partial_chunks = column_partials.shape[0]
            p.column_partial_ld = column_partials.shape[1] // 2
        return p

    def solve(self, cost32: torch.Tensor, u_out: torch.Tensor, v_out: torch.Tensor, record_ptr: int | None = None,
              column_partials: torch.Tensor | None = None):
        """One solve on the absorbed cost ``cost32`` (n x ld FP32): writes the dual
        increments u_out, v_out (FP32) and, if given, a device solve record.
        ``column_partials``: the column statistics ``fugal_fw_gradient_column_stats``
        wrote with this cost (skips the solve's own pass over it)."""
        N.require_cuda(cost32, "cost32", torch.float32)
        p = self.params(cost32, u_out, v_out, record_ptr, column_partials)
        N.call("fugal_sinkhorn_solve", ctypes.byref(p), self.workspace.data_ptr(), self.workspace.numel(),
               N.stream_handle(self.device))


def read_record(raw: torch.Tensor) -> SinkhornProfile:
    """SinkhornProfile from a host copy of one fugal_solve_record."""
    rec = N.SolveRecord.from_buffer_copy(raw.numpy().tobytes())
    if rec.status != 0:
        raise N.NativeError(f"Sinkhorn solve reported device status {rec.status} (bounded wait timed out)")
    errors = [rec.errors[k] for k in range(rec.n_errors)]
    final = rec.polish_error if rec.polish_count > 0 else rec.last_error
    return SinkhornProfile(errors=errors, iteration_count=rec.iteration_count, final_error=final)


class StandardSolver:
    """Workspace of the scaling-form solve (``fugal_sinkhorn_standard_solve``) for size n."""

    def __init__(self, n: int, config: Config, device):
        self.n = n
        self.config = config
        self.device = torch.device(device)
        ws = N.workspace_size("fugal_sinkhorn_standard_workspace_size", n)
        self.workspace = torch.empty(ws, dtype=torch.uint8, device=self.device)

    def solve(self, K: torch.Tensor, u: torch.Tensor, v: torch.Tensor, record_ptr: int | None = None):
        """Updates the FP32 scaling vectors u, v in place on the kernel matrix K."""
        N.require_cuda(K, "K", torch.float32)
        c = self.config
        N.call("fugal_sinkhorn_standard_solve", K.data_ptr(), N.matrix_ld(K, "K"), self.n, u.data_ptr(),
               v.data_ptr(), c.sinkhorn_iterations, c.sinkhorn_threshold, c.sinkhorn_eval_freq,
               -1 if c.sinkhorn_momentum_start is None else int(c.sinkhorn_momentum_start), record_ptr,
               self.workspace.data_ptr(), self.workspace.numel(), N.stream_handle(self.device))


def exp_scale(C: torch.Tensor, scale: float, out: torch.Tensor) -> torch.Tensor:
    """out = exp(scale * C) for square row-major FP32 device matrices."""
    n = C.shape[0]
    N.call("fugal_exp_scale", C.data_ptr(), N.matrix_ld(C, "C"), n, float(scale), out.data_ptr(),
           N.matrix_ld(out, "out"), N.stream_handle(C.device))
    return out


class SinkhornState:
    """Warm-started dual potentials (reference ``cugal/sinkhorn.py:51-65``).

    LOG: log-domain duals (FP64 internally, see the module docstring).  STANDARD:
    the scaling vectors u, v (FP32, start at 1/n) of ``solve_standard``."""

    def __init__(self, n: int, config: Config):
        if config.sinkhorn_method not in (SinkhornMethod.LOG, SinkhornMethod.STANDARD):
            raise NotImplementedError(f"{config.sinkhorn_method} is not available on the GPU path")
        if "cuda" not in config.device:
            raise ValueError("SinkhornState: only CUDA devices are supported")
        self.n = n
        self.config = config
        dev = torch.device(config.device)
        if config.sinkhorn_method == SinkhornMethod.STANDARD:
            self.method = SinkhornMethod.STANDARD
            self.u_std = torch.full((n,), 1.0 / n, dtype=torch.float32, device=dev)
            self.v_std = torch.full((n,), 1.0 / n, dtype=torch.float32, device=dev)
            self._std = StandardSolver(n, config, dev)
            self._rec = torch.empty(N.RECORD_BYTES, dtype=torch.uint8, device=dev)
            return
        self.method = SinkhornMethod.LOG
        self.U = torch.zeros(n, dtype=torch.float64, device=dev)
        self.V = torch.zeros(n, dtype=torch.float64, device=dev)
        self._solver = SinkhornSolver(n, config, dev)
        self._du = torch.empty(n, dtype=torch.float32, device=dev)
        self._dv = torch.empty(n, dtype=torch.float32, device=dev)
        self._rec = torch.empty(N.RECORD_BYTES, dtype=torch.uint8, device=dev)

    @property
    def u(self) -> torch.Tensor:
        if self.method == SinkhornMethod.STANDARD:
            return self.u_std
        return self.U.to(self.config.dtype)

    @property
    def v(self) -> torch.Tensor:
        if self.method == SinkhornMethod.STANDARD:
            return self.v_std
        return self.V.to(self.config.dtype)

    def solve_standard(self, C: torch.Tensor, config: Config | None = None, profile: SinkhornProfile | None = None):
        """``solve_standard`` (``cugal/sinkhorn.py:122-144``): returns (K, u, v), K = exp(-C/reg)."""
        config = config or self.config
        start = TimeStamp(config.device)
        N.require_cuda(C, "C")
        C32 = C.to(torch.float32).contiguous()
        K = exp_scale(C32, -1.0 / config.sinkhorn_regularization, torch.empty_like(C32))
        self._std.solve(K, self.u_std, self.v_std, self._rec.data_ptr())
        if profile is not None:
            rec = read_record(self._rec.cpu())
            profile.errors, profile.iteration_count = rec.errors, rec.iteration_count
            profile.final_error = rec.final_error
            profile.time = TimeStamp(config.device).elapsed_seconds(start)
        return K, self.u_std, self.v_std

    def plan(self, out: torch.Tensor | None = None) -> torch.Tensor:
        """The plan P = exp(K + u + v) of the last LOG solve (n x n FP32)."""
        if self.method != SinkhornMethod.LOG or not hasattr(self, "_cost32"):
            raise RuntimeError("plan(): run a LOG solve first")
        n = self.n
        out = torch.empty((n, n), dtype=torch.float32, device=self._cost32.device) if out is None else out
        N.call("fugal_sinkhorn_plan", self._cost32.data_ptr(), self._cost32.stride(0), n, self._du.data_ptr(),
               self._dv.data_ptr(), out.data_ptr(), N.matrix_ld(out, "out"), N.stream_handle(out.device))
        return out

    def solve(self, C: torch.Tensor, config: Config | None = None, profile: SinkhornProfile | None = None):
        """``solve`` / ``solve_log`` (``cugal/sinkhorn.py:90-120,146-156``): returns (K, u, v)."""
        config = config or self.config
        if self.method == SinkhornMethod.STANDARD:
            return self.solve_standard(C, config, profile)
        start = TimeStamp(config.device)
        n = self.n
        N.require_cuda(C, "C")
        K = (-C / config.sinkhorn_regularization).to(torch.float32)
        cost32 = torch.zeros((n, padded_ld(n)), dtype=torch.float32, device=C.device)  # finite padding
        cost32[:, :n] = (K.double() + self.U[:, None] + self.V[None, :]).float()
        self._solver.solve(cost32, self._du, self._dv, self._rec.data_ptr())
        self._cost32 = cost32
        self.U += self._du.double()
        self.V += self._dv.double()
        if profile is not None:
            rec = read_record(self._rec.cpu())
            profile.errors, profile.iteration_count = rec.errors, rec.iteration_count
            profile.time = TimeStamp(config.device).elapsed_seconds(start)
        return K, self.u.float(), self.v.float()

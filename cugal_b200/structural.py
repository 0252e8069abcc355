"""Structural term ``A P B`` of the Frank-Wolfe gradient kept across steps.

The reference forms ``-A P B`` from scratch every step with two sparse-dense
products (``cugal/pred.py:54-74``).  Its step is fixed, ``P' = (1 - a) P + a q``
(``cugal/pred.py:133-141``), so ``M = A P B`` follows

    M' = (1 - a) M + a A q B,

and after the first steps the Sinkhorn plan ``q`` has a handful of nonzero
entries per row (exactly one for a converged solve at the small
regularizations FUGAL uses), which makes ``A q B`` a sparse product.  The
gradient then becomes an elementwise pass over a stored ``M``
(``fugal_fw_gradient_structural``) instead of two gathers of ``P`` through
``A`` and ``B``.

``M`` is stored as int64 fixed point, ``M = Mq * 2^-frac_bits * scale``: the
``(1 - a)`` factors go into the host-held ``scale``, so a step only adds to the
entries ``A q B`` touches, and integer adds make the sums independent of the
order of the device's atomics (reruns are bit-identical).  The update records
the plan's nonzero entries per row (``fugal_fw_update_collect``); the scatter
flags a row with more than ``SLOTS`` of them, or a plan row sum above
``ROW_SUM_MAX``, and the next gradient recomputes ``Mq`` with the two SpMMs
(``fugal_structural_refresh``).  Nothing is dropped: every nonzero FP32 entry
of ``q`` is either added exactly (to 2^-frac_bits) or the term is recomputed.

This module holds the host side: the fixed-point bookkeeping (``FixedPoint``,
pure arithmetic, tested on the CPU) and the device buffers (``StructuralTerm``).
"""

from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import torch

from . import _native as N

SLOTS = 32                  # plan entries recorded per row
ROW_SUM_MAX = 32.0          # FUGAL_PLAN_ROW_SUM_MAX: larger plan rows flag the step
ROW_SUM_BITS = 5            # log2(ROW_SUM_MAX)
SCALE_BITS = 8              # scale stays >= 2^-SCALE_BITS between rescales
RESCALE_BELOW = 2.0 ** -6   # rescale Mq by a power of two once scale drops below this
MIN_FRAC_BITS = 24          # fewer fraction bits than this: keep the SpMM gradient
VALUE_BITS = 52             # 0 <= Mq < 2^52: its double is exact and cheap to form


def frac_bits(max_degree: int) -> int:
    """Fraction bits for a source graph of largest degree ``max_degree``.

    ``M[i][j] <= deg_A(i) * max row sum of P <= max_degree * ROW_SUM_MAX`` and
    ``Mq = M / scale * 2^F`` with ``scale >= 2^-SCALE_BITS``, so
    ``Mq < 2^52`` when ``F = 52 - SCALE_BITS - ROW_SUM_BITS - ceil(log2(max_degree + 1))``."""
    if max_degree < 0:
        raise ValueError("max_degree must be >= 0")
    return VALUE_BITS - SCALE_BITS - ROW_SUM_BITS - math.ceil(math.log2(max_degree + 1))


@dataclass
class FixedPoint:
    """Scale bookkeeping of ``M = Mq * 2^-bits * scale``."""

    bits: int
    scale: float = 1.0

    def refreshed(self) -> None:
        """Mq was just recomputed as round(A P B * 2^bits)."""
        self.scale = 1.0

    def m_scale(self) -> float:
        """Factor from Mq to M."""
        return math.ldexp(self.scale, -self.bits)

    def step(self, alpha: float) -> float | None:
        """Scale after a step of size ``alpha`` and the increment factor of its
        scatter (``round(q * factor)`` is added per plan entry), or None when the
        new scale would leave the range the bits were chosen for (the caller
        then recomputes Mq)."""
        new_scale = self.scale * (1.0 - alpha)
        if not (alpha >= 0.0) or not (new_scale >= 2.0 ** -SCALE_BITS):
            return None
        self.scale = new_scale
        return math.ldexp(alpha / new_scale, self.bits)

    def shift(self) -> int:
        """Power of two to divide Mq by at the next gradient (0: none), keeping
        scale in (1/2, 1] afterwards; the caller applies it with
        ``shifted(k)`` once the gradient has read Mq at the old scale."""
        if self.scale >= RESCALE_BELOW:
            return 0
        return int(math.floor(-math.log2(self.scale)))

    def shifted(self, k: int) -> None:
        self.scale = math.ldexp(self.scale, k)


def enabled_by_default() -> bool:
    """``FUGAL_GRAD_RECURRENCE=0`` keeps the two-SpMM gradient every step."""
    return os.environ.get("FUGAL_GRAD_RECURRENCE", "1") != "0"


@dataclass
class StructuralTerm:
    """Device state of the kept structural term of one alignment.

    Life cycle per Frank-Wolfe step: ``prepare`` (before the gradient: read the
    flags of the last update, recompute Mq when it is stale), the gradient from
    Mq, the solve, ``collect_update`` (the update that records the plan) and
    ``scatter`` (adds a A q B)."""

    A: object
    B: object
    n: int
    ld: int
    device: torch.device
    workspace: torch.Tensor
    fixed: FixedPoint = field(init=False)
    valid: bool = field(default=False, init=False)
    broken: bool = field(default=False, init=False)
    refreshes: int = field(default=0, init=False)
    scatters: int = field(default=0, init=False)

    def __post_init__(self):
        rp = self.A.row_pointers
        max_degree = int((rp[1:] - rp[:-1]).max().item()) if self.n > 0 else 0
        bits = frac_bits(max_degree)
        if bits < MIN_FRAC_BITS:
            raise ValueError(f"largest degree {max_degree} leaves {bits} fraction bits")
        self.fixed = FixedPoint(bits)
        dev = self.device
        self.Mq = torch.empty((self.n, self.ld), dtype=torch.int64, device=dev)
        self.counts = torch.zeros(self.n, dtype=torch.int32, device=dev)
        self.entries = torch.zeros((self.n, SLOTS, 2), dtype=torch.int32, device=dev)
        # [a plan row was not added, the fixed-point range was exceeded]
        self.flags = torch.zeros(2, dtype=torch.int32, device=dev)
        self.a_nnz = int(self.A.col_indices.numel())
        self.edge_rows = torch.empty(max(1, self.a_nnz), dtype=torch.int32, device=dev)
        N.call("fugal_csr_edge_rows", self.A.row_pointers.data_ptr(), self.n, self.a_nnz, self.edge_rows.data_ptr(),
               N.stream_handle(dev))

    def invalidate(self) -> None:
        """P changed outside ``collect_update``: recompute Mq at the next gradient."""
        self.valid = False

    def prepare(self, P_buf: torch.Tensor) -> bool:
        """Make Mq current for P; False when the term cannot be used (the caller
        takes the SpMM gradient).  Waits for the device once (the flags)."""
        if self.broken:
            return False
        if self.valid:
            f0, f1 = self.flags.tolist()
            if f1:
                self.broken = True
                return False
            if f0:
                self.valid = False
        if not self.valid:
            self.flags.zero_()
            stream = N.stream_handle(self.device)
            N.call("fugal_structural_refresh", self.n, self.A.row_pointers.data_ptr(), self.A.col_indices.data_ptr(),
                   self.B.row_pointers.data_ptr(), self.B.col_indices.data_ptr(), P_buf.data_ptr(), self.ld,
                   self.Mq.data_ptr(), self.ld, self.fixed.bits, self.workspace.data_ptr(), self.workspace.numel(),
                   self.flags.data_ptr(), stream)
            self.refreshes += 1
            if self.flags[1].item():
                self.broken = True
                return False
            self.fixed.refreshed()
            self.valid = True
        return True

    def collect_update(self, P_buf: torch.Tensor, cost32: torch.Tensor, u, v, U, V, alpha: float, reg: float,
                       gap: torch.Tensor, commit: int = 1) -> None:
        """``fugal_fw_update`` that records the plan, then the scatter of a A q B."""
        stream = N.stream_handle(self.device)
        N.call("fugal_fw_update_collect", self.n, P_buf.data_ptr(), self.ld, cost32.data_ptr(), self.ld, u.data_ptr(),
               v.data_ptr(), U.data_ptr(), V.data_ptr(), float(alpha), float(reg), gap.data_ptr(), commit,
               self.counts.data_ptr(), self.entries.data_ptr(), SLOTS, stream)
        factor = self.fixed.step(alpha)
        if factor is None:
            self.valid = False
            return
        N.call("fugal_structural_scatter", self.n, self.A.col_indices.data_ptr(), self.edge_rows.data_ptr(),
               self.a_nnz, self.B.row_pointers.data_ptr(), self.B.col_indices.data_ptr(), self.counts.data_ptr(),
               self.entries.data_ptr(), SLOTS, factor, self.Mq.data_ptr(), self.ld, self.flags.data_ptr(), stream)
        self.scatters += 1

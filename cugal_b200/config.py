"""Configuration of the FUGAL alignment (drop-in superset of cuGAL's ``Config``).

Mirrors ``cugal/config.py:11-141`` of the reference: every field keeps its name,
type and default, and ``to_dict``/``from_dict`` use the same dictionary format.
``from_dict`` reads the reference's dictionaries (fields it does not know are
dropped); the reference's ``from_dict`` accepts only its own fields, so result
files store ``split_dict()``: the reference's fields, and the fields added here
under a key of their own (``results.py``).  Fields added here are appended after
the reference's fields and default to behaviour that does not change the
reference's algorithm.
"""

from __future__ import annotations

import dataclasses
from dataclasses import dataclass
from enum import Enum
from typing import Optional

import torch


class SinkhornMethod(str, Enum):
    """Sinkhorn-Knopp variant (reference ``cugal/config.py:11-27``)."""

    STANDARD = "STANDARD"
    """Scaling-form Sinkhorn-Knopp on exp(-C/reg)."""

    LOG = "LOG"
    """Log-domain Sinkhorn-Knopp (the GPU path)."""

    MIX = "MIX"
    """Declared by the reference but never dispatched (``cugal/sinkhorn.py:152-156``)."""


class HungarianMethod(Enum):
    """Rounding of the quasi-permutation (reference ``cugal/config.py:30-52``)."""

    SCIPY = "SCIPY"
    GREEDY = "GREEDY"
    RAND = "RAND"
    MORE_RAND = "MORE_RAND"
    DOUBLE_GREEDY = "DOUBLE_GREEDY"
    PARALLEL_GREEDY = "PARALLEL_GREEDY"
    DENSE = "DENSE"
    SPARSE = "SPARSE"


def _dtype_name(dtype: Optional[torch.dtype]) -> Optional[str]:
    return None if dtype is None else str(dtype).removeprefix("torch.")


@dataclass(frozen=True)
class Config:
    """Configuration of the alignment (reference ``cugal/config.py:55-141``)."""

    # --- reference fields, same order, names and defaults -------------------
    safe_mode: bool = False
    device: str = "cpu"
    dtype: torch.dtype = torch.float64
    torch_sinkhorn: bool = False
    sinkhorn_regularization: float = 1.0
    sinkhorn_method: SinkhornMethod = SinkhornMethod.STANDARD
    sinkhorn_iterations: int = 500
    dynamic_sinkhorn_regularization: bool = False
    sinkhorn_scaling: float = 1.0
    sinkhorn_threshold: float = 1e-3
    sinkhorn_eval_freq: int = 10
    sinkhorn_momentum: bool = False
    mu: float = 0.5
    iter_count: int = 15
    frank_wolfe_iter_count: int = 10
    frank_wolfe_threshold: float | None = None
    use_sparse_adjacency: bool = False
    sinkhorn_cache_size: int = 0
    sinkhorn_momentum_start: Optional[int] = None
    recompute_distance: bool = False
    hungarian_method: HungarianMethod = HungarianMethod.DOUBLE_GREEDY

    # --- additions (B200 path) ----------------------------------------------
    stream_dtype: Optional[torch.dtype] = None
    """Element type the Sinkhorn sweeps stream the cost matrix in: ``None`` (same
    as the FP32 master), ``torch.bfloat16`` or ``torch.float16``.  Log-sum-exp,
    dual potentials and all accumulation stay in FP32; the convergence reduction
    is FP64."""

    polish_sweeps: int = 1
    """FP32 sweeps over the FP32 master cost after a reduced-precision solve."""

    fp32_warmup_sweeps: int = 0
    """FP32 sweeps of each solve before the reduced-precision copy is taken.  The
    copy is written by an absorb sweep, itself an FP32 sweep whose row update
    normalises the rows it writes, so no warm-up is needed: at n = 32768, 0, 1,
    2 and 10 warm-up sweeps gave the same node accuracy and final marginal
    errors, 0 in the least time."""

    reabsorb_every: int = 50
    """Refresh the reduced-precision copy from the FP32 master (folding the
    current duals into it) every this many sweeps."""

    lap_candidates: int = 8
    """Per-row candidate columns kept by the greedy rounding kernels."""

    line_search: bool = False
    """Frank-Wolfe step by exact line search instead of ``2 / (2 + it)``: the
    objective -<P, A P B> + <D, P> + lambda <P, 1 - P> is quadratic along the
    direction q - P, so the step is the minimiser of that parabola on [0, 1],
    computed on the device (one more pair of SpMM kernels per step)."""

    def convert_tensor(self, input: torch.Tensor) -> torch.Tensor:
        """Convert tensor to the configured dtype and device."""
        return input.to(dtype=self.dtype, device=self.device)

    def split_dict(self) -> tuple[dict, dict]:
        """(the reference's fields, the fields added here) of ``to_dict()``."""
        d = self.to_dict()
        ref = {k: d[k] for k in REFERENCE_FIELDS}
        return ref, {k: v for k, v in d.items() if k not in ref}

    def to_dict(self) -> dict:
        config_dict = dataclasses.asdict(self)
        config_dict["dtype"] = _dtype_name(self.dtype)
        config_dict["sinkhorn_method"] = self.sinkhorn_method.value
        config_dict["hungarian_method"] = self.hungarian_method.value
        config_dict["stream_dtype"] = _dtype_name(self.stream_dtype)
        return config_dict

    @classmethod
    def from_dict(cls, config_dict: dict):
        config_dict = dict(config_dict)
        config_dict["dtype"] = getattr(torch, config_dict["dtype"])
        config_dict["sinkhorn_method"] = SinkhornMethod(config_dict["sinkhorn_method"])
        config_dict["hungarian_method"] = HungarianMethod[config_dict["hungarian_method"]]
        if config_dict.get("stream_dtype") is not None:
            config_dict["stream_dtype"] = getattr(torch, config_dict["stream_dtype"])
        known = {f.name for f in dataclasses.fields(cls)}
        return cls(**{k: v for k, v in config_dict.items() if k in known})


# Field names of the reference's Config (cugal/config.py:55-120), in order.
REFERENCE_FIELDS = ("safe_mode", "device", "dtype", "torch_sinkhorn", "sinkhorn_regularization", "sinkhorn_method",
                    "sinkhorn_iterations", "dynamic_sinkhorn_regularization", "sinkhorn_scaling", "sinkhorn_threshold",
                    "sinkhorn_eval_freq", "sinkhorn_momentum", "mu", "iter_count", "frank_wolfe_iter_count",
                    "frank_wolfe_threshold", "use_sparse_adjacency", "sinkhorn_cache_size", "sinkhorn_momentum_start",
                    "recompute_distance", "hungarian_method")

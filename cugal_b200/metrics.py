"""Alignment quality metrics of the reference's experiment harness
(``benchmark/experiment.py:115-144``, ``Result`` at :340-368): edge correctness
(EC), induced conserved structure (ICS), symmetric substructure score (S3) and
node accuracy, with the reference's argument conventions
(``source_mapping`` = the computed answer, ``target_mapping`` = the planted one).

The reference counts the overlap on dense n x n numpy matrices; here it is one
integer counted on the device CSR graphs by ``fugal_alignment_overlap``.  An
answer that is not a permutation falls back to the dense definition, as does a
caller that passes numpy adjacency matrices.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .adjacency import Adjacency


def _as_device(mapping, device) -> torch.Tensor:
    if isinstance(mapping, torch.Tensor):
        return mapping.to(device=device, dtype=torch.int64).contiguous()
    return torch.as_tensor(np.asarray(mapping, dtype=np.int64), device=device)


def _dense_overlap(A: np.ndarray, B: np.ndarray, answer, truth) -> tuple[int, int, int]:
    adj1 = A[answer][:, answer]
    adj2 = B[truth][:, truth]
    return int(np.sum(adj1 + adj2 == 2)), int(np.sum(A == 1)), int(np.sum(adj2 == 1))


def overlap(source: Adjacency, target: Adjacency, answer, truth) -> tuple[int, int, int]:
    """(overlap, entries of the source adjacency, entries of the permuted target)."""
    n = source.number_of_nodes()
    dev = source.row_pointers.device
    a = _as_device(answer, dev)
    t = _as_device(truth, dev)
    if a.numel() != n or t.numel() != n:
        raise ValueError("answer and truth must have one entry per node")
    out = torch.zeros(1, dtype=torch.int64, device=dev)
    flag = torch.zeros(1, dtype=torch.int32, device=dev)
    ws = torch.empty(N.workspace_size("fugal_alignment_overlap_workspace_size", n), dtype=torch.uint8, device=dev)
    N.call("fugal_alignment_overlap", source.row_pointers.data_ptr(), N.ptr(source.col_indices),
           target.row_pointers.data_ptr(), N.ptr(target.col_indices), n, a.data_ptr(), t.data_ptr(), out.data_ptr(),
           flag.data_ptr(), ws.data_ptr(), ws.numel(), N.stream_handle(dev))
    f = int(flag.item())
    if f & 2:
        raise ValueError("truth mapping has entries outside 0..n-1")
    if f & 1:  # not a permutation: the reference's dense definition
        return _dense_overlap(source.as_dense(torch.float32).cpu().numpy(), target.as_dense(torch.float32).cpu().numpy(),
                              a.cpu().numpy(), t.cpu().numpy())
    return int(out.item()), int(source.col_indices.numel()), int(target.col_indices.numel())


def _counts(source_adjacency, target_adjacency, source_mapping, target_mapping):
    if isinstance(source_adjacency, Adjacency):
        return overlap(source_adjacency, target_adjacency, source_mapping, target_mapping)
    return _dense_overlap(np.asarray(source_adjacency), np.asarray(target_adjacency),
                          np.asarray(source_mapping), np.asarray(target_mapping))


def edge_correctness(source_adjacency, target_adjacency, source_mapping, target_mapping) -> float:
    inter, na, _ = _counts(source_adjacency, target_adjacency, source_mapping, target_mapping)
    return inter / na if na else 0.0


def induced_conserved_structure(source_adjacency, target_adjacency, source_mapping, target_mapping) -> float:
    inter, _, nb = _counts(source_adjacency, target_adjacency, source_mapping, target_mapping)
    return inter / nb if nb else 0.0


def symmetric_substructure(source_adjacency, target_adjacency, source_mapping, target_mapping) -> float:
    inter, na, nb = _counts(source_adjacency, target_adjacency, source_mapping, target_mapping)
    den = na + nb - inter
    return inter / den if den else 0.0


def alignment_accuracy(ground_truth, mapping) -> float:
    return float(np.mean(np.asarray(ground_truth) == np.asarray(mapping)))


@dataclass
class Result:
    """``benchmark/experiment.py:340-368`` (ics, ec, sss, accuracy, profile)."""
    ics: float
    ec: float
    sss: float
    accuracy: float
    profile: object

    @classmethod
    def calculate(cls, profile, source_adjacency, target_adjacency, answer, mapping) -> "Result":
        inter, na, nb = _counts(source_adjacency, target_adjacency, answer, mapping)
        den = na + nb - inter
        return cls(inter / nb if nb else 0.0, inter / na if na else 0.0, inter / den if den else 0.0,
                   alignment_accuracy(answer, mapping), profile)

    def to_dict(self) -> dict:
        """``benchmark/experiment.py:383-386``: the metrics plus ``profile.to_dict()``."""
        return {"ics": self.ics, "ec": self.ec, "sss": self.sss, "accuracy": self.accuracy,
                "profile": self.profile.to_dict()}

    @classmethod
    def from_dict(cls, d: dict) -> "Result":
        from .profile import Profile
        d = dict(d)
        d["profile"] = Profile.from_dict(d["profile"])
        return cls(**d)

    @staticmethod
    def average(results: list["Result"]) -> "Result":
        from .profile import Profile
        k = len(results)
        prof = Profile.average([r.profile for r in results])
        return Result(sum(r.ics for r in results) / k, sum(r.ec for r in results) / k,
                      sum(r.sss for r in results) / k, sum(r.accuracy for r in results) / k, prof)

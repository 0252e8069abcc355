"""Node features and their distances (reference ``cugal/feature_extraction.py``).

``extract_features_cuda`` runs the integer triangle-count kernel and the two
neighbour averages (``feature_extraction.py:15-38``); ``Features`` keeps the
mu-scaled source/target feature rows (``feature_extraction.py:67-108``).  The
distance matrix is never stored on the Frank-Wolfe path: the gradient kernel
recomputes ||Fs_i - Ft_j|| from the n x 4 rows.  ``add_distance`` /
``distance_matrix`` exist for callers of the reference API and use the same
direct-difference kernel (``cuda_kernels/distance.cu``) rather than
``torch.cdist``'s matrix-product expansion.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _native as N
from .adjacency import Adjacency
from .config import Config


def graph_features(adjacency: Adjacency, with_counts: bool = False):
    """(degrees, clustering[, degree_counts int32, triangle_counts int64]) of a CSR graph."""
    n = adjacency.number_of_nodes()
    dev = adjacency.row_pointers.device
    clustering = torch.empty(n, dtype=torch.float32, device=dev)
    degrees = torch.empty(n, dtype=torch.float32, device=dev)
    dc = torch.empty(n, dtype=torch.int32, device=dev) if with_counts else None
    tc = torch.empty(n, dtype=torch.int64, device=dev) if with_counts else None
    N.call("fugal_graph_features", adjacency.col_indices.data_ptr(), adjacency.row_pointers.data_ptr(), n,
           clustering.data_ptr(), degrees.data_ptr(), N.ptr(dc), N.ptr(tc), N.stream_handle(dev))
    return (degrees, clustering, dc, tc) if with_counts else (degrees, clustering)


def average_neighbor_features(adjacency: Adjacency, values: torch.Tensor) -> torch.Tensor:
    n = adjacency.number_of_nodes()
    N.require_cuda(values, "values", torch.float32)
    out = torch.empty(n, dtype=torch.float32, device=values.device)
    N.call("fugal_average_neighbor_features", adjacency.col_indices.data_ptr(), adjacency.row_pointers.data_ptr(),
           n, values.contiguous().data_ptr(), out.data_ptr(), N.stream_handle(values.device))
    return out


def extract_features_cuda(graph, config: Config) -> torch.Tensor:
    """[deg, clust, nbr_deg, nbr_clust] as an n x 4 FP32 tensor (``feature_extraction.py:15-38``)."""
    adjacency = graph if isinstance(graph, Adjacency) else Adjacency.from_graph(graph, config.device)
    degrees, clustering = graph_features(adjacency)
    if config.safe_mode:
        assert clustering.isfinite().all(), "clustering tensor has NaN values"
        assert degrees.isfinite().all(), "degrees tensor has NaN values"
    neighbor_clustering = average_neighbor_features(adjacency, clustering)
    neighbor_degrees = average_neighbor_features(adjacency, degrees)
    return torch.stack((degrees, clustering, neighbor_degrees, neighbor_clustering)).T.contiguous()


@dataclass
class Features:
    """Features of source and target graph (already multiplied by mu)."""

    source: torch.Tensor
    target: torch.Tensor

    @classmethod
    def create(cls, source, target, config: Config) -> "Features":
        """``Features.create`` (``cugal/feature_extraction.py:74-96``)."""
        if "cuda" not in config.device:
            raise ValueError("Features.create: only CUDA devices are supported")
        s = extract_features_cuda(source, config)
        t = extract_features_cuda(target, config)
        if config.safe_mode:
            assert s.isfinite().all(), "source feature tensor has NaN values"
            assert t.isfinite().all(), "target feature tensor has NaN values"
        s = (s * config.mu).contiguous()
        t = (t * config.mu).contiguous()
        if config.safe_mode:
            assert s.isfinite().all(), "source feature tensor has NaN values"
            assert t.isfinite().all(), "target feature tensor has NaN values"
        return cls(s, t)

    def add_distance(self, out: torch.Tensor) -> torch.Tensor:
        """out += distance matrix (``feature_extraction.py:98-104``), in place."""
        N.require_cuda(out, "out", torch.float32)
        n = out.shape[0]
        N.call("fugal_add_distance", self.source.float().contiguous().data_ptr(),
               self.target.float().contiguous().data_ptr(), n, out.data_ptr(), N.matrix_ld(out, "out"),
               N.stream_handle(out.device))
        return out

    def distance_matrix(self) -> torch.Tensor:
        """Euclidean distance matrix (``feature_extraction.py:106-108``)."""
        n = self.source.shape[0]
        out = torch.zeros((n, n), dtype=torch.float32, device=self.source.device)
        return self.add_distance(out)

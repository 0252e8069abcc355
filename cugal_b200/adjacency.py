"""Sparse adjacency (CSR) container (reference ``cugal/adjacency.py:18-156``).

Same fields and methods as the reference's ``Adjacency``.  Construction from a
networkx graph flattens the edge list on the host with numpy (the reference
builds a Python list of pairs, ``adjacency.py:50-69``), adds the reversed copy
of every edge of an undirected graph, and builds the CSR on the device with
``fugal_create_adjacency`` (count, scan, scatter, per-row sort).  ``mul`` is the
``adjacency_matmul`` kernel.  CUDA only.
"""

from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N


def edge_array(graph) -> np.ndarray:
    """int32 (x, y) pairs of ``nx.edges(graph)``, plus reversed pairs if undirected
    (``cugal/adjacency.py:50-55``)."""
    m = graph.number_of_edges()
    flat = None
    if not graph.is_directed() and not graph.is_multigraph():
        # each undirected edge once as (min, max), read straight off the adjacency dicts
        # (about a third faster than graph.edges(); the pairs are the same up to order and
        # orientation, and the CSR build sorts and adds both directions anyway)
        try:
            flat = np.fromiter(itertools.chain.from_iterable(
                (u, v) for u, nbrs in graph.adjacency() for v in nbrs if u <= v), dtype=np.int64, count=2 * m)
        except TypeError:  # labels that do not compare: the generic path reports them
            flat = None
    if flat is None:
        flat = np.fromiter((v for e in graph.edges() for v in e), dtype=np.int64, count=2 * m)
    flat = flat.reshape(-1, 2)
    if not graph.is_directed():
        flat = np.concatenate([flat, flat[:, ::-1]], axis=0)
    if flat.size and (flat.min() < 0 or flat.max() >= graph.number_of_nodes()):
        raise ValueError("node labels must be integers 0 .. n-1")
    return np.ascontiguousarray(flat, dtype=np.int32)


@dataclass
class Adjacency:
    col_indices: torch.Tensor
    """Column index of every non-zero, rows concatenated (int32)."""

    row_pointers: torch.Tensor
    """Offset of each row in ``col_indices`` (int32, n + 1 entries)."""

    @classmethod
    def from_edges(cls, edges: torch.Tensor, node_count: int) -> "Adjacency":
        """CSR from a device int32 tensor of (x, y) pairs: row y gets column x
        (``create_adjacency``, ``cuda_kernels/adjacency.cu:228-259``)."""
        N.require_cuda(edges, "edges", torch.int32)
        edges = edges.contiguous().view(-1, 2)
        m = edges.shape[0]
        dev = edges.device
        col = torch.empty(max(m, 1), dtype=torch.int32, device=dev)
        rp = torch.empty(node_count + 1, dtype=torch.int32, device=dev)
        ws = torch.empty(N.workspace_size("fugal_create_adjacency_workspace_size", m, node_count),
                         dtype=torch.uint8, device=dev)
        N.call("fugal_create_adjacency", edges.data_ptr(), m, node_count, col.data_ptr(), rp.data_ptr(),
               ws.data_ptr(), ws.numel(), N.stream_handle(dev))
        return cls(col[:m], rp)

    @classmethod
    def from_graph(cls, graph, device) -> "Adjacency":
        """Create from a networkx graph with nodes 0 .. n-1 (``cugal/adjacency.py:46-92``)."""
        if "cuda" not in str(device):
            raise ValueError("Adjacency.from_graph: only CUDA devices are supported")
        flat = edge_array(graph)
        edges = torch.from_numpy(flat).to(device, non_blocking=False)
        return cls.from_edges(edges, graph.number_of_nodes())

    @classmethod
    def from_dense(cls, dense: torch.Tensor) -> "Adjacency":
        """Create from a dense 0/1 matrix (``cugal/adjacency.py:26-44``)."""
        rows, cols = torch.nonzero(dense, as_tuple=True)
        rp = torch.zeros(len(dense) + 1, dtype=torch.int64, device=dense.device)
        rp[1:] = torch.cumsum(torch.bincount(rows, minlength=len(dense)), 0)
        return cls(cols.to(torch.int32), rp.to(torch.int32))

    def as_dense(self, dtype: torch.dtype) -> torch.Tensor:
        """Dense representation (``cugal/adjacency.py:94-106``)."""
        n = self.number_of_nodes()
        counts = (self.row_pointers[1:] - self.row_pointers[:-1]).to(torch.int64)
        rows = torch.repeat_interleave(torch.arange(n, device=counts.device), counts)
        dense = torch.zeros((n, n), dtype=dtype, device=self.col_indices.device)
        dense[rows, self.col_indices.to(torch.int64)] = 1
        return dense

    def byte_size(self) -> int:
        return 4 * len(self.col_indices) + 4 * len(self.row_pointers)

    def number_of_nodes(self) -> int:
        return len(self.row_pointers) - 1

    def number_of_edges(self) -> int:
        return len(self.col_indices)

    def validate(self):
        """Structural checks of ``cugal/adjacency.py:113-126``."""
        col = self.col_indices.cpu().numpy()
        rp = self.row_pointers.cpu().numpy()
        assert np.all(np.diff(rp) >= 0), "row_pointers isn't sorted"
        assert rp[0] == 0, "row_pointers doesn't start with 0"
        assert rp[-1] == len(col), "row_pointers doesn't end correctly"
        for r in range(len(rp) - 1):
            cols = col[rp[r]:rp[r + 1]]
            assert np.all(np.diff(cols) >= 0), "col_indices isn't sorted"
            assert np.all(cols <= self.number_of_nodes()), "invalid entries in col_indices"

    def mul(self, matrix: torch.Tensor, negate_lhs: bool = False) -> torch.Tensor:
        """self @ matrix (``cugal/adjacency.py:128-156``).  A non-contiguous
        ``matrix`` is taken to be the transpose of a contiguous one, and the
        result then has the transposed (column-major) layout, as in the reference."""
        n = self.number_of_nodes()
        assert matrix.shape[0] == n and matrix.shape[1] == n, "matrix must match size"
        N.require_cuda(matrix, "matrix", torch.float32)
        out = torch.empty_like(matrix)
        if matrix.is_contiguous():
            N.call("fugal_adjacency_matmul", self.col_indices.data_ptr(), self.row_pointers.data_ptr(), n,
                   matrix.data_ptr(), matrix.stride(0), 0, out.data_ptr(), out.stride(0), int(negate_lhs),
                   N.stream_handle(matrix.device))
        else:
            q = matrix.t()
            if not q.is_contiguous():
                q = q.contiguous()
                out = torch.empty_like(matrix.t().contiguous().t())
            N.call("fugal_adjacency_matmul", self.col_indices.data_ptr(), self.row_pointers.data_ptr(), n,
                   q.data_ptr(), q.stride(0), 1, out.data_ptr(), out.t().stride(0), int(negate_lhs),
                   N.stream_handle(matrix.device))
        return out

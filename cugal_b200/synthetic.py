"""Seeded synthetic alignment workloads (no dataset downloads).

Each workload is a source graph from a networkx generator and a target made by
relabelling the source with ``numpy.random.default_rng(seed).permutation(n)``
and then applying edge noise: remove round_down(x |E| / 2) uniformly chosen
edges and add the same number of uniformly chosen non-edges (x = the noise
fraction).  The 1000-node Newman-Watts-Strogatz case removes 1% of |E| and adds
as many.  Ground truth: source node i corresponds to target node perm[i].

Workloads (name: generator, seed, noise, Frank-Wolfe schedule, rounding):
  nws1000   newman_watts_strogatz(1000, 10, 0.1)   seed 0  1% remove + 1% add  15 x 10  SCIPY
  ba8192    barabasi_albert(8192, 5)               seed 1  5%                  15 x 10  SCIPY
  er32768   fast_gnp_random(32768, 16/32767)       seed 2  2%                  15 x 10  DOUBLE_GREEDY
  nws4096   newman_watts_strogatz(4096, 12, 0.05)  seed 3  3%                  15 x 10  SCIPY
  ba65536   barabasi_albert(65536, 8)              seed 4  2%                  10 x 10  DOUBLE_GREEDY
All use mu = 1, log-domain Sinkhorn with reg 1e-3, up to 500 sweeps, marginal
tolerance 1e-4 checked every 10 sweeps.  ``n`` can be overridden to run a
workload's generator and settings at a smaller size.
"""

from __future__ import annotations

from dataclasses import dataclass

import networkx as nx
import numpy as np


@dataclass(frozen=True)
class Workload:
    name: str
    generator: str
    n: int
    seed: int
    noise: float
    iter_count: int
    lap: str
    args: tuple = ()


WORKLOADS = {
    "nws1000": Workload("nws1000", "nws", 1000, 0, 0.01, 15, "SCIPY", (10, 0.1)),
    "ba8192": Workload("ba8192", "ba", 8192, 1, 0.05, 15, "SCIPY", (5,)),
    "er32768": Workload("er32768", "er", 32768, 2, 0.02, 15, "DOUBLE_GREEDY", (16.0,)),
    "nws4096": Workload("nws4096", "nws", 4096, 3, 0.03, 15, "SCIPY", (12, 0.05)),
    "ba65536": Workload("ba65536", "ba", 65536, 4, 0.02, 10, "DOUBLE_GREEDY", (8,)),
}


def source_graph(w: Workload, n: int | None = None) -> nx.Graph:
    n = w.n if n is None else n
    if w.generator == "nws":
        k, p = w.args
        return nx.newman_watts_strogatz_graph(n, k, p, seed=w.seed)
    if w.generator == "ba":
        return nx.barabasi_albert_graph(n, w.args[0], seed=w.seed)
    if w.generator == "er":
        return nx.fast_gnp_random_graph(n, w.args[0] / (n - 1), seed=w.seed)
    raise ValueError(w.generator)


def noisy_permuted_copy(graph: nx.Graph, rng: np.random.Generator, remove: int, add: int):
    """Relabel by a random permutation, remove `remove` edges, add `add` non-edges."""
    n = graph.number_of_nodes()
    perm = rng.permutation(n)
    edges = np.array(list(graph.edges()), dtype=np.int64).reshape(-1, 2)
    edges = perm[edges]
    keep = np.ones(len(edges), dtype=bool)
    if remove > 0:
        keep[rng.choice(len(edges), size=remove, replace=False)] = False
    edges = edges[keep]
    present = set(map(tuple, np.sort(edges, axis=1).tolist()))
    added = []
    while len(added) < add:
        u, v = rng.integers(0, n, size=2)
        a, b = (int(u), int(v)) if u < v else (int(v), int(u))
        if a == b or (a, b) in present:
            continue
        present.add((a, b))
        added.append((a, b))
    target = nx.Graph()
    target.add_nodes_from(range(n))
    target.add_edges_from(map(tuple, edges.tolist()))
    target.add_edges_from(added)
    return target, perm


def make_pair(name: str, n: int | None = None):
    """(source, target, perm, workload) for a named workload."""
    w = WORKLOADS[name]
    src = source_graph(w, n)
    m = src.number_of_edges()
    rng = np.random.default_rng(w.seed)
    if w.name == "nws1000":
        k = int(w.noise * m)
        tgt, perm = noisy_permuted_copy(src, rng, k, k)
    else:
        k = int(w.noise * m / 2)
        tgt, perm = noisy_permuted_copy(src, rng, k, k)
    return src, tgt, perm, w


def node_accuracy(mapping, perm: np.ndarray) -> float:
    cols = np.array([c for _, c in mapping])
    return float(np.mean(cols == perm[: len(cols)]))


def config_for(w: Workload, **overrides):
    """cugal_b200 Config of a workload (GPU FP32 path unless overridden)."""
    import torch
    from .config import Config, HungarianMethod, SinkhornMethod
    kw = dict(device="cuda", dtype=torch.float32, mu=1.0, iter_count=w.iter_count, frank_wolfe_iter_count=10,
              sinkhorn_method=SinkhornMethod.LOG, sinkhorn_regularization=1e-3, sinkhorn_iterations=500,
              sinkhorn_threshold=1e-4, sinkhorn_eval_freq=10, use_sparse_adjacency=True,
              hungarian_method=HungarianMethod[w.lap])
    kw.update(overrides)
    return Config(**kw)

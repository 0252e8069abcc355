"""CPU FP64 restatement of cuGAL's FUGAL Frank-Wolfe alignment path (the oracle).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never part of it.

Every function cites the reference file:line it restates (paths are relative to
the cuGAL repository).  Two reference quirks are exposed as explicit flags so a
parity test can pick "as the reference does it" or "as the algorithm intends":

* ``mutating_marginal`` (default False): ``SinkhornState.marginal_error_log``
  (``cugal/sinkhorn.py:67-74``) evaluates ``exp(K+u+v)`` *in place* on K and
  subtracts u, v after the exp, so K is corrupted for the rest of the solve.
* ``double_lambda``: ``dense_gradient`` (``cugal/pred.py:45-50``) adds the
  ``lambda*(1-2P)`` term twice; ``sparse_gradient`` (``cugal/pred.py:69-73``)
  adds it once.  The dense path of the oracle follows the dense reference (twice)
  unless told otherwise.

Parity pinned against the reference: ``tests/golden/make_golden.py`` runs the
reference's own Python functions on seeded inputs and ``tests/test_oracle_golden.py``
checks this module against those vectors.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.optimize
import scipy.sparse


# --------------------------------------------------------------------------
# Graph -> CSR                                      (cugal/adjacency.py:46-92)
# --------------------------------------------------------------------------

def csr_from_edges(edges: np.ndarray, node_count: int, undirected: bool = True):
    """CSR (row_pointers int32 [n+1], col_indices int32 [nnz]) from an edge list.

    ``Adjacency.from_graph`` adds the reversed copy of every edge of an
    undirected graph (``cugal/adjacency.py:54-55``) and sorts (row, col) pairs
    (``adjacency.py:75-83`` on CPU, a radix sort of row<<32|col in
    ``cuda_kernels/adjacency.cu:207-226`` on CUDA); columns within a row are
    therefore ascending and duplicates are kept.
    """
    edges = np.asarray(edges, dtype=np.int64).reshape(-1, 2)
    if undirected:
        edges = np.concatenate([edges, edges[:, ::-1]], axis=0)
    order = np.lexsort((edges[:, 1], edges[:, 0]))
    rows, cols = edges[order, 0], edges[order, 1]
    counts = np.bincount(rows, minlength=node_count)
    row_pointers = np.zeros(node_count + 1, dtype=np.int64)
    np.cumsum(counts, out=row_pointers[1:])
    return row_pointers.astype(np.int32), cols.astype(np.int32)


def csr_from_graph(graph):
    """``Adjacency.from_graph`` (``cugal/adjacency.py:46-92``) for an nx.Graph with 0..n-1 labels."""
    n = graph.number_of_nodes()
    edges = np.array(list(graph.edges()), dtype=np.int64).reshape(-1, 2)
    return csr_from_edges(edges, n, undirected=not graph.is_directed())


def csr_to_scipy(row_pointers, col_indices, n, dtype=np.float64):
    data = np.ones(len(col_indices), dtype=dtype)
    return scipy.sparse.csr_matrix((data, np.asarray(col_indices), np.asarray(row_pointers)), shape=(n, n))


# --------------------------------------------------------------------------
# Features                      (cuda_kernels/feature_extraction.cu:13-125)
# --------------------------------------------------------------------------

def triangle_counts(row_pointers, col_indices) -> tuple[np.ndarray, np.ndarray]:
    """Degrees and t(v) = sum over u in N(v) of |N(v) & N(u)| (twice the triangles).

    Restates ``vertex_features`` / ``intersection_size``
    (``cuda_kernels/feature_extraction.cu:13-65``): a sorted-merge intersection
    count for every CSR neighbour entry, integer arithmetic throughout.
    """
    rp = np.asarray(row_pointers, dtype=np.int64)
    col = np.asarray(col_indices, dtype=np.int64)
    n = len(rp) - 1
    deg = np.diff(rp)
    tri = np.zeros(n, dtype=np.int64)
    nbrs = [col[rp[v]:rp[v + 1]] for v in range(n)]
    for v in range(n):
        a = nbrs[v]
        total = 0
        for u in a:
            b = nbrs[u]
            # merge-count of two ascending lists, duplicates matched pairwise
            i = j = 0
            while i < len(a) and j < len(b):
                if a[i] == b[j]:
                    total += 1
                    i += 1
                    j += 1
                elif a[i] > b[j]:
                    j += 1
                else:
                    i += 1
        tri[v] = total
    return deg, tri


def clustering_from_counts(deg: np.ndarray, tri: np.ndarray) -> np.ndarray:
    """clust = t / (d(d-1)), 0 when t == 0 or d < 2 (``feature_extraction.cu:59-64``).

    ``d*(d-1)`` is an integer product converted to float; the division is the
    IEEE-rounded FP32 quotient.  (The reference compiles with
    ``--use_fast_math``, whose approximate division may differ by <= 2 ulp.)
    """
    deg = np.asarray(deg, dtype=np.int64)
    tri = np.asarray(tri, dtype=np.int64)
    denom = (deg * (deg - 1)).astype(np.float32)
    out = np.zeros(len(deg), dtype=np.float32)
    ok = (tri != 0) & (deg >= 2)
    out[ok] = tri[ok].astype(np.float32) / denom[ok]
    return out


def average_neighbor(row_pointers, col_indices, values: np.ndarray) -> np.ndarray:
    """avg[v] = (sum over CSR neighbours in CSR order, sequential FP32) / deg, 0 if deg == 0.

    Restates ``vertex_average_neighbor_features`` (``feature_extraction.cu:86-106``).
    """
    rp = np.asarray(row_pointers, dtype=np.int64)
    col = np.asarray(col_indices, dtype=np.int64)
    vals = np.asarray(values, dtype=np.float32)
    n = len(rp) - 1
    out = np.zeros(n, dtype=np.float32)
    for v in range(n):
        s = np.float32(0.0)
        for e in range(rp[v], rp[v + 1]):
            s = np.float32(s + vals[col[e]])
        d = rp[v + 1] - rp[v]
        out[v] = np.float32(0.0) if d == 0 else np.float32(s / np.float32(d))
    return out


def features_cuda_semantics(row_pointers, col_indices) -> np.ndarray:
    """[deg, clust, nbr_deg, nbr_clust] (n x 4, FP32) as ``extract_features_cuda``
    builds it (``cugal/feature_extraction.py:15-38``)."""
    deg, tri = triangle_counts(row_pointers, col_indices)
    clust = clustering_from_counts(deg, tri)
    degf = deg.astype(np.float32)
    nbr_deg = average_neighbor(row_pointers, col_indices, degf)
    nbr_clust = average_neighbor(row_pointers, col_indices, clust)
    return np.stack([degf, clust, nbr_deg, nbr_clust]).T.copy()


def features_nx_semantics(graph) -> np.ndarray:
    """``extract_features_nx`` (``cugal/feature_extraction.py:41-64``), FP64."""
    import networkx as nx
    nodes = sorted(graph.nodes())
    deg = dict(graph.degree())
    clust = nx.clustering(graph)
    degs = [deg[v] for v in nodes]
    clusts = [clust[v] for v in nodes]
    nbr_degs, nbr_clusts = [], []
    for v in nodes:
        ego = [m for m in nx.ego_graph(graph, v).nodes if m != v]
        nbr_degs.append(np.mean([deg[m] for m in ego]) if deg[v] > 0 else 0)
        nbr_clusts.append(np.mean([clust[m] for m in ego]) if deg[v] > 0 else 0)
    return np.nan_to_num(np.stack((degs, clusts, nbr_degs, nbr_clusts)).T.astype(np.float64))


def distance_matrix(source_features: np.ndarray, target_features: np.ndarray) -> np.ndarray:
    """Euclidean distances D[i,j] = ||F1_i - F2_j|| by direct differences, FP64.

    ``Features.distance_matrix`` (``cugal/feature_extraction.py:106-108``, torch.cdist)
    and ``add_distance`` (``cuda_kernels/distance.cu:11-33``).
    """
    a = np.asarray(source_features, dtype=np.float64)
    b = np.asarray(target_features, dtype=np.float64)
    diff = a[:, None, :] - b[None, :, :]
    return np.sqrt(np.sum(diff * diff, axis=-1))


# --------------------------------------------------------------------------
# Gradient                                          (cugal/pred.py:30-74)
# --------------------------------------------------------------------------

def sparse_gradient(A, B, P: np.ndarray, D: np.ndarray, lam: float) -> np.ndarray:
    """-2 A P B + D + lam (1 - 2P) for symmetric sparse A, B (``cugal/pred.py:54-74``).

    The reference computes ``B.mul(A.mul(P).T).T * -2`` (= -2 A P B for symmetric
    B), adds the distance (``add_feature_distance``, ``pred.py:30-35``), then
    ``regularize`` (``cuda_kernels/regularize.cu:10-22``): G += lam - 2 lam P.
    """
    AP = np.asarray(A @ P)
    G = -2.0 * np.asarray(B.T @ AP.T).T
    G = G + D
    G = G + (lam - lam * 2.0 * P)
    return G


def dense_gradient(A: np.ndarray, B: np.ndarray, P: np.ndarray, D: np.ndarray, lam: float,
                   double_lambda: bool = True) -> np.ndarray:
    """-A^T P B - A P B^T + D + lam(1-2P) [+ lam(1-2P) again] (``cugal/pred.py:38-51``)."""
    G = -A.T @ P @ B - A @ P @ B.T
    G = G + D + lam * (1 - 2 * P)
    if double_lambda:
        G = G + (lam - lam * 2 * P)
    return G


# --------------------------------------------------------------------------
# Sinkhorn                                          (cugal/sinkhorn.py:51-156)
# --------------------------------------------------------------------------

def logsumexp(x: np.ndarray, axis: int) -> np.ndarray:
    """torch.logsumexp semantics (max-shifted; all -inf gives -inf)."""
    m = np.max(x, axis=axis, keepdims=True)
    m_safe = np.where(np.isfinite(m), m, 0.0)
    with np.errstate(divide="ignore", over="ignore", invalid="ignore"):
        s = np.sum(np.exp(x - m_safe), axis=axis, keepdims=True)
        out = np.log(s) + m_safe
    return np.squeeze(out, axis=axis)


def lehmann_momentum(errors: list[float], momentum_start, eval_freq: int) -> float:
    """``SinkhornState.lehmann_momentum`` (``cugal/sinkhorn.py:78-88``).

    Indexes the error list with Python semantics, including negative indices
    (``errors[index - 2]`` with index == 1 reads the last element).
    """
    if momentum_start is None or len(errors) * eval_freq < momentum_start:
        return 1.0
    index = momentum_start // eval_freq
    if len(errors) < index - 1:
        return 1.0
    num, den = errors[index - 1], errors[index - 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        ratio = np.float64(num) / np.float64(den)
    ratio = min(float(ratio), 0.99)
    if math.isnan(ratio):
        ratio = 0.99
    power = 1.0 / eval_freq
    return 2.0 / (1.0 + math.sqrt(1 - ratio ** power))


@dataclass
class SinkhornResult:
    K: np.ndarray
    u: np.ndarray
    v: np.ndarray
    iteration_count: int
    errors: list = field(default_factory=list)


def marginal_error_log(K, u, v, mutate: bool) -> float:
    """Column-marginal L1 error (``cugal/sinkhorn.py:67-76``).

    ``mutate=True`` reproduces the reference method exactly: K becomes
    exp(K+u+v) - u - v *in place* and the error is taken from that.
    """
    if mutate:
        K += u[:, None]
        K += v[None, :]
        np.exp(K, out=K)
        K -= u[:, None]
        K -= v[None, :]
        return float(np.sum(np.abs(np.sum(K, axis=0) - 1)))
    return float(np.sum(np.abs(np.sum(np.exp(K + u[:, None] + v[None, :]), axis=0) - 1)))


def sinkhorn_log_solve(C: np.ndarray, u: np.ndarray, v: np.ndarray, reg: float,
                       max_iter: int, threshold: float, eval_freq: int,
                       momentum_start=None, mutating_marginal: bool = False) -> SinkhornResult:
    """``SinkhornState.solve_log`` CPU branch (``cugal/sinkhorn.py:90-120``).

    Column update then row update each iteration (both with momentum w); the
    column-marginal error is checked at iterations eval_freq, 2*eval_freq, ...
    (never at 0), after the row update.  u and v are warm starts and are
    returned updated.
    """
    K = -C / reg
    u = np.array(u, dtype=np.float64)
    v = np.array(v, dtype=np.float64)
    errors: list[float] = []
    momentum = 1.0
    iteration = 0
    for iteration in range(max_iter):
        v = v * (1 - momentum) - momentum * logsumexp(K + u[:, None], 0)
        u = u * (1 - momentum) - momentum * logsumexp(K + v[None, :], 1)
        if iteration % eval_freq == 0 and iteration != 0:
            errors.append(marginal_error_log(K, u, v, mutating_marginal))
            if errors[-1] < threshold:
                break
            momentum = lehmann_momentum(errors, momentum_start, eval_freq)
    return SinkhornResult(K, u, v, iteration + 1, errors)


M_EPS = 1e-16


def sinkhorn_standard_solve(C: np.ndarray, u: np.ndarray, v: np.ndarray, reg: float,
                            max_iter: int, threshold: float, eval_freq: int,
                            momentum_start=None) -> SinkhornResult:
    """``SinkhornState.solve_standard`` (``cugal/sinkhorn.py:122-144``): scaling form,
    error checked at iteration 0 and every eval_freq after (``sinkhorn.py:136``)."""
    K = np.exp(C / -reg)
    u = np.array(u, dtype=np.float64)
    v = np.array(v, dtype=np.float64)
    errors: list[float] = []
    momentum = 1.0
    iteration = 0
    for iteration in range(max_iter):
        v = v ** (1 - momentum) * (1 / (u @ K + M_EPS)) ** momentum
        u = u ** (1 - momentum) * (1 / (K @ v + M_EPS)) ** momentum
        if iteration % eval_freq == 0:
            errors.append(float(np.sum(np.abs(np.sum(K * v[None, :] * u[:, None], axis=0) - 1))))
            if errors[-1] < threshold:
                break
            momentum = lehmann_momentum(errors, momentum_start, eval_freq)
    return SinkhornResult(K, u, v, iteration + 1, errors)


def sinkhorn_log_step(K: np.ndarray, add: np.ndarray, out: np.ndarray, momentum: float) -> np.ndarray:
    """``sinkhorn_log_step`` (``cuda_kernels/sinkhorn_log.cu:8-66,100-114``):
    out[r] = (1-w) out[r] - w LSE_c(K[r,c] + add[c]); with |w - 1| < 1e-4 the
    plain kernel writes out[r] = -LSE."""
    lse = logsumexp(K + add[None, :], 1)
    if abs(momentum - 1.0) < 1e-4:
        return -lse
    return (1.0 - momentum) * out - momentum * lse


# --------------------------------------------------------------------------
# Frank-Wolfe update                              (cugal/pred.py:77-86,133-141)
# --------------------------------------------------------------------------

def update_quasi_permutation(P: np.ndarray, K: np.ndarray, u: np.ndarray, v: np.ndarray,
                             alpha: float, log: bool = True) -> np.ndarray:
    """P += alpha (q - P) with q = exp(K+u+v) (log) or u K v (standard); returns the
    step alpha (q - P) (``cugal/pred.py:77-86``).  P is updated in place."""
    q = np.exp(K + u[:, None] + v[None, :]) if log else K * v[None, :] * u[:, None]
    diff = alpha * (q - P)
    P += diff
    return diff


def duality_gap(G: np.ndarray, diff: np.ndarray, alpha: float) -> float:
    """|sum G * (diff / alpha)| (``cugal/pred.py:139-141``; the CUDA kernel
    ``update_quasi_permutation.cu:20-33`` sums (q-P) * (K * -reg) = (q-P) * C)."""
    return abs(float(np.sum(G * (diff / alpha))))


def apb(A, B, X: np.ndarray) -> np.ndarray:
    """A X B for sparse or dense symmetric A, B (the product ``sparse_gradient`` forms)."""
    AX = np.asarray(A @ X)
    return np.asarray(B.T @ AX.T).T


def fw_objective(A, B, P: np.ndarray, D: np.ndarray, lam_eff: float) -> float:
    """-<P, A P B> + <D, P> + lam_eff <P, 1 - P>: the objective whose gradient is
    ``sparse_gradient`` (``cugal/pred.py:54-74``) for symmetric A, B."""
    return float(-np.sum(P * apb(A, B, P)) + np.sum(D * P) + lam_eff * np.sum(P * (1.0 - P)))


def line_search_alpha(g: float, Q: float) -> float:
    """argmin over a in [0, 1] of a g + a^2 Q."""
    if Q > 0:
        return min(1.0, max(0.0, -g / (2.0 * Q)))
    return 1.0 if g + Q < 0 else 0.0


def line_search_step(A, B, P: np.ndarray, G: np.ndarray, q: np.ndarray, lam_eff: float):
    """Exact line search along d = q - P (opt-in; the reference steps with
    2/(2+it), ``cugal/pred.py:133``): f(P + a d) - f(P) = a g + a^2 Q with
    g = <G, d>, Q = -<d, A d B> - lam_eff <d, d>.  Returns (a, g, Q)."""
    d = q - P
    g = float(np.sum(G * d))
    Q = -float(np.sum(d * apb(A, B, d))) - lam_eff * float(np.sum(d * d))
    return line_search_alpha(g, Q), g, Q


# --------------------------------------------------------------------------
# Rounding                          (cugal/greedy_lap.py:7-85, pred.py:151-193)
# --------------------------------------------------------------------------

def double_greedy_order(P: np.ndarray) -> np.ndarray:
    """Rows by descending row maximum (``greedy_lap.py:51-52``).  The reference's
    ``argsort(descending=True)`` is unstable; this order breaks ties by lower row
    index (a stable sort), which is the order the CUDA kernels use."""
    return np.argsort(-P.max(axis=1), kind="stable")


def greedy_lap(P: np.ndarray, method: str, order=None, uniforms=None):
    """Greedy rounding of P (mutated in place as the reference does, Q4).

    method in GREEDY, RAND, MORE_RAND, DOUBLE_GREEDY, PARALLEL_GREEDY
    (``cugal/greedy_lap.py:10-85``).  ``order`` is the random row order of
    RAND / MORE_RAND (``torch.randperm``), ``uniforms`` the ``random.uniform``
    draws of MORE_RAND divided by the row total (values in [0, 1)).
    """
    n = P.shape[1]
    taken = np.ones(n, dtype=P.dtype)
    if method == "GREEDY":
        res = []
        for r in range(P.shape[0]):
            P[r] *= taken
            m = int(np.argmax(P[r]))
            taken[m] = 0
            res.append(m)
        return np.array(res, dtype=np.int64)
    if method == "RAND" or method == "DOUBLE_GREEDY":
        if method == "DOUBLE_GREEDY":
            order = double_greedy_order(P)
        res = np.zeros(n, dtype=np.int64)
        for r in order:
            P[r] *= taken
            m = int(np.argmax(P[r]))
            taken[m] = 0
            res[r] = m
        return res
    if method == "MORE_RAND":
        res = np.zeros(n, dtype=np.int64)
        for k, r in enumerate(order):
            P[r] *= taken
            cumsum = np.cumsum(P[r])
            x = uniforms[k] * cumsum[-1]
            m = int(np.nonzero(x <= cumsum)[0][0])
            taken[m] = 0
            res[r] = m
        return res
    if method == "PARALLEL_GREEDY":
        max_values = P.max(axis=1)
        max_cols = P.argmax(axis=1)
        order = np.argsort(-max_values, kind="stable")
        half = max_values[order] > 0.5
        parallel_rows = order[half]
        res = np.zeros(n, dtype=np.int64)
        res[parallel_rows] = max_cols[parallel_rows]
        taken[max_cols[parallel_rows]] = 0
        for r in order[~half]:
            P[r] *= taken
            m = int(np.argmax(P[r]))
            taken[m] = 0
            res[r] = m
        return res
    raise ValueError(method)


def sparsity(P: np.ndarray, eps: float | None = None) -> float:
    """Fraction of entries <= machine epsilon of P's dtype (``cugal/pred.py:152-153``)."""
    eps = np.finfo(P.dtype).eps if eps is None else eps
    return float(np.sum(P <= eps)) / P.size


def hungarian(P: np.ndarray, method: str, **kw) -> np.ndarray:
    """``hungarian`` (``cugal/pred.py:151-178``) for SCIPY and the greedy methods."""
    if method == "SCIPY":
        _, cols = scipy.optimize.linear_sum_assignment(P, maximize=True)
        return cols
    return greedy_lap(P, method, **kw)


# --------------------------------------------------------------------------
# Frank-Wolfe driver                               (cugal/pred.py:89-148)
# --------------------------------------------------------------------------

@dataclass
class OracleParams:
    """The live ``Config`` fields of the path (names as in ``cugal/config.py``)."""
    sinkhorn_regularization: float = 1.0
    sinkhorn_method: str = "LOG"
    sinkhorn_iterations: int = 500
    sinkhorn_threshold: float = 1e-3
    sinkhorn_eval_freq: int = 10
    sinkhorn_momentum_start: int | None = None
    mu: float = 0.5
    iter_count: int = 15
    frank_wolfe_iter_count: int = 10
    frank_wolfe_threshold: float | None = None
    use_sparse_adjacency: bool = True
    hungarian_method: str = "SCIPY"
    mutating_marginal: bool = False
    double_lambda: bool = True   # only read by the dense gradient
    line_search: bool = False    # exact line search instead of 2/(2+it) (no reference counterpart)


@dataclass
class FWTrace:
    sinkhorn_iterations: list = field(default_factory=list)
    sinkhorn_errors: list = field(default_factory=list)
    gaps: list = field(default_factory=list)
    alphas: list = field(default_factory=list)
    frank_wolfe_iterations: int = 0


def find_quasi_permutation_matrix(A_csr, B_csr, D: np.ndarray, p: OracleParams,
                                  trace: FWTrace | None = None) -> np.ndarray:
    """``find_quasi_permutation_matrix`` (``cugal/pred.py:89-148``), FP64."""
    n = D.shape[0]
    A = csr_to_scipy(*A_csr, n)
    B = csr_to_scipy(*B_csr, n)
    if p.sinkhorn_method == "LOG":
        u, v = np.zeros(n), np.zeros(n)
    else:
        u, v = np.full(n, 1.0 / n), np.full(n, 1.0 / n)
    P = np.full((n, n), 1.0 / n)
    for lam in range(p.iter_count):
        for it in range(1, p.frank_wolfe_iter_count + 1):
            if p.use_sparse_adjacency:
                G = sparse_gradient(A, B, P, D, lam)
            else:
                G = dense_gradient(A.toarray(), B.toarray(), P, D, lam, p.double_lambda)
            if p.sinkhorn_method == "LOG":
                res = sinkhorn_log_solve(G, u, v, p.sinkhorn_regularization, p.sinkhorn_iterations,
                                         p.sinkhorn_threshold, p.sinkhorn_eval_freq,
                                         p.sinkhorn_momentum_start, p.mutating_marginal)
            else:
                res = sinkhorn_standard_solve(G, u, v, p.sinkhorn_regularization, p.sinkhorn_iterations,
                                              p.sinkhorn_threshold, p.sinkhorn_eval_freq,
                                              p.sinkhorn_momentum_start)
            u, v = res.u, res.v
            if p.line_search:
                if p.sinkhorn_method == "LOG":
                    q = np.exp(res.K + u[:, None] + v[None, :])
                else:
                    q = res.K * v[None, :] * u[:, None]
                dense_twice = not p.use_sparse_adjacency and p.double_lambda
                alpha, g, _ = line_search_step(A, B, P, G, q, lam * (2.0 if dense_twice else 1.0))
                P += alpha * (q - P)
                gap = abs(g)
            else:
                alpha = 2.0 / float(2.0 + it)
                diff = update_quasi_permutation(P, res.K, u, v, alpha, p.sinkhorn_method == "LOG")
                gap = duality_gap(G, diff, alpha)
            if trace is not None:
                trace.sinkhorn_iterations.append(res.iteration_count)
                trace.sinkhorn_errors.append(res.errors)
                trace.gaps.append(gap)
                trace.alphas.append(alpha)
                trace.frank_wolfe_iterations += 1
            if p.frank_wolfe_threshold is not None and gap < p.frank_wolfe_threshold:
                break
    return P


def pad_graphs(source, target):
    """Node padding of ``cugal()`` (``cugal/pred.py:209-212``); adds range(max label)."""
    node_count = max(max(source.nodes()), max(target.nodes()))
    source.add_nodes_from(set(range(node_count)) - set(source.nodes()))
    target.add_nodes_from(set(range(node_count)) - set(target.nodes()))


def cugal(source, target, p: OracleParams, features: str = "cuda", trace: FWTrace | None = None,
          sparsity_eps: float | None = None, **lap_kw):
    """``cugal`` (``cugal/pred.py:196-249``): returns (P, mapping, sparsity).

    ``features='cuda'`` uses the integer-count semantics of the CUDA kernels
    (``extract_features_cuda``), ``'nx'`` the networkx CPU path.
    """
    pad_graphs(source, target)
    A_csr, B_csr = csr_from_graph(source), csr_from_graph(target)
    if features == "cuda":
        F1 = features_cuda_semantics(*A_csr).astype(np.float64)
        F2 = features_cuda_semantics(*B_csr).astype(np.float64)
    else:
        F1, F2 = features_nx_semantics(source), features_nx_semantics(target)
    D = distance_matrix(p.mu * F1, p.mu * F2)
    P = find_quasi_permutation_matrix(A_csr, B_csr, D, p, trace)
    sp = sparsity(P, sparsity_eps)
    cols = hungarian(P, p.hungarian_method, **lap_kw)
    mapping = [(i, int(cols[i])) for i in range(len(P))]
    return P, mapping, sp


# ----------------------------------------------------------------- metrics
def alignment_overlap(A: np.ndarray, B: np.ndarray, answer, truth) -> tuple[int, int, int]:
    """(overlap, entries of A, entries of the permuted B) behind the metrics of
    ``benchmark/experiment.py:115-141``: adj1 = A[answer][:, answer],
    adj2 = B[truth][:, truth], overlap = #(adj1 + adj2 == 2)."""
    adj1 = A[np.asarray(answer)][:, np.asarray(answer)]
    adj2 = B[np.asarray(truth)][:, np.asarray(truth)]
    return int(np.sum(adj1 + adj2 == 2)), int(np.sum(A == 1)), int(np.sum(adj2 == 1))


def edge_correctness(A, B, answer, truth) -> float:
    """``benchmark/experiment.py:115-121``."""
    inter, na, _ = alignment_overlap(A, B, answer, truth)
    return inter / na


def induced_conserved_structure(A, B, answer, truth) -> float:
    """``benchmark/experiment.py:124-130``."""
    inter, _, nb = alignment_overlap(A, B, answer, truth)
    return inter / nb


def symmetric_substructure(A, B, answer, truth) -> float:
    """``benchmark/experiment.py:133-140``."""
    inter, na, nb = alignment_overlap(A, B, answer, truth)
    return inter / (na + nb - inter)


# ------------------------------------------------------------ differentiation
def sinkhorn_plan_log(C: np.ndarray, reg: float, max_iter: int = 5000, threshold: float = 1e-14,
                      eval_freq: int = 10) -> np.ndarray:
    """Converged plan P = exp(-C/reg + u + v) of the log-domain solve
    (``cugal/sinkhorn.py:90-120``) from zero potentials, FP64."""
    n = C.shape[0]
    res = sinkhorn_log_solve(C, np.zeros(n), np.zeros(n), reg, max_iter, threshold, eval_freq, None, False)
    return np.exp(res.K + res.u[:, None] + res.v[None, :])


def sinkhorn_implicit_adjoint(P: np.ndarray, G: np.ndarray, reg: float) -> np.ndarray:
    """dL/dC at a converged plan P for G = dL/dP (implicit differentiation of the
    unit row / column sums): solve [I P; P^T I][a; b] = [(G o P) 1; (G o P)^T 1]
    (least squares: one null vector), dL/dC = -(1/reg) P o (G - a 1^T - 1 b^T)."""
    n = P.shape[0]
    GP = G * P
    M = np.block([[np.eye(n), P], [P.T, np.eye(n)]])
    z = np.linalg.lstsq(M, np.concatenate([GP.sum(1), GP.sum(0)]), rcond=None)[0]
    return -(P * (G - z[:n, None] - z[None, n:])) / reg

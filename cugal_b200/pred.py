"""FUGAL alignment driver (reference ``cugal/pred.py``), drop-in ``cugal()``.

``cugal(source, target, config, profile)`` has the reference's signature and
return value ``(P as a host numpy array, [(i, column_i)])``.  The Frank-Wolfe
loop (``pred.py:89-148``) runs as three kernel-library calls per step, all
asynchronous on the current CUDA stream:

  gradient  ``fugal_fw_gradient_structural``  -2 A P B + D + lambda (1 - 2P), written
                                      as the absorbed Sinkhorn input K + U_i + V_j, and the
                                      solve's first column update, with A P B read from the
                                      term kept across steps (structural.py); the two-SpMM
                                      ``fugal_fw_gradient_column_stats`` when that term is
                                      off or has to be recomputed
  solve     ``fugal_sinkhorn_solve``  whole log-domain solve, decisions on device
  update    ``fugal_fw_update_collect``  P += alpha (q - P), FP64 duality gap, duals folded,
                                      the plan's nonzero entries recorded; then
                                      ``fugal_structural_scatter`` adds alpha A q B
            (``fugal_fw_direction`` + ``fugal_fw_line_search_update`` with line_search,
            which keeps the two-SpMM gradient)

The host waits inside a solve (to stop enqueuing sweeps after convergence),
once per gradient for the kept term's two flags, and, when
``frank_wolfe_threshold`` is set, for the gap.  Only CUDA devices are
supported; a CPU config raises.
"""

from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse
import scipy.sparse.csgraph
import torch

from . import _native as N
from .adjacency import Adjacency
from .config import Config, HungarianMethod, SinkhornMethod
from .feature_extraction import Features
from .exact_lap import FUGAL_ITER_LIMIT, FUGAL_OK, default_max_steps, exact_assign
from .greedy_lap import greedy_assign
from .profile import Phase, Profile, SinkhornProfile, TimeStamp
from .sinkhorn import SinkhornSolver, StandardSolver, exp_scale, padded_ld, read_record
from .structural import StructuralTerm, enabled_by_default as structural_enabled_by_default


def check_config(config: Config) -> None:
    if "cuda" not in str(config.device):
        raise ValueError("cugal_b200 runs on CUDA devices only (config.device must be 'cuda[:k]')")
    if config.sinkhorn_method not in (SinkhornMethod.LOG, SinkhornMethod.STANDARD):
        raise NotImplementedError(f"sinkhorn_method={config.sinkhorn_method.value} is not available; "
                                  "use LOG or STANDARD")
    if config.sinkhorn_method == SinkhornMethod.STANDARD and config.stream_dtype is not None:
        raise NotImplementedError("stream_dtype (reduced-precision streaming) needs sinkhorn_method=LOG")
    if config.dtype != torch.float32:
        raise NotImplementedError("config.dtype must be torch.float32 on the GPU path "
                                  "(set stream_dtype for BF16/FP16 streaming)")
    if config.stream_dtype not in N.STREAM_DTYPES:
        raise ValueError(f"unsupported stream_dtype {config.stream_dtype}")


@dataclass
class FrankWolfeEngine:
    """Device state of one alignment: P, the absorbed cost, duals, workspaces."""

    A: Adjacency
    B: Adjacency
    features: Features | torch.Tensor
    config: Config
    max_solves: int = 0
    n: int = field(init=False)

    def __post_init__(self):
        n = self.A.number_of_nodes()
        if self.B.number_of_nodes() != n:
            raise ValueError("source and target must have the same number of nodes")
        self.n = n
        dev = torch.device(self.config.device)
        self.device = dev
        self.ld = padded_ld(n)
        self.P_buf = torch.zeros((n, self.ld), dtype=torch.float32, device=dev)
        self.P_buf[:, :n] = 1.0 / n
        # padding columns [n, ld) stay zero: the sweeps need them finite
        self.cost32 = torch.zeros((n, self.ld), dtype=torch.float32, device=dev)
        self.U = torch.zeros(n, dtype=torch.float64, device=dev)
        self.V = torch.zeros(n, dtype=torch.float64, device=dev)
        self.u = torch.zeros(n, dtype=torch.float32, device=dev)
        self.v = torch.zeros(n, dtype=torch.float32, device=dev)
        self.gap = torch.zeros(1, dtype=torch.float64, device=dev)
        self.grad_ws = torch.empty(N.workspace_size("fugal_gradient_workspace_size", n), dtype=torch.uint8,
                                   device=dev)
        self.standard = self.config.sinkhorn_method == SinkhornMethod.STANDARD
        if self.standard:
            # scaling form: plain gradient C in cost32, K = exp(-C/reg), scaling vectors from 1/n
            self.K_buf = torch.zeros((n, self.ld), dtype=torch.float32, device=dev)
            self.u.fill_(1.0 / n)
            self.v.fill_(1.0 / n)
            self.solver = StandardSolver(n, self.config, dev)
        else:
            self.solver = SinkhornSolver(n, self.config, dev)
            # column statistics of the cost, written by the gradient for the solve's
            # first column update: (chunks, ld) (max, sum) pairs
            chunks = ctypes.c_int32()
            N.call("fugal_gradient_column_chunks", n, ctypes.byref(chunks))
            self.colpart = torch.empty((chunks.value, 2 * self.ld), dtype=torch.float32, device=dev)
            self.colpart_valid = False
        self.records = torch.empty((max(1, self.max_solves), N.RECORD_BYTES), dtype=torch.uint8, device=dev)
        self.solves = 0
        self.updates = 0
        self._fixed_alphas: list[float] = []
        if self.config.line_search:
            # direction q - P (padding columns stay zero: the SpMM reads whole rows),
            # the three FP64 sums and the step of every update
            self.dir_buf = torch.zeros((n, self.ld), dtype=torch.float32, device=dev)
            self.ls_sums = torch.zeros(3, dtype=torch.float64, device=dev)
            self.alphas = torch.zeros(max(1, self.max_solves), dtype=torch.float64, device=dev)
        if isinstance(self.features, Features):
            self.fs = self.features.source.float().contiguous()
            self.ft = self.features.target.float().contiguous()
            self.D = None
        else:
            self.fs = self.ft = None
            self.D = self.features.float().contiguous()
        # dense reference path adds the lambda term twice (cugal/pred.py:46-50)
        self.lambda_scale = 1.0 if self.config.use_sparse_adjacency else 2.0
        # A P B kept across steps (structural.py), made at the first gradient that uses it
        self.structural: StructuralTerm | None = None
        self._structural_on = (not self.standard and not self.config.line_search
                               and structural_enabled_by_default())

    @property
    def P(self) -> torch.Tensor:
        return self.P_buf[:, :self.n]

    def gradient(self, lam: float, out_scale: float | None = None, out: torch.Tensor | None = None,
                 absorbed: bool = True) -> torch.Tensor:
        reg = self.config.sinkhorn_regularization
        if self.standard and out is None and out_scale is None:
            C = self.gradient(lam, out_scale=1.0, out=self.cost32, absorbed=False)
            exp_scale(C, -1.0 / reg, self.K_buf)
            return C
        to_cost = out is None
        out = self.cost32 if out is None else out
        scale = (-1.0 / reg) if out_scale is None else out_scale
        if to_cost and absorbed and out_scale is None and not self.standard:
            st = self._structural_term()
            if st is not None and st.prepare(self.P_buf):
                # the Sinkhorn input from the kept A P B (one elementwise pass)
                k = st.fixed.shift()
                N.call("fugal_fw_gradient_structural", self.n, st.Mq.data_ptr(), self.ld, st.fixed.m_scale(), k,
                       self.P_buf.data_ptr(), self.ld, N.ptr(self.fs), N.ptr(self.ft), N.ptr(self.D),
                       self.n if self.D is not None else 0, float(lam), self.lambda_scale, scale, N.ptr(self.U),
                       N.ptr(self.V), out.data_ptr(), N.matrix_ld(out, "out"), self.colpart.data_ptr(), self.ld,
                       N.stream_handle(self.device))
                if k:
                    st.fixed.shifted(k)
                self.colpart_valid = True
                return out
        args = (self.n, self.A.row_pointers.data_ptr(), self.A.col_indices.data_ptr(),
                self.B.row_pointers.data_ptr(), self.B.col_indices.data_ptr(), self.P_buf.data_ptr(), self.ld,
                N.ptr(self.fs), N.ptr(self.ft), N.ptr(self.D), self.n if self.D is not None else 0,
                float(lam), self.lambda_scale, scale, N.ptr(self.U) if absorbed else None,
                N.ptr(self.V) if absorbed else None, out.data_ptr(), N.matrix_ld(out, "out"),
                self.grad_ws.data_ptr(), self.grad_ws.numel())
        if to_cost and not self.standard:
            # the solve input: also hand the solve its first column update
            N.call("fugal_fw_gradient_column_stats", *args, self.colpart.data_ptr(), self.ld,
                   N.stream_handle(self.device))
            self.colpart_valid = True
        else:
            N.call("fugal_fw_gradient", *args, N.stream_handle(self.device))
        return out

    def solve(self) -> int:
        k = self.solves
        if k >= self.records.shape[0]:
            self.records = torch.cat([self.records, torch.empty_like(self.records)])
        if self.standard:
            self.solver.solve(self.K_buf, self.u, self.v, self.records[k].data_ptr())
        else:
            self.solver.solve(self.cost32, self.u, self.v, self.records[k].data_ptr(),
                              self.colpart if self.colpart_valid else None)
            self.colpart_valid = False
        self.solves += 1
        return k

    def update(self, alpha: float, lam: float = 0.0) -> torch.Tensor:
        """P += alpha (q - P) and the duality gap; with ``config.line_search`` the
        step is the exact line-search minimiser (``alpha`` unused, ``lam`` the
        gradient's lambda)."""
        self.updates += 1
        if self.config.line_search:
            return self._line_search_update(lam)
        self._fixed_alphas.append(float(alpha))
        if self.standard:
            N.call("fugal_fw_update_standard", self.n, self.P_buf.data_ptr(), self.ld, self.K_buf.data_ptr(), self.ld,
                   self.u.data_ptr(), self.v.data_ptr(), self.cost32.data_ptr(), self.ld, float(alpha),
                   self.gap.data_ptr(), N.stream_handle(self.device))
            return self.gap
        st = self.structural
        if st is not None and st.valid:
            st.collect_update(self.P_buf, self.cost32, self.u, self.v, self.U, self.V, float(alpha),
                              float(self.config.sinkhorn_regularization), self.gap)
            return self.gap
        N.call("fugal_fw_update", self.n, self.P_buf.data_ptr(), self.ld, self.cost32.data_ptr(), self.ld,
               self.u.data_ptr(), self.v.data_ptr(), self.U.data_ptr(), self.V.data_ptr(), float(alpha),
               float(self.config.sinkhorn_regularization), self.gap.data_ptr(), 1, N.stream_handle(self.device))
        if st is not None:
            st.invalidate()
        return self.gap

    def _structural_term(self) -> StructuralTerm | None:
        """The kept A P B, allocated on first use (8 bytes per entry of P); None
        when switched off or when its buffers do not fit."""
        if self.structural is None and self._structural_on:
            try:
                self.structural = StructuralTerm(self.A, self.B, self.n, self.ld, self.device, self.grad_ws)
            except (torch.OutOfMemoryError, ValueError):
                self._structural_on = False
        return self.structural

    def _line_search_update(self, lam: float) -> torch.Tensor:
        k = self.updates - 1
        if k >= self.alphas.numel():
            self.alphas = torch.cat([self.alphas, torch.zeros_like(self.alphas)])
        stream = N.stream_handle(self.device)
        d = self.dir_buf
        if self.standard:
            N.call("fugal_fw_direction", self.n, self.P_buf.data_ptr(), self.ld, self.cost32.data_ptr(), self.ld,
                   self.K_buf.data_ptr(), self.ld, self.u.data_ptr(), self.v.data_ptr(), None, None,
                   float(self.config.sinkhorn_regularization), d.data_ptr(), self.ld, self.ls_sums.data_ptr(), 0,
                   stream)
        else:
            N.call("fugal_fw_direction", self.n, self.P_buf.data_ptr(), self.ld, self.cost32.data_ptr(), self.ld,
                   None, 0, self.u.data_ptr(), self.v.data_ptr(), self.U.data_ptr(), self.V.data_ptr(),
                   float(self.config.sinkhorn_regularization), d.data_ptr(), self.ld, self.ls_sums.data_ptr(), 1,
                   stream)
        # W = -2 A d B into cost32, which the next gradient rewrites
        W = self.cost32
        N.call("fugal_fw_gradient", self.n, self.A.row_pointers.data_ptr(), self.A.col_indices.data_ptr(),
               self.B.row_pointers.data_ptr(), self.B.col_indices.data_ptr(), d.data_ptr(), self.ld,
               None, None, None, 0, 0.0, 1.0, 1.0, None, None, W.data_ptr(), self.ld,
               self.grad_ws.data_ptr(), self.grad_ws.numel(), stream)
        N.call("fugal_fw_line_search_update", self.n, self.P_buf.data_ptr(), self.ld, d.data_ptr(), self.ld,
               W.data_ptr(), self.ld, float(lam) * self.lambda_scale, self.ls_sums.data_ptr(),
               self.alphas[k:].data_ptr(), self.gap.data_ptr(), stream)
        return self.gap

    def step_lengths(self) -> np.ndarray:
        """Steps of the updates so far (the line-search minimisers, or 2/(2+it))."""
        if self.config.line_search:
            return self.alphas[:self.updates].cpu().numpy()
        return np.asarray(self._fixed_alphas)

    def sinkhorn_profiles(self) -> list[SinkhornProfile]:
        raw = self.records[:self.solves].cpu()
        return [read_record(raw[k]) for k in range(self.solves)]


def sparse_gradient(A: Adjacency, B: Adjacency, A_transpose, B_transpose, P: torch.Tensor,
                    features: Features | torch.Tensor, iteration: int) -> torch.Tensor:
    """Plain gradient -2 A P B + D + iteration (1 - 2P) (``cugal/pred.py:54-74``), symmetric A, B."""
    if A is not A_transpose or B is not B_transpose:
        raise NotImplementedError("only undirected graphs (symmetric adjacency) are supported")
    config = Config(device=str(P.device), dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                    use_sparse_adjacency=True)
    eng = FrankWolfeEngine(A, B, features, config)
    eng.P_buf[:, :eng.n] = P
    return eng.gradient(iteration, out_scale=1.0, out=torch.empty_like(eng.P_buf), absorbed=False)[:, :eng.n]


GREEDY_METHODS = (HungarianMethod.GREEDY, HungarianMethod.DOUBLE_GREEDY, HungarianMethod.PARALLEL_GREEDY,
                  HungarianMethod.RAND, HungarianMethod.MORE_RAND)


def round_on_device(P: torch.Tensor, config: Config, profile: Profile):
    """Sparsity count and rounding; returns (count tensor, columns as a device
    tensor for the greedy methods or a host array for the scipy methods)."""
    n = P.shape[0]
    count = torch.zeros(1, dtype=torch.int64, device=P.device)
    N.call("fugal_count_le", P.data_ptr(), N.matrix_ld(P, "P"), n, float(torch.finfo(P.dtype).eps),
           count.data_ptr(), N.stream_handle(P.device))
    start_time = TimeStamp(config.device)
    method = config.hungarian_method
    if method == HungarianMethod.SCIPY:
        cols, _, status = exact_assign(P, maximize=True)
        st = int(status.item())
        if st == FUGAL_ITER_LIMIT:
            raise N.NativeError(f"fugal_exact_lap: the search exceeded {default_max_steps(n)} Dijkstra steps, "
                                "more than a shortest-augmenting-path run can take")
        if st != FUGAL_OK:
            raise N.NativeError(f"fugal_exact_lap: device status {st}")
    elif method in GREEDY_METHODS:
        cols = greedy_assign(P, method, config.lap_candidates)
    elif method == HungarianMethod.SPARSE:
        # the reference's own host algorithm (cugal/pred.py:170-177): scipy's sparse
        # matching has tie rules of its own, which a device search would not share
        host = scipy.sparse.csr_matrix(P.cpu().numpy())
        _, cols = scipy.sparse.csgraph.min_weight_full_bipartite_matching(host, maximize=True)
    else:
        raise NotImplementedError(f"hungarian_method={method.value} is not available on the GPU path")
    profile.log_time(start_time, Phase.HUNGARIAN)
    return count, cols


def hungarian(quasi_permutation: torch.Tensor, config: Config, profile: Profile) -> np.ndarray:
    """Rounding step (``cugal/pred.py:151-178``)."""
    n = quasi_permutation.shape[0]
    count, cols = round_on_device(quasi_permutation, config, profile)
    if isinstance(cols, torch.Tensor):
        cols = cols.cpu().numpy()
    profile.sparsity = int(count.item()) / (n * n)
    return cols


_STAGE_BYTES = 256 << 20
_COPY_THREADS = 8


def matrix_to_host(M: torch.Tensor) -> np.ndarray:
    """A new host numpy copy of the device matrix M (rows may be strided).

    A plain ``M.cpu()`` copies into pageable memory at about 2 GB/s here (the
    driver stages it and the fresh pages fault in one by one).  Instead, blocks of
    rows go device -> pinned staging buffer (two 256 MB buffers from torch's
    caching host allocator, so later calls reuse them) on a side stream, and
    host threads move each block into the numpy array while the next block is
    in flight."""
    from concurrent.futures import ThreadPoolExecutor
    n_rows, n_cols = M.shape
    out = np.empty((n_rows, n_cols), dtype=np.float32)
    if n_rows == 0 or n_cols == 0:
        return out
    rows = max(1, min(n_rows, _STAGE_BYTES // (n_cols * 4)))
    try:
        stages = [torch.empty((rows, n_cols), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    except RuntimeError:  # no page-locked memory to be had: the plain (slower) copy
        return M.cpu().numpy()
    copy_stream = torch.cuda.Stream(device=M.device)
    copy_stream.wait_stream(torch.cuda.current_stream(M.device))
    done = [torch.cuda.Event() for _ in range(2)]
    pending = [None, None]

    def host_copy(pool, k, r0, r1):
        done[k].synchronize()
        src = stages[k].numpy()
        bounds = np.linspace(r0, r1, _COPY_THREADS + 1).astype(int)
        parts = [pool.submit(np.copyto, out[a:b], src[a - r0:b - r0]) for a, b in zip(bounds[:-1], bounds[1:]) if b > a]
        for f in parts:
            f.result()

    with ThreadPoolExecutor(max_workers=_COPY_THREADS + 1) as pool:
        for blk, r0 in enumerate(range(0, n_rows, rows)):
            k = blk & 1
            r1 = min(n_rows, r0 + rows)
            if pending[k] is not None:
                pending[k].result()  # staging buffer k is free again
            with torch.cuda.stream(copy_stream):
                stages[k][:r1 - r0].copy_(M[r0:r1], non_blocking=True)
                done[k].record(copy_stream)
            pending[k] = pool.submit(host_copy, pool, k, r0, r1)
        for f in pending:
            if f is not None:
                f.result()
    return out


def convert_to_permutation_matrix(quasi_permutation: torch.Tensor, config: Config,
                                  profile: Profile) -> tuple[np.ndarray, list[tuple[int, int]]]:
    """(P on the host, [(i, col[i])]) (``cugal/pred.py:181-193``)."""
    cols = hungarian(quasi_permutation, config, profile)
    mapping = [(i, int(c)) for i, c in enumerate(cols)]
    return matrix_to_host(quasi_permutation), mapping


def find_quasi_permutation_matrix(A: Adjacency, B: Adjacency, features: Features | torch.Tensor,
                                  config: Config, profile: Profile) -> torch.Tensor:
    """Frank-Wolfe loop (``cugal/pred.py:89-148``)."""
    check_config(config)
    engine = FrankWolfeEngine(A, B, features, config, max_solves=config.iter_count * config.frank_wolfe_iter_count)
    solve_times = []
    for lam in range(config.iter_count):
        for it in range(1, config.frank_wolfe_iter_count + 1):
            start_time = TimeStamp(config.device)
            engine.gradient(lam)
            profile.log_time(start_time, Phase.GRADIENT)

            start_time = TimeStamp(config.device)
            engine.solve()
            end_time = TimeStamp(config.device)
            solve_times.append((start_time, end_time))
            profile.log_time(start_time, Phase.SINKHORN)

            alpha = 2.0 / float(2.0 + it)
            gap = engine.update(alpha, lam)
            profile.frank_wolfe_iterations += 1
            if config.frank_wolfe_threshold is not None and abs(float(gap.item())) < config.frank_wolfe_threshold:
                break
    for (s, e), sp in zip(solve_times, engine.sinkhorn_profiles()):
        sp.time = e.elapsed_seconds(s)
        profile.sinkhorn_profiles.append(sp)
    profile._steps.extend(float(a) for a in engine.step_lengths())
    if config.safe_mode:
        assert engine.P.isfinite().all(), "quasi_permutation tensor has NaN values"
    return engine.P


def pad_graphs(source, target) -> None:
    """Node padding of ``cugal()`` (``cugal/pred.py:209-212``), including its use of
    range(max label), which leaves the larger label itself to the graph that has it."""
    node_count = max(max(source.nodes()), max(target.nodes()))
    source.add_nodes_from(set(range(node_count)) - set(source.nodes()))
    target.add_nodes_from(set(range(node_count)) - set(target.nodes()))


def align(A: Adjacency, B: Adjacency, config: Config, profile: Profile | None = None):
    """Whole alignment on device-resident CSR graphs: features, Frank-Wolfe,
    rounding.  Returns (P view, columns, sparsity-count tensor) without any
    device-to-host copy for the greedy rounding methods."""
    check_config(config)
    profile = Profile() if profile is None else profile
    start_time = TimeStamp(config.device)
    features = Features.create(A, B, config)
    profile.log_time(start_time, Phase.FEATURE_EXTRACTION)
    P = find_quasi_permutation_matrix(A, B, features, config, profile)
    count, cols = round_on_device(P, config, profile)
    return P, cols, count


def cugal(source, target, config: Config, profile: Profile | None = None
          ) -> tuple[np.ndarray, list[tuple[int, int]]]:
    """Run the alignment (``cugal/pred.py:196-249``).

    Returns the quasi-permutation matrix (host numpy, FP32) and the mapping from
    source to target node.  ``profile`` is filled in place; unlike the reference,
    the default is a fresh Profile per call rather than one shared default."""
    check_config(config)
    profile = Profile() if profile is None else profile
    before = time.time()
    pad_graphs(source, target)
    A = Adjacency.from_graph(source, config.device)
    B = Adjacency.from_graph(target, config.device)

    start_time = TimeStamp(config.device)
    features = Features.create(A, B, config)
    profile.log_time(start_time, Phase.FEATURE_EXTRACTION)

    quasi_permutation = find_quasi_permutation_matrix(A, B, features, config, profile)
    output = convert_to_permutation_matrix(quasi_permutation, config, profile)
    if config.safe_mode:
        assert np.isfinite(output[0]).all(), "output permutation matrix has NaN values"
    profile.resolve()
    profile.time = time.time() - before
    dev = torch.device(config.device)
    profile.max_memory = torch.cuda.max_memory_allocated(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    return output

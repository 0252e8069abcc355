"""Failure detection without a GPU fault: a bounded device wait that runs out.

The row-owned 16-bit Sinkhorn sweep waits on shared-memory barriers for its
bulk copies; every wait gives up after a time limit, records
FUGAL_DEVICE_TIMEOUT in the solve state and lets the kernel drain its copies,
free its tensor memory and return.  The test arms one copy of CTA 0 for 16
bytes more than it delivers (``FUGAL_TEST_FAULT_ROW``) with a 1 ms limit
(``FUGAL_TEST_WAIT_LIMIT_NS``): the alignment must end with a clean host-side
error that names the device status, and the same context must then run a
normal alignment."""

import os
import time

import networkx as nx
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _align(n=512):
    from cugal_b200 import Profile, cugal
    from cugal_b200.config import Config, HungarianMethod, SinkhornMethod
    from cugal_b200.synthetic import noisy_permuted_copy
    g = nx.newman_watts_strogatz_graph(n, 8, 0.1, seed=21)
    h, perm = noisy_permuted_copy(g, np.random.default_rng(21), 4, 4)
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                 sinkhorn_regularization=1e-2, sinkhorn_iterations=60, sinkhorn_threshold=1e-4, sinkhorn_eval_freq=10,
                 mu=1.0, iter_count=1, frank_wolfe_iter_count=2, use_sparse_adjacency=True,
                 hungarian_method=HungarianMethod.DOUBLE_GREEDY, stream_dtype=torch.bfloat16)
    P, mapping = cugal(nx.Graph(g), nx.Graph(h), cfg, Profile())
    return P, mapping


def test_row_sweep_wait_timeout_is_reported_and_context_survives(monkeypatch):
    from cugal_b200 import _native as N
    from cugal_b200.sinkhorn import SinkhornSolver  # noqa: F401  (row sweep path is the BF16 default)
    plan = N.sinkhorn_plan(512, N.FUGAL_BF16)
    assert plan["threads"] == 512 and plan["cluster"] == 1, plan  # the row-owned kernel runs these sweeps
    P_ok, map_ok = _align()
    monkeypatch.setenv("FUGAL_TEST_FAULT_ROW", "0")
    monkeypatch.setenv("FUGAL_TEST_WAIT_LIMIT_NS", "1000000")
    t0 = time.perf_counter()
    with pytest.raises(N.NativeError, match="device status 6"):
        _align()
    torch.cuda.synchronize()
    assert time.perf_counter() - t0 < 60.0
    monkeypatch.delenv("FUGAL_TEST_FAULT_ROW")
    monkeypatch.delenv("FUGAL_TEST_WAIT_LIMIT_NS")
    # the context is intact: the same alignment runs and gives the same answer
    P2, map2 = _align()
    assert [m[1] for m in map2] == [m[1] for m in map_ok]
    np.testing.assert_array_equal(P2, P_ok)
    assert os.environ.get("FUGAL_TEST_FAULT_ROW") is None


def test_safe_mode_rejects_nonfinite_features():
    """Host-injected fault: a NaN feature weight with safe_mode set stops the
    alignment with the reference's assertion (cugal/pred.py:222-224)."""
    from cugal_b200 import Profile, cugal
    from cugal_b200.config import Config, SinkhornMethod
    g = nx.newman_watts_strogatz_graph(64, 6, 0.1, seed=3)
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG, mu=float("nan"),
                 safe_mode=True, iter_count=1, frank_wolfe_iter_count=1)
    with pytest.raises(AssertionError, match="NaN"):
        cugal(nx.Graph(g), nx.Graph(g), cfg, Profile())


def test_mismatched_sizes_are_rejected_before_any_launch():
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.config import Config, SinkhornMethod
    from cugal_b200.pred import FrankWolfeEngine
    A = Adjacency.from_graph(nx.path_graph(30), "cuda")
    B = Adjacency.from_graph(nx.path_graph(31), "cuda")
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG)
    with pytest.raises(ValueError, match="same number of nodes"):
        FrankWolfeEngine(A, B, torch.zeros((30, 30), device="cuda"), cfg)

"""Device exact assignment (fugal_exact_lap) against scipy.optimize.linear_sum_assignment
on the same FP32 matrix: identical mappings, including matrices full of ties, where
the answer depends on scipy's candidate order and tie rules."""

import numpy as np
import pytest
import scipy.optimize
import torch

pytestmark = pytest.mark.gpu


def _ours(P_host, maximize=True, ld_pad=0, max_steps=None):
    from cugal_b200.exact_lap import exact_assign
    n = P_host.shape[0]
    buf = torch.zeros((n, n + ld_pad), dtype=torch.float32, device="cuda")
    buf[:, :n] = torch.tensor(P_host, device="cuda")
    cols, steps, status = exact_assign(buf[:, :n], maximize=maximize, max_steps=max_steps)
    torch.cuda.synchronize()
    return cols.cpu().numpy(), int(steps.item()), int(status.item())


def _scipy(P_host, maximize=True):
    return scipy.optimize.linear_sum_assignment(P_host.astype(np.float64), maximize=maximize)[1]


def _noisy_permutation(n, seed, noise):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(n)
    P = rng.random((n, n)) * noise / n
    P[np.arange(n), perm] += 1.0
    return P.astype(np.float32)


@pytest.mark.parametrize("case", ["uniform300", "uniform1000", "near_perm2000", "near_perm8", "constant64",
                                  "small_ints200", "binary300", "duplicate_rows120", "one"])
@pytest.mark.parametrize("maximize", [True, False])
def test_exact_lap_matches_scipy(case, maximize):
    rng = np.random.default_rng(7)
    if case == "uniform300":
        P = rng.random((300, 300)).astype(np.float32)
    elif case == "uniform1000":
        P = rng.random((1000, 1000)).astype(np.float32)
    elif case == "near_perm2000":
        # minimising over a near-permutation is a hard instance (long augmenting paths): smaller n
        P = _noisy_permutation(2000 if maximize else 400, 3, 5.0)
    elif case == "near_perm8":
        P = _noisy_permutation(8, 4, 50.0)
    elif case == "constant64":
        P = np.full((64, 64), 0.25, dtype=np.float32)
    elif case == "small_ints200":
        P = rng.integers(0, 4, size=(200, 200)).astype(np.float32)
    elif case == "binary300":
        P = (rng.random((300, 300)) < 0.02).astype(np.float32)
    elif case == "duplicate_rows120":
        base = rng.integers(0, 3, size=(40, 120)).astype(np.float32)
        P = np.repeat(base, 3, axis=0)
    else:
        P = np.array([[3.0]], dtype=np.float32)
    n = P.shape[0]
    cols, steps, status = _ours(P, maximize=maximize, ld_pad=5, max_steps=n * n + 1024)
    assert status == 0
    assert steps >= P.shape[0]
    np.testing.assert_array_equal(cols, _scipy(P, maximize=maximize))


def test_exact_lap_on_a_frank_wolfe_plan():
    """P from a real alignment (the rounding input of the SCIPY method)."""
    import networkx as nx
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.config import Config, HungarianMethod, SinkhornMethod
    from cugal_b200.pred import align
    n = 400
    g = nx.newman_watts_strogatz_graph(n, 8, 0.1, seed=11)
    h = nx.relabel_nodes(g, dict(zip(range(n), np.random.default_rng(11).permutation(n).tolist())))
    cfg = Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG, iter_count=3,
                 sinkhorn_regularization=1e-2, use_sparse_adjacency=True, hungarian_method=HungarianMethod.SCIPY)
    P, cols, _ = align(Adjacency.from_graph(g, "cuda"), Adjacency.from_graph(h, "cuda"), cfg)
    P_host = P.cpu().numpy()
    cols = cols.cpu().numpy() if isinstance(cols, torch.Tensor) else np.asarray(cols)
    np.testing.assert_array_equal(cols, _scipy(P_host))


def test_exact_lap_reports_nan_and_step_cap():
    P = np.random.default_rng(1).random((50, 50)).astype(np.float32)
    _, _, status = _ours(P, max_steps=10)
    assert status == 4  # FUGAL_ITER_LIMIT
    P[3, 7] = np.nan
    _, _, status = _ours(P)
    assert status == 5  # FUGAL_NONFINITE


def test_rounding_raises_when_the_search_exceeds_its_bound(monkeypatch):
    """The SCIPY rounding has no host fallback: a search that reaches its step
    bound (here forced down to 5 steps) is an error, not a silent scipy call."""
    import cugal_b200.exact_lap as EL
    from cugal_b200 import _native as N
    from cugal_b200.config import Config, HungarianMethod
    from cugal_b200.pred import round_on_device
    from cugal_b200.profile import Profile
    P = torch.tensor(np.random.default_rng(2).random((64, 64)).astype(np.float32), device="cuda")
    cfg = Config(device="cuda", dtype=torch.float32, hungarian_method=HungarianMethod.SCIPY)
    _, cols = round_on_device(P, cfg, Profile())
    np.testing.assert_array_equal(np.asarray(cols.cpu() if isinstance(cols, torch.Tensor) else cols),
                                  _scipy(P.cpu().numpy()))
    monkeypatch.setattr(EL, "default_max_steps", lambda n: 5)
    with pytest.raises(N.NativeError, match="Dijkstra steps"):
        round_on_device(P, cfg, Profile())

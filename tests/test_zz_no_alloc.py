"""fugal_fw_gradient_fixed_scratch (the gradient entry point that allocates
nothing) against fugal_fw_gradient with a caller workspace, through the C-ABI.

Two calls in a row on the shared scratch array: a larger graph pair first, then
a smaller one whose n is not a multiple of 4, so the second call runs on what
the first left behind.  The comparison uses the gradient tests' tolerance.
"""

import networkx as nx
import numpy as np
import pytest
import torch

from cugal_b200 import _native as N

MAX_N = 2048


def _csr(graph):
    from cugal_b200.adjacency import Adjacency
    return Adjacency.from_graph(graph, "cuda")


def _inputs(n, seed, with_features, with_duals):
    rng = np.random.default_rng(seed)
    g = nx.newman_watts_strogatz_graph(n, 8, 0.1, seed=seed)
    perm = rng.permutation(n)
    h = nx.relabel_nodes(g, dict(zip(range(n), perm.tolist())))
    A, B = _csr(g), _csr(h)
    ld = (n + 7) // 8 * 8
    P = torch.zeros((n, ld), dtype=torch.float32, device="cuda")
    P[:, :n] = torch.tensor(rng.random((n, n)) / n, dtype=torch.float32, device="cuda")
    fs = ft = D = None
    if with_features:
        fs = torch.tensor(rng.random((n, 4)) * 5, dtype=torch.float32, device="cuda")
        ft = torch.tensor(rng.random((n, 4)) * 5, dtype=torch.float32, device="cuda")
    else:
        D = torch.tensor(rng.random((n, n)) * 3, dtype=torch.float32, device="cuda")
    U = V = None
    if with_duals:
        U = torch.tensor(rng.standard_normal(n) * 1e3, dtype=torch.float64, device="cuda")
        V = torch.tensor(rng.standard_normal(n) * 1e3, dtype=torch.float64, device="cuda")
    return dict(n=n, A=A, B=B, P=P, ld=ld, fs=fs, ft=ft, D=D, U=U, V=V)


def _args(x, lam, out_scale, out):
    p = N.ptr
    return (x["n"], p(x["A"].row_pointers), p(x["A"].col_indices), p(x["B"].row_pointers), p(x["B"].col_indices),
            p(x["P"]), x["ld"], p(x["fs"]), p(x["ft"]), p(x["D"]), x["n"] if x["D"] is not None else 0,
            lam, 1.0, out_scale, p(x["U"]), p(x["V"]), p(out), x["ld"])


def _both(x, lam, out_scale):
    stream = N.stream_handle(torch.device("cuda"))
    ws = torch.empty(N.workspace_size("fugal_gradient_workspace_size", x["n"]), dtype=torch.uint8, device="cuda")
    expect = torch.full((x["n"], x["ld"]), float("nan"), dtype=torch.float32, device="cuda")
    got = torch.full_like(expect, float("nan"))
    N.call("fugal_fw_gradient", *_args(x, lam, out_scale, expect), ws.data_ptr(), ws.numel(), stream)
    N.call("fugal_fw_gradient_fixed_scratch", *_args(x, lam, out_scale, got), stream)
    torch.cuda.synchronize()
    n = x["n"]
    return got[:, :n].double().cpu(), expect[:, :n].double().cpu()


@pytest.mark.gpu
def test_fixed_scratch_gradient_matches_workspace_gradient_twice_in_a_row():
    first = _inputs(1500, 11, with_features=True, with_duals=True)
    got, expect = _both(first, lam=0.7, out_scale=-0.5)
    assert torch.isfinite(got).all()
    torch.testing.assert_close(got, expect, rtol=1e-5, atol=1e-5 * expect.abs().max().item())
    second = _inputs(301, 12, with_features=False, with_duals=False)
    got, expect = _both(second, lam=2.0, out_scale=1.0)
    assert torch.isfinite(got).all()
    torch.testing.assert_close(got, expect, rtol=1e-5, atol=1e-5 * expect.abs().max().item())


@pytest.mark.gpu
def test_fixed_scratch_gradient_at_its_size_limit():
    """n = FUGAL_FIXED_SCRATCH_MAX_N, a multiple of 4: the intermediate fills the
    scratch array exactly."""
    x = _inputs(MAX_N, 13, with_features=True, with_duals=True)
    assert MAX_N * ((MAX_N + 3) // 4 * 4) * 4 == 16 * 1024 * 1024
    got, expect = _both(x, lam=1.5, out_scale=-1.0)
    assert torch.isfinite(got).all()
    torch.testing.assert_close(got, expect, rtol=1e-5, atol=1e-5 * expect.abs().max().item())


def test_fixed_scratch_rejects_sizes_above_its_limit():
    with pytest.raises(N.NativeError, match="fixed scratch limit"):
        N.call("fugal_fw_gradient_fixed_scratch", MAX_N + 1, *([None] * 5), MAX_N + 1, None, None, None, 0,
               0.0, 1.0, 1.0, None, None, None, MAX_N + 1, None)

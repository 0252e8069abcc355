"""The oracle's implicit Sinkhorn adjoint against the reference's solve_log
differentiated by torch autograd (tests/golden/reference_adjoint.npz, written by
tests/golden/make_adjoint_golden.py) and against central finite differences."""

from pathlib import Path

import numpy as np
import pytest

from oracle import fugal_fp64 as O

GOLD = np.load(Path(__file__).resolve().parent / "golden" / "reference_adjoint.npz")


@pytest.mark.parametrize("k", [0, 1])
def test_implicit_adjoint_matches_reference_autograd(k):
    C, W, reg = GOLD[f"C{k}"], GOLD[f"W{k}"], float(GOLD[f"reg{k}"])
    P = O.sinkhorn_plan_log(C, reg)
    np.testing.assert_allclose(P, GOLD[f"P{k}"], rtol=1e-9, atol=1e-12)
    dC = O.sinkhorn_implicit_adjoint(P, W, reg)
    np.testing.assert_allclose(dC, GOLD[f"dC{k}"], rtol=1e-6, atol=1e-9)


def test_implicit_adjoint_matches_finite_differences():
    rng = np.random.default_rng(3)
    n, reg, h = 8, 0.4, 1e-6
    C = rng.random((n, n)) * 2
    W = rng.standard_normal((n, n))
    dC = O.sinkhorn_implicit_adjoint(O.sinkhorn_plan_log(C, reg), W, reg)
    fd = np.zeros_like(C)
    for i in range(n):
        for j in range(n):
            Cp, Cm = C.copy(), C.copy()
            Cp[i, j] += h
            Cm[i, j] -= h
            fd[i, j] = (np.sum(W * O.sinkhorn_plan_log(Cp, reg)) - np.sum(W * O.sinkhorn_plan_log(Cm, reg))) / (2 * h)
    np.testing.assert_allclose(dC, fd, rtol=1e-5, atol=1e-7)

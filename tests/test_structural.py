"""Host logic of the kept structural term A P B (cugal_b200/structural.py), on the CPU.

The fixed-point recurrence is restated here in integer numpy arithmetic, the way
the device kernels apply it (refresh = round(A P B 2^F); per step
Mq[i][j] += round(q_kl * factor) for i in N(k), j in N(l); the gradient reads
Mq * m_scale, then divides Mq by 2^shift), and checked against A P B formed
densely in FP64 from the same P sequence (P' = (1 - a) P + a q)."""

import math

import networkx as nx
import numpy as np
import pytest

from cugal_b200 import structural as S


def test_frac_bits_keep_values_below_2_52():
    for d in [0, 1, 2, 15, 16, 17, 1000, 65535]:
        F = S.frac_bits(d)
        bound = d * S.ROW_SUM_MAX * 2.0 ** F * 2.0 ** S.SCALE_BITS
        assert bound < 2.0 ** 52, (d, F)
        # the bound is tight: the next power of two of the degree reaches 2^52 exactly
        assert (2 ** math.ceil(math.log2(d + 1))) * S.ROW_SUM_MAX * 2.0 ** (F + S.SCALE_BITS) == 2.0 ** 52
    assert S.frac_bits(16) == 52 - 8 - 5 - 5
    with pytest.raises(ValueError):
        S.frac_bits(-1)


def test_fixed_point_schedule_rescales_by_powers_of_two():
    fp = S.FixedPoint(40)
    scales = []
    for lam in range(6):
        for it in range(1, 11):
            k = fp.shift()
            assert k == 0 or fp.scale < S.RESCALE_BELOW
            if k:
                fp.shifted(k)
                assert 0.5 < fp.scale <= 1.0
            factor = fp.step(2.0 / (2.0 + it))
            assert factor is not None
            assert fp.scale >= 2.0 ** -S.SCALE_BITS
            scales.append(fp.scale)
    assert min(scales) >= 2.0 ** -S.SCALE_BITS
    # a step that would leave the range is refused (the caller recomputes)
    fp2 = S.FixedPoint(40)
    assert fp2.step(1.0) is None and fp2.scale == 1.0
    fp2.scale = 2.0 ** -7
    assert fp2.step(0.75) is None


def _sym_csr(g, n):
    rp = np.zeros(n + 1, dtype=np.int64)
    nbrs = [sorted(g.neighbors(i)) for i in range(n)]
    rp[1:] = np.cumsum([len(x) for x in nbrs])
    return rp, np.concatenate([np.asarray(x, dtype=np.int64) for x in nbrs]) if rp[-1] else np.zeros(0, np.int64)


def _simulate(n, g, h, plans, alphas, seed):
    """Integer restatement of refresh / scatter / shift, against dense FP64 A P B."""
    A = nx.to_numpy_array(g, nodelist=range(n))
    B = nx.to_numpy_array(h, nodelist=range(n))
    a_rp, a_ci = _sym_csr(g, n)
    b_rp, b_ci = _sym_csr(h, n)
    dmax = int(np.diff(a_rp).max())
    fp = S.FixedPoint(S.frac_bits(dmax))
    P = np.full((n, n), 1.0 / n)
    Mq = np.rint(A @ P @ B * 2.0 ** fp.bits).astype(np.int64)   # refresh
    fp.refreshed()
    worst = 0.0
    for q, a in zip(plans, alphas):
        # gradient reads M at the current scale, then the optional shift
        k = fp.shift()
        M = Mq.astype(np.float64) * fp.m_scale()
        exact = A @ P @ B
        worst = max(worst, float(np.max(np.abs(M - exact))))
        if k:
            Mq = (Mq + (1 << (k - 1))) >> k
            fp.shifted(k)
        # update + scatter
        P = (1.0 - a) * P + a * q
        factor = fp.step(a)
        assert factor is not None
        rows, cols = np.nonzero(q)
        for kk, l in zip(rows, cols):
            inc = int(np.rint(q[kk, l] * factor))
            for i in a_ci[a_rp[kk]:a_rp[kk + 1]]:
                Mq[i, b_ci[b_rp[l]:b_rp[l + 1]]] += inc
        assert Mq.max() < 2 ** 52 and Mq.min() >= 0
    M = Mq.astype(np.float64) * fp.m_scale()
    worst = max(worst, float(np.max(np.abs(M - A @ P @ B))))
    return worst, fp


@pytest.mark.parametrize("seed", [0, 1])
def test_recurrence_matches_dense_product(seed):
    rng = np.random.default_rng(seed)
    n = 60
    g = nx.gnp_random_graph(n, 0.15, seed=seed)
    h = nx.relabel_nodes(g, dict(zip(range(n), rng.permutation(n))))
    plans, alphas = [], []
    for lam in range(4):
        for it in range(1, 11):
            q = np.zeros((n, n))
            perm = rng.permutation(n)
            q[np.arange(n), perm] = 1.0
            # a few rows split over two or three columns, as unconverged plans are
            for r in rng.choice(n, 5, replace=False):
                w = rng.dirichlet(np.ones(3))
                q[r] = 0.0
                q[r, rng.choice(n, 3, replace=False)] = w
            plans.append(q)
            alphas.append(2.0 / (2.0 + it))
    worst, fp = _simulate(n, g, h, plans, alphas, seed)
    # each increment is rounded to 2^-F of its scale; 40 steps, up to deg^2 adds per entry
    assert worst < 1e-9, worst
    assert fp.scale > 2.0 ** -S.SCALE_BITS


def test_hub_graph_uses_fewer_fraction_bits_and_stays_in_range():
    n = 80
    g = nx.star_graph(n - 1)
    h = nx.star_graph(n - 1)
    rng = np.random.default_rng(5)
    plans = []
    for _ in range(12):
        q = np.zeros((n, n))
        q[np.arange(n), rng.permutation(n)] = 1.0
        plans.append(q)
    worst, fp = _simulate(n, g, h, plans, [2.0 / (2.0 + it) for it in range(1, 13)], 5)
    assert fp.bits == S.frac_bits(n - 1)
    assert worst < 1e-8, worst

"""Generate golden vectors by running the reference's own Python implementation.

Run where the cuGAL reference is checked out (``CUGAL_REFERENCE``; default: a
directory ``reference`` beside this repository)::

    python tests/golden/make_golden.py

The reference imports ``cudf``, ``cugraph`` (``cugal/pred.py:8-9``) and
``matplotlib`` (``cugal/profile.py:5``) at module level; none is needed on the
CPU path, so empty stand-in modules are registered before the import.  The
reference's ``has_cuda`` flags are forced to False: with the repository root on
``sys.path`` the source directory ``cuda_kernels/`` imports as an empty
namespace package and would otherwise switch the CPU code onto CUDA branches.

The fixtures are small ``.npz`` files committed next to this script; the tests
never read the reference at run time.
"""

from __future__ import annotations

import json
import os
import random
import sys
import types
from pathlib import Path

import networkx as nx
import numpy as np
import torch

HERE = Path(__file__).resolve().parent
REF = os.environ.get("CUGAL_REFERENCE") or str(HERE.parent.parent.parent / "reference")


def import_reference():
    for name in ["cudf", "cugraph", "matplotlib", "matplotlib.pyplot"]:
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.path.insert(0, REF)
    import cugal
    import cugal.adjacency
    import cugal.feature_extraction
    import cugal.pred
    import cugal.sinkhorn
    import cugal.greedy_lap
    for mod in [cugal.adjacency, cugal.feature_extraction, cugal.pred, cugal.sinkhorn]:
        mod.has_cuda = False
    return cugal


def patched_marginal_error_log(self, K):
    # The non-mutating form the reference leaves unreachable at cugal/sinkhorn.py:76.
    Q = torch.exp(K + self.u[:, None] + self.v[None, :])
    return torch.sum(abs(torch.sum(Q, dim=0) - 1)).item()


def main():
    cugal = import_reference()
    from cugal.adjacency import Adjacency
    from cugal.config import Config, SinkhornMethod, HungarianMethod
    from cugal.feature_extraction import extract_features_nx, Features
    from cugal.greedy_lap import greedy_lap
    from cugal.pred import dense_gradient, update_quasi_permutation, cugal as ref_cugal
    from cugal.profile import Profile, SinkhornProfile
    from cugal.sinkhorn import SinkhornState

    original_marginal = SinkhornState.marginal_error_log
    out = {}

    # ---- CSR from graphs (cugal/adjacency.py:46-92, CPU branch) -------------
    graphs = {
        "nws16": nx.newman_watts_strogatz_graph(16, 7, 0.01, seed=11),
        "ba40": nx.barabasi_albert_graph(40, 3, seed=12),
        "gaps": nx.Graph([(0, 3), (3, 5), (5, 9), (1, 3), (9, 2)]),
    }
    graphs["gaps"].add_nodes_from(range(12))
    for name, g in graphs.items():
        adj = Adjacency.from_graph(g, "cpu")
        out[f"csr_{name}_edges"] = np.array(list(g.edges()), dtype=np.int64).reshape(-1, 2)
        out[f"csr_{name}_n"] = np.int64(g.number_of_nodes())
        out[f"csr_{name}_row_pointers"] = adj.row_pointers.numpy().astype(np.int64)
        out[f"csr_{name}_col_indices"] = adj.col_indices.numpy().astype(np.int64)

    # ---- networkx features (cugal/feature_extraction.py:41-64) ------------
    feat_graphs = {
        "nws32": nx.newman_watts_strogatz_graph(32, 10, 0.1, seed=13),
        "ba40": graphs["ba40"],
        "gaps": graphs["gaps"],
    }
    for name, g in feat_graphs.items():
        out[f"feat_{name}_edges"] = np.array(list(g.edges()), dtype=np.int64).reshape(-1, 2)
        out[f"feat_{name}_n"] = np.int64(g.number_of_nodes())
        out[f"feat_{name}_nx"] = extract_features_nx(g)

    # ---- distance (cugal/feature_extraction.py:106-108) ---------------------
    rng = np.random.default_rng(21)
    F1 = torch.tensor(rng.random((20, 4)) * 5)
    F2 = torch.tensor(rng.random((20, 4)) * 5)
    out["dist_F1"], out["dist_F2"] = F1.numpy(), F2.numpy()
    out["dist_D"] = Features(F1, F2).distance_matrix().numpy()

    # ---- dense gradient with the doubled lambda term (cugal/pred.py:38-51) -
    n = 14
    A = torch.tensor(nx.to_numpy_array(nx.newman_watts_strogatz_graph(n, 4, 0.2, seed=14)))
    B = torch.tensor(nx.to_numpy_array(nx.newman_watts_strogatz_graph(n, 4, 0.2, seed=15)))
    P = torch.tensor(rng.random((n, n)))
    D = torch.tensor(rng.random((n, n)))
    out["grad_A"], out["grad_B"], out["grad_P"], out["grad_D"] = A.numpy(), B.numpy(), P.numpy(), D.numpy()
    for lam in [0, 3]:
        out[f"grad_dense_l{lam}"] = dense_gradient(A, B, P.clone(), D.clone(), lam).numpy()

    # ---- Sinkhorn (cugal/sinkhorn.py:51-156) ----------------------------------
    n = 24
    C = torch.tensor(rng.random((n, n)) * 4)
    out["sk_C"] = C.numpy()
    cases = {
        "log_patched": dict(method=SinkhornMethod.LOG, reg=0.1, thr=1e-6, freq=10, mstart=None, patch=True),
        "log_mutating": dict(method=SinkhornMethod.LOG, reg=0.1, thr=1e-6, freq=10, mstart=None, patch=False),
        "log_momentum": dict(method=SinkhornMethod.LOG, reg=0.05, thr=1e-9, freq=5, mstart=10, patch=True),
        "log_momentum_neg": dict(method=SinkhornMethod.LOG, reg=0.05, thr=1e-9, freq=10, mstart=10, patch=True),
        "std": dict(method=SinkhornMethod.STANDARD, reg=0.5, thr=1e-8, freq=10, mstart=None, patch=True),
    }
    for name, c in cases.items():
        SinkhornState.marginal_error_log = patched_marginal_error_log if c["patch"] else original_marginal
        config = Config(sinkhorn_method=c["method"], sinkhorn_regularization=c["reg"],
                        sinkhorn_threshold=c["thr"], sinkhorn_eval_freq=c["freq"],
                        sinkhorn_momentum_start=c["mstart"], sinkhorn_iterations=200)
        state = SinkhornState(n, config)
        # warm start: run one solve, then a second solve on a perturbed cost
        prof = SinkhornProfile()
        K, u, v = state.solve(C.clone(), config, prof)
        out[f"sk_{name}_u1"], out[f"sk_{name}_v1"] = u.numpy().copy(), v.numpy().copy()
        out[f"sk_{name}_K1"] = K.numpy().copy()
        out[f"sk_{name}_it1"] = np.int64(prof.iteration_count)
        out[f"sk_{name}_err1"] = np.array(prof.errors, dtype=np.float64)
        C2 = C + 0.3 * torch.tensor(np.sin(np.arange(n * n)).reshape(n, n))
        prof2 = SinkhornProfile()
        K, u, v = state.solve(C2.clone(), config, prof2)
        out[f"sk_{name}_C2"] = C2.numpy()
        out[f"sk_{name}_u2"], out[f"sk_{name}_v2"] = u.numpy().copy(), v.numpy().copy()
        out[f"sk_{name}_K2"] = K.numpy().copy()
        out[f"sk_{name}_it2"] = np.int64(prof2.iteration_count)
        out[f"sk_{name}_err2"] = np.array(prof2.errors, dtype=np.float64)
        out[f"sk_{name}_params"] = np.array([c["reg"], c["thr"], c["freq"], -1 if c["mstart"] is None else c["mstart"]])
    SinkhornState.marginal_error_log = original_marginal

    # ---- update (cugal/pred.py:77-86) -----------------------------------------
    n = 16
    P = torch.tensor(rng.random((n, n)))
    K = torch.tensor(rng.normal(size=(n, n)))
    u, v = torch.tensor(rng.normal(size=n)), torch.tensor(rng.normal(size=n))
    out["upd_P"], out["upd_K"], out["upd_u"], out["upd_v"] = P.numpy(), K.numpy(), u.numpy(), v.numpy()
    for name, method in [("log", SinkhornMethod.LOG), ("std", SinkhornMethod.STANDARD)]:
        P2 = P.clone()
        q = update_quasi_permutation(P2, K.clone(), u, v, 0.4, method)
        out[f"upd_{name}_P"], out[f"upd_{name}_q"] = P2.numpy(), q.numpy()

    # ---- greedy rounding (cugal/greedy_lap.py:7-85) -----------------------------
    n = 30
    base = torch.tensor(rng.random((n, n)) ** 4)
    base[3, :] = base[3, :] * 0.0 + torch.tensor(rng.random(n)) * 1e-3
    base[7, 5] = 0.9
    base[8, 5] = 0.8
    out["lap_P"] = base.numpy()
    for method in ["GREEDY", "DOUBLE_GREEDY", "PARALLEL_GREEDY", "RAND", "MORE_RAND"]:
        cfg = Config(hungarian_method=HungarianMethod[method])
        Pm = base.clone()
        torch.manual_seed(5)
        random.seed(6)
        res = greedy_lap(Pm, cfg)
        out[f"lap_{method}_cols"] = np.array([int(x) for x in res], dtype=np.int64)
        out[f"lap_{method}_P"] = Pm.numpy()
    torch.manual_seed(5)
    out["lap_RAND_order"] = torch.randperm(n).numpy()
    torch.manual_seed(5)
    out["lap_MORE_RAND_order"] = torch.randperm(n).numpy()
    random.seed(6)
    out["lap_MORE_RAND_uniforms"] = np.array([random.random() for _ in range(n)])

    # ---- full alignment, CPU FP64 dense path (cugal/pred.py:196-249) --------
    g = nx.newman_watts_strogatz_graph(40, 6, 0.1, seed=16)
    perm = np.random.default_rng(17).permutation(40)
    h = nx.relabel_nodes(g, {i: int(perm[i]) for i in range(40)})
    h = nx.Graph(sorted(h.edges()))
    h.add_nodes_from(range(40))
    out["e2e_src_edges"] = np.array(list(g.edges()), dtype=np.int64)
    out["e2e_tgt_edges"] = np.array(list(h.edges()), dtype=np.int64)
    out["e2e_perm"] = perm
    for name, patch, lap in [("patched_scipy", True, HungarianMethod.SCIPY),
                             ("patched_dgreedy", True, HungarianMethod.DOUBLE_GREEDY),
                             ("mutating_scipy", False, HungarianMethod.SCIPY)]:
        SinkhornState.marginal_error_log = patched_marginal_error_log if patch else original_marginal
        config = Config(device="cpu", dtype=torch.float64, sinkhorn_method=SinkhornMethod.LOG,
                        sinkhorn_regularization=0.05, sinkhorn_iterations=200, sinkhorn_threshold=1e-6,
                        sinkhorn_eval_freq=10, mu=1.0, iter_count=3, frank_wolfe_iter_count=10,
                        use_sparse_adjacency=False, hungarian_method=lap)
        profile = Profile()
        src = nx.Graph(g)
        tgt = nx.Graph(h)
        Pout, mapping = ref_cugal(src, tgt, config, profile)
        out[f"e2e_{name}_P"] = Pout
        out[f"e2e_{name}_cols"] = np.array([m[1] for m in mapping], dtype=np.int64)
        out[f"e2e_{name}_sk_iters"] = np.array([p.iteration_count for p in profile.sinkhorn_profiles])
        out[f"e2e_{name}_fw"] = np.int64(profile.frank_wolfe_iterations)
        out[f"e2e_{name}_sparsity"] = np.float64(profile.sparsity)
    SinkhornState.marginal_error_log = original_marginal

    np.savez_compressed(HERE / "reference_golden.npz", **out)

    # ---- Config dictionaries (cugal/config.py:128-141) ------------------------
    configs = [Config(), Config(device="cuda", dtype=torch.float32, sinkhorn_method=SinkhornMethod.LOG,
                                sinkhorn_regularization=1e-3, use_sparse_adjacency=True, mu=1.0,
                                hungarian_method=HungarianMethod.SCIPY, frank_wolfe_threshold=0.5,
                                sinkhorn_momentum_start=20)]
    with open(HERE / "reference_configs.json", "w") as f:
        json.dump([c.to_dict() for c in configs], f, indent=1, sort_keys=True)
    print("wrote", HERE / "reference_golden.npz", len(out), "arrays")


if __name__ == "__main__":
    main()

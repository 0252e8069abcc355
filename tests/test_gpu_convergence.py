"""Why some Sinkhorn solves run to the 500-iteration cap: the FP32 floor of the
column-marginal error.

On the Barabasi-Albert n=8192 workload (m 5, seed 1, 5% noise; reg 1e-3,
tolerance 1e-4 on the L1 column error summed over n columns) the Frank-Wolfe
engine is run for a few steps; the absorbed cost of the next step (FP32, exactly
as the solve receives it) is then solved twice from the same start: by this
path (FP32 stream) and by the FP64 restatement of the reference's solve_log
(oracle/fugal_torch64.py) on the same FP32 values.  The FP64 solve reaches the
tolerance; the FP32 one cannot, because the L1 error of an FP32-evaluated plan
does not fall below a floor of about n x (FP32 rounding of a column sum), which
at n=8192 is above 1e-4 -- the same floor the reference's own FP32 GPU path
meets.  The plans agree closely once both have converged as far as they can,
so the extra iterations change the answer only at rounding level."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_capped_fp32_solve_is_the_fp32_error_floor():
    from cugal_b200.adjacency import Adjacency
    from cugal_b200.feature_extraction import Features
    from cugal_b200.pred import FrankWolfeEngine
    from cugal_b200.synthetic import WORKLOADS, config_for, make_pair
    from oracle import fugal_torch64 as T
    src, tgt, _, w = make_pair("ba8192")
    n = src.number_of_nodes()
    config = config_for(w, device="cuda")
    A, B = Adjacency.from_graph(src, "cuda"), Adjacency.from_graph(tgt, "cuda")
    eng = FrankWolfeEngine(A, B, Features.create(A, B, config), config, max_solves=16)
    for it in range(1, 6):
        eng.gradient(0.0)
        eng.solve()
        eng.update(2.0 / (2.0 + it))
    eng.gradient(0.0)
    K = eng.cost32[:, :n].double().clone()  # the solve's input, exactly
    k = eng.solve()
    torch.cuda.synchronize()
    prof = eng.sinkhorn_profiles()[k]
    u32, v32 = eng.u.double(), eng.v.double()
    P32 = torch.exp(K + u32[:, None] + v32[None, :])
    u = torch.zeros(n, dtype=torch.float64, device="cuda")
    v = torch.zeros(n, dtype=torch.float64, device="cuda")
    rec = T.sinkhorn_log_solve_(K, u, v, 500, 1e-4, 10, block=1024)
    P64 = torch.exp(K + u[:, None] + v[None, :])
    floor = n * 2.0 ** -24
    err_exact = T.marginal_error(K, u32.clone(), v32.clone(), 1024)  # the FP32 duals' error evaluated in FP64
    diff = float((P32 - P64).abs().max().item())
    print(f"\n[ba8192 step 6] FP32 stream: {prof.iteration_count} iterations, recorded errors min "
          f"{min(prof.errors):.2e} last {prof.errors[-1]:.2e}; its duals' error in FP64 {err_exact:.2e}; "
          f"FP64 solve: {rec.iterations} iterations, last error {rec.errors[-1]:.2e}; n 2^-24 = {floor:.2e}; "
          f"max|P32 - P64| {diff:.2e}")
    assert rec.iterations < 500 and rec.errors[-1] < 1e-4       # FP64 reaches the tolerance
    assert prof.iteration_count == 500                          # FP32 runs to the cap ...
    assert min(prof.errors) > 1e-4 and min(prof.errors) < 50 * floor  # ... stuck at the FP32 floor
    assert diff < 1e-3

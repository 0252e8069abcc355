"""bench.py's multi-rank logic on CPU with world size 2 (gloo): the max-over-ranks
timing and barrier that the replica bench uses, and the reference arm launched
the way a multi-GPU run launches it (torchrun), where rank 0 alone prints."""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime
    import torch
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    torch.distributed.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    bench.dist_init(world, "gloo")  # already initialised: a no-op
    bench.barrier(world)
    got = bench.max_over_ranks(1.5 + rank, world, "cpu")
    Path(out_dir, f"rank{rank}.txt").write_text(repr(got))
    torch.distributed.destroy_process_group()


def test_max_over_ranks_world_size_two(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        assert float((tmp_path / f"rank{r}.txt").read_text()) == 2.5


def test_reference_arm_under_torchrun_prints_one_line():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--workload", "nws1000",
           "--cpu-seconds", "0.3"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    res = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [ln for ln in res.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, res.stdout
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference" and rec["n_gpus"] == 2
    assert rec["cpu_baseline"]["kind"] == "port" and rec["value"] > 0
    assert rec["e2e"]["h2d_bytes_per_step"] == 0


if __name__ == "__main__":
    pytest.main([__file__, "-q"])

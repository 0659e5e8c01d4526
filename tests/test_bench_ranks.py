"""The bench's multi-GPU path is replicas only: every rank runs its own grid,
the ranks' times are reduced to the slowest, and the whole-job value counts
the cells of all ranks.  These run the host side of that path as two `gloo`
ranks on the CPU, and check that only rank 0 of the reference arm works."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

from conftest import REPO


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        slowest = bench.max_over_ranks(values[rank], dist, device="cpu")
        dist.barrier()
        value = bench.replica_value(world, 1000, 10, slowest)
        with open(os.path.join(out, f"rank{rank}.txt"), "w") as f:
            f.write(f"{slowest!r} {value!r}\n")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_on_two_gloo_ranks(tmp_path):
    values = [0.25, 0.75]
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, values, str(tmp_path)))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for r in range(2):
        slowest, value = map(float, (tmp_path / f"rank{r}.txt").read_text().split())
        assert slowest == 0.75
        # 2 replicas x 1000 cells x 10 steps in the slowest rank's time
        assert value == pytest.approx(2 * 1000 * 10 / 0.75)


def test_max_over_ranks_without_a_process_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks(1.5, None) == 1.5
    assert bench.replica_value(1, 100, 4, 2.0) == 200.0


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun every rank starts the reference arm; the ranks other
    than 0 leave at once without output (and without running the
    reference)."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "2", "--warmup", "3"],
                       capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""

"""CPU: the multi-rank plumbing of bench.py with the gloo backend
(world size 2): times are reduced to the slowest rank, and the reference arm
prints one line from rank 0 while the other rank exits without output."""
import json
import os
import subprocess
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, REPO)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    v = bench.max_over_ranks_of(1.0 + 2.5 * rank, "cpu")
    with open(os.path.join(out, f"r{rank}"), "w") as fh:
        fh.write(repr(v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    assert [float(open(tmp_path / f"r{r}").read()) for r in range(2)] == [3.5, 3.5]


def test_max_over_ranks_without_a_group():
    sys.path.insert(0, REPO)
    import bench
    assert bench.max_over_ranks_of(4.25, "cpu") == 4.25


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun():
    port = 30500 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
           "--impl", "reference", "--config", "c2", "--size", "16x16x8", "--ref-sample-iters", "1",
           "--ref-iterations", "10", "--gpus", "2", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0

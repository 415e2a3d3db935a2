"""Multi-process (world size 2, gloo on CPU) tests of the bench's replica
plumbing: the depthmap path shards by reconstruction with no exchange, so
N GPUs run N replicas; the ranks meet only at barriers and a max-reduce of
their device times, and the whole-job throughput counts every rank's maps
over the slowest rank's time."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    g = bench.Group(world, rank, backend="gloo")
    g.barrier()
    ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
    ms_max = g.max(ms)
    value = bench.replica_throughput(world, 24, 5, ms_max)
    g.barrier()
    g.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ms_max": ms_max, "value": value}, f)


def test_two_rank_max_and_throughput(tmp_path):
    torch = pytest.importorskip("torch")
    mp = torch.multiprocessing.get_context("spawn")
    port = _free_port()
    procs = [mp.Process(target=_rank_main, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for r in res:
        assert r["ms_max"] == 150.0  # every rank sees the slowest rank's time
        assert r["value"] == pytest.approx(2 * 24 * 5 / 0.150)


def test_reference_arm_under_torchrun_prints_on_rank_zero_only():
    """With N > 1 the reference arm runs on rank 0 alone; other ranks exit 0
    without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1",
               MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=120, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""

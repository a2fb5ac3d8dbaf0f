"""bench.py's multi-rank plumbing on CPU (gloo, world size 2): the timed region
is the slowest rank's, the value is the aggregate over replicas, and the
reference arm prints from rank 0 only."""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [120.0, 310.0][rank]
        t = bench.max_over_ranks(local_ms, dist)
        out[rank] = (t, bench.replica_value(world, 4, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_aggregate_value_gloo():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, 29517, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    for r in (0, 1):
        t, v = res[r]
        assert t == 310.0
        assert v == pytest.approx(2 * 4 / 0.310)


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.replica_value(1, 5, 1000.0) == pytest.approx(5.0)


@pytest.mark.parametrize("rank", [1])
def test_reference_arm_is_silent_on_other_ranks(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_line_shape_when_unavailable(tmp_path):
    # with the reference library absent the arm prints its one-line reason
    code = ("import sys, json; sys.path.insert(0, %r); import oracle.ref as r; "
            "r.LIB_PATH = %r; import bench; "
            "from libisdf_b200 import synth; "
            "a = type('A', (), dict(gpus=1, steps=1, warmup=0))(); "
            "bench.run_reference(a, synth.SI8)") % (ROOT, str(tmp_path / "missing.so"))
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120,
                       env=dict(os.environ, RANK="0", WORLD_SIZE="1"))
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line

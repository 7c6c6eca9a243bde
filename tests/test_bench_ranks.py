"""The benchmark's multi-process path on the CPU: ranks are independent
replicas, the step time is the maximum over ranks (gloo, world size 2), the
reported value is the whole job's keys/s, and the reference arm runs on rank 0
only."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.reduce_max(dist, world, times[rank], "cpu")
        dist.barrier()
        out.put((rank, ms, bench.weak_value(1000, world, ms)))
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_maximum_over_ranks_and_value_is_whole_job():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    times = [2.0, 5.0]
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, times, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [5.0, 5.0]                 # both ranks see the slowest
    assert all(abs(g[2] - 2 * 1000 / 5e-3) < 1e-6 for g in got)


def test_single_rank_reduce_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(None, 1, 3.5, "cpu") == 3.5
    assert bench.weak_value(4194304, 1, 24.0) == pytest.approx(4194304 / 24e-3)


@pytest.mark.parametrize("rank", [0, 1])
def test_reference_arm_prints_on_rank_zero_only(rank):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--workload", "records_n32", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    if rank:
        assert lines == []
    else:
        line = json.loads(lines[-1])
        assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
        assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] in ("reference", "port")

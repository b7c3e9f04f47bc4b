"""The multi-rank host logic of bench.py on the CPU: world-size-2 `gloo`
process groups over 127.0.0.1 stand in for the NCCL ranks of a
`torchrun --nproc-per-node N bench.py` launch.  The render path does not
shard (every rank renders the whole frame: replicas), so the only
cross-rank steps are the barrier before each timed region and the max over
ranks of the step time; the reported value is world x paths over that
slowest time."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, out):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        r, w, local = bench.dist_env()
        assert (r, w, local) == (rank, world, rank)
        dist.barrier()
        slowest = bench.max_over_ranks(times[rank])
        # the same collective sequence twice, as the timed and e2e regions take it
        dist.barrier()
        slowest_e2e = bench.max_over_ranks(2 * times[rank])
        out.put((rank, slowest, slowest_e2e, bench.job_rate(1920 * 1080 * 64, slowest, w)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_gloo_world2():
    world, times = 2, [12.5, 31.25]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0, p.exitcode
    got = sorted(q.get(timeout=10) for _ in range(world))
    paths = 1920 * 1080 * 64
    for rank, slowest, slowest_e2e, rate in got:
        assert slowest == max(times)
        assert slowest_e2e == 2 * max(times)
        assert rate == pytest.approx(world * paths / (max(times) / 1000) / 1e6)


def test_without_process_group():
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.job_rate(1e6, 1000.0, 1) == pytest.approx(1.0)
    assert bench.job_rate(1e6, 1000.0, 4) == pytest.approx(4.0)


@pytest.mark.parametrize("argv", [["--impl", "reference"], ["--workload", "batched"], ["--workload", "adjoint"]])
def test_other_ranks_exit_without_work(argv):
    """rank 1 of 2 of the reference arm and of the one-GPU workloads prints
    nothing and exits 0 (no process group, no device)"""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--gpus", "2", *argv], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""

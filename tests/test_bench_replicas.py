"""The N>1 plumbing of bench.py on CPU: two gloo ranks take the max of their
step times (every rank calls the reduction at the same point), the whole-job
value counts every replica, and the reference arm prints from rank 0 only."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, r, _ = bench.dist_env()
    ms = bench.max_over_ranks(10.0 + 5.0 * r, w, device="cpu")
    ms2 = bench.max_over_ranks(3.0 - r, w, device="cpu")  # same order on every rank
    dist.barrier()
    dist.destroy_process_group()
    out.put((r, w, ms, ms2))


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == [(0, 2, 15.0, 3.0), (1, 2, 15.0, 3.0)]


def test_aggregate_counts_every_replica():
    assert bench.aggregate_steps_per_s(20.0, 1) == pytest.approx(50.0)
    assert bench.aggregate_steps_per_s(20.0, 4) == pytest.approx(200.0)
    assert bench.max_over_ranks(7.5, 1) == 7.5


def test_reference_arm_prints_on_rank0_only():
    code = ("import sys; sys.argv=['bench.py','--impl','reference','--steps','1','--warmup','0'];"
            "import bench; a=bench.parse(); bench.main_reference(a, 2, 1)")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_launch_count_matches_the_profiled_step():
    """gpu_launches counts 64 kernels per chosen step on ring8_1m (35,392 tiles of 16 px over 8 views), the
    number the ncu launch list of that step shows; the plain form launches per view."""
    import bench
    assert bench.launches_per_step(35392, 8, "chosen") == 64
    # two tile-sort passes for up to 65,536 tiles; a third beyond that
    assert bench.launches_per_step(70000, 16, "chosen") == 64 + 2 * 5
    assert bench.launches_per_step(35392, 8, "plain") == 8 * (38 + 2 + 1 + 1) + 5

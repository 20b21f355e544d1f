"""bench.py's multi-process plumbing on CPU (gloo, world size 2): replicas
exchange no data; the step time is the maximum over ranks and the reported
value is the rays of all ranks over that time.  The reference arm runs on
rank 0 alone."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch

    import bench
    dev = torch.device("cpu")
    w, r = bench.dist_setup(dev)
    assert (w, r) == (world, rank)
    bench.barrier()
    # rank r took (r + 1) ms per step for the first quantity, (10 - r) for the second
    got = bench.max_over_ranks([rank + 1.0, 10.0 - rank], dev)
    rate = bench.whole_job_mrays(1_000_000, w, got[0])
    bench.dist_teardown()
    q.put((rank, got, rate))


@pytest.mark.timeout(120)
def test_max_over_ranks_and_whole_job_rate_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, got, rate in res:
        assert got == [2.0, 10.0]          # element-wise max over both ranks
        assert rate == pytest.approx(2 * 1e6 / 2e-3 / 1e6)  # 2 ranks x 1M rays / 2 ms


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl",
                          "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"],
                         env=env, capture_output=True, text=True, timeout=120)
    assert out.returncode == 0
    assert out.stdout.strip() == ""


def test_single_rank_helpers_without_a_group():
    import torch

    import bench
    assert bench.dist_setup(torch.device("cpu")) == (1, 0) or os.environ.get("WORLD_SIZE")
    assert bench.max_over_ranks([3.0, 4.0], torch.device("cpu")) == [3.0, 4.0]
    assert bench.whole_job_mrays(262144, 1, 1.0) == pytest.approx(262.144)


@pytest.mark.parametrize("workload", ["texture", "lines", "solids"])
def test_reference_arm_of_the_newer_workloads(workload):
    """bench.py --impl reference for the texture, line and solid workloads:
    one JSON line with the contract's keys from the reference's own CPU code."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--workload", workload, "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    import json
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
    assert line["e2e"]["h2d_bytes_per_step"] == 0

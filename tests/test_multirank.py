"""The multi-GPU path of bench.py on CPU: two ranks on the gloo backend.

Under torchrun every rank runs its own codewords (replicas: the path has no
data-path collective); the only cross-rank steps are the barrier and the
max-over-ranks reduction of the timed region, and the whole-job throughput is
all ranks' bytes over the slowest rank's time.  The reference arm runs on
rank 0 alone; other ranks exit without work."""
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mine = 10.0 + 5.0 * rank  # the slower rank's time must win
        dist.barrier()
        slowest = bench.max_over_ranks(mine, world, "cpu")
        out.put((rank, slowest, bench.aggregate_gbs(1e9, world, 4, slowest)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_to_the_slowest_rank():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in res] == [0, 1]
    for _, slowest, gbs in res:
        assert slowest == 15.0
        assert gbs == pytest.approx(world * 1e9 * 4 / 15.0 / 1e9)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                        "--warmup", "3"], cwd=ROOT, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""

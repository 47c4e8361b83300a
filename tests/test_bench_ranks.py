"""bench.py's multi-rank plumbing on CPU: two gloo ranks, each with its own
time, agree on the slowest one (the replica runs report max-over-ranks)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        dist.barrier()
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 15.0, 1: 15.0}


def test_max_over_ranks_single():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5


def test_reference_arm_other_ranks_exit(monkeypatch):
    """Under torchrun only rank 0 runs the CPU reference; the others return 0."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(steps=1, warmup=1, gpus=2, precision="fp32")
    assert bench.run_reference(args) == 0


def test_reference_model_extrapolation():
    """The reference arm fits t(p) = F + p P to its 1- and 2-projection samples
    and extrapolates one apply as 4 gammas x (F + 361 P)."""
    sys.path.insert(0, ROOT)
    import bench
    F, P, apply_s = bench.reference_model([(1, 10.0), (2, 12.0), (1, 10.0), (2, 12.0)])
    assert (F, P) == pytest.approx((8.0, 2.0))
    assert apply_s == pytest.approx(4 * (8.0 + 361 * 2.0))
    with pytest.raises(RuntimeError):
        bench.reference_model([(1, 10.0), (1, 11.0)])

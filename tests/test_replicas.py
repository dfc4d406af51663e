"""The multi-GPU path of bench.py (one process per GPU, replicas only) on the CPU: two ranks over
gloo on 127.0.0.1, each with its own timings.  Every rank sees the slowest rank's time (the value a
bench line divides all ranks' cell updates by), and the barrier and the teardown complete."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas(world, rank, backend="gloo", timeout_s=60)
    rep.barrier()
    one = rep.max(1.5 + rank)                                   # a time
    several = rep.max({"mixed": 3.0 - rank, "fp64": 7.0 + 2 * rank})   # times of several legs
    rep.close()
    q.put((rank, one, several))


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r for r, _, _ in results] == [0, 1]
    for _, one, several in results:
        assert one == 2.5
        assert several == {"mixed": 3.0, "fp64": 9.0}


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    rep = bench.Replicas(1, 0)
    rep.barrier()
    assert rep.max(4.0) == 4.0
    assert rep.max({"a": 1.0}) == {"a": 1.0}
    rep.close()

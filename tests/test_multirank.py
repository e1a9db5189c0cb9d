"""The replicated multi-GPU path on CPU: two gloo ranks.

bench.py runs one independent replica per GPU (the path does not shard) and reports the whole-job
throughput as the particle-steps of all ranks over the slowest rank's time.  Here two processes
on the gloo backend exercise that reduction with different per-rank times and work, and rank
failure before the reduction surfaces as an error on the other rank instead of a hang.
"""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q, fail_rank):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise SystemExit(3)  # leaves between steps: no collective of this rank is in flight
        secs, units = bench.reduce_over_ranks(1.0 + rank, 1000 * (rank + 1), device="cpu")
        q.put((rank, secs, units))
    except SystemExit:
        raise
    except Exception as e:  # the surviving rank's collective times out
        q.put((rank, "error", type(e).__name__))
    finally:
        if rank != fail_rank:
            dist.destroy_process_group()


def _run(world, fail_rank=-1):
    import random

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    out = []
    while not q.empty():
        out.append(q.get())
    for p in procs:
        if p.is_alive():
            p.kill()
    return sorted(out, key=lambda x: x[0]), [p.exitcode for p in procs]


def test_two_ranks_reduce_time_max_and_work_sum():
    out, codes = _run(2)
    assert codes == [0, 0]
    assert [o[1:] for o in out] == [(2.0, 3000.0), (2.0, 3000.0)]


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.reduce_over_ranks(1.5, 42) == (1.5, 42.0)


@pytest.mark.timeout(180)
def test_rank_that_leaves_is_reported_not_hung():
    out, codes = _run(2, fail_rank=1)
    assert codes[1] == 3
    assert out and out[0][0] == 0 and out[0][1] == "error"

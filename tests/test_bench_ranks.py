"""The multi-process path of bench.py on the host: two gloo ranks, as
torchrun starts them for `bench.py --gpus 2` (one process per GPU, each an
independent replica).  The ranks meet at the barriers around the timed
window, the job's time is the max over ranks, and the reference arm runs on
rank 0 only."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench
    r, w, local = bench.dist_init()
    bench.dist_barrier(w)
    ms = 10.0 + 5.0 * r                     # this rank's timed window
    ms_max = bench.dist_max(ms, w)
    # the reference arm: rank 0 runs it, the others return without work
    ref = bench.run_reference(None, r, w) if r != 0 else "rank0"
    bench.dist_close(w)
    out.put((r, w, local, ms_max, ref))


def test_two_gloo_ranks_barrier_and_max_over_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(k, 2, port, q)) for k in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[:3] for r in res] == [(0, 2, 0), (1, 2, 1)]
    assert all(r[3] == pytest.approx(15.0) for r in res)      # slowest rank's time on every rank
    assert res[1][4] is None                                  # rank 1 does no reference work

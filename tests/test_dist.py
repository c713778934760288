"""The multi-rank path on CPU (gloo, world size 2 and 3): row sharding covers
the batch exactly once, and per-rank results gathered with
cospdnn_b200.dist equal the single-process result (categories and per-layer
survivor counts from the FP64 oracle on each rank's shard)."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from cospdnn_b200.dist import shard_rows  # noqa: E402


def test_shard_rows_cover_batch():
    for total in (0, 1, 7, 1000, 60001):
        for world in (1, 2, 3, 8):
            ranges = [shard_rows(total, world, r) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == total
            for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
                assert a1 == b0 and a0 <= a1
            sizes = [b - a for a, b in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_rows(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=60))
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        from netgen import make_net, oracle_run
        from cospdnn_b200 import dist as cd
        csc, y0, b = make_net(1024, 6, 400, seed=61, dlo=0.2, dhi=0.4)
        r0, r1 = cd.shard_rows(len(y0), world, rank)
        local = oracle_run(csc, y0[r0:r1], b)  # this rank's rows only
        cats = cd.gather_categories(local["categories"], r0)
        alive = cd.sum_alive(local["alive"])
        t = cd.max_over_ranks(1.0 + rank)
        if rank == 0:
            q.put((cats.tolist(), alive.tolist(), t))
        dist.destroy_process_group()
    except Exception as ex:  # surface the failure to the parent
        q.put(("error", repr(ex), 0))


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_results_equal_single_process(world):
    from netgen import make_net, oracle_run
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        cats, alive, t = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.terminate()
    assert cats != "error", alive
    csc, y0, b = make_net(1024, 6, 400, seed=61, dlo=0.2, dhi=0.4)
    ref = oracle_run(csc, y0, b)
    assert len(ref["categories"]) > 0
    np.testing.assert_array_equal(cats, ref["categories"])
    np.testing.assert_array_equal(alive, ref["alive"])
    assert t == float(world)

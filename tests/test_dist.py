"""The multi-rank path on CPU (gloo, world size 2 and 3): row sharding covers
the batch exactly once, and per-rank results gathered with
cospdnn_b200.dist equal the single-process result (categories and per-layer
survivor counts from the FP64 oracle on each rank's shard).  A second test
runs each rank's host path of the reference's API mirror
(cospdnn_b200.test_graph_challenge_tc with gpu_id = rank, gpu_num = world:
its row slice, the BCSC and fuse rows handed to the engine, categories moved
to batch row ids) up to the engine, which a stand-in evaluating the FP64
oracle on exactly what it was given replaces (no GPU here)."""
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


class OracleEngine:
    """Stand-in for cospdnn_b200.Engine without a GPU: keeps what the caller
    hands over (sizes, BCSC layers with their fuse rows, input rows) and
    answers result() with the FP64 oracle run on exactly that, each BCSC
    layer folded as the engine folds it (W[fuse[start + ro]][bid*16 + co] +=
    value[co*16 + ro])."""

    def __init__(self, device=0):
        self.nets, self.layers, self.inputs = [], {}, {}

    def add_net(self, neuron, layers, rows, bias=None, threshold=1e-5, precision=1, kernel=0):
        self.nets.append(dict(neuron=neuron, layers=layers, rows=rows, bias=bias, threshold=threshold))
        return len(self.nets) - 1

    def set_layer_bcsc(self, net, layer, col_ptr, row_index, values, blocksize=16, fuse=None):
        n, bs = self.nets[net]["neuron"], blocksize
        W = np.zeros((n, n), np.float64)
        V = np.asarray(values, np.float32).reshape(-1, bs, bs)  # [block][co][ro]
        for bid in range(len(col_ptr) - 1):
            for blk in range(col_ptr[bid], col_ptr[bid + 1]):
                co, ro = np.nonzero(V[blk])
                rows = np.asarray(row_index[blk] + ro)
                src = rows if fuse is None else np.asarray(fuse)[rows]
                np.add.at(W, (src, bid * bs + co), V[blk][co, ro])
        self.layers[(net, layer)] = W

    def build(self):
        pass

    def set_input(self, net, y0, fmt=None, stream=None):
        self.inputs[net] = np.asarray(y0)

    def run(self, stream=None):
        pass

    def result(self, net, stream=None):
        from oracle import pyoracle as po
        d = self.nets[net]
        csc = []
        for l in range(d["layers"]):
            W = self.layers[(net, l)]
            r, c = np.nonzero(W)
            csc.append(po.coo_to_csc(r.astype(np.int32), c.astype(np.int32), W[r, c].astype(np.float32),
                                     d["neuron"]))
        ref = po.infer_fp64(csc, self.inputs[net], np.float32(d["bias"]), tau=d["threshold"])
        L = d["layers"]
        return dict(categories=np.nonzero(ref["death"] == L)[0].astype(np.int32),
                    alive=po.survivors_per_layer(ref["death"], L))

    def close(self):
        pass


def _bcsc_net(seed):
    """A small network in the reference's BCSC form with random fuse rows."""
    from netgen import make_net
    from oracle import pyoracle as po
    csc, y0, b = make_net(256, 5, 301, seed=seed, dlo=0.25, dhi=0.45)
    rng = np.random.default_rng(seed)
    weight, row_idx, ptr, fuse = [], [], [], []
    for cp, ri, vv in csc:
        row, col, val = po.csc_to_coo(cp, ri, vv)
        perm = rng.permutation(256).astype(np.int32)
        inv = np.argsort(perm).astype(np.int32)
        # weight row u is read from activation row fuse[u]: relabel the rows
        # so that the folded product is the original layer
        row2 = inv[row]
        bcp, bri, _, bvals = po.bcsc_greedy(row2, col, val, 16)
        weight.append(bvals)
        row_idx.append(bri)
        ptr.append(bcp)
        fuse.append(perm)
    return y0, weight, row_idx, ptr, fuse, np.float32(b), csc


def _mirror_worker(rank, world, port, q):
    try:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world,
                                timeout=__import__("datetime").timedelta(seconds=60))
        import sys
        sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
        import cospdnn_b200 as cs
        from cospdnn_b200 import dist as cd
        cs.Engine = OracleEngine  # the host path only: no GPU on this machine
        y0, weight, row_idx, ptr, fuse, b, _ = _bcsc_net(67)
        res = cs.test_graph_challenge_tc(y0, weight, row_idx, ptr, fuse, len(y0), 256, float(b),
                                         gpu_id=rank, gpu_num=world, verbose=False)
        cats = cd.gather_categories(res["categories"], 0)  # already batch row ids
        alive = cd.sum_alive(res["alive"])
        if rank == 0:
            q.put((cats.tolist(), alive.tolist()))
        dist.destroy_process_group()
    except Exception as ex:  # surface the failure to the parent
        q.put(("error", repr(ex)))


@pytest.mark.parametrize("world", [2, 3])
def test_mirror_host_path_per_rank_equals_whole_batch(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_mirror_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        cats, alive = q.get(timeout=240)
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.terminate()
    assert cats != "error", alive
    # the whole batch in one process: the same stand-in, every row at once
    # (the reference builder's greedy BCSC is what the engine folds, so the
    # expected result comes from the folded layers, not from the CSC)
    y0, weight, row_idx, ptr, fuse, b, _ = _bcsc_net(67)
    e = OracleEngine()
    e.add_net(256, len(weight), len(y0), float(b))
    for l in range(len(weight)):
        e.set_layer_bcsc(0, l, ptr[l], row_idx[l], weight[l], 16, fuse[l])
    e.set_input(0, y0)
    ref = e.result(0)
    assert len(ref["categories"]) > 0
    np.testing.assert_array_equal(cats, ref["categories"])
    np.testing.assert_array_equal(alive, ref["alive"])

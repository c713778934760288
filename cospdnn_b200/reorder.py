"""Similarity-based reordering of each layer's input rows, producing the
reordered weight files and dataset/fuse_matrix that the reference's command
line expects (README.md:9; read at src/cospdnn.cpp:14-44) and leaves to the
user to make.

The reference cuts every layer into 16x16 blocks greedily along each block
column of 16 outputs: a block starts at the first row not yet covered and
spans 16 rows (src/utils/matrix.h:1200-1269), and its kernel reads block row
r from activation row fuse[l][r] (src/kernels/kernel.cu:257-275).  Putting
rows that feed the same output block columns next to each other therefore
packs the non-zeros into fewer, denser blocks.  Here a row's signature is
the set of output block columns it feeds; rows are sorted by two seeded
MinHash values of the signature and then the signature itself, so rows with
equal signatures end up side by side and rows with similar ones (high
Jaccard similarity) close together; each group of equal signatures starts on
a 16-row boundary where rows that feed nothing can fill the gap, so blocks
come out aligned and no block of one group spills into the next (the
reference's kernel reads exactly two blocks per column,
src/kernels/kernel.cu:257).  The reordered layer is
W'[u'][v] = W[order[u']][v] with fuse[l][u'] = order[u'], the same product.
A layer keeps the identity order when the reordering does not reduce its
greedy block count.

    python -m cospdnn_b200.reorder SRC DST neuron layers [--workers N]

reads SRC/sparse-images-N.tsv and SRC/neuronN/N-l{l}.tsv (raw weights, rows =
inputs, 1-based) and writes DST with the reordered weights, the same images
and DST/fuse_matrix/neuronN/N_L_fuse.tsv; layers are reordered in N processes
(default: one per layer, up to the host's cores).
"""
import os
import shutil
import sys

import numpy as np

BLOCK = 16


def _coo(colptr, rowidx, vals):
    colptr = np.asarray(colptr, np.int64)
    col = np.repeat(np.arange(len(colptr) - 1, dtype=np.int64), np.diff(colptr))
    return np.asarray(rowidx, np.int64), col, np.asarray(vals, np.float32)


def greedy_blocks(rows, cols, neuron, block=BLOCK):
    """Number of blocks the reference's greedy builder makes for the
    non-zeros at (rows, cols) (src/utils/matrix.h:1200-1269): non-zeros in
    column-major order; a block column starts at the first column past the
    previous one and spans `block` columns; a non-zero whose row no block of
    its block column covers opens a block at that row, spanning `block` rows.

    Block columns are independent, so step t takes the t-th non-zero of every
    block column at once and tests it against that block column's starts so
    far (the walk within a block column stays in the builder's order)."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    if rows.size == 0:
        return 0
    idx = np.lexsort((rows, cols))
    r, c = rows[idx], cols[idx]
    # block column of every distinct column (a walk over columns, not non-zeros)
    ucols = np.unique(c)
    bcid = np.empty(len(ucols), np.int64)
    c0, g = None, -1
    for i, col in enumerate(ucols.tolist()):
        if c0 is None or col - c0 >= block:
            c0, g = col, g + 1
        bcid[i] = g
    gid = bcid[np.searchsorted(ucols, c)]
    gstart = np.flatnonzero(np.r_[True, gid[1:] != gid[:-1]])
    glen = np.diff(np.r_[gstart, len(r)])
    never = np.iinfo(np.int64).min // 2  # a start that covers no row
    starts = np.full((len(gstart), 8), never, np.int64)
    nstart = np.zeros(len(gstart), np.int64)
    for t in range(int(glen.max())):
        act = np.flatnonzero(glen > t)
        rr = r[gstart[act] + t]
        w = int(nstart[act].max())
        d = rr[:, None] - starts[act, :w]
        opened = act[~((d >= 0) & (d < block)).any(axis=1)] if w else act
        if opened.size:
            if int(nstart[opened].max()) >= starts.shape[1]:
                grown = np.full((len(gstart), 2 * starts.shape[1]), never, np.int64)
                grown[:, :starts.shape[1]] = starts
                starts = grown
            starts[opened, nstart[opened]] = r[gstart[opened] + t]
            nstart[opened] += 1
    return int(nstart.sum())


def mma_regions(colptr, rowidx, neuron, k=16, n=16):
    """Number of aligned k x n regions (k inputs x n outputs) holding a
    non-zero of one layer (CSC over input rows x outputs): the MMAs that a
    tensor-core layer kernel of MMA depth k and width n issues per row tile,
    whatever the fill of each region."""
    colptr = np.asarray(colptr, np.int64)
    rows = np.asarray(rowidx, np.int64)
    cols = np.repeat(np.arange(neuron, dtype=np.int64), np.diff(colptr))
    return int(np.unique((rows // k) * (neuron // n + 1) + cols // n).size)


def similarity_order(rows, cols, neuron, block=BLOCK, seed=0, align=True):
    """Row order (new position -> original row) grouping rows by the output
    block columns they feed.  With `align`, every group of rows with equal
    signatures starts on a multiple of `block`, the gaps filled with rows
    that feed nothing while such rows are left (they go last otherwise)."""
    rows = np.asarray(rows, np.int64)
    nbc = (neuron + block - 1) // block
    bc = np.asarray(cols, np.int64) // block
    key = np.unique(rows * nbc + bc)
    r, b = key // nbc, key % nbc
    rng = np.random.default_rng(seed)
    h1, h2 = rng.permutation(nbc), rng.permutation(nbc)
    starts = np.flatnonzero(np.r_[True, np.diff(r) != 0]) if len(r) else np.zeros(0, np.int64)
    present = r[starts]
    sigs = np.split(b, starts[1:]) if len(r) else []
    m1 = np.minimum.reduceat(h1[b], starts) if len(r) else []
    m2 = np.minimum.reduceat(h2[b], starts) if len(r) else []
    keyed = sorted(zip(m1, m2, (tuple(x.tolist()) for x in sigs), present.tolist()))
    empty = np.setdiff1d(np.arange(neuron), present).tolist()
    order, e, prev = [], 0, None
    for k1, k2, sig, u in keyed:
        if align and sig != prev and len(order) % block:
            fill = block - len(order) % block
            if len(empty) - e >= fill:
                order += empty[e:e + fill]
                e += fill
        order.append(u)
        prev = sig
    order += empty[e:]
    return np.asarray(order, np.int64)


def reorder_layer(colptr, rowidx, vals, neuron, block=BLOCK, seed=0, align=True):
    """Reorders one layer (CSC over input rows x outputs).  Returns
    (order, (colptr, rowidx, vals) of W', blocks before, blocks after)."""
    rows, cols, v = _coo(colptr, rowidx, vals)
    before = greedy_blocks(rows, cols, neuron, block)
    order = similarity_order(rows, cols, neuron, block, seed, align)
    pos = np.empty(neuron, np.int64)
    pos[order] = np.arange(neuron)
    after = greedy_blocks(pos[rows], cols, neuron, block)
    if after >= before:
        order, after = np.arange(neuron, dtype=np.int64), before
        pos = order
    nrows = pos[rows]
    idx = np.lexsort((nrows, cols))
    cp = np.zeros(neuron + 1, np.int32)
    np.add.at(cp, cols[idx] + 1, 1)
    cp = np.cumsum(cp).astype(np.int32)
    return order, (cp, nrows[idx].astype(np.int32), v[idx]), before, after


def reorder_network(csc_layers, neuron, block=BLOCK, seed=0):
    """Every layer: returns (reordered CSC layers, fuse rows, [(before, after)])."""
    out, fuse, stats = [], [], []
    for cp, ri, vv in csc_layers:
        order, csc, b0, b1 = reorder_layer(cp, ri, vv, neuron, block, seed)
        out.append(csc)
        fuse.append(order.astype(np.int32))
        stats.append((b0, b1))
    return out, fuse, stats


def _load_triples(path):
    """(n, 3) array of a whitespace-separated "u v val" file."""
    if os.path.getsize(path) == 0:
        return np.zeros((0, 3))
    try:
        import pandas as pd
    except ImportError:
        return np.loadtxt(path, ndmin=2)
    return pd.read_csv(path, sep=r"\s+", header=None, engine="c").to_numpy(np.float64)


def _read_layer(path, neuron):
    t = _load_triples(path)
    u, v, val = t[:, 0].astype(np.int64) - 1, t[:, 1].astype(np.int64) - 1, t[:, 2].astype(np.float32)
    if len(u) and (u.min() < 0 or u.max() >= neuron or v.min() < 0 or v.max() >= neuron):
        raise ValueError(f"{path}: index out of range")
    idx = np.lexsort((u, v))
    cp = np.zeros(neuron + 1, np.int64)
    np.add.at(cp, v[idx] + 1, 1)
    return np.cumsum(cp).astype(np.int32), u[idx].astype(np.int32), val[idx]


def _reorder_file(src, dst, neuron, l, block, seed):
    """Reads layer l of the dataset at src, writes its reordered weights under
    dst; returns (fuse row, blocks before, blocks after)."""
    name = os.path.join(f"neuron{neuron}", f"{neuron}-l{l + 1}.tsv")
    cp, ri, vv = _read_layer(os.path.join(src, name), neuron)
    order, (ncp, nri, nvv), b0, b1 = reorder_layer(cp, ri, vv, neuron, block, seed)
    col = np.repeat(np.arange(neuron), np.diff(ncp))
    with open(os.path.join(dst, name), "w") as f:
        for a, b, v in zip((nri + 1).tolist(), (col + 1).tolist(), nvv.tolist()):
            f.write(f"{a}\t{b}\t{v:.9g}\n")
    return order, b0, b1


def reorder_dataset(src, dst, neuron, layers, block=BLOCK, seed=0, workers=1):
    """Writes the reordered dataset (weights, images, fuse matrix) to dst;
    returns [(blocks before, blocks after)] per layer.  Layers are
    independent: with workers > 1 they are reordered in that many processes
    (started with spawn, so a caller that has initialised CUDA is safe); the
    files written are the same."""
    os.makedirs(os.path.join(dst, f"neuron{neuron}"), exist_ok=True)
    os.makedirs(os.path.join(dst, "fuse_matrix", f"neuron{neuron}"), exist_ok=True)
    img = f"sparse-images-{neuron}.tsv"
    if os.path.abspath(os.path.join(src, img)) != os.path.abspath(os.path.join(dst, img)):
        shutil.copyfile(os.path.join(src, img), os.path.join(dst, img))
    jobs = [(src, dst, neuron, l, block, seed) for l in range(layers)]
    if workers > 1 and layers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=min(workers, layers), mp_context=mp.get_context("spawn")) as ex:
            done = list(ex.map(_reorder_file, *zip(*jobs)))
    else:
        done = [_reorder_file(*j) for j in jobs]
    with open(os.path.join(dst, "fuse_matrix", f"neuron{neuron}", f"{neuron}_{layers}_fuse.tsv"), "w") as f:
        for order, _, _ in done:
            f.write("\t".join(str(int(x)) for x in order) + "\n")
    return [(b0, b1) for _, b0, b1 in done]


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    workers = None
    if "--workers" in argv:
        i = argv.index("--workers")
        if i + 1 >= len(argv):
            argv = []
        else:
            workers = int(argv[i + 1])
            del argv[i:i + 2]
    if len(argv) != 4:
        print("usage: python -m cospdnn_b200.reorder SRC DST neuron layers [--workers N]")
        return 1
    layers = int(argv[3])
    if workers is None:  # one process per layer, up to the host's cores
        workers = min(layers, os.cpu_count() or 1)
    try:
        stats = reorder_dataset(argv[0], argv[1], int(argv[2]), layers, workers=workers)
    except (OSError, ValueError) as e:  # missing or damaged dataset files
        print(f"reorder: {e}")
        return 1
    b0 = sum(s[0] for s in stats)
    b1 = sum(s[1] for s in stats)
    print(f"greedy 16x16 blocks: {b0} -> {b1} over {len(stats)} layers")
    return 0


if __name__ == "__main__":
    sys.exit(main())

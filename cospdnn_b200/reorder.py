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

    python -m cospdnn_b200.reorder SRC DST neuron layers

reads SRC/sparse-images-N.tsv and SRC/neuronN/N-l{l}.tsv (raw weights, rows =
inputs, 1-based) and writes DST with the reordered weights, the same images
and DST/fuse_matrix/neuronN/N_L_fuse.tsv.
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
    its block column covers opens a block at that row, spanning `block` rows."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    idx = np.lexsort((rows, cols))
    r_all, c_all = rows[idx].tolist(), cols[idx].tolist()
    total, c0, starts = 0, None, []
    for r, c in zip(r_all, c_all):
        if c0 is None or c - c0 >= block:
            c0, starts = c, []
        for s0 in starts:
            if 0 <= r - s0 < block:
                break
        else:
            starts.append(r)
            total += 1
    return total


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


def reorder_dataset(src, dst, neuron, layers, block=BLOCK, seed=0):
    """Writes the reordered dataset (weights, images, fuse matrix) to dst;
    returns [(blocks before, blocks after)] per layer."""
    os.makedirs(os.path.join(dst, f"neuron{neuron}"), exist_ok=True)
    os.makedirs(os.path.join(dst, "fuse_matrix", f"neuron{neuron}"), exist_ok=True)
    img = f"sparse-images-{neuron}.tsv"
    if os.path.abspath(os.path.join(src, img)) != os.path.abspath(os.path.join(dst, img)):
        shutil.copyfile(os.path.join(src, img), os.path.join(dst, img))
    stats, fuse = [], []
    for l in range(layers):
        name = os.path.join(f"neuron{neuron}", f"{neuron}-l{l + 1}.tsv")
        cp, ri, vv = _read_layer(os.path.join(src, name), neuron)
        order, (ncp, nri, nvv), b0, b1 = reorder_layer(cp, ri, vv, neuron, block, seed)
        col = np.repeat(np.arange(neuron), np.diff(ncp))
        with open(os.path.join(dst, name), "w") as f:
            for a, b, v in zip((nri + 1).tolist(), (col + 1).tolist(), nvv.tolist()):
                f.write(f"{a}\t{b}\t{v:.9g}\n")
        fuse.append(order)
        stats.append((b0, b1))
    with open(os.path.join(dst, "fuse_matrix", f"neuron{neuron}", f"{neuron}_{layers}_fuse.tsv"), "w") as f:
        for order in fuse:
            f.write("\t".join(str(int(x)) for x in order) + "\n")
    return stats


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if len(argv) != 4:
        print("usage: python -m cospdnn_b200.reorder SRC DST neuron layers")
        return 1
    stats = reorder_dataset(argv[0], argv[1], int(argv[2]), int(argv[3]))
    b0 = sum(s[0] for s in stats)
    b1 = sum(s[1] for s in stats)
    print(f"greedy 16x16 blocks: {b0} -> {b1} over {len(stats)} layers")
    return 0


if __name__ == "__main__":
    sys.exit(main())

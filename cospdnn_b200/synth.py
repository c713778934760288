"""Seeded synthetic networks in the shapes of the Graph Challenge sparse DNNs.

Weights W_l: 32 distinct masks m_k drawn uniformly from [0, N) per (net,
layer); W[i][i ^ m_k] = 1/16, i.e. exactly 32 nonzeros per row and column.
Inputs Y0: binary rows, row r with density U[dlo, dhi), generated on the GPU
(cospdnn_synth_input).  Streams are SplitMix64 (Steele, Lea & Flood 2014):
stream_seed(seed, kind, net, x) with kind 1 = masks (x = layer), 2 = input
rows (x = row), 3 = the multi-network mix, 4 = reference-compatible masks.
Also writes the reference's file formats (src/cospdnn.cpp:14-79).
"""
import ctypes as C
import os

import numpy as np

M64 = (1 << 64) - 1
GAMMA = 0x9E3779B97F4A7C15


def _mix(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


class SplitMix64:
    def __init__(self, state):
        self.s = state & M64

    def next(self):
        self.s = (self.s + GAMMA) & M64
        return _mix(self.s)


def stream_seed(seed, a, b, c):
    g = SplitMix64(seed ^ 0x5851F42D4C957F2D)
    x = g.next()
    g.s = x ^ ((a + 0x632BE59BD9B4E019) & M64)
    x = g.next()
    g.s = x ^ ((b + 0x9E3779B97F4A7C15) & M64)
    x = g.next()
    g.s = x ^ ((c + 0xD1B54A32D192ED03) & M64)
    return g.next()


def xor_masks(seed, net, layer, neuron, nmask=32):
    g = SplitMix64(stream_seed(seed, 1, net, layer))
    out = []
    while len(out) < nmask:
        m = g.next() % neuron
        if m not in out:
            out.append(m)
    return np.array(out, np.int32)


def r1_masks(seed, net, layer, neuron):
    """Masks {16*h0+t, 16*h1+t}: two aligned dense 16x16 blocks per block column."""
    nb = neuron // 16
    g = SplitMix64(stream_seed(seed, 4, net, layer))
    h0 = g.next() % nb
    h1 = g.next() % nb
    while h1 == h0:
        h1 = g.next() % nb
    return np.array([16 * h0 + t for t in range(16)] + [16 * h1 + t for t in range(16)], np.int32)


def masks_to_csc(masks, neuron, val=0.0625):
    """CSC (row = input, column = output): output j <- inputs j ^ m_k, ascending."""
    masks = np.asarray(masks, np.int64)
    j = np.arange(neuron, dtype=np.int64)[:, None]
    rows = np.sort(j ^ masks[None, :], axis=1).astype(np.int32)
    k = len(masks)
    colptr = (np.arange(neuron + 1, dtype=np.int64) * k).astype(np.int32)
    return colptr, rows.reshape(-1), np.full(neuron * k, val, np.float32)


def mix_config(seed, nnet=8, nchoices=(1024, 4096, 16384), lchoices=(120, 480), bmin=2000,
               bmax=60000):
    g = SplitMix64(stream_seed(seed, 3, 0, 0))
    out = []
    for _ in range(nnet):
        n = nchoices[g.next() % len(nchoices)]
        l = lchoices[g.next() % len(lchoices)]
        b = bmin + g.next() % (bmax - bmin + 1)
        out.append((int(n), int(l), int(b)))
    return out


def network(neuron, layers, seed, net=0, kind="xor"):
    """List of per-layer CSC triplets."""
    f = r1_masks if kind == "r1" else xor_masks
    return [masks_to_csc(f(seed, net, l, neuron), neuron) for l in range(layers)]


def input_rows(rows, neuron, seed, net=0, dlo=0.08, dhi=0.25, row0=0, fmt=0, device=0, stream=None):
    """Binary inputs generated on the GPU; returns a torch uint8 CUDA tensor
    [rows][neuron] (fmt 0) or packed bits [rows][neuron/8] (fmt 2)."""
    import torch

    from . import _check, _stream, lib
    cols = neuron if fmt == 0 else neuron // 8
    out = torch.empty((rows, cols), dtype=torch.uint8, device=f"cuda:{device}")
    _check(lib().cospdnn_synth_input(out.data_ptr(), rows, neuron, seed, net, row0, dlo, dhi, fmt, _stream(stream)))
    return out


def _mix64(z):
    """SplitMix64's output function on a uint64 array (wrapping arithmetic)."""
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def input_rows_host(rows, neuron, seed, net=0, dlo=0.08, dhi=0.25, row0=0, chunk=256):
    """The rows input_rows generates on the GPU, computed on the host with
    numpy (the same bytes, [rows][neuron] uint8), for machines without a GPU:
    draw 1 of row r's stream gives its density d = dlo + (dhi - dlo) * u,
    draw j + 2 gives element j = (u < d), u = (draw >> 11) * 2^-53."""
    out = np.empty((rows, neuron), np.uint8)
    g = np.uint64(GAMMA)
    draws = (np.arange(neuron, dtype=np.uint64) + np.uint64(2)) * g
    scale = 1.0 / 9007199254740992.0
    for r0 in range(0, rows, chunk):
        r1 = min(rows, r0 + chunk)
        s0 = np.array([stream_seed(seed, 2, net, row0 + r) for r in range(r0, r1)], np.uint64)
        d = dlo + (dhi - dlo) * ((_mix64(s0 + g) >> np.uint64(11)).astype(np.float64) * scale)
        u = (_mix64(s0[:, None] + draws[None, :]) >> np.uint64(11)).astype(np.float64) * scale
        out[r0:r1] = u < d[:, None]
    return out


# ---------------------------------------------------------- reference files
def write_reference_dataset(dirname, neuron, layers, y0, csc_layers, fuse=None):
    """Writes dir/sparse-images-N.tsv, dir/neuronN/N-l{l+1}.tsv and
    dir/fuse_matrix/neuronN/N_L_fuse.tsv in the reference's formats."""
    os.makedirs(os.path.join(dirname, f"neuron{neuron}"), exist_ok=True)
    os.makedirs(os.path.join(dirname, "fuse_matrix", f"neuron{neuron}"), exist_ok=True)
    y0 = np.asarray(y0)
    r, c = np.nonzero(y0)
    vals = y0[r, c].astype(np.float32).tolist()
    with open(os.path.join(dirname, f"sparse-images-{neuron}.tsv"), "w") as f:
        for a, b, v in zip((r + 1).tolist(), (c + 1).tolist(), vals):
            f.write(f"{a}\t{b}\t{v:.9g}\n")  # "1" for binary images
    for l, (cp, ri, vv) in enumerate(csc_layers):
        col = np.repeat(np.arange(neuron), np.diff(cp))
        with open(os.path.join(dirname, f"neuron{neuron}", f"{neuron}-l{l + 1}.tsv"), "w") as f:
            for a, b, v in zip((ri + 1).tolist(), (col + 1).tolist(), vv.tolist()):
                f.write(f"{a}\t{b}\t{v:.9g}\n")  # 9 digits: every float32 reads back exactly
    with open(os.path.join(dirname, "fuse_matrix", f"neuron{neuron}",
                           f"{neuron}_{layers}_fuse.tsv"), "w") as f:
        for l in range(layers):
            row = np.arange(neuron) if fuse is None else fuse[l]
            f.write("\t".join(str(int(x)) for x in row) + "\n")


def main(argv=None):
    """python -m cospdnn_b200.synth OUT_DIR neuron layers batch [--seed S]
    [--kind xor|r1] [--dlo D] [--dhi D]: a seeded synthetic network and its
    input rows in the reference's dataset format (identity fuse), generated on
    the host, for both command lines (ours and the reference's)."""
    import argparse
    ap = argparse.ArgumentParser(prog="python -m cospdnn_b200.synth")
    ap.add_argument("out_dir")
    ap.add_argument("neuron", type=int)
    ap.add_argument("layers", type=int)
    ap.add_argument("batch", type=int)
    ap.add_argument("--seed", type=int, default=20240611)
    ap.add_argument("--kind", choices=["xor", "r1"], default="xor")
    ap.add_argument("--dlo", type=float, default=0.08)
    ap.add_argument("--dhi", type=float, default=0.25)
    a = ap.parse_args(argv)
    if a.neuron <= 0 or a.layers <= 0 or a.batch <= 0 or (a.kind == "r1" and a.neuron % 16):
        ap.error("neuron, layers and batch must be positive (neuron a multiple of 16 for r1)")
    y0 = input_rows_host(a.batch, a.neuron, a.seed, dlo=a.dlo, dhi=a.dhi)
    try:
        write_reference_dataset(a.out_dir, a.neuron, a.layers, y0, network(a.neuron, a.layers, a.seed, kind=a.kind))
    except OSError as e:
        print(f"synth: {e}")
        return 1
    print(f"wrote {a.out_dir}: {a.neuron} neurons x {a.layers} layers ({a.kind}), {a.batch} rows, "
          f"{int(y0.sum())} input non-zeros")
    return 0


if __name__ == "__main__":
    import sys
    sys.exit(main())


"""Seeded synthetic networks for the tests (built with the oracle's generators)."""
import numpy as np

from oracle import pyoracle as po

BIAS = {1024: -0.3, 4096: -0.35, 16384: -0.4, 65536: -0.45}


def make_net(neuron, layers, rows, seed=1, net=0, dlo=0.08, dhi=0.25, kind="xor", nmask=32,
             bias=None):
    """XOR-mask (or reference-compatible R1) weights as CSC per layer, binary
    Y0 with per-row density U[dlo, dhi), float32 bias."""
    csc = []
    for l in range(layers):
        if kind == "r1":
            m = po.r1_masks(seed, net, l, neuron)
        else:
            m = po.xor_masks(seed, net, l, neuron, nmask)
        csc.append(po.masks_to_csc(m, neuron))
    y0 = po.input_binary(seed, net, rows, neuron, dlo, dhi)
    b = np.float32(BIAS.get(neuron, -0.3) if bias is None else bias)
    return csc, y0, b


def oracle_run(csc, y0, bias, tau=1e-5, want_final=False):
    res = po.infer_fp64(csc, y0, bias, tau=tau, want_final=want_final)
    L = len(csc)
    alive = po.survivors_per_layer(res["death"], L)
    cats = np.nonzero(res["death"] == L)[0].astype(np.int32)
    return dict(alive=alive, categories=cats, death=res["death"], final=res["final"])


def half_block_layer(neuron, seed, net, layer, val=0.125):
    """Reference-kernel-friendly layer: output block column g (outputs
    16g..16g+7) reads the first 8 rows of two aligned input blocks
    g^a and g^b (a != b per layer), value `val`; outputs 16g+8..16g+15 have no
    inputs.  The reference kernel's last pipeline stage (second half of the
    second block) then carries only zero weights, so its race cannot change
    the result, and the all-equal 8x8 quadrants are symmetric."""
    nb = neuron // 16
    g = SplitMix(seed * 1000003 + net * 1009 + layer)
    a = g.next() % nb
    b = g.next() % nb
    while b == a:
        b = g.next() % nb
    cols, rows = [], []
    for blk in range(nb):
        src = sorted([blk ^ a, blk ^ b])
        for r in range(8):
            ins = [16 * src[0] + k for k in range(8)] + [16 * src[1] + k for k in range(8)]
            cols.append((16 * blk + r, ins))
    colptr = np.zeros(neuron + 1, np.int32)
    rowidx, vals = [], []
    per = {c: ins for c, ins in cols}
    for j in range(neuron):
        ins = per.get(j, [])
        rowidx += ins
        vals += [val] * len(ins)
        colptr[j + 1] = colptr[j] + len(ins)
    return colptr, np.array(rowidx, np.int32), np.array(vals, np.float32)


class SplitMix:
    def __init__(self, s):
        self.s = s & ((1 << 64) - 1)

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & ((1 << 64) - 1)
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & ((1 << 64) - 1)
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & ((1 << 64) - 1)
        return z ^ (z >> 31)


def make_half_block_net(neuron, layers, rows, seed=1, dlo=0.1, dhi=0.3, bias=-0.3):
    csc = [half_block_layer(neuron, seed, 0, l) for l in range(layers)]
    y0 = po.input_binary(seed, 0, rows, neuron, dlo, dhi)
    return csc, y0, np.float32(bias)


def random_layer(neuron, seed, layer, kmin=12, kmax=44, wlo=0.02, whi=0.12, neg=0.1):
    """Unstructured weights: column j has U[kmin, kmax] distinct random inputs
    (so the per-column entry counts differ), values multiples of 1/256 in
    [wlo, whi], a fraction `neg` of them negated."""
    rng = np.random.default_rng(seed * 7919 + layer)
    colptr = np.zeros(neuron + 1, np.int32)
    rows, vals = [], []
    for j in range(neuron):
        k = int(rng.integers(kmin, kmax + 1))
        r = np.sort(rng.choice(neuron, size=k, replace=False)).astype(np.int32)
        v = np.round(rng.uniform(wlo, whi, size=k) * 256) / 256
        v[rng.random(k) < neg] *= -1
        rows.append(r)
        vals.append(v.astype(np.float32))
        colptr[j + 1] = colptr[j] + k
    return colptr, np.concatenate(rows), np.concatenate(vals)


def make_random_net(neuron, layers, rows, seed=1, dlo=0.2, dhi=0.4, bias=-0.2, **kw):
    csc = [random_layer(neuron, seed, l, **kw) for l in range(layers)]
    y0 = po.input_binary(seed, 0, rows, neuron, dlo, dhi)
    return csc, y0, np.float32(bias)


def shift_half_block_layer(neuron, seed, layer, val=0.125):
    """Like half_block_layer with output block column g reading the first 8
    rows of input blocks (g + a) and (g + b) mod N/16 (2(a - b) != 0 mod
    N/16), so no two input row groups feed the same pair of block columns."""
    nb = neuron // 16
    g = SplitMix(seed * 7919 + layer)
    while True:
        a, b = g.next() % nb, g.next() % nb
        if a != b and (2 * (a - b)) % nb != 0:
            break
    colptr = np.zeros(neuron + 1, np.int32)
    rowidx = []
    for j in range(neuron):
        blk, r = divmod(j, 16)
        ins = []
        if r < 8:
            for s in sorted([(blk + a) % nb, (blk + b) % nb]):
                ins += [16 * s + k for k in range(8)]
        rowidx += ins
        colptr[j + 1] = colptr[j] + len(ins)
    return colptr, np.array(rowidx, np.int32), np.full(len(rowidx), val, np.float32)


def permute_rows(csc, neuron, seed):
    """The layer with its input rows renamed by a seeded permutation (a
    different network with the same hidden block structure)."""
    cp, ri, vv = csc
    col = np.repeat(np.arange(neuron), np.diff(cp))
    perm = np.random.default_rng(seed).permutation(neuron)
    return po.coo_to_csc(perm[np.asarray(ri)], col, np.asarray(vv, np.float32), neuron)

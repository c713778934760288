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

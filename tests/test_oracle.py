"""The CPU oracle against the reference's own outputs (golden fixtures) and
against straightforward restatements on tiny cases."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "bcsc_*.npz"))))
def test_bcsc_builder_matches_reference_builder(oracle, path):
    """orc_bcsc_greedy == the reference's BCSRCSCMatrix (src/utils/matrix.h:1200-1269)."""
    g = np.load(path)
    cp, ri, ci, vals = oracle.bcsc_greedy(g["row"], g["col"], g["val"], int(g["bs"]))
    np.testing.assert_array_equal(cp, g["col_ptr"])
    np.testing.assert_array_equal(ri, g["row_index"])
    np.testing.assert_array_equal(ci, g["col_index"])
    np.testing.assert_array_equal(vals, g["values"])


def test_golden_covers_misplaced_block_start(oracle):
    """At least one fixture exercises the reference builder storing the value
    that opens a block at offset 0 although its column offset is not 0."""
    g = np.load(os.path.join(GOLDEN, "bcsc_xor_n128_m32.npz"))
    bs = int(g["bs"])
    cp, ri, vals = g["col_ptr"], g["row_index"], g["values"].reshape(-1, bs, bs)
    dense = {}
    for r, c, v in zip(g["row"], g["col"], g["val"]):
        dense[(int(r), int(c))] = float(v)
    misplaced = 0
    for bc in range(len(cp) - 1):
        c0 = int(g["col_index"][bc])
        for blk in range(cp[bc], cp[bc + 1]):
            r0 = int(ri[blk])
            for co in range(bs):
                for ro in range(bs):
                    v = vals[blk, co, ro]
                    if v != 0 and dense.get((r0 + ro, c0 + co)) != v:
                        misplaced += 1
    assert misplaced > 0


def _dense_w(cp, ri, vv, n):
    w = np.zeros((n, n), np.float64)
    for j in range(n):
        for p in range(cp[j], cp[j + 1]):
            w[ri[p], j] = vv[p]
    return w


def test_fp64_recurrence_matches_python_loop(oracle):
    n, L, rows, bias = 64, 6, 40, -0.3
    layers = [oracle.masks_to_csc(oracle.xor_masks(3, 0, l, n, 8), n) for l in range(L)]
    y0 = oracle.input_binary(5, 0, rows, n, 0.25, 0.6)
    res = oracle.infer_fp64(layers, y0, np.float32(bias), tau=1e-5, want_max=True)
    b = float(np.float32(bias))
    for r in range(rows):
        y = y0[r].astype(np.float64)
        death = L
        for l, (cp, ri, vv) in enumerate(layers):
            z = np.empty(n)
            for j in range(n):
                acc = 0.0
                for p in range(cp[j], cp[j + 1]):
                    if y[ri[p]] != 0:
                        acc = acc + float(vv[p]) * y[ri[p]]
                z[j] = acc + b
            y = np.clip(z, 0.0, 32.0)
            assert res["maxval"][r, l] == y.max()
            if not y.max() > 1e-5:
                death = l
                break
        assert res["death"][r] == death


def test_ref_layer_equals_true_product_on_reference_compatible_blocks(oracle):
    """With two aligned symmetric dense blocks per block column (the R1 masks),
    the reference kernel's 2-block, transposed-block arithmetic is the true
    product."""
    n, batch = 256, 128
    cp, ri, vv = oracle.masks_to_csc(oracle.r1_masks(7, 0, 0, n), n)
    row, col, val = oracle.csc_to_coo(cp, ri, vv)
    bcp, bri, bci, bvals = oracle.bcsc_greedy(row, col, val, 16)
    assert np.all(np.diff(bcp) == 2)
    rng = np.random.default_rng(0)
    a = rng.integers(0, 2, (n, batch)).astype(np.float32)
    hilo = np.concatenate([a, np.zeros_like(a)])
    fuse = np.arange(n, dtype=np.int32)
    c_ref = oracle.ref_layer(hilo, bvals, fuse, bcp, bri, -0.3, batch, n)
    c_true = oracle.bcsc_layer(a, bvals, fuse, bcp, bri, -0.3, batch, n)
    w = _dense_w(cp, ri, vv, n)
    c_dense = np.clip(w.T @ a.astype(np.float64) + np.float32(-0.3), 0, 32)
    np.testing.assert_allclose(c_true, c_dense, rtol=0, atol=1e-6)
    np.testing.assert_allclose(c_ref, c_dense, rtol=0, atol=1e-6)


def test_ref_layer_transposes_asymmetric_blocks(oracle):
    """An asymmetric block shows the reference kernel's orientation: value
    [k*16+r] is the weight from input start+k to output r."""
    n, batch = 32, 128
    values = np.zeros((2, 256), np.float32)
    values[0, 3 * 16 + 5] = 1.0  # stored as (col_off 3, row_off 5)
    idx_ptr = np.array([0, 2, 4], np.int32)
    index = np.array([0, 16, 0, 16], np.int32)
    allv = np.concatenate([values, np.zeros((2, 256), np.float32)]).reshape(-1)
    a = np.zeros((n, batch), np.float32)
    a[3, :] = 2.0  # input row 3
    hilo = np.concatenate([a, np.zeros_like(a)])
    fuse = np.arange(n, dtype=np.int32)
    c = oracle.ref_layer(hilo, allv, fuse, idx_ptr, index, 0.0, batch, n)
    assert np.all(c[5] == 2.0) and np.count_nonzero(c) == batch
    t = oracle.bcsc_layer(a, allv, fuse, idx_ptr, index, 0.0, batch, n)
    b = np.zeros((n, batch), np.float32)
    b[5, :] = 2.0
    a2 = np.zeros_like(a)
    a2[5, :] = 2.0
    t2 = oracle.bcsc_layer(a2, allv, fuse, idx_ptr, index, 0.0, batch, n)
    assert np.count_nonzero(t) == 0 and np.all(t2[3] == 2.0)


@pytest.mark.parametrize("tau", [1e-5, 0.0])
def test_fp64_recurrence_clamp_signs_and_real_inputs(oracle, tau):
    """The same pin where the plain loop reaches every branch: unstructured
    weights of both signs up to 4 (outputs above the clamp at 32 and below
    0), non-binary inputs, threshold 1e-5 or 0; per-layer maxima, the layer a
    row dies at and the final activations of surviving rows all equal."""
    n, L, rows, bias = 48, 5, 30, -6.0  # rows die at layers 1 and 2, 18 survive
    rng = np.random.default_rng(11)
    layers = []
    for l in range(L):
        cp = np.zeros(n + 1, np.int32)
        ri, vv = [], []
        for j in range(n):
            k = int(rng.integers(0, 12))
            ri += sorted(rng.choice(n, k, replace=False).tolist())
            vv += (rng.uniform(-4, 4, k) * rng.choice([1, 1, 0.01], k)).astype(np.float32).tolist()
            cp[j + 1] = cp[j] + k
        layers.append((cp, np.array(ri, np.int32), np.array(vv, np.float32)))
    y0 = (rng.random((rows, n)) < 0.5) * rng.uniform(0, 3, (rows, n))
    y0 = y0.astype(np.float32)
    res = oracle.infer_fp64(layers, y0, np.float32(bias), tau=tau, want_max=True, want_final=True)
    b = float(np.float32(bias))
    clamped = False
    for r in range(rows):
        y = y0[r].astype(np.float64)
        death = L
        for l, (cp, ri, vv) in enumerate(layers):
            z = np.empty(n)
            for j in range(n):
                acc = 0.0
                for p in range(cp[j], cp[j + 1]):
                    if y[ri[p]] != 0:
                        acc = acc + float(vv[p]) * y[ri[p]]
                z[j] = acc + b
            clamped |= bool((z > 32).any())
            y = np.clip(z, 0.0, 32.0)
            assert res["maxval"][r, l] == y.max()
            if not y.max() > tau:
                death = l
                break
        assert res["death"][r] == death
        if death == L:
            np.testing.assert_array_equal(res["final"][r], y)
    assert clamped and 0 < int((res["death"] == L).sum()) < rows


def test_cpu_csr_baseline_agrees_with_fp64(oracle):
    n, L, rows = 256, 12, 300
    csc = [oracle.masks_to_csc(oracle.xor_masks(9, 0, l, n), n) for l in range(L)]
    csr = [oracle.coo_to_csr(*oracle.csc_to_coo(*c), n) for c in csc]
    y0 = oracle.input_binary(9, 0, rows, n, 0.25, 0.45)
    bias = np.float32(-0.3)
    ref = oracle.infer_fp64(csc, y0, bias)
    alive, death = oracle.infer_fp32_csr(csr, y0, bias)
    assert alive == int((ref["death"] == L).sum())
    assert (death == ref["death"]).mean() > 0.99


def test_generators_are_seeded_and_prefix_stable(oracle):
    a = oracle.input_binary(1, 2, 50, 128)
    b = oracle.input_binary(1, 2, 80, 128)
    np.testing.assert_array_equal(a, b[:50])
    c = oracle.input_binary(1, 2, 30, 128, row0=50)
    np.testing.assert_array_equal(c, b[50:80])
    m = oracle.xor_masks(4, 1, 3, 1024)
    assert len(set(m.tolist())) == 32 and m.min() >= 0 and m.max() < 1024
    np.testing.assert_array_equal(m, oracle.xor_masks(4, 1, 3, 1024))
    mix = oracle.mix_config(5)
    assert len(mix) == 8 and all(2000 <= b <= 60000 for _, _, b in mix)

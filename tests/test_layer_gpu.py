"""The drop-in operator entries (cospdnn_layer, cospdnn_prune_compact) against
the oracle, and the oracle's restatement of the reference kernel against the
reference's own kernel compiled for sm_100a (oracle/_ref)."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_cospdnn.so")


@pytest.fixture(scope="module")
def cs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200
    cospdnn_b200.lib()
    return cospdnn_b200


def bcsc_case(oracle, n, seed, kind="xor"):
    m = oracle.r1_masks(seed, 0, 0, n) if kind == "r1" else oracle.xor_masks(seed, 0, 0, n)
    cp, ri, vv = oracle.masks_to_csc(m, n)
    row, col, val = oracle.csc_to_coo(cp, ri, vv)
    return oracle.bcsc_greedy(row, col, val, 16)


def hilo(a):
    hi = a.astype(np.float16)
    lo = (a - hi.astype(np.float32)).astype(np.float16)
    return np.concatenate([hi, lo])


def dev(x, dt=None):
    t = torch.from_numpy(np.ascontiguousarray(x))
    if dt is not None:
        t = t.to(dt)
    return t.cuda()


@pytest.mark.parametrize("batch", [128, 300, 301])  # 301: not a multiple of 4, the general kernel
@pytest.mark.parametrize("kind", ["xor", "r1"])
def test_layer_true_product(cs, oracle, batch, kind):
    n = 256
    bcp, bri, _, bvals = bcsc_case(oracle, n, 21, kind)
    rng = np.random.default_rng(1)
    a = (rng.random((n, batch)) * 3).astype(np.float32)
    a[rng.random((n, batch)) < 0.5] = 0
    fuse = rng.permutation(n).astype(np.int32)
    ah = hilo(a)
    want = oracle.bcsc_layer(ah[:n].astype(np.float32) + ah[n:].astype(np.float32), bvals, fuse,
                             bcp, bri, -0.3, batch, n)
    out = torch.empty((n, batch), dtype=torch.float32, device="cuda")
    cs.layer(dev(ah), dev(bvals, torch.float16), out, dev(fuse), dev(bcp), dev(bri), -0.3, batch, n)
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=2e-5)
    # float activations / float weights
    out2 = torch.empty_like(out)
    cs.layer(dev(a), dev(bvals), out2, dev(fuse), dev(bcp), dev(bri), -0.3, batch, n,
             flags=cs.LAYER_A_FLOAT | cs.LAYER_B_FLOAT)
    torch.cuda.synchronize()
    want2 = oracle.bcsc_layer(a, bvals, fuse, bcp, bri, -0.3, batch, n)
    np.testing.assert_allclose(out2.cpu().numpy(), want2, rtol=0, atol=2e-5)


def test_layer_reference_arithmetic(cs, oracle):
    n, batch = 256, 256
    bcp, bri, _, bvals = bcsc_case(oracle, n, 22)
    rng = np.random.default_rng(2)
    a = (rng.random((n, batch)) * 2).astype(np.float32)
    ah = hilo(a)
    fuse = np.arange(n, dtype=np.int32)
    want = oracle.ref_layer(ah.astype(np.float32), bvals.astype(np.float16).astype(np.float32),
                            fuse, bcp, bri, -0.3, batch, n)
    out = torch.empty((n, batch), dtype=torch.float32, device="cuda")
    cs.layer(dev(ah), dev(bvals, torch.float16), out, dev(fuse), dev(bcp), dev(bri), -0.3, batch,
             n, flags=cs.LAYER_REFERENCE_ARITH)
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=2e-5)


def _ref_kernel():
    ref = C.CDLL(REF_SO)
    ref.ref_cospdnn_single.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_int, C.c_int, C.c_int, C.c_void_p]
    return ref


def _run_ref_kernel(ref, A, B, F, P, I, bias, batch, n, nbc):
    out = torch.full((n, batch), -1.0, dtype=torch.float32, device="cuda")
    rc = ref.ref_cospdnn_single(A.data_ptr(), B.data_ptr(), out.data_ptr(), F.data_ptr(),
                                P.data_ptr(), I.data_ptr(), bias, batch, n, nbc, None)
    assert rc == 0
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference kernel not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", [23, 24])
def test_reference_kernel_pins_oracle(cs, oracle, seed):
    """The reference's own cospdnn_single (built from its sources for sm_100a)
    equals the oracle's restatement of its arithmetic and cospdnn_layer's
    REFERENCE_ARITH mode, on the BCSC its own builder makes, with asymmetric
    random block values.  The weights sit in the first 8 block rows of each
    block (k < 8), so the kernel's last pipeline stage multiplies only zero
    weights and its race (see the next test) cannot change the result."""
    import netgen
    ref = _ref_kernel()
    n, batch = 512, 256
    row, col, val = oracle.csc_to_coo(*netgen.half_block_layer(n, seed, 0, 0))
    bcp, bri, _, bvals = oracle.bcsc_greedy(row, col, val, 16)
    rng = np.random.default_rng(seed)
    V = bvals.reshape(-1, 16, 16)
    V[:, :8, :] = 0
    V[:, :, 8:] = 0
    # asymmetric values in the [k<8][r<8] quadrant (k = value index // 16)
    vq = np.zeros_like(V)
    vq[:, :8, :8] = rng.integers(1, 9, (V.shape[0], 8, 8)) / 16.0
    bvals = np.ascontiguousarray(vq.reshape(-1), np.float32)
    a = rng.integers(0, 2, (n, batch)).astype(np.float32) * (rng.random((n, batch)) * 4).astype(np.float32)
    ah = hilo(a)
    fuse = rng.permutation(n).astype(np.int32)
    want = oracle.ref_layer(ah.astype(np.float32), bvals, fuse, bcp, bri, -0.35, batch, n)
    A, B = dev(ah), dev(bvals, torch.float16)
    F, P, I = dev(fuse), dev(bcp), dev(bri)
    got_ref = _run_ref_kernel(ref, A, B, F, P, I, -0.35, batch, n, len(bcp) - 1)
    out = torch.empty((n, batch), dtype=torch.float32, device="cuda")
    cs.layer(A, B, out, F, P, I, -0.35, batch, n, flags=cs.LAYER_REFERENCE_ARITH)
    torch.cuda.synchronize()
    np.testing.assert_allclose(got_ref, want, rtol=0, atol=5e-5)
    np.testing.assert_allclose(out.cpu().numpy(), got_ref, rtol=0, atol=5e-5)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference kernel not built (make -C oracle ref)")
def test_reference_kernel_last_stage_race(cs, oracle):
    """src/kernels/kernel.cu:344-357: after the k=2 iteration no cp.async group
    is committed, so `cp.async.wait_group 1` does not wait for stage 3, whose
    shared-memory tiles (second half of the column's second block) may still be
    in flight when the MMAs read them.  With weights and activations that are
    non-zero only in stage 3 (block rows 24..31 of blocks starting at rows 0
    and 16), a stale tile can only remove contributions, so every reference
    output is <= the value its arithmetic intends; the race-free layer entry
    reproduces the intended value exactly."""
    ref = _ref_kernel()
    n, batch = 256, 1024
    nbc = n // 16
    idx_ptr = np.arange(0, 2 * nbc + 1, 2, dtype=np.int32)
    index = np.tile(np.array([0, 16], np.int32), nbc)
    rng = np.random.default_rng(3)
    V = np.zeros((2 * nbc, 16, 16), np.float32)
    V[1::2, 8:, :] = rng.integers(1, 9, (nbc, 8, 16)) / 16.0  # block p+1, k >= 8
    bvals = np.ascontiguousarray(V.reshape(-1))
    a = np.zeros((n, batch), np.float32)
    a[24:32] = rng.integers(1, 4, (8, batch))
    ah = hilo(a)
    fuse = np.arange(n, dtype=np.int32)
    want = oracle.ref_layer(ah.astype(np.float32), bvals, fuse, idx_ptr, index, 0.0, batch, n)
    A, B, F, P, I = dev(ah), dev(bvals, torch.float16), dev(fuse), dev(idx_ptr), dev(index)
    stale = 0
    for _ in range(5):
        got = _run_ref_kernel(ref, A, B, F, P, I, 0.0, batch, n, nbc)
        assert np.all(got <= want + 1e-5)
        stale += int((got < want - 1e-5).sum())
    out = torch.empty((n, batch), dtype=torch.float32, device="cuda")
    cs.layer(A, B, out, F, P, I, 0.0, batch, n, flags=cs.LAYER_REFERENCE_ARITH)
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=0, atol=1e-5)
    print(f"reference outputs short of the intended value (stale stage-3 tiles), 5 runs: {stale}")


@pytest.mark.parametrize("batch", [1, 200, 1000])
@pytest.mark.parametrize("hilo_out", [False, True])
def test_prune_compact(cs, batch, hilo_out):
    n = 64
    rng = np.random.default_rng(batch)
    c = (rng.random((n, batch)) - 0.7).astype(np.float32).clip(0, None)
    dead = rng.random(batch) < 0.4
    c[:, dead] = 0
    c[0, dead & (rng.random(batch) < 0.5)] = 5e-6  # below the 1e-5 threshold
    map_in = rng.permutation(10 * batch)[:batch].astype(np.int32)
    keep = np.nonzero((c > 1e-5).any(axis=0))[0]
    stride = (len(keep) + 127) // 128 * 128
    ws = torch.empty(cs.prune_workspace_bytes(batch) // 4, dtype=torch.int32, device="cuda")
    if hilo_out:
        A = torch.full((2 * n, max(stride, batch)), 7.0, dtype=torch.float16, device="cuda")
    else:
        A = torch.full((n, max(stride, batch)), 7.0, dtype=torch.float32, device="cuda")
    cat = torch.full((batch,), -1, dtype=torch.int32, device="cuda")
    mo = torch.full((batch,), -1, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
    cs.prune_compact(dev(c), n, batch, 1e-5, A, cat, dev(map_in), mo, cnt, ws,
                     flags=cs.PRUNE_OUT_HALF_HILO if hilo_out else 0)
    torch.cuda.synchronize()
    k = int(cnt.item())
    assert k == len(keep)
    np.testing.assert_array_equal(cat.cpu().numpy()[:k], keep)
    np.testing.assert_array_equal(mo.cpu().numpy()[:k], map_in[keep])
    flat = A.cpu().numpy().reshape(-1)
    if hilo_out:
        hi = flat[:n * stride].reshape(n, stride)
        lo = flat[n * stride:2 * n * stride].reshape(n, stride)
        want_hi = c[:, keep].astype(np.float16)
        want_lo = (c[:, keep] - want_hi.astype(np.float32)).astype(np.float16)
        np.testing.assert_array_equal(hi[:, :k], want_hi)
        np.testing.assert_array_equal(lo[:, :k], want_lo)
        got = hi.astype(np.float32) + lo.astype(np.float32)
    else:
        got = flat[:n * stride].reshape(n, stride)
        np.testing.assert_array_equal(got[:, :k], c[:, keep])
    assert np.all(got[:, k:stride] == 0)

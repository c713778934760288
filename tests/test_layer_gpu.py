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


@pytest.mark.parametrize("batch", [128, 300])
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


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference kernel not built (make -C oracle ref)")
@pytest.mark.parametrize("kind,seed", [("xor", 23), ("xor", 24), ("r1", 25)])
def test_reference_kernel_pins_oracle(cs, oracle, kind, seed):
    """The reference's own cospdnn_single (built from its sources for sm_100a)
    agrees with the oracle's restatement, with asymmetric blocks and more than
    two blocks per column, and with cospdnn_layer's REFERENCE_ARITH mode."""
    ref = C.CDLL(REF_SO)
    ref.ref_cospdnn_single.argtypes = [C.c_void_p] * 6 + [C.c_float, C.c_int, C.c_int, C.c_int, C.c_void_p]
    n, batch = 512, 256
    bcp, bri, _, bvals = bcsc_case(oracle, n, seed, kind)
    rng = np.random.default_rng(seed)
    a = rng.integers(0, 2, (n, batch)).astype(np.float32) * (rng.random((n, batch)) * 4).astype(np.float32)
    ah = hilo(a)
    fuse = np.arange(n, dtype=np.int32)
    want = oracle.ref_layer(ah.astype(np.float32), bvals.astype(np.float16).astype(np.float32),
                            fuse, bcp, bri, -0.35, batch, n)
    A, B = dev(ah), dev(bvals, torch.float16)
    F, P, I = dev(fuse), dev(bcp), dev(bri)
    out_ref = torch.full((n, batch), -1.0, dtype=torch.float32, device="cuda")
    rc = ref.ref_cospdnn_single(A.data_ptr(), B.data_ptr(), out_ref.data_ptr(), F.data_ptr(),
                                P.data_ptr(), I.data_ptr(), -0.35, batch, n, len(bcp) - 1, None)
    assert rc == 0
    out = torch.empty_like(out_ref)
    cs.layer(A, B, out, F, P, I, -0.35, batch, n, flags=cs.LAYER_REFERENCE_ARITH)
    torch.cuda.synchronize()
    got_ref = out_ref.cpu().numpy()
    np.testing.assert_allclose(got_ref, want, rtol=0, atol=5e-5)
    np.testing.assert_allclose(out.cpu().numpy(), got_ref, rtol=0, atol=5e-5)
    if kind == "r1":  # valid inputs: the reference kernel computes the true product
        true = torch.empty_like(out)
        cs.layer(A, B, true, F, P, I, -0.35, batch, n)
        torch.cuda.synchronize()
        np.testing.assert_allclose(true.cpu().numpy(), got_ref, rtol=0, atol=5e-5)


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
        hi = flat[:n * stride].reshape(n, stride).astype(np.float32)
        lo = flat[n * stride:2 * n * stride].reshape(n, stride).astype(np.float32)
        got = hi + lo
        np.testing.assert_allclose(got[:, :k], c[:, keep], rtol=2e-6, atol=1e-9)
    else:
        got = flat[:n * stride].reshape(n, stride)
        np.testing.assert_array_equal(got[:, :k], c[:, keep])
    assert np.all(got[:, k:stride] == 0)

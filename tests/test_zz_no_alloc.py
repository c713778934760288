"""cospdnn_prune_compact_noalloc: the allocation-free pruning entry, for
callers that cannot call cudaMalloc, checked through the C ABI against the
allocating cospdnn_prune_compact on two calls in a row (different inputs, so
the second call also shows the shared scratch is cleared between calls).

Collected last on purpose: the scratch is a device array owned by the
library, and this test must pass both alone in a fresh process and after
every other test."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _case(seed, n, batch):
    rng = np.random.default_rng(seed)
    c = (rng.random((n, batch)) - 0.6).astype(np.float32).clip(0, None)
    dead = rng.random(batch) < 0.5
    c[:, dead] = 0
    c[3, dead & (rng.random(batch) < 0.3)] = 5e-6  # at or below the threshold
    map_in = rng.permutation(4 * batch)[:batch].astype(np.int32)
    return c, map_in


def _run(cs, fn_noalloc, c, map_in, hilo):
    n, batch = c.shape
    cols = (batch + 127) // 128 * 128
    outs = []
    for use_noalloc in (False, True):
        dt = torch.float16 if hilo else torch.float32
        A = torch.full(((2 if hilo else 1) * n, cols), 3.0, dtype=dt, device="cuda")
        cat = torch.full((batch,), -1, dtype=torch.int32, device="cuda")
        mo = torch.full((batch,), -1, dtype=torch.int32, device="cuda")
        cnt = torch.zeros(1, dtype=torch.int32, device="cuda")
        Cd = torch.from_numpy(c).cuda()
        Md = torch.from_numpy(map_in).cuda()
        flags = cs.PRUNE_OUT_HALF_HILO if hilo else 0
        if use_noalloc:
            rc = fn_noalloc(C.c_void_p(Cd.data_ptr()), n, batch, C.c_float(1e-5), C.c_void_p(A.data_ptr()),
                            C.c_void_p(cat.data_ptr()), C.c_void_p(Md.data_ptr()), C.c_void_p(mo.data_ptr()),
                            C.c_void_p(cnt.data_ptr()), flags, None)
            assert rc == cs.OK, cs.lib().cospdnn_last_error()
        else:
            ws = torch.empty(cs.prune_workspace_bytes(batch) // 4, dtype=torch.int32, device="cuda")
            cs.prune_compact(Cd, n, batch, 1e-5, A, cat, Md, mo, cnt, ws, flags=flags)
        torch.cuda.synchronize()
        k = int(cnt.item())
        outs.append((k, cat.cpu().numpy()[:k], mo.cpu().numpy()[:k], A.cpu().numpy()))
    return outs


def test_noalloc_prune_matches_allocating_entry_twice():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200 as cs
    fn = cs.lib().cospdnn_prune_compact_noalloc
    for call, (seed, n, batch, hilo) in enumerate([(1, 64, 3000, False), (2, 48, 1700, True)]):
        c, map_in = _case(seed, n, batch)
        (k0, cat0, mo0, a0), (k1, cat1, mo1, a1) = _run(cs, fn, c, map_in, hilo)
        keep = np.nonzero((c > 1e-5).any(axis=0))[0]
        assert k0 == k1 == len(keep), f"call {call}"
        np.testing.assert_array_equal(cat1, cat0)
        np.testing.assert_array_equal(cat1, keep)
        np.testing.assert_array_equal(mo1, mo0)
        stride = (k0 + 127) // 128 * 128
        rows = (2 if hilo else 1) * n
        np.testing.assert_array_equal(a1.reshape(-1)[:rows * stride], a0.reshape(-1)[:rows * stride])


def test_noalloc_prune_rejects_oversized_batch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200 as cs
    fn = cs.lib().cospdnn_prune_compact_noalloc
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = C.c_void_p(dummy.data_ptr())
    rc = fn(p, 4, (1 << 20) + 1, C.c_float(1e-5), p, p, None, p, p, 0, None)
    assert rc == cs.ERR_INVALID
    assert b"1048576" in cs.lib().cospdnn_last_error()

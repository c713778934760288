"""Per-layer survivor counts of the reference's own host loop
(test_graph_challenge_tc, src/cospdnn.cu:172-307, built from its sources into
oracle/_ref) against the FP64 oracle and the engine, on reference-compatible
weights: two aligned 16x16 blocks per block column whose non-zeros fill the
symmetric top-left 8x8 quadrant, so the reference kernel computes the true
recurrence and its last-stage race multiplies only zero weights."""
import ctypes as C
import os

import numpy as np
import pytest

from netgen import make_half_block_net, oracle_run

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_cospdnn.so")


def run_reference_loop(oracle, csc, y0, bias, want_wall=False, fuse=None):
    """The reference's host loop on the greedy BCSC of each layer's CSC (rows
    = block rows, read through fuse[l] when given, else the identity)."""
    ref = C.CDLL(REF_SO)
    L, n = len(csc), y0.shape[1]
    vals, rows, ptrs = [], [], []
    for cp, ri, vv in csc:
        row, col, val = oracle.csc_to_coo(cp, ri, vv)
        bcp, bri, _, bvals = oracle.bcsc_greedy(row, col, val, 16)
        # the kernel reads fuse[start + 15] of the first two blocks of every
        # column: run it only where both exist and stay inside the fuse row
        assert np.all(np.diff(bcp) >= 2)
        assert bri[bcp[:-1]].max() <= n - 16 and bri[bcp[:-1] + 1].max() <= n - 16
        vals.append(np.ascontiguousarray(bvals, np.float32))
        rows.append(np.ascontiguousarray(bri, np.int32))
        ptrs.append(np.ascontiguousarray(bcp, np.int32))
    fp = C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    V = (fp * L)(*[v.ctypes.data_as(fp) for v in vals])
    RI = (ip * L)(*[r.ctypes.data_as(ip) for r in rows])
    P = (ip * L)(*[p.ctypes.data_as(ip) for p in ptrs])
    nv = np.array([len(v) for v in vals], np.int64)
    nr = np.array([len(r) for r in rows], np.int64)
    npp = np.array([len(p) for p in ptrs], np.int64)
    feats = np.full(64, -1, np.int32)
    kms, wms = C.c_double(), C.c_double()
    last = C.c_int()
    tail = C.create_string_buffer(4096)
    ref.ref_run_network.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_float, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_int, C.c_char_p, C.c_int, C.c_void_p]
    fz = None
    if fuse is not None:
        fuse = [np.ascontiguousarray(f, np.int32) for f in fuse]
        assert len(fuse) == L and all(f.shape == (n,) and f.min() >= 0 and f.max() < n for f in fuse)
        fz = (ip * L)(*[f.ctypes.data_as(ip) for f in fuse])
    y = np.ascontiguousarray(y0, np.uint8)
    rc = ref.ref_run_network(y.ctypes.data, y.shape[0], n, L, C.addressof(V), nv.ctypes.data,
                             C.addressof(RI), nr.ctypes.data, C.addressof(P), npp.ctypes.data,
                             float(bias), C.addressof(kms), C.addressof(wms), C.addressof(last),
                             feats.ctypes.data, 64, tail, 4096, None if fz is None else C.addressof(fz))
    assert rc == 0, tail.value.decode()
    if want_wall:
        return feats, kms.value, wms.value
    return feats, kms.value


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference not built (make -C oracle ref)")
def test_reference_loop_counts_match_oracle_and_engine(oracle):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200 as cs
    n, L, rows = 1024, 16, 2048
    csc, y0, b = make_half_block_net(n, L, rows, seed=31)
    feats, kms = run_reference_loop(oracle, csc, y0, b)
    ref = oracle_run(csc, y0, b)
    # the reference prints counts for the layers it compacts (l <= 21)
    np.testing.assert_array_equal(feats[:L], ref["alive"])
    eng = cs.Engine(0)
    nid = eng.add_net(n, L, rows, float(b), 1e-5, cs.PREC_FP16, cs.KERNEL_AUTO)
    for l, (cp, ri, vv) in enumerate(csc):
        eng.set_layer_csc(nid, l, cp, ri, vv)
    eng.build()
    eng.set_input(nid, y0)
    eng.run()
    res = eng.result(nid)
    eng.close()
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    assert kms > 0


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference not built (make -C oracle ref)")
def test_reference_last_layer_reuses_previous_weights(oracle):
    """src/cospdnn.cu:177-209: the layer loop points B_d, index_d, col_ptr_d
    and fuse_d at layer l's buffers only inside `if (l + 1 < layer)`, so the
    last layer runs on the buffers of layer L-2.  With a last layer whose
    weights are too small for any output to pass the bias, the true
    recurrence prunes every row there; the reference's printed count equals
    the oracle's count for layer L-2's weights applied twice."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from netgen import half_block_layer
    n, L, rows = 1024, 4, 1024
    csc, y0, b = make_half_block_net(n, L, rows, seed=37)
    csc[L - 1] = half_block_layer(n, 37, 0, L - 1, val=1e-7)
    feats, _ = run_reference_loop(oracle, csc, y0, b)
    true = oracle_run(csc, y0, b)
    assert true["alive"][L - 1] == 0 and true["alive"][L - 2] > 0
    stale = oracle_run(csc[:L - 1] + [csc[L - 2]], y0, b)
    np.testing.assert_array_equal(feats[:L - 1], true["alive"][:L - 1])
    assert feats[L - 1] == stale["alive"][L - 1] > 0


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference not built (make -C oracle ref)")
def test_reference_runs_reordered_network(oracle):
    """A network with hidden block structure (each layer's input rows renamed
    by a permutation, so the greedy blocks are scattered and the reference's
    two-block kernel would truncate the product): after cospdnn_b200.reorder
    every block column has two aligned blocks again, and the reference's own
    host loop, reading activations through the fuse rows, prints the true
    recurrence's counts -- for every layer but the last, which runs on layer
    L-2's buffers (previous test)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from netgen import permute_rows, shift_half_block_layer
    from cospdnn_b200 import reorder
    n, L, rows = 1024, 6, 2048
    layers = [permute_rows(shift_half_block_layer(n, 13, l, val=0.25), n, 130 + l) for l in range(L)]
    y0 = oracle.input_binary(13, 0, rows, n, 0.1, 0.3)
    b = np.float32(-0.3)
    true = oracle_run(layers, y0, b)
    assert 0 < true["alive"][L - 2] < rows  # rows die along the way, not all
    # as given: about 13 scattered blocks per column, of which the kernel reads two
    plain, _ = run_reference_loop(oracle, layers, y0, b)
    assert not np.array_equal(plain[:L - 1], true["alive"][:L - 1])
    out, fuse, stats = reorder.reorder_network(layers, n)
    assert all(after == 2 * (n // 16) < before for before, after in stats)
    feats, _ = run_reference_loop(oracle, out, y0, b, fuse=fuse)
    np.testing.assert_array_equal(feats[:L - 1], true["alive"][:L - 1])

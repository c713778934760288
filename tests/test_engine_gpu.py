"""Parity of the whole-network engine with the FP64 oracle (GPU)."""
import numpy as np
import pytest

from netgen import make_net, oracle_run

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def cs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200
    cospdnn_b200.lib()
    return cospdnn_b200


def run_engine(cs, nets, precision, kernel=0, tau=1e-5, runs=1):
    """nets: list of (csc, y0, bias).  Returns per-net result dicts."""
    eng = cs.Engine(0)
    ids = []
    for csc, y0, bias in nets:
        nid = eng.add_net(y0.shape[1], len(csc), y0.shape[0], float(bias), tau, precision, kernel)
        for l, (cp, ri, vv) in enumerate(csc):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
    out = None
    for _ in range(runs):
        for nid, (_, y0, _) in zip(ids, nets):
            eng.set_input(nid, y0)
        eng.run()
        out = [eng.result(nid) for nid in ids]
    out_launches = eng.launch_count()
    finals = [eng.final_values(nid, len(r["categories"])) for nid, r in zip(ids, out)]
    eng.close()
    for r, f in zip(out, finals):
        r["final"] = f
        r["launches"] = out_launches
    return out


def check_parity(res, ref, layers):
    np.testing.assert_array_equal(res["alive"], ref["alive"][:layers])
    np.testing.assert_array_equal(res["categories"], ref["categories"])


@pytest.mark.parametrize("prec,kernel", [(0, 1), (1, 1), (2, 1), (1, 2), (2, 2)])
def test_engine_xor_1024_matches_fp64(cs, prec, kernel):
    csc, y0, b = make_net(1024, 12, 3000, seed=3)
    ref = oracle_run(csc, y0, b)
    res = run_engine(cs, [(csc, y0, b)], prec, kernel)[0]
    check_parity(res, ref, 12)
    assert res["launches"] > 0


@pytest.mark.parametrize("prec,kernel", [(0, 1), (1, 1), (2, 1), (1, 2), (2, 2)])
def test_engine_sustained_activity_matches_fp64(cs, prec, kernel):
    """Input density U[0.25,0.45]: most rows stay alive, categories non-trivial."""
    csc, y0, b = make_net(1024, 24, 1500, seed=5, dlo=0.25, dhi=0.45)
    ref = oracle_run(csc, y0, b, want_final=True)
    assert len(ref["categories"]) > 100
    res = run_engine(cs, [(csc, y0, b)], prec, kernel)[0]
    check_parity(res, ref, 24)
    fin_ref = ref["final"][ref["categories"]]
    tol = {0: 1e-3, 1: 0.25, 2: 2.0}[prec]
    assert np.abs(res["final"] - fin_ref).max() <= tol


@pytest.mark.parametrize("kernel", [1, 2])
def test_engine_multi_network_uneven(cs, kernel):
    nets = [make_net(1024, 10, 2500, seed=7, net=0),
            make_net(2048, 6, 700, seed=7, net=1, dlo=0.25, dhi=0.45),
            make_net(1024, 15, 1200, seed=7, net=2, dlo=0.2, dhi=0.4)]
    refs = [oracle_run(*n) for n in nets]
    res = run_engine(cs, nets, 1, kernel)
    for r, f, n in zip(res, refs, nets):
        check_parity(r, f, len(n[0]))


def test_engine_repeat_runs_identical(cs):
    csc, y0, b = make_net(1024, 8, 1000, seed=9, dlo=0.2, dhi=0.4)
    ref = oracle_run(csc, y0, b)
    res = run_engine(cs, [(csc, y0, b)], 1, 1, runs=3)[0]
    check_parity(res, ref, 8)


def test_engine_zero_threshold_rule(cs):
    csc, y0, b = make_net(1024, 10, 2000, seed=11)
    ref = oracle_run(csc, y0, b, tau=0.0)
    res = run_engine(cs, [(csc, y0, b)], 0, 1, tau=0.0)[0]
    check_parity(res, ref, 10)


def test_engine_bcsc_input_with_fuse(cs):
    """Weights given as the reference's greedy BCSC plus a fuse permutation."""
    from oracle import pyoracle as po
    n, L, rows = 512, 6, 800
    csc, y0, b = make_net(n, L, rows, seed=13, dlo=0.2, dhi=0.4)
    rng = np.random.default_rng(0)
    eng = cs.Engine(0)
    nid = eng.add_net(n, L, rows, float(b), 1e-5, 0, 1)
    folded = []
    for l, (cp, ri, vv) in enumerate(csc):
        fuse = rng.permutation(n).astype(np.int32)
        row, col, val = po.csc_to_coo(cp, ri, vv)
        bcp, bri, _, bvals = po.bcsc_greedy(row, col, val, 16)
        eng.set_layer_bcsc(nid, l, bcp, bri, bvals, 16, fuse)
        # the same layer with the fuse folded in, as the oracle sees it
        bs = 16
        V = bvals.reshape(-1, bs, bs)
        rr, cc, ww = [], [], []
        for bid in range(len(bcp) - 1):
            for blk in range(bcp[bid], bcp[bid + 1]):
                co, ro = np.nonzero(V[blk])
                rr += list(fuse[bri[blk] + ro])
                cc += list(bid * bs + co)
                ww += list(V[blk][co, ro])
        folded.append(po.coo_to_csc(np.array(rr, np.int32), np.array(cc, np.int32),
                                    np.array(ww, np.float32), n))
    eng.build()
    eng.set_input(nid, y0)
    eng.run()
    res = eng.result(nid)
    eng.close()
    ref = oracle_run(folded, y0, b)
    check_parity(res, ref, L)


@pytest.mark.parametrize("n,rows", [(4096, 700), (512, 130), (256, 1)])
def test_engine_tcgen05_shapes(cs, n, rows):
    """Ragged row tiles (rows not a multiple of 128), narrow and wide layers."""
    csc, y0, b = make_net(n, 6, rows, seed=17, dlo=0.2, dhi=0.45, bias=-0.3)
    ref = oracle_run(csc, y0, b, want_final=True)
    res = run_engine(cs, [(csc, y0, b)], 1, 2)[0]
    check_parity(res, ref, 6)


def test_engine_tcgen05_layer_values_match_cuda_core(cs):
    """Same net, same FP16 storage: the tcgen05 and CUDA-core kernels produce
    final activations within the FP16 rounding of each other."""
    csc, y0, b = make_net(1024, 8, 600, seed=19, dlo=0.25, dhi=0.45)
    r_tc = run_engine(cs, [(csc, y0, b)], 1, 2)[0]
    r_cc = run_engine(cs, [(csc, y0, b)], 1, 1)[0]
    np.testing.assert_array_equal(r_tc["categories"], r_cc["categories"])
    assert np.abs(r_tc["final"] - r_cc["final"]).max() <= 0.125


# Row-tile heights of the CUDA-core tile kernel (tile = N x TR values in at
# most 200 KB of shared memory): each case exercises a different number of
# lanes per output (G) and outputs per shared-memory wavefront (P); 16384
# features take 8-byte lane pieces (P = 16).
@pytest.mark.parametrize("n,prec", [(512, 1), (1000, 1), (2048, 2), (3000, 1), (8192, 1), (16384, 2),
                                    (512, 0), (1000, 0), (4096, 0), (16384, 0)])
def test_engine_cc_tile_shapes(cs, n, prec):
    from netgen import make_random_net
    csc, y0, b = make_random_net(n, 5, 333, seed=23)
    ref = oracle_run(csc, y0, b, want_final=True)
    res = run_engine(cs, [(csc, y0, b)], prec, 1)[0]
    check_parity(res, ref, 5)
    if len(ref["categories"]):
        tol = {0: 1e-3, 1: 0.25, 2: 2.0}[prec]
        assert np.abs(res["final"] - ref["final"][ref["categories"]]).max() <= tol


@pytest.mark.parametrize("n,prec", [(2048, 1), (4096, 2), (8192, 1), (4096, 0)])
def test_engine_cc_random_weights_sustained(cs, n, prec):
    """Unequal entry counts per output (12..44): zero-weight padding and the
    bank-conflict-free entry order with uneven residue loads; rows pruned in
    the middle layers exercise the row-tile compaction copy."""
    from netgen import make_random_net
    csc, y0, b = make_random_net(n, 8, 700, seed=29)
    ref = oracle_run(csc, y0, b)
    assert ref["alive"][0] > 0
    res = run_engine(cs, [(csc, y0, b)], prec, 1)[0]
    check_parity(res, ref, 8)


def test_engine_row_major_gather_kernel_wide_fp32(cs):
    """FP32 rows of 32768 features do not fit a row tile in shared memory:
    the net runs on the row-major gather kernel."""
    csc, y0, b = make_net(32768, 4, 200, seed=31, dlo=0.2, dhi=0.4)
    ref = oracle_run(csc, y0, b)
    res = run_engine(cs, [(csc, y0, b)], 0, 1)[0]
    check_parity(res, ref, 4)


def test_engine_mixed_kernels_one_graph(cs):
    """Row-tile, row-major and tcgen05 nets advance in the same graph."""
    from netgen import make_random_net
    nets = [make_random_net(2048, 6, 500, seed=37),
            make_net(16384, 3, 150, seed=37, net=1, dlo=0.2, dhi=0.4),
            make_net(1024, 7, 400, seed=37, net=2, dlo=0.2, dhi=0.4)]
    refs = [oracle_run(*n) for n in nets]
    eng = cs.Engine(0)
    ids = []
    for (csc, y0, b), prec, kern in zip(nets, (1, 0, 1), (1, 1, 2)):
        nid = eng.add_net(y0.shape[1], len(csc), y0.shape[0], float(b), 1e-5, prec, kern)
        for l, (cp, ri, vv) in enumerate(csc):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
    for nid, (_, y0, _) in zip(ids, nets):
        eng.set_input(nid, y0)
    eng.run()
    res = [eng.result(nid) for nid in ids]
    eng.close()
    for r, f, n in zip(res, refs, nets):
        check_parity(r, f, len(n[0]))


@pytest.mark.parametrize("n,prec,kernel", [(1000, 1, 1), (4096, 1, 1), (1024, 0, 1), (4096, 2, 2), (16384, 1, 1),
                                           (32768, 0, 1)])
def test_engine_input_formats_agree(cs, n, prec, kernel):
    """Bytes, packed bits (little-endian within a byte) and float32 inputs of
    the same binary rows give identical results (row tiles, MMA tiles and
    row-major layouts), equal to the oracle's."""
    if n & (n - 1):  # XOR masks need a power of two; N/8 odd = unaligned bit rows
        from netgen import make_random_net
        csc, y0, b = make_random_net(n, 4, 333, seed=41)
    else:
        csc, y0, b = make_net(n, 4, 333, seed=41, dlo=0.2, dhi=0.4)
    ref = oracle_run(csc, y0, b)
    bits = np.packbits(y0, axis=1, bitorder="little")
    eng = cs.Engine(0)
    nid = eng.add_net(n, 4, y0.shape[0], float(b), 1e-5, prec, kernel)
    for l, (cp, ri, vv) in enumerate(csc):
        eng.set_layer_csc(nid, l, cp, ri, vv)
    eng.build()
    outs = []
    for x, fmt in ((y0, cs.INPUT_U8), (bits, cs.INPUT_BITS), (y0.astype(np.float32), cs.INPUT_F32)):
        eng.set_input(nid, x, fmt=fmt)
        eng.run()
        r = eng.result(nid)
        outs.append((r, eng.final_values(nid, len(r["categories"]))))
    eng.close()
    for r, f in outs:
        check_parity(r, ref, 4)
        np.testing.assert_array_equal(f, outs[0][1])


def _empty_columns_layer(n, seed):
    """Random weights where a quarter of the outputs have no inputs at all."""
    from netgen import random_layer
    cp, ri, vv = random_layer(n, seed, 0)
    rng = np.random.default_rng(seed)
    empty = rng.random(n) < 0.25
    keep = np.repeat(~empty, np.diff(cp))
    counts = np.where(empty, 0, np.diff(cp))
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int32), ri[keep], vv[keep]


@pytest.mark.parametrize("prec,kernel", [(1, 1), (0, 1), (1, 2)])
def test_engine_edge_cases(cs, prec, kernel):
    """In one engine: a net with no rows, a one-layer net, a net whose layers
    have outputs without inputs, and a net whose second layer has no weights
    at all (every row pruned there)."""
    from netgen import make_random_net
    n = 1024
    c_a, y_a, b_a = make_random_net(n, 3, 200, seed=71)
    c_b, y_b, b_b = make_random_net(n, 1, 150, seed=72)
    c_c = [_empty_columns_layer(n, 73 + l) for l in range(4)]
    _, y_c, b_c = make_random_net(n, 1, 250, seed=73)
    c_d, y_d, b_d = make_random_net(n, 3, 120, seed=74)
    c_d[1] = (np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    nets = [(c_a, y_a[:0], b_a), (c_b, y_b, b_b), (c_c, y_c, b_c), (c_d, y_d, b_d)]
    eng = cs.Engine(0)
    ids = []
    for csc, y0, b in nets:
        nid = eng.add_net(n, len(csc), y0.shape[0], float(b), 1e-5, prec, kernel)
        for l, (cp, ri, vv) in enumerate(csc):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
    for nid, (_, y0, _) in zip(ids, nets):
        if y0.shape[0]:
            eng.set_input(nid, y0)
    eng.run()
    res = [eng.result(nid) for nid in ids]
    eng.close()
    assert len(res[0]["categories"]) == 0
    for r, (csc, y0, b) in zip(res[1:], nets[1:]):
        check_parity(r, oracle_run(csc, y0, b), len(csc))
    assert res[3]["alive"][1] == 0 and len(res[3]["categories"]) == 0


def test_engine_next_input_set_during_run(cs):
    """Inputs are double buffered: the next batch is copied and converted on
    a second stream while a run on the first stream still reads the current
    batch; both runs equal the oracle's."""
    from netgen import make_random_net
    n, L = 1024, 6
    csc, y_a, b = make_random_net(n, L, 800, seed=81)
    _, y_b, _ = make_random_net(n, 1, 800, seed=82, dlo=0.3, dhi=0.5)
    ref_a, ref_b = oracle_run(csc, y_a, b), oracle_run(csc, y_b, b)
    assert not np.array_equal(ref_a["categories"], ref_b["categories"])
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    eng = cs.Engine(0)
    nid = eng.add_net(n, L, 800, float(b), 1e-5, 1, 0)
    for l, (cp, ri, vv) in enumerate(csc):
        eng.set_layer_csc(nid, l, cp, ri, vv)
    eng.build()
    got = []
    for rep in range(2):
        eng.set_input(nid, torch.from_numpy(np.packbits(y_a, axis=1, bitorder="little")).pin_memory(),
                      fmt=cs.INPUT_BITS, stream=s1)
        eng.run(s1)                                   # batch A
        eng.set_input(nid, y_b, stream=s2)            # batch B, while A runs
        ev = torch.cuda.Event()
        ev.record(s2)
        got.append(eng.result(nid, s1))               # A's result
        s1.wait_event(ev)
        eng.run(s1)                                   # batch B
        got.append(eng.result(nid, s1))
    eng.close()
    for r, ref in zip(got, [ref_a, ref_b, ref_a, ref_b]):
        check_parity(r, ref, L)


@pytest.mark.parametrize("n,prec,rows,kernel,scale", [
    (1024, 1, 333, 1, 1), (4096, 1, 5, 1, 1), (16384, 2, 97, 1, 1), (1024, 0, 333, 1, 1), (2048, 0, 64, 1, 1),
    (512, 1, 333, 1, 1), (4096, 1, 333, 2, 1), (2048, 2, 17, 2, 1), (1024, 1, 200, 2, 1),
    (1024, 1, 333, 1, 16), (2048, 0, 64, 1, 16), (4096, 2, 97, 1, 16), (1024, 1, 200, 2, 16)])
def test_layer0_bit_count_matches_general_kernel(cs, n, prec, rows, kernel, scale):
    """Layer 0 by bit counting (binary inputs, one weight value per output)
    stores exactly what the general row-tile kernel stores: a one-layer net
    run on U8 and packed-bit inputs (counted) and on the same rows as FP32
    (never counted); row tiles of 64, 32, 16, 8 and 4 rows (CUDA-core nets,
    32-row units) and MMA tiles (tcgen05 nets, 16-row units).  Per-output
    weight values differ (1/16 times 1, 2 or 3), so the kernel reads each
    output's own weight; scale 16 makes them 1, 2 or 3, so that outputs pass
    16 and the clamp at 32 (the kernel's path for |z| > 16)."""
    from oracle import pyoracle as po
    cp, ri, vv = po.masks_to_csc(po.xor_masks(59, 0, 0, n), n)
    col = np.repeat(np.arange(n), np.diff(cp))
    vv = (vv * (1 + col % 3) * scale).astype(np.float32)
    y0 = po.input_binary(59, 0, rows, n, 0.1, 0.3)
    b = np.float32(-0.3)
    ref = oracle_run([(cp, ri, vv)], y0, b)
    eng = cs.Engine(0)
    nid = eng.add_net(n, 1, rows, float(b), 1e-5, prec, kernel)
    eng.set_layer_csc(nid, 0, cp, ri, vv)
    eng.build()
    outs = []
    bits = np.packbits(y0, axis=1, bitorder="little")
    for x, fmt in ((y0, cs.INPUT_U8), (bits, cs.INPUT_BITS), (y0.astype(np.float32), cs.INPUT_F32)):
        eng.set_input(nid, x, fmt=fmt)
        eng.run()
        r = eng.result(nid)
        check_parity(r, ref, 1)
        outs.append(eng.final_values(nid, len(r["categories"])))
    eng.close()
    np.testing.assert_array_equal(outs[0], outs[2])
    np.testing.assert_array_equal(outs[1], outs[2])


def test_layer0_bit_count_falls_back(cs):
    """Inputs with a value above 1, and layers whose outputs mix weight
    values, take the general kernel; results stay exact."""
    from netgen import random_layer
    from oracle import pyoracle as po
    n, rows = 1024, 200
    xor = po.masks_to_csc(po.xor_masks(61, 0, 0, n), n)
    mixed = random_layer(n, 61, 0)
    y0 = po.input_binary(61, 0, rows, n, 0.1, 0.3)
    y2 = y0.copy()
    y2[::7] *= 2  # values 0 and 2 in every seventh row
    for layer, x in ((xor, y2), (mixed, y0)):
        ref = oracle_run([layer, xor], x, np.float32(-0.3))
        eng = cs.Engine(0)
        nid = eng.add_net(n, 2, rows, -0.3, 1e-5, 1, 1)
        eng.set_layer_csc(nid, 0, *layer)
        eng.set_layer_csc(nid, 1, *xor)
        eng.build()
        eng.set_input(nid, x)
        eng.run()
        check_parity(eng.result(nid), ref, 2)
        eng.close()


def test_run_networks_one_call(cs):
    """cospdnn_run_networks: three networks of different widths, depths,
    precisions and kernels (row tiles, MMA tiles) in one call, U8 and FP32
    inputs, each equal to the FP64 oracle."""
    from netgen import make_random_net
    a_csc, a_y0, a_b = make_net(1024, 5, 300, seed=71, dlo=0.2, dhi=0.4)
    b_csc, b_y0, b_b = make_random_net(512, 3, 120, seed=72)
    c_csc, c_y0, c_b = make_net(4096, 4, 200, seed=73, dlo=0.2, dhi=0.4, kind="r1")
    nets = [dict(neuron=1024, layers=a_csc, y0=a_y0, bias=a_b, precision=cs.PREC_FP16),
            dict(neuron=512, layers=b_csc, y0=b_y0.astype(np.float32), bias=b_b, precision=cs.PREC_FP32),
            dict(neuron=4096, layers=c_csc, y0=c_y0, bias=c_b, precision=cs.PREC_BF16, kernel=cs.KERNEL_TCGEN05)]
    res, ms = cs.run_networks(nets)
    assert ms > 0
    for r, (csc, y0, b) in zip(res, ((a_csc, a_y0, a_b), (b_csc, b_y0, b_b), (c_csc, c_y0, c_b))):
        check_parity(r, oracle_run(csc, y0, b), len(csc))

"""Parity with the FP64 oracle at the sizes the benchmark configurations use
(GPU): the widest layers (65536 neurons, counted layer 0 then the tcgen05
kernel), the eight-network uneven mix with its 480-layer networks, a
sustained-activity network of 10000 rows x 120 layers whose categories are
not empty, and a batch split over two engines (row shards) against one.
Besides survivor counts and categories, the outputs of selected layers are
compared value by value with the oracle's FP64 replay of the same rows and
must lie within the error bound the engine carries for each row."""
import numpy as np
import pytest

from netgen import make_net, oracle_run

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
SEED = 20240611


@pytest.fixture(scope="module")
def cs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200
    cospdnn_b200.lib()
    return cospdnn_b200


def build(cs, nets, precision, kernel=0):
    """nets: list of (csc, y0, bias) -> engine with inputs set, ids."""
    eng = cs.Engine(0)
    ids = []
    for csc, y0, bias in nets:
        nid = eng.add_net(y0.shape[1], len(csc), y0.shape[0], float(bias), 1e-5, precision, kernel)
        for l, (cp, ri, vv) in enumerate(csc):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
    for nid, (_, y0, _) in zip(ids, nets):
        eng.set_input(nid, y0)
    return eng, ids


def check_values(oracle, eng, nid, csc, y0, bias, layer, max_rows=512):
    """Layer `layer`'s outputs of up to max_rows kept rows against the FP64
    replay: every row's max |dY| within the engine's bound for it; returns
    the max |dY| (0 when no row survived the layer)."""
    vals, ids, bnd = eng.layer_values(nid, layer, max_rows=max_rows, bounds=True)
    if len(ids) == 0:
        return 0.0
    assert np.all(np.diff(ids) > 0)
    want = oracle.replay_fp64(csc, y0, bias, ids.astype(np.int64), layer)
    d = np.abs(vals.astype(np.float64) - want).max(axis=1)
    assert np.all(d <= bnd.astype(np.float64)), (layer, float(d.max()), float(bnd[np.argmax(d - bnd)]))
    return float(d.max())


def test_65536_neurons_counted_layer0_and_feature_split(cs, oracle):
    """The C4 shape on 1024 rows x 120 layers: no row tile of 65536 FP16
    features fits one CTA's shared memory, so the engine splits 2-row tiles
    by feature over the two CTAs of a cluster (k_layer_cs) and counts layer 0
    from bit planes into 2-row tiles (k_layer0_bits16)."""
    csc, y0, b = make_net(65536, 120, 1024, seed=SEED, dlo=0.08, dhi=0.25)
    ref = oracle_run(csc, y0, b)
    eng, (nid,) = build(cs, [(csc, y0, b)], cs.PREC_FP16)
    eng.run()
    res = eng.result(nid)
    info = eng.net_info(nid)
    assert info["kernel"] == cs.KERNEL_CUDA_CORE and info["row_tile"] == 2 and info["layer0_counted"]
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    assert ref["alive"][0] > 0  # layer 1 runs on the split kernel
    dy0 = check_values(oracle, eng, nid, csc, y0, b, 0, max_rows=256)
    # layer 0 is counted exactly: the only error is the FP16 rounding of the output
    assert dy0 <= 32 * 2.0 ** -11
    if ref["alive"][1] > 0:
        check_values(oracle, eng, nid, csc, y0, b, 1, max_rows=256)
    eng.close()


def test_65536_neurons_sustained_feature_split_bf16_fp32_input(cs, oracle):
    """Layer 0 on the split kernel as well (FP32 inputs are not counted),
    BF16, 600 rows x 4 layers with denser inputs, so that rows survive into
    layers 2 and 3; odd row count (the last 2-row tile has one row)."""
    csc, y0, b = make_net(65536, 4, 601, seed=SEED + 3, dlo=0.3, dhi=0.45)
    rng = np.random.default_rng(5)
    y0f = (y0 * rng.uniform(0.5, 1.5, size=y0.shape)).astype(np.float32)
    ref = oracle_run(csc, y0f, b)
    eng, (nid,) = build(cs, [(csc, y0f, b)], cs.PREC_BF16)
    eng.run()
    res = eng.result(nid)
    info = eng.net_info(nid)
    assert info["row_tile"] == 2 and not info["layer0_counted"]
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    for l in range(4):
        if ref["alive"][l] > 0:
            check_values(oracle, eng, nid, csc, y0f, b, l, max_rows=128)
    eng.close()


def test_65536_neurons_feature_split_mixed_weights(cs, oracle):
    """Weights of several values (no compact entry lists: column and weight
    per entry) on the split kernel, FP16, 300 rows x 3 layers."""
    csc, y0, b = make_net(65536, 3, 300, seed=SEED + 4, dlo=0.2, dhi=0.35)
    rng = np.random.default_rng(9)
    csc = [(cp, ri, (vv * rng.choice([0.5, 1.0, 1.5], size=vv.shape)).astype(np.float32)) for cp, ri, vv in csc]
    ref = oracle_run(csc, y0, b)
    eng, (nid,) = build(cs, [(csc, y0, b)], cs.PREC_FP16)
    eng.run()
    res = eng.result(nid)
    assert eng.net_info(nid)["row_tile"] == 2
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    for l in range(3):
        if ref["alive"][l] > 0:
            check_values(oracle, eng, nid, csc, y0, b, l, max_rows=128)
    eng.close()


def test_65536_neurons_tcgen05_forced(cs, oracle):
    """tcgen05 at 65536 neurons on request (layer 0 counted into MMA tiles,
    then k_layer_tc), 512 rows x 6 layers."""
    csc, y0, b = make_net(65536, 6, 512, seed=SEED, dlo=0.08, dhi=0.25)
    ref = oracle_run(csc, y0, b)
    eng, (nid,) = build(cs, [(csc, y0, b)], cs.PREC_FP16, kernel=cs.KERNEL_TCGEN05)
    eng.run()
    res = eng.result(nid)
    info = eng.net_info(nid)
    assert info["kernel"] == cs.KERNEL_TCGEN05 and info["layer0_counted"]
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    if ref["alive"][0] > 0:
        check_values(oracle, eng, nid, csc, y0, b, 1, max_rows=128)
    eng.close()


def test_eight_network_mix_with_480_layer_networks(cs, oracle):
    """The seeded eight-network mix (1024/4096/16384 neurons, 120/480 layers)
    with each batch scaled down 40x: one graph, every network exact."""
    from cospdnn_b200 import synth
    mix = synth.mix_config(SEED)
    assert any(L == 480 for _, L, _ in mix)
    nets = []
    for i, (n, L, rows) in enumerate(mix):
        csc = synth.network(n, L, SEED, net=i)
        y0 = oracle.input_binary(SEED, i, max(64, rows // 40), n, 0.08, 0.25)
        nets.append((csc, y0, np.float32(cs.BIAS[n])))
    eng, ids = build(cs, nets, cs.PREC_FP16)
    eng.run()
    for nid, (csc, y0, b) in zip(ids, nets):
        res = eng.result(nid)
        ref = oracle_run(csc, y0, b)
        np.testing.assert_array_equal(res["alive"], ref["alive"])
        np.testing.assert_array_equal(res["categories"], ref["categories"])
    eng.close()


@pytest.mark.parametrize("prec", [0, 1, 2])
def test_sustained_activity_10000_rows_120_layers(cs, oracle, prec):
    """Input density U[0.25,0.45]: most rows survive all 120 layers, so the
    categories are not empty; survivor counts, categories and the values of
    the first, a middle and the last layer against the FP64 oracle."""
    csc, y0, b = make_net(1024, 120, 10000, seed=SEED, dlo=0.25, dhi=0.45)
    ref = oracle_run(csc, y0, b)
    assert len(ref["categories"]) > 1000
    eng, (nid,) = build(cs, [(csc, y0, b)], prec)
    eng.run()
    res = eng.result(nid)
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    for l in (0, 60, 119):
        check_values(oracle, eng, nid, csc, y0, b, l, max_rows=256)
    final = eng.final_values(nid, 10)
    assert final.shape == (10, 1024)
    eng.close()


def test_row_shards_on_two_engines_equal_one_engine(cs):
    """The batch split into contiguous row shards (cospdnn_b200.dist), one
    engine per shard on the same GPU: categories concatenated in shard order
    and survivor counts summed equal the unsharded run."""
    from cospdnn_b200.dist import shard_rows
    csc, y0, b = make_net(1024, 24, 3001, seed=SEED, dlo=0.2, dhi=0.45)
    eng, (nid,) = build(cs, [(csc, y0, b)], cs.PREC_FP16)
    eng.run()
    whole = eng.result(nid)
    eng.close()
    assert len(whole["categories"]) > 0
    cats, alive = [], np.zeros(24, np.int64)
    for rank in range(2):
        r0, r1 = shard_rows(len(y0), 2, rank)
        e, (k,) = build(cs, [(csc, y0[r0:r1], b)], cs.PREC_FP16)
        e.run()
        r = e.result(k)
        e.close()
        cats.append(r["categories"] + r0)
        alive += r["alive"]
    np.testing.assert_array_equal(np.concatenate(cats), whole["categories"])
    np.testing.assert_array_equal(alive, whole["alive"])


def test_layer_values_and_final_values_bounds(cs, oracle):
    """layer_values returns the kept rows of a layer in ascending id order
    with the same values as the graph run's final values at the last layer;
    final_values writes min(max_rows, count) rows and nothing for 0."""
    csc, y0, b = make_net(1024, 6, 700, seed=SEED + 7, dlo=0.25, dhi=0.45)
    eng, (nid,) = build(cs, [(csc, y0, b)], cs.PREC_FP16)
    eng.run()
    res = eng.result(nid)
    n = len(res["categories"])
    assert n > 10
    fin = eng.final_values(nid, n)
    vals, ids = eng.layer_values(nid, 5)
    np.testing.assert_array_equal(ids, res["categories"])
    np.testing.assert_array_equal(vals, fin)
    few = eng.final_values(nid, 3)
    np.testing.assert_array_equal(few, fin[:3])
    assert eng.final_values(nid, 0).shape == (0, 1024)
    # a layer before the last: rows kept after it, and every value within bound
    check_values(oracle, eng, nid, csc, y0, b, 2, max_rows=700)
    eng.close()


def test_layer_values_leaves_every_network_finished(cs):
    """layer_values of one network stops the eager pass at that layer to copy
    its rows, then runs the pass on to the end: afterwards every network's
    result equals the graph run's (the parity check of a multi-network
    configuration reads results after values)."""
    nets = [make_net(1024, 8, 900, seed=SEED + 11, dlo=0.25, dhi=0.45),
            make_net(4096, 10, 700, seed=SEED + 12, dlo=0.2, dhi=0.4)]
    eng, ids = build(cs, nets, cs.PREC_FP16)
    eng.run()
    want = [eng.result(nid) for nid in ids]
    vals, rid = eng.layer_values(ids[0], 1)
    assert len(rid) > 0
    for nid, w in zip(ids, want):
        r = eng.result(nid)
        np.testing.assert_array_equal(r["alive"], w["alive"])
        np.testing.assert_array_equal(r["categories"], w["categories"])
    eng.close()

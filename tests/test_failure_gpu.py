"""Device-side failure paths, exercised without a GPU fault (GPU).

Every wait of the engine's kernels is bounded and the layer loop has an
iteration guard.  These tests make one of them run out on purpose through
the engine's test hooks (cospdnn_engine_set_test_limits): a copy that the
tcgen05 kernel's producer never issues (its consumer's bounded wait gives up
after about 10 ms), a message that one CTA of the feature-split kernel's
cluster never sends to the other, and a loop guard of two iterations.  The run then stops,
the result call reports COSPDNN_ERR_DEVICE, and the next run with the default
limits is clean and exact against the FP64 oracle.  Nothing traps, faults or
hangs: the kernels return and the context stays usable."""
import numpy as np
import pytest

from netgen import make_net, oracle_run

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

WAIT = 20_000_000  # SM cycles, about 10 ms


@pytest.fixture(scope="module")
def cs():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200
    cospdnn_b200.lib()
    return cospdnn_b200


def build(cs, csc, y0, b, prec, kernel):
    eng = cs.Engine(0)
    nid = eng.add_net(y0.shape[1], len(csc), y0.shape[0], float(b), 1e-5, prec, kernel)
    for l, (cp, ri, vv) in enumerate(csc):
        eng.set_layer_csc(nid, l, cp, ri, vv)
    eng.build()
    eng.set_input(nid, y0)
    return eng, nid


def test_rejects_limits_that_would_fail_correct_runs(cs):
    csc, y0, b = make_net(256, 2, 64, seed=1)
    eng, _ = build(cs, csc, y0, b, cs.PREC_FP16, cs.KERNEL_AUTO)
    for args in ((1000, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, 2)):
        with pytest.raises(cs.CospdnnError) as e:
            eng.set_test_limits(*args)
        assert e.value.code == cs.ERR_INVALID
    eng.close()


@pytest.mark.parametrize("fp32_input", [False, True])
def test_tcgen05_wait_for_a_withheld_copy_runs_out(cs, fp32_input):
    """Binary inputs: layer 0 is counted and layer 1 is the first tcgen05
    launch; FP32 inputs: layer 0 already runs on tcgen05."""
    csc, y0, b = make_net(1024, 6, 2000, seed=71, dlo=0.2, dhi=0.4)
    if fp32_input:
        y0 = y0.astype(np.float32)
    ref = oracle_run(csc, y0, b)
    assert ref["alive"][0] > 0
    eng, nid = build(cs, csc, y0, b, cs.PREC_FP16, cs.KERNEL_TCGEN05)
    eng.set_test_limits(wait_cycles=WAIT, withhold_stage=1)
    for _ in range(2):  # the failure repeats on every run while the hook is set
        eng.run()
        with pytest.raises(cs.CospdnnError) as e:
            eng.result(nid)
        assert e.value.code == cs.ERR_DEVICE
    eng.set_test_limits()  # defaults again: the next run is clean and exact
    eng.run()
    res = eng.result(nid)
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    eng.close()


def test_loop_guard_stops_the_run(cs):
    csc, y0, b = make_net(1024, 8, 1500, seed=73, dlo=0.25, dhi=0.45)
    ref = oracle_run(csc, y0, b)
    assert ref["alive"][-1] > 0  # all 8 layers run
    eng, nid = build(cs, csc, y0, b, cs.PREC_FP16, cs.KERNEL_CUDA_CORE)
    eng.set_test_limits(max_iters=2)
    eng.run()
    with pytest.raises(cs.CospdnnError) as e:
        eng.result(nid)
    assert e.value.code == cs.ERR_DEVICE
    # the eager pass stops at the same guard
    ms = eng.profile_layers()
    assert len(ms) == 3
    with pytest.raises(cs.CospdnnError):
        eng.result(nid)
    eng.set_test_limits()
    eng.run()
    res = eng.result(nid)
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    eng.close()


def test_feature_split_wait_for_a_withheld_message_runs_out(cs):
    """65536 neurons take the feature-split kernel (two CTAs of a cluster
    exchange partial sums): the first CTA of the first cluster skips its
    first message, the other CTA's bounded wait for it runs out, then the
    first CTA's wait for the buffer's release; both stop and meet at the
    cluster barrier, the run reports COSPDNN_ERR_DEVICE, and the next run
    with the default limits is exact."""
    csc, y0, b = make_net(65536, 3, 600, seed=75, dlo=0.08, dhi=0.25)
    ref = oracle_run(csc, y0, b)
    assert ref["alive"][0] > 0  # layer 1 runs on the split kernel
    eng, nid = build(cs, csc, y0, b, cs.PREC_FP16, cs.KERNEL_AUTO)
    assert eng.net_info(nid)["row_tile"] == 2
    eng.set_test_limits(wait_cycles=WAIT, withhold_stage=1)
    eng.run()
    with pytest.raises(cs.CospdnnError) as e:
        eng.result(nid)
    assert e.value.code == cs.ERR_DEVICE
    eng.set_test_limits()
    eng.run()
    res = eng.result(nid)
    np.testing.assert_array_equal(res["alive"], ref["alive"])
    np.testing.assert_array_equal(res["categories"], ref["categories"])
    eng.close()

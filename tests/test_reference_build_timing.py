"""The reference's own CUDA build (its host loop test_graph_challenge_tc and
kernels, compiled from its sources for sm_100a into oracle/_ref) timed on
the same synthetic workloads as bench.py: XOR-mask weights and seeded binary
inputs with 60000 rows.

Timing only: on these weights the reference's kernel reads two 16x16 blocks
per block column (src/kernels/kernel.cu:257) while the XOR masks give about
19-32, so its product is truncated and its survivor counts differ from the
true recurrence's.  Prints one JSON line per workload with the reference's
own "Kernel Exec Time" (its CUDA events around the layer kernels) and the
wall time of its whole host loop (allocation, copies, per-layer host
compaction), and appends it to $COSPDNN_REF_TIMING_OUT when that is set."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libref_cospdnn.so")
SEED = 20240611
BIAS = {1024: -0.3, 4096: -0.35, 16384: -0.4}


# the 16384-neuron workload spends about 90 s in the reference's host code:
# only with COSPDNN_REF_TIMING_FULL=1
WORKLOADS = [("c1", 1024, "xor"), ("c2", 4096, "xor"), ("r1", 4096, "r1")]
if os.environ.get("COSPDNN_REF_TIMING_FULL") == "1":
    WORKLOADS.insert(2, ("c3", 16384, "xor"))


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("name,neuron,kind", WORKLOADS)
def test_reference_build_timing(oracle, name, neuron, kind):
    """r1: two aligned dense 16x16 blocks per block column, the structure the
    reference's kernel computes in full (its last-stage race can still make
    its outputs timing-dependent); the others are timing only."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cospdnn_b200 import synth
    from test_reference_loop_gpu import run_reference_loop
    layers, rows = 120, 60000
    csc = synth.network(neuron, layers, SEED, net=0, kind=kind)
    y0 = oracle.input_binary(SEED, 0, rows, neuron, 0.08, 0.25)
    feats, kms, wms = run_reference_loop(oracle, csc, y0, BIAS[neuron], want_wall=True)
    assert kms > 0 and wms > 0
    edges = float(rows) * layers * 32 * neuron
    line = {"workload": f"{name}: {neuron} neurons x {layers} layers, {rows} rows, {kind} W, "
                        f"binary Y0 density U[0.08,0.25]",
            "impl": "reference CUDA build (sm_100a), timing only",
            "kernel_exec_ms": kms, "wall_ms": wms,
            "edges_per_s_kernel": edges / (kms * 1e-3), "edges_per_s_wall": edges / (wms * 1e-3),
            "printed_features": [int(x) for x in feats[:8] if x >= 0]}
    print(json.dumps(line))
    out = os.environ.get("COSPDNN_REF_TIMING_OUT")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(line) + "\n")


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference not built (make -C oracle ref)")
@pytest.mark.parametrize("neuron", [1024, 4096])
def test_layer_entry_timing_vs_reference_kernel(oracle, neuron):
    """The drop-in layer entry beside the reference's cospdnn_single on the
    same buffers: its BCSC of one R1 layer (two dense blocks per column, what
    its kernel computes in full), hi/lo FP16 activations of 60032 columns.
    CUDA-event time per launch (median of 20, after 5 warm-up launches); the
    outputs agree in the reference-arithmetic mode where the reference's
    last-stage race cannot act (weights only in one quadrant of each block)."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import cospdnn_b200 as cs
    from test_layer_gpu import _ref_kernel, dev, hilo
    from cospdnn_b200 import synth
    batch = 60032  # 60000 padded to the reference kernel's 64-column tile, as its host loop does (src/cospdnn.cu:24)
    cp, ri, vv = synth.network(neuron, 1, SEED, net=0, kind="r1")[0]
    row, col, val = oracle.csc_to_coo(cp, ri, vv)
    bcp, bri, _, bvals = oracle.bcsc_greedy(row, col, val, 16)
    V = bvals.reshape(-1, 16, 16)
    V[:, 8:, :] = 0  # race-free (as in the reference pin of test_layer_gpu.py):
    V[:, :, 8:] = 0  # only the [k<8][r<8] quadrant of each block is non-zero
    bvals = np.ascontiguousarray(V.reshape(-1))
    rng = np.random.default_rng(5)
    a = (rng.random((neuron, batch)) < 0.2).astype(np.float32)
    A, B = dev(hilo(a)), dev(bvals, torch.float16)
    F = dev(np.arange(neuron, dtype=np.int32))
    P, I = dev(bcp), dev(bri)
    nbc = len(bcp) - 1
    ref = _ref_kernel()
    out_ref = torch.empty((neuron, batch), dtype=torch.float32, device="cuda")
    out = torch.empty_like(out_ref)

    def time_it(fn):
        for _ in range(5):
            fn()
        ts = []
        for _ in range(20):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    t_ref = time_it(lambda: ref.ref_cospdnn_single(A.data_ptr(), B.data_ptr(), out_ref.data_ptr(), F.data_ptr(),
                                                   P.data_ptr(), I.data_ptr(), -0.35, batch, neuron, nbc, None))
    t_ra = time_it(lambda: cs.layer(A, B, out, F, P, I, -0.35, batch, neuron, flags=cs.LAYER_REFERENCE_ARITH))
    torch.cuda.synchronize()
    np.testing.assert_allclose(out.cpu().numpy(), out_ref.cpu().numpy(), rtol=0, atol=5e-5)
    t_true = time_it(lambda: cs.layer(A, B, out, F, P, I, -0.35, batch, neuron))
    line = {"workload": f"one R1 layer, {neuron} neurons, batch {batch}, hi/lo FP16 activations",
            "reference_cospdnn_single_ms": t_ref, "cospdnn_layer_reference_arith_ms": t_ra,
            "cospdnn_layer_true_product_ms": t_true}
    print(json.dumps(line))
    out_path = os.environ.get("COSPDNN_REF_TIMING_OUT")
    if out_path:
        with open(out_path, "a") as f:
            f.write(json.dumps(line) + "\n")

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

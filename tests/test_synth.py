"""The product's synthetic generator (cospdnn_b200.synth, cospdnn_synth_input)
produces exactly the oracle's seeded streams."""
import numpy as np
import pytest

from cospdnn_b200 import synth


@pytest.mark.parametrize("n", [1024, 4096, 65536])
def test_masks_match_oracle(oracle, n):
    for l in range(3):
        np.testing.assert_array_equal(synth.xor_masks(5, 2, l, n), oracle.xor_masks(5, 2, l, n))
        np.testing.assert_array_equal(synth.r1_masks(5, 2, l, n), oracle.r1_masks(5, 2, l, n))


def test_csc_matches_oracle(oracle):
    m = synth.xor_masks(1, 0, 0, 2048)
    for a, b in zip(synth.masks_to_csc(m, 2048), oracle.masks_to_csc(m, 2048)):
        np.testing.assert_array_equal(a, b)


def test_mix_config_matches_oracle(oracle):
    assert synth.mix_config(77) == oracle.mix_config(77)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", [0, 2])
def test_gpu_input_generator_matches_oracle(oracle, fmt):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rows, n = 300, 1024
    want = oracle.input_binary(9, 3, rows, n, 0.08, 0.25, row0=1000)
    got = synth.input_rows(rows, n, 9, net=3, row0=1000, fmt=fmt).cpu().numpy()
    if fmt == 2:
        got = np.unpackbits(got, axis=1, bitorder="little")
    np.testing.assert_array_equal(got, want)

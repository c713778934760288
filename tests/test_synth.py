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


@pytest.mark.parametrize("seed,net,rows,n,dlo,dhi,row0", [(9, 3, 300, 1024, 0.08, 0.25, 1000),
                                                          (1, 0, 700, 4096, 0.2, 0.4, 0),
                                                          (7, 5, 37, 64, 0.0, 1.0, 123456)])
def test_host_input_generator_matches_oracle(oracle, seed, net, rows, n, dlo, dhi, row0):
    """The host (numpy) generator makes the bytes the GPU generator makes:
    both equal the oracle's streams."""
    np.testing.assert_array_equal(synth.input_rows_host(rows, n, seed, net=net, dlo=dlo, dhi=dhi, row0=row0),
                                  oracle.input_binary(seed, net, rows, n, dlo, dhi, row0=row0))


def test_dataset_command(oracle, tmp_path, capsys):
    """python -m cospdnn_b200.synth writes the seeded network and rows in the
    reference's formats (1-based "b n 1" images, "u v 0.0625" weights,
    identity fuse)."""
    out = tmp_path / "d"
    assert synth.main([str(out), "64", "3", "20", "--seed", "5", "--kind", "r1"]) == 0
    assert "64 neurons x 3 layers (r1), 20 rows" in capsys.readouterr().out
    img = np.loadtxt(out / "sparse-images-64.tsv", ndmin=2)
    y = np.zeros((20, 64), np.uint8)
    y[img[:, 0].astype(int) - 1, img[:, 1].astype(int) - 1] = 1
    np.testing.assert_array_equal(y, oracle.input_binary(5, 0, 20, 64))
    for l in range(3):
        w = np.loadtxt(out / "neuron64" / f"64-l{l + 1}.tsv", ndmin=2)
        cp, ri, vv = oracle.masks_to_csc(oracle.r1_masks(5, 0, l, 64), 64)
        col = np.repeat(np.arange(64), np.diff(cp))
        got = sorted(zip((w[:, 0] - 1).astype(int), (w[:, 1] - 1).astype(int)))
        assert got == sorted(zip(ri.tolist(), col.tolist())) and np.all(w[:, 2] == 0.0625)
    fuse = np.loadtxt(out / "fuse_matrix" / "neuron64" / "64_3_fuse.tsv", dtype=np.int64)
    np.testing.assert_array_equal(fuse, np.tile(np.arange(64), (3, 1)))
    with pytest.raises(SystemExit):
        synth.main([str(out), "60", "1", "1", "--kind", "r1"])
    blocker = tmp_path / "file"
    blocker.write_text("")
    assert synth.main([str(blocker / "d"), "64", "1", "2"]) == 1  # cannot create the directory

"""The similarity reordering (cospdnn_b200.reorder) on CPU: it recovers hidden
block structure (rows of dense-block layers renamed by a permutation) down to
the aligned blocks the reference's greedy builder makes for the unpermuted
layer, never increases the block count, keeps the product (W' read through
the fuse row equals W), and its block count is the reference builder's."""
import numpy as np
import pytest

from netgen import half_block_layer, permute_rows, random_layer, shift_half_block_layer
from cospdnn_b200 import reorder as ro


def _fold(csc, fuse, n, oracle):
    """W[fuse[u']][v] = W'[u'][v]: the product the reference computes."""
    row, col, val = oracle.csc_to_coo(*csc)
    return oracle.coo_to_csc(np.asarray(fuse)[row], col, val, n)


def _same(a, b):
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


@pytest.mark.parametrize("n,seed", [(1024, 3), (4096, 8)])
def test_hidden_r1_blocks_recovered(oracle, n, seed):
    layer = oracle.masks_to_csc(oracle.r1_masks(seed, 0, 0, n), n)
    hidden = permute_rows(layer, n, seed)
    order, csc, before, after = ro.reorder_layer(*hidden, n)
    row, col, val = oracle.csc_to_coo(*csc)
    bcp, bri, _, _ = oracle.bcsc_greedy(row, col, val, 16)
    assert np.all(np.diff(bcp) == 2) and np.all(bri % 16 == 0)
    assert after == len(bri) == 2 * (n // 16) < before
    _same(_fold(csc, order, n, oracle), hidden)


def test_shifted_half_blocks_two_aligned_blocks(oracle):
    n = 1024
    for l in range(4):
        hidden = permute_rows(shift_half_block_layer(n, 5, l), n, 50 + l)
        order, csc, before, after = ro.reorder_layer(*hidden, n)
        row, col, val = oracle.csc_to_coo(*csc)
        bcp, bri, _, _ = oracle.bcsc_greedy(row, col, val, 16)
        assert np.all(np.diff(bcp) == 2) and np.all(bri % 16 == 0) and after < before
        # the non-zeros sit in the first 8 rows of each block (offsets 0..7)
        assert np.all(np.isin(row % 16, np.arange(8)))
        _same(_fold(csc, order, n, oracle), hidden)


def test_xor_half_blocks_merge(oracle):
    """Under XOR structure the two row groups of a column have equal
    signatures and share one aligned block: one block per column."""
    n = 1024
    hidden = permute_rows(half_block_layer(n, 2, 0, 0), n, 7)
    order, csc, before, after = ro.reorder_layer(*hidden, n)
    assert after == n // 16 < before
    _same(_fold(csc, order, n, oracle), hidden)


@pytest.mark.parametrize("kind", ["xor", "random", "r1"])
def test_never_more_blocks_and_count_matches_builder(oracle, kind):
    n = 1024
    for l in range(3):
        if kind == "xor":
            layer = oracle.masks_to_csc(oracle.xor_masks(11, 0, l, n), n)
        elif kind == "random":
            layer = random_layer(n, 11, l)
        else:
            layer = oracle.masks_to_csc(oracle.r1_masks(11, 0, l, n), n)
        row, col, val = oracle.csc_to_coo(*layer)
        assert ro.greedy_blocks(row, col, n) == len(oracle.bcsc_greedy(row, col, val, 16)[1])
        order, csc, before, after = ro.reorder_layer(*layer, n)
        assert after <= before
        if after == before:
            np.testing.assert_array_equal(order, np.arange(n))
        r2, c2, v2 = oracle.csc_to_coo(*csc)
        assert ro.greedy_blocks(r2, c2, n) == len(oracle.bcsc_greedy(r2, c2, v2, 16)[1]) == after
        _same(_fold(csc, order, n, oracle), layer)


def test_reorder_network_and_main(oracle, tmp_path, capsys):
    from cospdnn_b200 import synth
    n, L = 1024, 3
    layers = [permute_rows(shift_half_block_layer(n, 9, l), n, 90 + l) for l in range(L)]
    out, fuse, stats = ro.reorder_network(layers, n)
    assert len(out) == len(fuse) == L and all(b < a for a, b in stats)
    y0 = (np.random.default_rng(1).random((20, n)) < 0.2).astype(np.uint8)
    synth.write_reference_dataset(str(tmp_path / "src"), n, L, y0, layers)
    assert ro.main([str(tmp_path / "src"), str(tmp_path / "dst"), str(n), str(L)]) == 0
    assert "greedy 16x16 blocks:" in capsys.readouterr().out
    f = np.loadtxt(tmp_path / "dst" / "fuse_matrix" / f"neuron{n}" / f"{n}_{L}_fuse.tsv", dtype=np.int64)
    for l in range(L):
        np.testing.assert_array_equal(f[l], fuse[l])


def test_block_count_random_layers_with_empty_columns(oracle):
    """The block count (block columns walked in step) equals the reference
    builder's on random patterns, including empty columns, so that block
    columns start off multiples of 16, and widths that are not multiples of 16."""
    rng = np.random.default_rng(5)
    for trial in range(120):
        n = int(rng.choice([16, 48, 100, 256, 1000]))
        nnz = int(rng.integers(1, 6 * n))
        rows, cols = rng.integers(0, n, nnz), rng.integers(0, n, nnz)
        if trial % 3 == 0:
            cols = cols // 7 * 7
        key = np.unique(rows * n + cols)
        rows, cols = key // n, key % n
        want = len(oracle.bcsc_greedy(rows, cols, np.ones(len(rows), np.float32), 16)[1])
        assert ro.greedy_blocks(rows, cols, n) == want, trial
    assert ro.greedy_blocks([], [], 64) == 0


def test_parallel_layers_write_the_same_files(tmp_path):
    from cospdnn_b200 import synth
    n, L = 1024, 3
    layers = [permute_rows(shift_half_block_layer(n, 13, l), n, 130 + l) for l in range(L)]
    y0 = (np.random.default_rng(2).random((10, n)) < 0.2).astype(np.uint8)
    synth.write_reference_dataset(str(tmp_path / "src"), n, L, y0, layers)
    one = ro.reorder_dataset(str(tmp_path / "src"), str(tmp_path / "one"), n, L, workers=1)
    assert ro.main([str(tmp_path / "src"), str(tmp_path / "many"), str(n), str(L), "--workers", "3"]) == 0
    rel = [f"neuron{n}/{n}-l{l + 1}.tsv" for l in range(L)] + [f"fuse_matrix/neuron{n}/{n}_{L}_fuse.tsv"]
    for r in rel:
        assert (tmp_path / "one" / r).read_bytes() == (tmp_path / "many" / r).read_bytes(), r
    assert all(b < a for a, b in one)
    assert ro.main([str(tmp_path / "src"), str(tmp_path / "x"), str(n), "--workers"]) == 1


@pytest.mark.parametrize("name", ["bcsc_r1_n256", "bcsc_rand_n80_gaps", "bcsc_rand_n96", "bcsc_xor_n128_m32",
                                  "bcsc_xor_n256_m32", "bcsc_xor_n64_bs8", "bcsc_xor_n64_m8"])
def test_block_count_matches_reference_builder_fixtures(name):
    """The block count equals the number of blocks the reference's own
    builder (compiled from its sources) made for the golden fixtures."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", name + ".npz"))
    n = int(max(g["row"].max(), g["col"].max())) + 1
    assert ro.greedy_blocks(g["row"], g["col"], n, int(g["bs"])) == len(g["row_index"])


def test_main_reports_missing_or_damaged_files(tmp_path, capsys):
    from cospdnn_b200 import synth
    n = 64
    assert ro.main([str(tmp_path / "none"), str(tmp_path / "out"), str(n), "2", "--workers", "1"]) == 1
    assert "reorder: " in capsys.readouterr().out
    layers = [random_layer(n, 3, l) for l in range(2)]
    synth.write_reference_dataset(str(tmp_path / "src"), n, 2, np.ones((2, n), np.uint8), layers)
    with open(tmp_path / "src" / f"neuron{n}" / f"{n}-l2.tsv", "a") as f:
        f.write("65\t1\t0.5\n")
    assert ro.main([str(tmp_path / "src"), str(tmp_path / "out"), str(n), "2", "--workers", "1"]) == 1
    assert "index out of range" in capsys.readouterr().out



def test_mma_regions_counts_aligned_regions():
    from cospdnn_b200 import synth
    # hand-made: output 0 <- inputs 0 and 17, output 20 <- input 3 (N = 32)
    colptr = np.zeros(33, np.int64)
    colptr[1:] = 2
    colptr[21:] = 3
    rowidx = np.array([0, 17, 3])
    assert ro.mma_regions(colptr, rowidx, 32, 16, 16) == 3   # (0,0) (1,0) (0,1)
    assert ro.mma_regions(colptr, rowidx, 32, 16, 32) == 2   # (0,0) (1,0)
    assert ro.mma_regions(colptr, rowidx, 32, 32, 32) == 1
    # two dense aligned 16x16 blocks per block column
    cp, ri, _ = synth.masks_to_csc(synth.r1_masks(7, 0, 0, 256), 256)
    assert ro.mma_regions(cp, ri, 256, 16, 16) == 2 * 256 // 16
    # XOR masks: both 8-output halves of a 16-output group read the same input blocks
    cp, ri, _ = synth.masks_to_csc(synth.xor_masks(7, 0, 0, 1024), 1024)
    assert ro.mma_regions(cp, ri, 1024, 16, 8) == 2 * ro.mma_regions(cp, ri, 1024, 16, 16)

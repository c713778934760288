"""Host logic of the Python mirrors of the reference's host functions
(cospdnn_b200.test_graph_challenge_tc and test_graph_challenge_tc_co,
src/cospdnn.cuh:14-35), on the CPU with a recording stand-in for the engine:
the rows of slice gpu_id of gpu_num (src/cospdnn.cu:23,35-44,
src/cospdnn_double.cu:236-274), every layer's BCSC arrays and fuse row
handed over, binary rows as bytes and others as floats, both networks of the
two-network call in one engine with one build and one run, categories moved
to batch row ids, and the reference's printed lines."""
import numpy as np
import pytest

import cospdnn_b200 as cs


class FakeEngine:
    """Records the calls the mirrors make; result() reports the first and
    last local row as categories and layer l with l + 1 survivors."""
    created = []

    def __init__(self, device=0):
        self.device, self.nets, self.layers, self.inputs = device, [], {}, {}
        self.builds = self.runs = 0
        self.closed = False
        FakeEngine.created.append(self)

    def add_net(self, neuron, layers, rows, bias=None, threshold=cs.THRESHOLD, precision=cs.PREC_FP16,
                kernel=cs.KERNEL_AUTO):
        self.nets.append(dict(neuron=neuron, layers=layers, rows=rows, bias=bias, threshold=threshold,
                              precision=precision))
        return len(self.nets) - 1

    def set_layer_bcsc(self, net, layer, col_ptr, row_index, values, blocksize=16, fuse=None):
        assert not self.builds
        self.layers[(net, layer)] = (col_ptr, row_index, values, blocksize, fuse)

    def build(self):
        self.builds += 1

    def set_input(self, net, y0, fmt=None, stream=None):
        assert self.builds == 1
        self.inputs[net] = y0

    def run(self, stream=None):
        self.runs += 1

    def result(self, net, stream=None):
        d = self.nets[net]
        return dict(categories=np.array([0, d["rows"] - 1], np.int32),
                    alive=np.arange(1, d["layers"] + 1, dtype=np.int64))

    def close(self):
        self.closed = True


def _net(rng, batch, neuron, layers, binary):
    x = (rng.random((batch, neuron)) < 0.3).astype(np.float32)
    if not binary:
        x *= 0.5
    w = [rng.random(256).astype(np.float32) for _ in range(layers)]
    ri = [np.array([0], np.int32) for _ in range(layers)]
    ptr = [np.array([0, 1], np.int32) for _ in range(layers)]
    fuse = [rng.permutation(neuron).astype(np.int32) for _ in range(layers)]
    return x, w, ri, ptr, fuse


@pytest.fixture
def fake(monkeypatch):
    FakeEngine.created = []
    monkeypatch.setattr(cs, "Engine", FakeEngine)
    return FakeEngine


def test_single_network_slice_and_output(fake, capsys):
    rng = np.random.default_rng(1)
    x, w, ri, ptr, fuse = _net(rng, 101, 64, 3, True)
    res = cs.test_graph_challenge_tc(x, w, ri, ptr, fuse, 101, 64, -0.3, gpu_id=1, gpu_num=2)
    (e,) = fake.created
    assert e.device == 1 and e.builds == 1 and e.runs == 1 and e.closed
    assert e.nets[0]["rows"] == 50 and e.nets[0]["layers"] == 3   # rows 51..100 of 101
    np.testing.assert_array_equal(e.inputs[0], x[51:101])
    assert e.inputs[0].dtype == np.uint8
    for l in range(3):
        assert e.layers[(0, l)][4] is fuse[l] and e.layers[(0, l)][0] is ptr[l]
    np.testing.assert_array_equal(res["categories"], [51, 100])
    assert capsys.readouterr().out.splitlines() == [f"layer {l}, feature = {l + 1}" for l in range(3)]


def test_two_networks_one_engine(fake, capsys):
    rng = np.random.default_rng(2)
    a = _net(rng, 90, 64, 2, True)
    b = _net(rng, 41, 128, 4, False)   # other width, depth and batch; non-binary rows
    r1, r2 = cs.test_graph_challenge_tc_co(*a, 90, 64, -0.3, *b, 41, 128, -0.35, gpu_id=0, gpu_num=1)
    (e,) = fake.created
    assert e.builds == 1 and e.runs == 1 and e.closed and e.device == 0
    assert [(d["neuron"], d["layers"], d["rows"], d["bias"]) for d in e.nets] == [(64, 2, 90, -0.3),
                                                                                   (128, 4, 41, -0.35)]
    assert e.inputs[0].dtype == np.uint8 and e.inputs[1].dtype == np.float32
    np.testing.assert_array_equal(e.inputs[1], b[0])
    assert sorted(e.layers) == [(0, 0), (0, 1), (1, 0), (1, 1), (1, 2), (1, 3)]
    assert e.layers[(1, 2)][4] is b[4][2] and e.layers[(1, 2)][2] is b[1][2]
    np.testing.assert_array_equal(r1["categories"], [0, 89])
    np.testing.assert_array_equal(r2["categories"], [0, 40])
    out = capsys.readouterr().out.splitlines()
    assert out == ([f"SpDNN 1 layer {l}, feature = {l + 1}" for l in range(2)] +
                   [f"SpDNN 2 layer {l}, feature = {l + 1}" for l in range(4)])


def test_two_networks_slices_and_no_fuse(fake):
    rng = np.random.default_rng(3)
    a = list(_net(rng, 10, 64, 1, True))
    b = list(_net(rng, 7, 64, 1, True))
    a[4] = b[4] = None
    r1, r2 = cs.test_graph_challenge_tc_co(*a, 10, 64, -0.3, *b, 7, 64, -0.3, gpu_id=2, gpu_num=3,
                                           verbose=False)
    (e,) = fake.created
    assert e.device == 2
    assert [d["rows"] for d in e.nets] == [2, 1]          # rows 8..9 of 10, row 6 of 7
    assert e.layers[(0, 0)][4] is None and e.layers[(1, 0)][4] is None
    np.testing.assert_array_equal(r1["categories"], [8, 9])
    np.testing.assert_array_equal(r2["categories"], [6, 6])


def test_square_blocks_only(fake):
    rng = np.random.default_rng(4)
    a = _net(rng, 4, 64, 1, True)
    with pytest.raises(cs.CospdnnError):
        cs.test_graph_challenge_tc_co(*a, 4, 64, -0.3, *a, 4, 64, -0.3, blocksize_c=16, blocksize_r=8)
    assert not fake.created


def test_mirrors_are_not_collected_as_tests():
    assert cs.test_graph_challenge_tc.__test__ is False
    assert cs.test_graph_challenge_tc_co.__test__ is False

"""The reference's command lines, rebuilt over the C ABI
(cospdnn_b200/cli/cospdnn.out and cospdnn_double.out): argv, dataset files
(src/cospdnn.cpp:13-79) and the per-layer survivor lines, checked against the
FP64 oracle on a dataset written in the reference's formats with a
non-trivial fuse permutation."""
import os
import re
import subprocess

import numpy as np
import pytest

from netgen import make_net, oracle_run

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "cospdnn_b200", "cli")


def _exe(name):
    p = os.path.join(CLI, name + ".out")
    if not os.path.exists(p):
        pytest.skip("command lines not built (python -m cospdnn_b200.build)")
    return p


@pytest.mark.parametrize("name,nargs", [("cospdnn", 6), ("cospdnn_double", 8)])
def test_cli_usage(name, nargs):
    out = subprocess.run([_exe(name)] + ["1"] * (nargs - 1), capture_output=True, text=True, timeout=60)
    assert out.returncode == 0
    assert out.stdout.startswith("Usage: exe neuron")


@pytest.mark.parametrize("nargs", [1, 4, 7])
def test_cli_multi_usage(nargs):
    """cospdnn_multi.out takes three numbers per network, then gpu_id and
    dataset_dir: any other count prints the usage line."""
    out = subprocess.run([_exe("cospdnn_multi")] + ["1"] * nargs, capture_output=True, text=True, timeout=60)
    assert out.returncode == 0
    assert out.stdout.startswith("Usage: exe neuron1 batch1 layer1 [neuron2 batch2 layer2 ...]")


def test_cli_multi_fails_without_a_device(tmp_path):
    """Three networks (two widths, one read twice) are parsed and cached; with
    no CUDA device visible the run then ends with an error, not a result."""
    from cospdnn_b200 import synth
    for n, seed in ((64, 5), (128, 6)):
        csc, y0, _ = make_net(n, 2, 10, seed=seed, dlo=0.2, dhi=0.4)
        synth.write_reference_dataset(str(tmp_path / "d"), n, 2, y0, csc)
    (tmp_path / "c").mkdir()
    out = subprocess.run([_exe("cospdnn_multi"), "64", "10", "2", "128", "10", "2", "64", "8", "2", "0",
                          str(tmp_path / "d")], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES="", COSPDNN_CACHE=str(tmp_path / "c")))
    assert out.returncode != 0
    assert "[Neuron3] :64" in out.stdout and "Total Kernel Exec Time" not in out.stdout
    assert (tmp_path / "c" / "cospdnn-n64-b10-l2.bin").stat().st_size > 0
    assert (tmp_path / "c" / "cospdnn-n128-b10-l2.bin").stat().st_size > 0
    # a zero or negative size is rejected before any file is read
    out = subprocess.run([_exe("cospdnn_multi"), "64", "10", "2", "128", "0", "2", "0", str(tmp_path / "d")],
                         capture_output=True, text=True, timeout=60)
    assert out.returncode != 0 and "bad arguments" in out.stdout


@pytest.mark.parametrize("gpu_num", [1, 2])
def test_cli_fails_without_a_device(tmp_path, gpu_num):
    """With no CUDA device visible the program exits with an error for one
    GPU and for several (it does not report an empty result)."""
    from cospdnn_b200 import synth
    csc, y0, _ = make_net(64, 2, 10, seed=1, dlo=0.2, dhi=0.4)
    synth.write_reference_dataset(str(tmp_path), 64, 2, y0, csc)
    out = subprocess.run([_exe("cospdnn"), "64", "10", "2", str(gpu_num), "0", str(tmp_path)], capture_output=True,
                         text=True, timeout=120, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert out.returncode != 0
    assert "Kernel Exec Time" not in out.stdout and "[Categories]" not in out.stdout


def test_cli_writes_cache_before_it_needs_a_device(tmp_path):
    """The dataset is parsed and cached before the first CUDA call, so a run
    on a host without a GPU prepares the cache (and then stops with an error)."""
    from cospdnn_b200 import synth
    csc, y0, _ = make_net(64, 2, 10, seed=2, dlo=0.2, dhi=0.4)
    synth.write_reference_dataset(str(tmp_path / "d"), 64, 2, y0, csc)
    (tmp_path / "c").mkdir()
    out = subprocess.run([_exe("cospdnn"), "64", "10", "2", "1", "0", str(tmp_path / "d")], capture_output=True,
                         text=True, timeout=120,
                         env=dict(os.environ, CUDA_VISIBLE_DEVICES="", COSPDNN_CACHE=str(tmp_path / "c")))
    assert out.returncode != 0
    assert (tmp_path / "c" / "cospdnn-n64-b10-l2.bin").stat().st_size > 0


@pytest.mark.parametrize("fault,message", [
    ("no_images", "sparse-images-64.tsv does not exists."),
    ("no_layer", "64-l2.tsv does not exists."),
    ("weight_index", "weight index out of range in"),
    ("fuse_entry", "fuse entry out of range in"),
    ("fuse_short", "read error"),
    ("image_neuron", "input neuron index out of range in"),
    ("layer_is_dir", "64-l2.tsv cannot be read."),
    ("images_is_dir", "sparse-images-64.tsv cannot be read."),
])
def test_cli_bad_dataset_files(tmp_path, fault, message):
    """Damaged dataset files end the run with the reference's kind of message
    and a non-zero exit status, before any device is needed."""
    from cospdnn_b200 import synth
    csc, y0, _ = make_net(64, 2, 10, seed=3, dlo=0.2, dhi=0.4)
    d = tmp_path / "d"
    synth.write_reference_dataset(str(d), 64, 2, y0, csc)
    fuse = d / "fuse_matrix" / "neuron64" / "64_2_fuse.tsv"
    if fault == "no_images":
        (d / "sparse-images-64.tsv").unlink()
    elif fault == "no_layer":
        (d / "neuron64" / "64-l2.tsv").unlink()
    elif fault == "weight_index":
        with open(d / "neuron64" / "64-l1.tsv", "a") as f:
            f.write("65\t1\t0.0625\n")
    elif fault == "fuse_entry":
        fuse.write_text("64 " + fuse.read_text())
    elif fault == "fuse_short":
        fuse.write_text(fuse.read_text().split("\n")[0] + "\n")
    elif fault == "layer_is_dir":
        (d / "neuron64" / "64-l2.tsv").unlink()
        (d / "neuron64" / "64-l2.tsv").mkdir()
    elif fault == "images_is_dir":
        (d / "sparse-images-64.tsv").unlink()
        (d / "sparse-images-64.tsv").mkdir()
    else:
        with open(d / "sparse-images-64.tsv", "a") as f:
            f.write("1\t65\t1\n")
    out = subprocess.run([_exe("cospdnn"), "64", "10", "2", "1", "0", str(d)], capture_output=True, text=True,
                         timeout=120, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert out.returncode != 0
    assert message in out.stdout, out.stdout


@pytest.mark.parametrize("var,value", [("COSPDNN_PRECISION", "fp8"), ("COSPDNN_KERNEL", "wgmma")])
def test_cli_rejects_unknown_settings(tmp_path, var, value):
    """An unknown precision or kernel name is an error, not the default."""
    from cospdnn_b200 import synth
    csc, y0, _ = make_net(64, 2, 10, seed=4, dlo=0.2, dhi=0.4)
    synth.write_reference_dataset(str(tmp_path), 64, 2, y0, csc)
    out = subprocess.run([_exe("cospdnn"), "64", "10", "2", "1", "0", str(tmp_path)], capture_output=True,
                         text=True, timeout=120, env=dict(os.environ, CUDA_VISIBLE_DEVICES="", **{var: value}))
    assert out.returncode != 0 and f"{var} must be" in out.stdout


def _dataset(tmp, n, L, rows, seed, net):
    """Writes a net in the reference's formats with a random fuse per layer and
    returns the oracle's view (weights folded through the fuse)."""
    from cospdnn_b200 import synth
    from oracle import pyoracle as po
    csc, y0, b = make_net(n, L, rows, seed=seed, net=net, dlo=0.2, dhi=0.4)
    rng = np.random.default_rng(seed)
    fuse = [rng.permutation(n).astype(np.int32) for _ in range(L)]
    synth.write_reference_dataset(str(tmp), n, L, y0, csc, fuse=fuse)
    folded = []
    for l, (cp, ri, vv) in enumerate(csc):
        row, col, val = po.csc_to_coo(cp, ri, vv)
        folded.append(po.coo_to_csc(fuse[l][row], col, val, n))
    return oracle_run(folded, y0, b)


def _alive(text, prefix):
    pat = re.compile(prefix + r"layer (\d+), feature = (\d+)")
    got = {}
    for m in pat.finditer(text):
        got[int(m.group(1))] = int(m.group(2))
    return [got[k] for k in sorted(got)]


def _per_layer(text, pat):
    return {int(m.group(1)): m.group(2) for m in re.finditer(pat, text)}


def _pad(n):
    return (int(n) + 127) // 128 * 128


@pytest.mark.gpu
def test_cli_single_matches_oracle(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cospdnn_b200 import categories as cat
    ref = _dataset(tmp_path, 1024, 6, 500, 43, 0)
    truth = tmp_path / "truth.tsv"
    cat.write(truth, ref["categories"])
    (tmp_path / "cache").mkdir()
    for prec in ("fp16", "fp32", "fp16"):  # the second fp16 run reads the binary cache
        ours = tmp_path / f"ours-{prec}.tsv"
        env = dict(os.environ, COSPDNN_PRECISION=prec, COSPDNN_CATEGORIES=str(ours), COSPDNN_TRUTH=str(truth),
                   COSPDNN_CACHE=str(tmp_path / "cache"))
        out = subprocess.run([_exe("cospdnn"), "1024", "500", "6", "1", "0", str(tmp_path)],
                             capture_output=True, text=True, timeout=600, env=env)
        assert out.returncode == 0, out.stdout + out.stderr
        assert _alive(out.stdout, "") == list(ref["alive"])
        assert "initial padding batch 512" in out.stdout
        batch = _per_layer(out.stdout, r"layer (\d+), batch = (\d+)")
        assert [int(batch[l]) for l in range(6)] == [_pad(a) for a in ref["alive"]]
        times = _per_layer(out.stdout, r"Layer (\d+) exec Time = ([0-9.e+-]+)\n")
        assert sorted(times) == list(range(6)) and float(times[0]) > 0
        assert "Kernel Exec Time = " in out.stdout
        assert f"[Categories] :{len(ref['categories'])}" in out.stdout
        assert "categories check: PASS" in out.stdout
        assert cat.read(ours).tolist() == list(ref["categories"])
    assert "Read cache success" in out.stdout
    # a truth file that differs: FAIL and exit status 2
    cat.write(truth, list(ref["categories"])[1:])
    out = subprocess.run([_exe("cospdnn"), "1024", "500", "6", "1", "0", str(tmp_path)],
                         capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 2 and "categories check: FAIL" in out.stdout and "extra 1" in out.stdout


@pytest.mark.gpu
def test_cli_layer_lines_past_layer_21(tmp_path):
    """The reference prints "feature" lines for the layers it compacts
    (l <= 21) and "batch" / "exec Time" lines for every layer
    (src/cospdnn.cu:262-264,302-305); the JSON line carries the proven bound
    on |final value - FP64 value|."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import json
    ref = _dataset(tmp_path, 1024, 24, 300, 59, 0)
    assert ref["alive"][-1] > 0
    env = dict(os.environ, COSPDNN_JSON="1")
    out = subprocess.run([_exe("cospdnn"), "1024", "300", "24", "1", "0", str(tmp_path)],
                         capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert _alive(out.stdout, "") == list(ref["alive"][:22])
    assert "layer 22, feature" not in out.stdout
    batch = _per_layer(out.stdout, r"layer (\d+), batch = (\d+)")
    assert [int(batch[l]) for l in range(24)] == [_pad(a) for a in ref["alive"]]
    times = _per_layer(out.stdout, r"Layer (\d+) exec Time = ([0-9.e+-]+)\n")
    assert sorted(times) == list(range(24)) and all(float(times[l]) > 0 for l in range(24))
    line = json.loads([x for x in out.stdout.splitlines() if x.startswith("{")][0])
    assert line["alive"] == list(ref["alive"]) and line["max_abs_dy_bound"] >= 0
    # without the timing pass the exec Time lines read 0
    env["COSPDNN_LAYER_TIMES"] = "0"
    out = subprocess.run([_exe("cospdnn"), "1024", "300", "24", "1", "0", str(tmp_path)],
                         capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0 and "Layer 23 exec Time = 0\n" in out.stdout


@pytest.mark.gpu
def test_cli_double_matches_oracle(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ref1 = _dataset(tmp_path, 1024, 5, 400, 47, 0)
    ref2 = _dataset(tmp_path, 2048, 7, 300, 53, 1)
    from cospdnn_b200 import categories as cat
    env = dict(os.environ)
    for i, r in ((1, ref1), (2, ref2)):
        cat.write(tmp_path / f"truth{i}.tsv", r["categories"])
        env[f"COSPDNN_TRUTH_{i}"] = str(tmp_path / f"truth{i}.tsv")
        env[f"COSPDNN_CATEGORIES_{i}"] = str(tmp_path / f"ours{i}.tsv")
    out = subprocess.run([_exe("cospdnn_double"), "1024", "400", "5", "2048", "300", "7", "0", str(tmp_path)],
                         capture_output=True, text=True, timeout=600, env=env)
    assert out.returncode == 0, out.stdout + out.stderr
    assert _alive(out.stdout, "SpDNN 1 ") == list(ref1["alive"])
    assert _alive(out.stdout, "SpDNN 2 ") == list(ref2["alive"])
    assert "initial padding batch 512 and 384" in out.stdout
    batch = {int(m.group(1)): (int(m.group(2)), int(m.group(3)))
             for m in re.finditer(r"layer (\d+), batch1 = (\d+), batch2 = (\d+)", out.stdout)}
    a1 = list(ref1["alive"]) + [0, 0]
    assert [batch[l] for l in range(7)] == [(_pad(a1[l]), _pad(ref2["alive"][l])) for l in range(7)]
    assert len(re.findall(r"Layer \d+ exec Time = [0-9.e+-]+ms", out.stdout)) == 7
    assert "Total Kernel Exec Time = " in out.stdout
    assert "SpDNN 1 categories check: PASS" in out.stdout and "SpDNN 2 categories check: PASS" in out.stdout
    assert cat.read(tmp_path / "ours2.tsv").tolist() == list(ref2["categories"])

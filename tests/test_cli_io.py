"""Host-side parts of the command lines, on CPU: the number reader of the
dataset files (the same numbers as the reference's stream extraction), the
binary dataset cache (COSPDNN_CACHE) and the categories files
(COSPDNN_CATEGORIES, COSPDNN_TRUTH),
through a small program built with g++ against cospdnn_b200/cli/reference_io.h,
and the Python categories module (cospdnn_b200.categories)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from netgen import make_net

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HARNESS = r"""
#include <cinttypes>
#include "reference_io.h"
using namespace cospdnn_cli;

static uint64_t mix(uint64_t h, const void *p, size_t n) {
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
    return h;
}
static uint64_t digest(const Network &n) {
    uint64_t h = 1469598103934665603ull;
    h = mix(h, n.input.rows.data(), n.input.rows.size() * sizeof(float));
    for (const auto &c : n.w) {
        h = mix(h, c.colptr.data(), c.colptr.size() * 4);
        h = mix(h, c.rowidx.data(), c.rowidx.size() * 4);
        h = mix(h, c.vals.data(), c.vals.size() * 4);
    }
    return h;
}
// (u, v, val) triples until the first that does not parse, as the stream
// extraction reads them and as NumReader reads them with `block`-byte reads
static void triples(const char *path, size_t block) {
    uint64_t hs = 1469598103934665603ull, hr = hs;
    long ns = 0, nr = 0, u, v;
    float val;
    std::ifstream f(path);
    while (f >> u >> v >> val) {
        hs = mix(mix(mix(hs, &u, sizeof u), &v, sizeof v), &val, sizeof val);
        ++ns;
    }
    NumReader r(path, block);
    while (r.next(u) && r.next(v) && r.next(val)) {
        hr = mix(mix(mix(hr, &u, sizeof u), &v, sizeof v), &val, sizeof val);
        ++nr;
    }
    printf("stream %" PRIu64 " %ld\nreader %" PRIu64 " %ld\n", hs, ns, hr, nr);
}
int main(int argc, char **argv) {
    const std::string mode = argv[1];
    if (mode == "nums") {
        triples(argv[2], (size_t)atol(argv[3]));
        return 0;
    }
    if (mode == "json") {  // json MS ROW... : a result line for a fixed 3-layer network
        RunReport r;
        r.program = "cospdnn";
        r.neuron = 1024;
        r.batch = 60000;
        r.layers = 3;
        r.precision = COSPDNN_PREC_BF16;
        r.kernel = COSPDNN_KERNEL_TCGEN05;
        r.gpus = 2;
        r.weights = 3 * 32768;
        r.ms = (float)atof(argv[2]);
        r.alive = {500, 40, 7};
        r.rechecked = {3, 0, 1};
        for (int i = 3; i < argc; ++i) r.categories.push_back(atoll(argv[i]));
        report_json(r);
        return 0;
    }
    if (mode == "load" || mode == "parse") {
        const int n = atoi(argv[2]), b = atoi(argv[3]), l = atoi(argv[4]);
        const Network net = mode == "load" ? load_network(n, b, l, argv[5]) : parse_network(n, b, l, argv[5]);
        printf("digest %" PRIu64 " integral %d read %ld layers %zu\n", digest(net), (int)net.input.integral,
               net.input.read, net.w.size());
        return 0;
    }
    std::vector<int64_t> rows;
    for (int i = 2; i < argc; ++i) rows.push_back(atoll(argv[i]));
    return report_categories(rows, "COSPDNN_CATEGORIES", "COSPDNN_TRUTH", "");
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    d = tmp_path_factory.mktemp("harness")
    src = d / "h.cpp"
    src.write_text(HARNESS)
    exe = d / "h"
    subprocess.run([gxx, "-O1", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
                    os.path.join(ROOT, "cospdnn_b200", "cli"), str(src), "-o", str(exe), "-pthread"], check=True)
    return str(exe)


def _run(exe, args, env=None):
    out = subprocess.run([exe] + [str(a) for a in args], capture_output=True, text=True, timeout=120,
                         env=dict(os.environ, **(env or {})))
    return out.returncode, out.stdout


def _digest(text):
    line = [x for x in text.splitlines() if x.startswith("digest ")][0]
    return line.split()[1]


def test_binary_cache(harness, tmp_path):
    from cospdnn_b200 import synth
    n, L, rows = 256, 4, 60
    data = tmp_path / "data"
    csc, y0, _ = make_net(n, L, rows, seed=71, dlo=0.2, dhi=0.4)
    rng = np.random.default_rng(71)
    fuse = [rng.permutation(n).astype(np.int32) for _ in range(L)]
    synth.write_reference_dataset(str(data), n, L, y0, csc, fuse=fuse)
    cache = tmp_path / "cache"
    cache.mkdir()
    env = {"COSPDNN_CACHE": str(cache)}
    rc, parsed = _run(harness, ["parse", n, rows, L, data])
    assert rc == 0 and "layers 4" in parsed and "integral 1" in parsed
    # first load parses and writes the cache, the second reads it
    rc, first = _run(harness, ["load", n, rows, L, data], env)
    assert rc == 0 and "Read cache success" not in first
    cfile = cache / f"cospdnn-n{n}-b{rows}-l{L}.bin"
    assert cfile.exists()
    rc, second = _run(harness, ["load", n, rows, L, data], env)
    assert rc == 0 and "Read cache success" in second
    assert _digest(first) == _digest(second) == _digest(parsed)
    # a changed source file invalidates the cache
    lay = data / f"neuron{n}" / f"{n}-l2.tsv"
    text = lay.read_text().splitlines()
    a, b, v = text[0].split("\t")
    text[0] = f"{a}\t{b}\t0.5"
    lay.write_text("\n".join(text) + "\n")
    rc, changed = _run(harness, ["load", n, rows, L, data], env)
    assert rc == 0 and "Read cache success" not in changed
    _, reparsed = _run(harness, ["parse", n, rows, L, data])
    assert _digest(changed) == _digest(reparsed) != _digest(parsed)
    rc, again = _run(harness, ["load", n, rows, L, data], env)
    assert "Read cache success" in again and _digest(again) == _digest(reparsed)
    # a damaged cache falls back to the files
    cfile.write_bytes(cfile.read_bytes()[:100])
    rc, damaged = _run(harness, ["load", n, rows, L, data], env)
    assert rc == 0 and "Read cache success" not in damaged and _digest(damaged) == _digest(reparsed)
    # another batch is another cache entry
    rc, fewer = _run(harness, ["load", n, rows - 10, L, data], env)
    assert rc == 0 and (cache / f"cospdnn-n{n}-b{rows - 10}-l{L}.bin").exists()


def test_reordered_dataset_same_product(harness, tmp_path):
    """cospdnn_b200.reorder rewrites the weights and the fuse matrix; the
    command lines fold the fuse back into W, so both datasets give the same
    network."""
    from cospdnn_b200 import reorder, synth
    from netgen import permute_rows, shift_half_block_layer
    n, L, rows = 1024, 3, 40
    layers = [permute_rows(shift_half_block_layer(n, 17, l), n, 170 + l) for l in range(L)]
    y0 = (np.random.default_rng(17).random((rows, n)) < 0.2).astype(np.uint8)
    synth.write_reference_dataset(str(tmp_path / "src"), n, L, y0, layers)
    stats = reorder.reorder_dataset(str(tmp_path / "src"), str(tmp_path / "dst"), n, L)
    assert all(b < a for a, b in stats)
    _, src = _run(harness, ["parse", n, rows, L, tmp_path / "src"])
    _, dst = _run(harness, ["parse", n, rows, L, tmp_path / "dst"])
    assert _digest(src) == _digest(dst)


def test_categories_cli_helpers(harness, tmp_path):
    out, truth = tmp_path / "ours.tsv", tmp_path / "truth.tsv"
    truth.write_text("3\n1\n10\n")
    env = {"COSPDNN_CATEGORIES": str(out), "COSPDNN_TRUTH": str(truth)}
    rc, text = _run(harness, ["cats", 0, 2, 9], env)
    assert rc == 0 and "categories check: PASS (ours 3, truth 3, missing 0, extra 0)" in text
    assert out.read_text() == "1\n3\n10\n"
    rc, text = _run(harness, ["cats", 0, 2, 8], env)
    assert rc == 2 and "FAIL (ours 3, truth 3, missing 1, extra 1)" in text
    rc, text = _run(harness, ["cats"], env)  # no survivors
    assert rc == 2 and "missing 3, extra 0" in text and out.read_text() == ""
    truth.write_text("1\nx\n")
    rc, text = _run(harness, ["cats", 0], env)
    assert rc != 0 and "cannot read truth file" in text
    rc, text = _run(harness, ["cats", 0], dict(env, COSPDNN_TRUTH=str(tmp_path)))  # a directory
    assert rc != 0 and "cannot read truth file" in text


def test_categories_module(tmp_path):
    from cospdnn_b200 import categories as cat
    p = tmp_path / "c.tsv"
    cat.write(p, [9, 0, 2, 2])
    assert p.read_text() == "1\n3\n10\n"
    assert cat.read(p).tolist() == [0, 2, 9]
    r = cat.check([0, 2, 9], p)
    assert r["ok"] and r["ours"] == 3 and r["truth"] == 3
    r = cat.check([0, 2, 8], p)
    assert not r["ok"] and r["missing"].tolist() == [9] and r["extra"].tolist() == [8]
    q = tmp_path / "d.tsv"
    cat.write(q, [0, 2, 9])
    assert cat.main([str(q), str(p)]) == 0
    cat.write(q, [0, 2])
    assert cat.main([str(q), str(p)]) == 2
    bad = tmp_path / "bad.tsv"
    bad.write_text("0\n")
    with pytest.raises(ValueError):
        cat.read(bad)
    assert cat.main([str(bad), str(p)]) == 1                  # malformed: an error, not a mismatch
    assert cat.main([str(tmp_path / "none.tsv"), str(p)]) == 1
    assert cat.main(["--hash", str(tmp_path / "none.tsv")]) == 1


def _fmt_triples(rng, n):
    """Lines of "u v val" with mixed white space and number forms."""
    ws = [" ", "\t", "  ", " \t ", "\t\t"]
    ends = ["\n", "\r\n", " \n", "\n\n", "\t\n"]
    out = []
    for _ in range(n):
        u, v = int(rng.integers(1, 5000)), int(rng.integers(1, 5000))
        val = float(rng.choice([0.0625, -0.25, 1.0, 3.0, 1e-5, 2.5e7]) * rng.choice([1, -1]))
        form = int(rng.integers(0, 6))
        txt = [f"{val}", f"{val:.9g}", f"{val:e}", f"{val:E}", f"{val:.3f}", f"+{abs(val)}"][form]
        if form == 4 and abs(val) < 1 and txt.startswith("0"):
            txt = txt[1:]  # ".062"
        us = f"+{u}" if rng.random() < 0.05 else str(u)
        out.append(us + rng.choice(ws) + str(v) + rng.choice(ws) + txt + rng.choice(ends))
    return out


@pytest.mark.parametrize("bad", [None, "abc", "1e", "1e+", "0x5", "-0x1p3", "inf", "nan", "5e3e2", "--3", "+.",
                                 ".", "7.5.3", "1.5e"])
def test_number_reader_matches_stream_extraction(harness, tmp_path, bad):
    """NumReader stops where `while (f >> u >> v >> val)` stops and reads the
    same numbers, across many 8 KB reads (tokens split between reads) and
    with a malformed token in the value or index position."""
    rng = np.random.default_rng(0 if bad is None else len(bad) * 7 + ord(bad[0]))
    lines = _fmt_triples(rng, 20000)
    if bad is not None:
        at = int(rng.integers(100, 19000))
        parts = lines[at].split()
        parts[int(rng.integers(0, 3))] = bad
        lines[at] = " ".join(parts) + "\n"
    path = tmp_path / "t.tsv"
    path.write_text("".join(lines).rstrip("\n"))  # no newline at the end
    for block in (8192, 1 << 24):
        rc, out = _run(harness, ["nums", path, block])
        got = dict(line.split(" ", 1) for line in out.strip().splitlines())
        assert rc == 0 and got["stream"] == got["reader"], (bad, block, got)
        if bad is None:
            assert got["reader"].split()[1] == "20000"
    for text in ("", "  \n\t\n", "1 2 0.5"):
        path.write_text(text)
        rc, out = _run(harness, ["nums", path, 8192])
        got = dict(line.split(" ", 1) for line in out.strip().splitlines())
        assert got["stream"] == got["reader"], text


def test_json_result_line(harness, tmp_path):
    """COSPDNN_JSON: one JSON line with sizes, device time, edges and
    edges/s, rows alive and rechecked per layer and the categories' count and
    hash (the FNV-1a hash of their categories file, as
    cospdnn_b200.categories computes it); printed for 1, appended to a named
    file, absent when unset."""
    import json
    from cospdnn_b200 import categories as cat
    rows = [9, 0, 2, 4096]
    rc, out = _run(harness, ["json", "1.5"] + rows, {"COSPDNN_JSON": "1"})
    assert rc == 0
    j = json.loads(out.strip())
    assert j["program"] == "cospdnn" and "network" not in j
    assert (j["neuron"], j["batch"], j["layers"], j["gpus"]) == (1024, 60000, 3, 2)
    assert j["precision"] == "bf16" and j["kernel"] == "tcgen05" and j["weights"] == 98304
    assert j["ms"] == 1.5 and j["edges"] == 60000 * 98304
    assert abs(j["edges_per_s"] - 60000 * 98304 / 1.5e-3) / j["edges_per_s"] < 1e-5
    assert j["alive"] == [500, 40, 7] and j["fp64_rechecked"] == [3, 0, 1]
    assert j["categories"] == 4 and j["category_hash"] == "fnv1a64:" + cat.digest(rows)
    f = tmp_path / "cats.tsv"
    cat.write(f, rows)
    assert cat.main(["--hash", str(f)]) == 0
    log = tmp_path / "r.jsonl"
    for _ in range(2):
        rc, out = _run(harness, ["json", "2"] + rows, {"COSPDNN_JSON": str(log)})
        assert rc == 0 and out == ""
    lines = log.read_text().splitlines()
    assert len(lines) == 2 and all(json.loads(x)["ms"] == 2 for x in lines)
    rc, out = _run(harness, ["json", "2"], {"COSPDNN_JSON": ""})
    assert rc == 0 and out == ""
    assert cat.digest([]) == "cbf29ce484222325"  # FNV-1a offset basis: no rows


def test_dataset_writer_keeps_float32_weights(harness, tmp_path):
    """Weights written by synth.write_reference_dataset read back bit for bit
    through the command lines' reader (random float32 values need 9 digits)."""
    from cospdnn_b200 import synth
    from netgen import random_layer
    n, L, rows = 128, 2, 8
    layers = []
    rng = np.random.default_rng(4)
    for l in range(L):
        cp, ri, vv = random_layer(n, 40, l)
        layers.append((cp, ri, rng.standard_normal(len(vv)).astype(np.float32)))
    y0 = (rng.random((rows, n)) < 0.3).astype(np.uint8)
    synth.write_reference_dataset(str(tmp_path), n, L, y0, layers)
    for l, (cp, ri, vv) in enumerate(layers):
        t = np.loadtxt(tmp_path / f"neuron{n}" / f"{n}-l{l + 1}.tsv", ndmin=2, dtype=str)
        back = np.array([np.float32(x) for x in t[:, 2]])
        np.testing.assert_array_equal(back.view(np.uint32), vv.view(np.uint32))
    rc, out = _run(harness, ["parse", n, rows, L, tmp_path])
    assert rc == 0 and f"layers {L}" in out and "integral 1" in out
    assert (tmp_path / f"sparse-images-{n}.tsv").read_text().split("\n")[0].endswith("\t1")
    # non-binary rows keep their values
    y1 = np.where(y0 > 0, rng.random((rows, n)).astype(np.float32) * 3, 0).astype(np.float32)
    synth.write_reference_dataset(str(tmp_path / "v"), n, L, y1, layers)
    t = np.loadtxt(tmp_path / "v" / f"sparse-images-{n}.tsv", ndmin=2, dtype=str)
    back = np.zeros((rows, n), np.float32)
    back[t[:, 0].astype(int) - 1, t[:, 1].astype(int) - 1] = [np.float32(x) for x in t[:, 2]]
    np.testing.assert_array_equal(back, y1)
    rc, out = _run(harness, ["parse", n, rows, L, tmp_path / "v"])
    assert rc == 0 and "integral 0" in out


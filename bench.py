#!/usr/bin/env python
"""edges/s of the whole L-layer sparse-DNN inference (Graph Challenge shapes).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2]
                    [--impl ours|reference]

One step = one complete inference of the configured network(s): Y0 resident
on the device -> all layers (pruned rows dropped, early exit when every row
is dead) -> categories on the device, as one CUDA-graph launch.
edges/s = rows x sum_l nnz(W_l) / step time.  Under torchrun every rank runs
its own batch of rows (weak scaling; no collective on the data path).
--impl reference times the CPU implementation of the same recurrence (the
multithreaded FP32 CSR port in oracle/) on this host's cores.
"""
import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edges/s (inputs×ΣnnzW / s) at 1 B200, FP16-TC vs plain FP32; categories exact"
UNIT = "edges/s"
SEED = 20240611
PREC = {"fp32": 0, "fp16": 1, "bf16": 2}
DTYPE = {"fp32": "f32", "fp16": "f16", "bf16": "bf16"}

# name -> (networks [(neuron, layers, rows)], precision, input density)
def config_nets(name):
    if name == "c1":
        return [(1024, 120, 60000)], "fp32", (0.08, 0.25)
    if name == "c2":
        return [(4096, 120, 60000)], "fp16", (0.08, 0.25)
    if name == "c3":
        return [(16384, 120, 60000)], "bf16", (0.08, 0.25)
    if name == "c4":
        return [(65536, 120, 60000)], "fp16", (0.08, 0.25)
    if name == "c5":
        from cospdnn_b200 import synth
        return synth.mix_config(SEED), "fp16", (0.08, 0.25)
    if name == "s1":
        return [(1024, 120, 60000)], "fp16", (0.25, 0.45)
    if name == "r1":
        return [(4096, 120, 60000)], "fp16", (0.08, 0.25)
    raise SystemExit(f"unknown config {name}")


def weight_kind(name):
    """r1: reference-compatible masks (two aligned dense 16x16 blocks per
    block column, the structure the reference's kernel expects); else XOR."""
    return "r1" if name == "r1" else "xor"


def workload_name(name, nets, prec, dens):
    if len(nets) == 1:
        n, l, b = nets[0]
        w = ("R1 W (two dense 16x16 blocks per block column, 32 nnz/col, 1/16)" if weight_kind(name) == "r1"
             else "XOR-mask W (32 nnz/col, 1/16)")
        return f"{n} neurons x {l} layers, {b} rows, {w}, binary Y0 density U[{dens[0]},{dens[1]}], {prec}"
    return (f"{len(nets)} networks {[(n, l, b) for n, l, b in nets]}, XOR-mask W, "
            f"binary Y0 density U[{dens[0]},{dens[1]}], {prec}")


def edges(nets):
    return float(sum(b * l * 32 * n for n, l, b in nets))


# DRAM bytes (read + write) per input row of one launch of the config's
# dominant layer kernel, from one ncu capture of a smaller case of the same
# kernel on the same weights (profiles/k_layer_*.md): traffic grows with the
# rows a launch processes.
DRAM_BYTES_PER_ROW = {
    "c2": (135.131136e6 + 88.350208e6) / 16384,  # k_layer_cc_4096n_16384rows_fp16.md
    "c1": (135.193088e6 + 88.413696e6) / 32768,  # k_layer_cc_1024n_32768rows_fp32.md
    "c3": (271.177216e6 + 224.850688e6) / 8192,  # k_layer_cc_16384n_8192rows_bf16.md
    "r1": (134.869248e6 + 83.793152e6) / 16384,  # k_layer_tc_4096n_16384rows_r1_fp16.md
    "c4": (280.101632e6 + 228.839424e6) / 2048,  # k_layer_cs_65536n_2048rows_fp16.md
}

def measured_peaks():
    """HBM copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json,
    burst figure: the layer kernels are timed alone), else the fallback."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback"


TNAME = {"fp32": "float", "fp16": "__half", "bf16": "__nv_bfloat16"}
# rows per network that the FP64 parity check replays (the whole batch where
# the oracle finishes in seconds, else the first rows of it)
PARITY_ROWS = {1024: 60000, 4096: 60000, 16384: 16384, 65536: 2048}
DY_ROWS = 2048  # rows per checked layer compared value by value


def is_split(info, prec):
    """Feature-split nets: CUDA cores with 2-row tiles of a 16-bit type (the
    one-CTA row-tile kernel takes 16-bit tiles of 4 rows or more)."""
    import cospdnn_b200 as cs
    return info["kernel"] == cs.KERNEL_CUDA_CORE and info["row_tile"] == 2 and prec != "fp32"


def layer_kernel_name(info, n, prec):
    """Name of the kernel that computes layers >= 1 of a net (engine's choice)."""
    import cospdnn_b200 as cs
    es = 4 if prec == "fp32" else 2
    if info["kernel"] == cs.KERNEL_TCGEN05:
        return f"k_layer_tc<{TNAME[prec]}>"
    tr = info["row_tile"]
    if tr == 0:
        return f"k_layer_plain<{TNAME[prec]}>"
    if is_split(info, prec):
        return f"k_layer_cs<{TNAME[prec]}>"
    nt = 256 if n * tr * es <= 96 * 1024 else 512
    lb = 16 if tr * es >= 16 else 8
    return f"k_layer_cc<{TNAME[prec]}, {nt}, {lb}>"


def layer0_kernel_name(info, prec):
    import cospdnn_b200 as cs
    if not info["layer0_counted"]:
        return None
    sixteen = info["kernel"] == cs.KERNEL_TCGEN05 or is_split(info, prec)
    return f"k_layer0_bits16<{TNAME[prec]}>" if sixteen else f"k_layer0_bits<{TNAME[prec]}>"


def weight_bytes(info, n, prec):
    """Bytes of W_l the layer kernel reads (32 entries per output)."""
    import cospdnn_b200 as cs
    if info["kernel"] == cs.KERNEL_TCGEN05:
        return 32.0 * (n // 16) * 512  # about one 16x16 operand per entry group of a block column
    if info["row_tile"] and prec != "fp32":
        return 32.0 * n * 4  # (input column << 16 | weight) per entry
    return 32.0 * n * 8      # int32 index + float weight per entry


def own_bound(names, prec, fma_per_launch, ms_per_launch, sms, sm_mhz):
    """The dominant CUDA-core layer kernel against its own bound: one 128-byte
    shared-load wavefront per clock per SM.  A wavefront carries 64 FMAs of
    16-bit rows (16- or 8-byte lanes of 8 or 4 rows; the feature-split
    kernel's 4-byte words of 2 rows) and 32 of FP32 rows.  Counts the
    algorithmic FMAs (one per non-zero weight and active row), not the
    zero-weight padding of the conflict-free schedule.  None for the other
    kernels (tcgen05, row-major gather) or without a time."""
    if not names or ms_per_launch <= 0 or sms <= 0 or sm_mhz <= 0:
        return None
    if not all(n.startswith(("k_layer_cc<", "k_layer_cs<")) for n in names):
        return None
    peak = 32.0 if prec == "fp32" else 64.0
    achieved = fma_per_launch / (ms_per_launch * 1e-3) / (sms * sm_mhz * 1e6)
    return {"bound": "shared-memory wavefronts (one 128-byte wavefront per clock per SM)",
            "achieved": achieved, "peak": peak, "unit": "FMA/clk/SM", "frac": achieved / peak,
            "fma_per_launch": fma_per_launch, "sms": sms, "sm_mhz": sm_mhz}


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        # raw samples: $COSPDNN_CLOCKS_DIR if set, else the temporary directory
        # (the JSON line carries their summary)
        out = os.environ.get("COSPDNN_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, f"cospdnn_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            time.sleep(0.2)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()

    def summary(self):
        if self.p is None or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def sample_rows(run, total, budget_s):
    """Largest row count (<= total) whose run takes about budget_s seconds,
    grown geometrically from a small probe."""
    rows = min(total, 512)
    while True:
        t0 = time.perf_counter()
        run(rows)
        dt = time.perf_counter() - t0
        if rows >= total or dt >= 0.5 * budget_s:
            return rows
        rows = int(min(total, rows * max(2.0, min(8.0, 0.8 * budget_s / max(dt, 1e-3)))))


def cpu_baseline(nets, dens, y0_host_fn, weights, budget_s=12.0, threads=None):
    """Multithreaded FP32 CSR recurrence (oracle/ port) on a bounded row sample."""
    from oracle import pyoracle as po
    threads = threads or os.cpu_count()
    total_edges, total_t, desc = 0.0, 0.0, []
    for i, (n, L, b) in enumerate(nets):
        csr = [po.coo_to_csr(*po.csc_to_coo(*c), n) for c in weights[i]]
        bias = np.float32({1024: -0.3, 4096: -0.35, 16384: -0.4, 65536: -0.45}[n])
        rows = sample_rows(lambda r: po.infer_fp32_csr(csr, y0_host_fn(i, r), bias, threads=threads),
                           b, budget_s / len(nets))
        y = y0_host_fn(i, rows)
        t0 = time.perf_counter()
        po.infer_fp32_csr(csr, y, bias, threads=threads)
        t = time.perf_counter() - t0
        total_edges += rows * L * 32.0 * n
        total_t += t
        desc.append(f"{rows} of {b} rows of net {i} ({n}x{L})")
    return {"value": total_edges / total_t, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "; ".join(desc) + f"; {total_t:.1f} s on {threads} threads, FP32 CSR, early exit"}


def parity_check(cs, nets, prec, kernel, dens, weights, local, stream, inputs):
    """The FP64 oracle as checker of the benched configuration: an engine of
    the same networks (weights, precision, kernel choice) on the first rows of
    each batch (all of them where the oracle finishes in seconds), whose
    per-layer survivor counts and categories are compared with the oracle's,
    and whose outputs at up to four layers with survivors (first, last and
    two between; up to DY_ROWS rows each) are compared value by value with
    the oracle's FP64 replay of the same rows (max |dY|, and whether every
    row's |dY| lies within the error bound the engine carries for it)."""
    from oracle import pyoracle as po
    threads = os.cpu_count()
    rows = [min(b, PARITY_ROWS.get(n, 2048)) for n, _, b in nets]
    eng = cs.Engine(local)
    ids = []
    for i, (n, L, b) in enumerate(nets):
        nid = eng.add_net(n, L, rows[i], cs.BIAS[n], cs.THRESHOLD, PREC[prec], kernel)
        for l, (cp, ri, vv) in enumerate(weights[i]):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
    for nid, y, r in zip(ids, inputs, rows):
        eng.set_input(nid, y[:r], stream=stream)
    eng.run(stream)
    alive_eq, cats_eq, dy, dy_rows, dy_layers, within = True, True, 0.0, 0, [], True
    for i, (nid, (n, L, b)) in enumerate(zip(ids, nets)):
        res = eng.result(nid, stream)
        y0 = inputs[i][:rows[i]].cpu().numpy()
        bias = np.float32(cs.BIAS[n])
        ref = po.infer_fp64(weights[i], y0, bias, threads=threads)
        alive_ref = po.survivors_per_layer(ref["death"], L)
        alive_eq &= bool(np.array_equal(res["alive"], alive_ref))
        cats_eq &= bool(np.array_equal(res["categories"], np.nonzero(ref["death"] == L)[0]))
        live = [l for l in range(L) if alive_ref[l] > 0]
        if live:
            pick = sorted({live[0], live[len(live) // 3], live[(2 * len(live)) // 3], live[-1]})
            for l in pick:
                vals, rid, bnd = eng.layer_values(nid, l, max_rows=DY_ROWS, stream=stream, bounds=True)
                if len(rid) == 0:
                    continue
                want = po.replay_fp64(weights[i], y0, bias, rid.astype(np.int64), l)
                d = np.abs(vals.astype(np.float64) - want).max(axis=1)
                dy = max(dy, float(d.max()))
                within &= bool(np.all(d <= bnd.astype(np.float64)))
                dy_rows += len(rid)
                dy_layers.append((i, l))
    eng.close()
    return {"rows_checked": [int(r) for r in rows], "alive_equal": alive_eq, "categories_equal": cats_eq,
            "max_abs_dy": dy, "dy_within_proven_bound": within,
            "dy_rows_checked": int(dy_rows), "dy_layers": [f"net {i} layer {l}" for i, l in dy_layers],
            "oracle": "FP64 recurrence, fixed summation order (oracle/oracle.c), "
                      f"{threads} threads; values compared after each listed layer for up to "
                      f"{DY_ROWS} of its kept rows"}


def reference_cuda_build(nets, kind, dens):
    """The reference's own host loop and kernels (test_graph_challenge_tc,
    compiled from its sources for sm_100a into oracle/_ref) on the same
    weights and inputs, one run; its printed "Kernel Exec Time" and the wall
    time of the call.  Single networks up to 4096 neurons (its host code
    takes minutes beyond that).  On XOR-mask weights its kernel reads two
    16x16 blocks per block column (src/kernels/kernel.cu:257), so its product
    is truncated: timing only."""
    import ctypes as C
    so = os.path.join(ROOT, "oracle", "_ref", "libref_cospdnn.so")
    if len(nets) != 1 or nets[0][0] > 4096:
        return {"unavailable": "measured for single networks of at most 4096 neurons"}
    if not os.path.exists(so):
        return {"unavailable": "oracle/_ref/libref_cospdnn.so not built (make -C oracle ref REF=...)"}
    from cospdnn_b200 import synth
    from oracle import pyoracle as po
    n, L, b = nets[0]
    csc = synth.network(n, L, SEED, net=0, kind=kind)
    vals, rws, ptrs = [], [], []
    for cp, ri, vv in csc:
        row, col, val = po.csc_to_coo(cp, ri, vv)
        bcp, bri, _, bvals = po.bcsc_greedy(row, col, val, 16)
        # its kernel reads the first two blocks of every column, 16 fuse rows each
        if not (np.all(np.diff(bcp) >= 2) and bri[bcp[:-1]].max() <= n - 16 and bri[bcp[:-1] + 1].max() <= n - 16):
            return {"unavailable": "weights outside what the reference kernel reads in bounds"}
        vals.append(np.ascontiguousarray(bvals, np.float32))
        rws.append(np.ascontiguousarray(bri, np.int32))
        ptrs.append(np.ascontiguousarray(bcp, np.int32))
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int)
    V = (fp * L)(*[v.ctypes.data_as(fp) for v in vals])
    RI = (ip * L)(*[r.ctypes.data_as(ip) for r in rws])
    P = (ip * L)(*[q.ctypes.data_as(ip) for q in ptrs])
    nv = np.array([len(v) for v in vals], np.int64)
    nr = np.array([len(r) for r in rws], np.int64)
    npp = np.array([len(q) for q in ptrs], np.int64)
    feats = np.full(64, -1, np.int32)
    kms, wms, last = C.c_double(), C.c_double(), C.c_int()
    tail = C.create_string_buffer(4096)
    ref = C.CDLL(so)
    ref.ref_run_network.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.c_void_p]
    y = np.ascontiguousarray(po.input_binary(SEED, 0, b, n, dens[0], dens[1]), np.uint8)
    bias = {1024: -0.3, 4096: -0.35, 16384: -0.4, 65536: -0.45}[n]
    rc = ref.ref_run_network(y.ctypes.data, b, n, L, C.addressof(V), nv.ctypes.data, C.addressof(RI),
                             nr.ctypes.data, C.addressof(P), npp.ctypes.data, float(bias), C.addressof(kms),
                             C.addressof(wms), C.addressof(last), feats.ctypes.data, 64, tail, 4096, None)
    if rc != 0:
        return {"unavailable": f"reference run failed: {tail.value.decode(errors='replace')[-200:]}"}
    e = float(b) * L * 32 * n
    return {"kernel_exec_ms": kms.value, "wall_ms": wms.value, "edges_per_s_kernel": e / (kms.value * 1e-3),
            "edges_per_s_wall": e / (wms.value * 1e-3),
            "printed_features": [int(x) for x in feats[:8] if x >= 0],
            "note": ("its Kernel Exec Time covers its SpMM kernels only (src/cospdnn.cu:303-310); wall "
                     "covers its whole host loop. " +
                     ("Timing only: XOR-mask weights have 19-32 blocks per block column and its kernel "
                      "reads two, so its product is truncated." if kind == "xor" else
                      "R1 weights: two aligned dense blocks per block column, computed in full."))}


def _ref_build_child(q, nets, kind, dens):
    try:
        q.put(reference_cuda_build(nets, kind, dens))
    except Exception as ex:
        q.put({"unavailable": f"{type(ex).__name__}: {ex}"})


def reference_cuda_build_isolated(nets, kind, dens, timeout_s=600.0):
    """reference_cuda_build in a child process (spawned): the reference's host
    code ends its process on any CUDA error (Safe_Call -> exit,
    src/gpu_lib/gpu_runtime.h:6-17), which must not take this arm's line
    with it.  Bounded by timeout_s."""
    import multiprocessing as mp
    import queue
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    p = ctx.Process(target=_ref_build_child, args=(q, nets, kind, dens), daemon=True)
    p.start()
    t_end = time.time() + timeout_s
    res = None
    while res is None and time.time() < t_end:
        try:
            res = q.get(timeout=1.0)
        except queue.Empty:
            if not p.is_alive():
                try:
                    res = q.get(timeout=1.0)
                except queue.Empty:
                    break
    p.join(10)
    if p.is_alive():
        p.kill()
        p.join()
    if res is None:
        return {"unavailable": f"the reference's host code ended without a result (exit status {p.exitcode}: "
                               f"it exits on a CUDA error, or ran over {timeout_s:.0f} s)"}
    return res


def run_reference(args, nets, prec, dens):
    """--impl reference: the CPU implementation of the recurrence, timed here."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from cospdnn_b200 import synth
    from oracle import pyoracle as po
    threads = os.cpu_count()

    def host_rows(i, rows):
        return po.input_binary(SEED, i, rows, nets[i][0], dens[0], dens[1])

    layers = [[po.coo_to_csr(*po.csc_to_coo(*c), n) for c in synth.network(n, L, SEED, net=i,
                                                                         kind=weight_kind(args.config))]
              for i, (n, L, b) in enumerate(nets)]
    # size one step to a bounded sample: ~budget seconds per step
    budget = max(2.0, 60.0 / max(1, args.steps + args.warmup))
    samples = []
    for i, (n, L, b) in enumerate(nets):
        bias = np.float32({1024: -0.3, 4096: -0.35, 16384: -0.4, 65536: -0.45}[n])
        rows = sample_rows(lambda r: po.infer_fp32_csr(layers[i], host_rows(i, r), bias,
                                                       threads=threads), b, budget / len(nets))
        samples.append((i, rows, host_rows(i, rows), bias))
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        for i, rows, y, bias in samples:
            po.infer_fp32_csr(layers[i], y, bias, threads=threads)
        if step >= args.warmup:
            times.append(time.perf_counter() - t0)
    step_edges = sum(rows * nets[i][1] * 32.0 * nets[i][0] for i, rows, _, _ in samples)
    t = sum(times) / len(times)
    value = step_edges / t
    sample = ", ".join(f"{rows} of {nets[i][2]} rows of net {i}" for i, rows, _, _ in samples)
    ref_build = None
    if not args.no_reference_build:
        # reported, not fatal: the arm's value is the CPU port
        ref_build = reference_cuda_build_isolated(nets, weight_kind(args.config), dens)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded; Graph Challenge shapes)",
        "config": {"workload": workload_name(args.config, nets, prec, dens), "config": args.config,
                   "seed": SEED},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample + f" per step; FP32 CSR recurrence, OpenMP over rows, "
                                            f"early exit; the reference has no CPU implementation "
                                            f"of this path"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda_build": ref_build,
    }
    print(json.dumps(line), flush=True)


def build_engine(cs, nets, prec, kernel, weights, local, rows=None):
    eng = cs.Engine(local)
    ids = []
    for i, (n, L, b) in enumerate(nets):
        nid = eng.add_net(n, L, b if rows is None else rows[i], cs.BIAS[n], cs.THRESHOLD, PREC[prec], kernel)
        for l, (cp, ri, vv) in enumerate(weights[i]):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
    return eng, ids


def time_device(torch, eng, stream, steps, warmup, flush, clocks=None):
    """Mean device time of one run over `steps` runs (CUDA events on the
    launching stream around each run), after `warmup` runs; between timed runs
    (outside the events) a write of `flush` evicts L2."""
    for _ in range(warmup):
        eng.run(stream)
    stream.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        for e0, e1 in evs:
            with torch.cuda.stream(stream):
                flush.zero_()
            e0.record(stream)
            eng.run(stream)
            e1.record(stream)
        stream.synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in evs) / steps


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="c2")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=[None, "fp32", "fp16", "bf16"])
    ap.add_argument("--kernel", type=int, default=0, help="0 auto, 1 CUDA cores, 2 tcgen05")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline and the FP64 parity check")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp32", action="store_true", help="skip the plain-FP32 arm of the same engine")
    ap.add_argument("--no-reference-build", action="store_true",
                    help="--impl reference: skip timing the reference's own CUDA build")
    ap.add_argument("--rows", type=int, default=None, help="override the rows per network (profiling)")
    ap.add_argument("--layers", type=int, default=None,
                    help="override the layers per network (profiling: the XOR-mask configurations have no "
                         "rows left after a few layers, and the device loop stops there)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    nets, prec, dens = config_nets(args.config)
    if args.rows:
        nets = [(n, l, args.rows) for n, l, _ in nets]
    if args.layers:
        nets = [(n, args.layers, b) for n, _, b in nets]
    if args.precision:
        prec = args.precision
    if args.impl == "reference":
        return run_reference(args, nets, prec, dens)

    import torch
    import torch.distributed as dist

    import cospdnn_b200 as cs
    from cospdnn_b200 import synth

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device(f"cuda:{local}"))
    stream = torch.cuda.Stream()
    # L2 is 126 MB: a 256 MB write between timed runs evicts it
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    # ---- setup (untimed): weights replicated, each rank its own rows
    kind = weight_kind(args.config)
    weights = [synth.network(n, L, SEED, net=i, kind=kind) for i, (n, L, b) in enumerate(nets)]
    eng, ids = build_engine(cs, nets, prec, args.kernel, weights, local)
    inputs = []
    with torch.cuda.stream(stream):
        for i, (n, L, b) in enumerate(nets):
            inputs.append(synth.input_rows(b, n, SEED, net=i, dlo=dens[0], dhi=dens[1],
                                           row0=rank * b, device=local, stream=stream))
        stream.synchronize()
    for nid, y in zip(ids, inputs):
        eng.set_input(nid, y, stream=stream)
    stream.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        from cospdnn_b200 import dist as cd
        return cd.max_over_ranks(x, device=f"cuda:{local}")

    # ---- device-resident timing: one graph launch per step, L2 evicted between steps
    barrier()
    clk = Clocks(local)
    ms = max_over_ranks(time_device(torch, eng, stream, args.steps, args.warmup, flush, clocks=clk))
    barrier()
    launches_per_run = eng.launch_count(stream)
    results = [eng.result(nid, stream) for nid in ids]
    infos = [eng.net_info(nid, stream) for nid in ids]
    step_edges = edges(nets)
    value = step_edges * world / (ms * 1e-3)

    # ---- roofline of the dominant kernel from the per-iteration layer-kernel
    # times of an eager pass of the same kernels (CUDA events on `stream`)
    lms = eng.profile_layers(stream=stream)
    nit = len(lms)
    es = 4 if prec == "fp32" else 2
    b_l0 = np.zeros(nit)
    b_ly = np.zeros(nit)
    rows_ly = np.zeros(nit)
    fma_ly = np.zeros(nit)
    for r, info, (n, L, b), w in zip(results, infos, nets, weights):
        rows_in = np.concatenate([[b], r["alive"][:-1]])
        for it in range(min(nit, L)):
            R = float(rows_in[it])
            if R <= 0:
                continue
            if it == 0 and info["layer0_counted"]:
                # bit planes read, outputs written, the layer-0 schedule
                b_l0[it] += R * n / 8 + R * n * es + 32.0 * n * 2 + 4.0 * n
            else:
                # active input rows read, their outputs written, W
                b_ly[it] += 2.0 * R * n * es + weight_bytes(info, n, prec)
                rows_ly[it] += R
                fma_ly[it] += R * float(w[it][0][-1])  # nnz(W_l) FMAs per active row
    # iteration 0 is the counting kernel when every net counted layer 0
    l0_iter = all(i["layer0_counted"] for i in infos)
    t_l0 = float(lms[0]) if (nit and l0_iter) else 0.0
    it_ly = [i for i in range(nit) if not (i == 0 and l0_iter) and b_ly[i] > 0]
    t_ly = float(sum(lms[i] for i in it_ly))
    peak, peak_kind = measured_peaks()
    names = sorted({layer_kernel_name(i, n, prec) for i, (n, _, _) in zip(infos, nets)})
    l0_names = sorted({x for x in (layer0_kernel_name(i, prec) for i in infos) if x})
    per_layer = []
    for i in range(min(nit, 8)):
        bb = b_l0[i] + b_ly[i]
        per_layer.append({"iter": i, "kernel": (" + ".join(l0_names) if (i == 0 and l0_iter) else " + ".join(names)),
                          "ms": float(lms[i]), "bytes": bb,
                          "GBps": float(bb / (lms[i] * 1e-3) / 1e9) if lms[i] > 0 else 0.0})
    dominant_is_l0 = l0_iter and t_l0 > t_ly
    if dominant_is_l0:
        kname, kb, kt, klaunch = " + ".join(l0_names), float(b_l0[0]), t_l0, 1
    else:
        kname, kb, kt, klaunch = " + ".join(names), float(sum(b_ly[i] for i in it_ly)), t_ly, max(1, len(it_ly))
    achieved = kb / (kt * 1e-3) / 1e9 if kt > 0 else 0.0
    traffic = None
    if (not dominant_is_l0 and args.config in DRAM_BYTES_PER_ROW and args.precision in (None, prec)
            and args.kernel == 0 and it_ly):
        traffic = DRAM_BYTES_PER_ROW[args.config] * float(sum(rows_ly[i] for i in it_ly)) / len(it_ly)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "kernel": kname, "launches": klaunch, "bytes_per_launch": kb / klaunch,
                "ms_per_launch": kt / klaunch,
                "bytes_rule": ("per launch: active input rows x N x elem read + their outputs written + W_l "
                               "(layer 0 counted from bits: R x N / 8 bytes of bit planes + outputs + schedule)"),
                "traffic_note": ("DRAM bytes per launch scaled from an ncu capture of a smaller case of the same "
                                 "kernel (per input row) to this workload's rows per launch; null where no "
                                 "capture of this kernel and config is committed"),
                "layer0": ({"kernel": " + ".join(l0_names), "ms": t_l0, "bytes": float(b_l0[0]),
                            "GBps": float(b_l0[0] / (t_l0 * 1e-3) / 1e9) if t_l0 > 0 else 0.0,
                            "frac": float(b_l0[0] / (t_l0 * 1e-3) / 1e9 / peak) if t_l0 > 0 else 0.0}
                           if l0_iter else None),
                "per_layer": per_layer}
    if not dominant_is_l0:
        # a secondary figure: it must not cost the line when a clock sample is odd
        try:
            csum = clk.summary() or {}
            roofline["own_bound"] = own_bound(
                names, prec, float(sum(fma_ly[i] for i in it_ly)) / max(1, len(it_ly)), kt / klaunch,
                torch.cuda.get_device_properties(local).multi_processor_count,
                float(csum.get("sm_mhz") or csum.get("sm_max_mhz") or 0.0))
        except (TypeError, ValueError, KeyError) as ex:
            roofline["own_bound"] = {"error": repr(ex)}

    # ---- end to end through the public API: pinned host Y0 -> H2D -> run -> D2H result
    e2e = None
    if not args.no_e2e:
        import ctypes as C
        # the rows are binary: hand them over as packed bits (1 bit per feature,
        # COSPDNN_INPUT_BITS), the compact form of a Graph Challenge input
        host_in = [torch.from_numpy(np.packbits(y.cpu().numpy(), axis=1, bitorder="little")).pin_memory()
                   for y in inputs]
        outbufs = [torch.empty(8 * (1 + L) + 4 * b, dtype=torch.uint8).pin_memory()
                   for (n, L, b) in nets]
        h2d = sum(int(x.numel()) for x in host_in)
        d2h = sum(int(x.numel()) for x in outbufs)
        lib = cs.lib()

        # Pipelined steps: step k's input (H2D of the packed bits and the
        # conversion) runs on a copy stream while step k-1 runs; the engine's
        # inputs are double buffered, so input k waits only for run k-2.
        copy = torch.cuda.Stream()
        ev_in = [torch.cuda.Event() for _ in range(2)]
        ev_done = [torch.cuda.Event() for _ in range(2)]

        def set_inputs(k):
            if k >= 2:
                copy.wait_event(ev_done[k % 2])
            for nid, x in zip(ids, host_in):
                cs._check(lib.cospdnn_engine_set_input(eng._h, nid, C.c_void_p(x.data_ptr()),
                                                       cs.INPUT_BITS, 0, cs._stream(copy)))
            ev_in[k % 2].record(copy)

        def e2e_steps(nsteps, start=None):
            if start is not None:
                copy.wait_event(start)
            set_inputs(0)
            for k in range(nsteps):
                stream.wait_event(ev_in[k % 2])
                eng.run(stream)
                for nid, o in zip(ids, outbufs):
                    cs._check(lib.cospdnn_engine_result_async(eng._h, nid, C.c_void_p(o.data_ptr()),
                                                              o.numel(), cs._stream(stream)))
                ev_done[k % 2].record(stream)
                if k + 1 < nsteps:
                    set_inputs(k + 1)
            stream.synchronize()

        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps(args.warmup)
        barrier()
        t0 = time.perf_counter()
        ev0.record(stream)
        e2e_steps(args.steps, start=ev0)
        ev1.record(stream)
        ev1.synchronize()
        wall = (time.perf_counter() - t0) / args.steps
        barrier()
        e2e_ms = max_over_ranks(max(ev0.elapsed_time(ev1) / args.steps, wall * 1e3))
        cnt = int(np.frombuffer(outbufs[0].numpy().tobytes(), np.int64, 1)[0])
        assert cnt == len(results[0]["categories"]), "e2e result differs from device-resident run"
        e2e = {"value": step_edges * world / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
               "input": "binary rows as packed bits (COSPDNN_INPUT_BITS) copied from pinned host memory "
                        "every step; result (count, alive per layer, categories) read back every step; the "
                        "next step's copy and conversion overlap the current run (double-buffered inputs)"}
    eng.close()
    del eng

    # ---- the plain FP32 path of the same engine on the same workload
    fp32 = None
    if not args.no_fp32 and prec != "fp32":
        e32, ids32 = build_engine(cs, nets, "fp32", 0, weights, local)
        for nid, y in zip(ids32, inputs):
            e32.set_input(nid, y, stream=stream)
        k32 = min(args.steps, 10)
        ms32 = max_over_ranks(time_device(torch, e32, stream, k32, 3, flush))
        r32 = [e32.result(nid, stream) for nid in ids32]
        info32 = [e32.net_info(nid, stream) for nid in ids32]
        same = all(np.array_equal(a["categories"], b["categories"]) and np.array_equal(a["alive"], b["alive"])
                   for a, b in zip(results, r32))
        fp32 = {"value": step_edges * world / (ms32 * 1e-3), "unit": UNIT, "ms_per_step": ms32, "steps": k32,
                "kernel": sorted({layer_kernel_name(i, n, "fp32") for i, (n, _, _) in zip(info32, nets)}),
                "same_categories_and_alive": bool(same)}
        e32.close()
        del e32

    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the CPU leg: the multithreaded FP32 CSR port timed as the baseline,
        # and the FP64 oracle as the checker of this configuration
        cpu = cpu_baseline(nets, dens, lambda i, rows: inputs[i][:rows].cpu().numpy(), weights)
        parity = parity_check(cs, nets, prec, args.kernel, dens, weights, local, stream, inputs)

    clocks = clk.summary()
    if rank == 0:
        r0 = results[0]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": DTYPE[prec], "data": "synthetic (seeded; Graph Challenge shapes)",
            "config": {
                "workload": workload_name(args.config, nets, prec, dens), "config": args.config,
                "seed": SEED, "accumulate": "f32", "parallelism": f"rows sharded, {world} rank(s)",
                "l2": "L2 flushed between timed steps (256 MB write outside the events)",
                "kernel": {0: "auto", 1: "cuda-core", 2: "tcgen05"}[args.kernel],
                "layer_kernels": names, "layer0_kernels": l0_names,
                "categories": [len(r["categories"]) for r in results],
                "alive_per_layer_net0": [int(x) for x in r0["alive"][:8]],
                "rechecked_fp64_net0": int(r0["rechecked"].sum()),
                "parity": parity,
            },
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "fp32": fp32, "vs_fp32": (value / fp32["value"]) if fp32 else None,
            "gpu_launches": int(launches_per_run * args.steps),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

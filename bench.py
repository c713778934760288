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


# DRAM bytes (read + write) per input row of one layer launch of the
# dominant kernel, from one ncu capture of a smaller case of the same
# workload (profiles/k_layer_*.md): traffic grows with the rows processed.
DRAM_BYTES_PER_ROW = {
    "c2": (135.131136e6 + 88.350208e6) / 16384,  # k_layer_cc_4096n_16384rows_fp16.md
    "c1": (135.193088e6 + 88.413696e6) / 32768,  # k_layer_cc_1024n_32768rows_fp32.md
    "c3": (271.177216e6 + 224.850688e6) / 8192,  # k_layer_cc_16384n_8192rows_bf16.md
    "r1": (134.869248e6 + 83.793152e6) / 16384,  # k_layer_tc_4096n_16384rows_r1_fp16.md
}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


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


def cpu_baseline(nets, dens, y0_host_fn, budget_s=12.0, threads=None, kind="xor"):
    """Multithreaded FP32 CSR recurrence (oracle/ port) on a bounded row sample."""
    from cospdnn_b200 import synth
    from oracle import pyoracle as po
    threads = threads or os.cpu_count()
    total_edges, total_t, desc = 0.0, 0.0, []
    for i, (n, L, b) in enumerate(nets):
        csr = [po.coo_to_csr(*po.csc_to_coo(*c), n) for c in synth.network(n, L, SEED, net=i, kind=kind)]
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
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="c2")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default=None, choices=[None, "fp32", "fp16", "bf16"])
    ap.add_argument("--kernel", type=int, default=0, help="0 auto, 1 CUDA cores, 2 tcgen05")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--rows", type=int, default=None, help="override the rows per network (profiling)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    nets, prec, dens = config_nets(args.config)
    if args.rows:
        nets = [(n, l, args.rows) for n, l, _ in nets]
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

    # ---- setup (untimed): weights replicated, each rank its own rows
    eng = cs.Engine(local)
    ids, inputs = [], []
    for i, (n, L, b) in enumerate(nets):
        nid = eng.add_net(n, L, b, cs.BIAS[n], cs.THRESHOLD, PREC[prec], args.kernel)
        for l, (cp, ri, vv) in enumerate(synth.network(n, L, SEED, net=i, kind=weight_kind(args.config))):
            eng.set_layer_csc(nid, l, cp, ri, vv)
        ids.append(nid)
    eng.build()
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

    # ---- device-resident timing
    for _ in range(args.warmup):
        eng.run(stream)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            eng.run(stream)
        ev1.record(stream)
        ev1.synchronize()
        barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps)
    launches_per_run = eng.launch_count(stream)
    results = [eng.result(nid, stream) for nid in ids]
    step_edges = edges(nets)
    value = step_edges * world / (ms * 1e-3)

    # ---- per-layer kernel times (eager pass of the same kernels) -> roofline
    iters_max = max(L for _, L, _ in nets) + 1
    import ctypes as C
    lms = np.zeros(iters_max, np.float32)
    nit = C.c_int()
    cs._check(cs.lib().cospdnn_engine_profile_layers(
        eng._h, cs._stream(stream), iters_max, lms.ctypes.data_as(C.POINTER(C.c_float)),
        C.byref(nit)))
    nit = nit.value
    es = 4 if prec == "fp32" else 2
    layer_bytes = np.zeros(nit)
    for r, (n, L, b) in zip(results, nets):
        rows_in = np.concatenate([[b], r["alive"][:-1]])
        for it in range(min(nit, L)):
            R = rows_in[it]
            if R > 0:
                # algorithmic bytes: active input rows read + their outputs written + W
                layer_bytes[it] += 2.0 * R * n * es + 32.0 * n * 8
    per_layer = [{"iter": i, "ms": float(lms[i]), "GBps": float(layer_bytes[i] / (lms[i] * 1e-3) / 1e9)
                  if lms[i] > 0 else 0.0} for i in range(nit)]
    peak, peak_kind = measured_peaks()
    tot_b, tot_t = float(layer_bytes.sum()), float(lms[:nit].sum()) * 1e-3
    achieved = tot_b / tot_t / 1e9 if tot_t > 0 else 0.0
    rows_per_launch = 0.0
    for r, (n, L, b) in zip(results, nets):
        rows_in = np.concatenate([[b], r["alive"][:-1]])
        rows_per_launch += float(rows_in[:min(nit, L)].sum()) / max(1, nit)
    traffic = None
    if args.config in DRAM_BYTES_PER_ROW and args.precision in (None, prec) and args.kernel == 0:
        traffic = DRAM_BYTES_PER_ROW[args.config] * rows_per_launch
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                "kernel": "layer kernels of the net (bit-count layer 0 for binary inputs; row-tile CUDA-core, "
                          "tcgen05 or row-major gather)",
                "traffic_note": "DRAM bytes per launch scaled from an ncu capture of a smaller case "
                                "(per input row) to this workload's average rows per layer launch",
                "bytes_per_launch": tot_b / max(1, nit),
                "ms_per_launch": float(lms[:nit].mean()) if nit else 0.0,
                "per_layer": per_layer[:8]}

    # ---- end to end through the public API: pinned host Y0 -> H2D -> run -> D2H result
    e2e = None
    if not args.no_e2e:
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
               "input": "binary rows as packed bits (COSPDNN_INPUT_BITS) from pinned host memory; "
                        "result (count, alive per layer, categories) read back every step; the next "
                        "step's copy and conversion overlap the current run (double-buffered inputs)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(nets, dens, lambda i, rows: inputs[i][:rows].cpu().numpy(), kind=weight_kind(args.config))

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
                "l2": "inputs larger than L2 (no flush)",
                "kernel": {0: "auto", 1: "cuda-core", 2: "tcgen05"}[args.kernel],
                "categories": [len(r["categories"]) for r in results],
                "alive_per_layer_net0": [int(x) for x in r0["alive"][:8]],
                "rechecked_fp64_net0": int(r0["rechecked"].sum()),
            },
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": int(launches_per_run * args.steps),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

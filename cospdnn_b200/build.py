"""Builds libcospdnn_b200.so in-tree with nvcc for sm_100a.

    python -m cospdnn_b200.build            # incremental
    python -m cospdnn_b200.build --force    # rebuild everything
"""
import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcospdnn_b200.so")
SOURCES = ["layer_ref.cu", "engine.cu", "tc_layer.cu", "cc_layer.cu", "cs_layer.cu", "bits_layer.cu", "synth.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
         "--expt-relaxed-constexpr", "-diag-suppress", "177"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "cospdnn_b200.h"))
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _stale(o, [s] + headers):
            cmd = [nvcc(), *ARCH, *FLAGS, "-c", s, "-o", o]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        subprocess.run([nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs], check=True)
    build_cli(force)
    return LIB


CLI = os.path.join(HERE, "cli")
CLI_PROGRAMS = ["cospdnn", "cospdnn_double", "cospdnn_multi"]


def build_cli(force=False):
    """The reference's command lines (cli/cospdnn.out, cli/cospdnn_double.out) and
    their k-network form (cli/cospdnn_multi.out):
    host C++ over the C ABI, linked against the in-tree library."""
    cxx = shutil.which("g++") or "g++"
    inc = os.path.join(os.path.dirname(HERE), "include")
    deps = [os.path.join(CLI, "reference_io.h"), os.path.join(inc, "cospdnn_b200.h"), LIB]
    for prog in CLI_PROGRAMS:
        src = os.path.join(CLI, prog + ".cpp")
        out = os.path.join(CLI, prog + ".out")
        if force or _stale(out, [src] + deps):
            subprocess.run([cxx, "-O2", "-std=c++17", "-Wall", "-I", inc, src, "-o", out, "-L", HERE,
                            "-lcospdnn_b200", "-Wl,-rpath,$ORIGIN/..", "-pthread"], check=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="pass -Xptxas -v")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
    sys.exit(0)

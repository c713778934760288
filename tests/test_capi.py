"""The C-ABI library loads and exports every function include/*.h declares,
each with its argument types declared in the ctypes layer (no compute calls:
this runs without a GPU)."""
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(cospdnn_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("cospdnn_layer", "cospdnn_prune_compact", "cospdnn_engine_run"):
        assert n in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    import cospdnn_b200
    L = cospdnn_b200.lib()
    assert hasattr(L, name), f"{name} declared in include/ but not exported"
    # the Python layer declares the argument types of every entry point, so
    # no size_t or pointer argument goes through as a C int
    assert getattr(L, name).argtypes is not None, name


def test_version_and_error_string():
    import cospdnn_b200
    L = cospdnn_b200.lib()
    assert L.cospdnn_version() >= 100
    assert isinstance(L.cospdnn_last_error(), bytes)


def test_invalid_arguments_fail_cleanly_without_gpu():
    import cospdnn_b200 as cs
    L = cs.lib()
    rc = L.cospdnn_layer(None, None, None, None, None, None, 0.0, 0, 0, 16, 16, 0, 0, None)
    assert rc == cs.ERR_INVALID
    assert b"null" in L.cospdnn_last_error()
    assert L.cospdnn_prune_workspace_bytes(1000) >= 4000


def test_run_networks_rejects_bad_arguments_without_gpu():
    import ctypes as C
    import cospdnn_b200 as cs
    L = cs.lib()
    assert L.cospdnn_run_networks(None, 1, 0, None) == cs.ERR_INVALID
    net = cs.NetworkC()  # all pointers NULL
    net.desc.neuron, net.desc.layers, net.desc.rows = 64, 1, 10
    assert L.cospdnn_run_networks(C.addressof(net), 1, 0, None) == cs.ERR_INVALID
    assert b"run_networks" in L.cospdnn_last_error()


def test_header_is_plain_c(tmp_path):
    """include/cospdnn_b200.h compiles as C99 (no C++ in the boundary) and a C
    program links against the library and calls it."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    libdir = os.path.join(ROOT, "cospdnn_b200")
    if gcc is None or not os.path.exists(os.path.join(libdir, "libcospdnn_b200.so")):
        pytest.skip("gcc or the built library missing")
    src = tmp_path / "c.c"
    src.write_text('#include "cospdnn_b200.h"\n'
                   'int main(void) { return cospdnn_version() >= 100 && cospdnn_last_error() ? 0 : 1; }\n')
    exe = tmp_path / "c"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", os.path.join(ROOT, "include"),
                    str(src), "-o", str(exe), "-L", libdir, "-lcospdnn_b200", f"-Wl,-rpath,{libdir}"], check=True,
                   timeout=120)
    assert subprocess.run([str(exe)], timeout=60).returncode == 0

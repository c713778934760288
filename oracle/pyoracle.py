"""ctypes wrapper around the CPU oracle (liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  It is the checker, never the product path.  See oracle.h for the
reference file:line each function restates.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
u8p = C.POINTER(C.c_uint8)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = C.CDLL(path)
        L.orc_stream_seed.restype = C.c_uint64
        L.orc_stream_seed.argtypes = [C.c_uint64] * 4
        L.orc_xor_masks.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, i32p]
        L.orc_r1_masks.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, i32p]
        L.orc_input_binary.argtypes = [C.c_uint64, C.c_int, C.c_int64, C.c_int64, C.c_int,
                                       C.c_double, C.c_double, u8p]
        L.orc_mix_config.argtypes = [C.c_uint64, C.c_int, i32p, C.c_int, i32p, C.c_int, C.c_int,
                                     C.c_int, i32p, i32p, i32p]
        L.orc_masks_to_csc.argtypes = [i32p, C.c_int, C.c_int, C.c_float, i32p, i32p, f32p]
        L.orc_bcsc_greedy.argtypes = [C.c_int64, i32p, i32p, f32p, C.c_int, C.c_int,
                                      C.POINTER(i32p), i32p, C.POINTER(i32p), i32p,
                                      C.POINTER(i32p), C.POINTER(f32p)]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_ref_layer.argtypes = [f32p, f32p, f32p, i32p, i32p, i32p, C.c_float, C.c_int, C.c_int]
        L.orc_bcsc_layer.argtypes = [f32p, f32p, f32p, i32p, i32p, i32p, C.c_int, C.c_float,
                                     C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_infer_fp64.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(i32p),
                                     C.POINTER(i32p), C.POINTER(f32p), u8p, f32p, C.c_float,
                                     C.c_double, C.c_int, i32p, f64p, f64p]
        L.orc_replay_fp64.argtypes = [C.c_int, C.c_int, C.c_int64, i64p, C.POINTER(i32p),
                                      C.POINTER(i32p), C.POINTER(f32p), u8p, f32p, C.c_float,
                                      f64p]
        L.orc_infer_fp32_csr.restype = C.c_int64
        L.orc_infer_fp32_csr.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(i32p),
                                         C.POINTER(i32p), C.POINTER(f32p), u8p, C.c_float,
                                         C.c_float, C.c_int, i32p]
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(t)


# ---------------------------------------------------------------- generators
def xor_masks(seed, net, layer, neuron, nmask=32):
    m = np.empty(nmask, np.int32)
    if lib().orc_xor_masks(seed, net, layer, neuron, nmask, _p(m, i32p)) != 0:
        raise ValueError("bad mask request")
    return m


def r1_masks(seed, net, layer, neuron):
    m = np.empty(32, np.int32)
    if lib().orc_r1_masks(seed, net, layer, neuron, _p(m, i32p)) != 0:
        raise ValueError("bad R1 mask request")
    return m


def input_binary(seed, net, rows, neuron, dlo=0.08, dhi=0.25, row0=0):
    y = np.empty((rows, neuron), np.uint8)
    lib().orc_input_binary(seed, net, row0, rows, neuron, dlo, dhi, _p(y, u8p))
    return y


def mix_config(seed, nnet=8, nchoices=(1024, 4096, 16384), lchoices=(120, 480), bmin=2000,
               bmax=60000):
    nc = np.array(nchoices, np.int32)
    lc = np.array(lchoices, np.int32)
    n = np.empty(nnet, np.int32)
    l = np.empty(nnet, np.int32)
    b = np.empty(nnet, np.int32)
    lib().orc_mix_config(seed, nnet, _p(nc, i32p), len(nc), _p(lc, i32p), len(lc), bmin, bmax,
                         _p(n, i32p), _p(l, i32p), _p(b, i32p))
    return [(int(n[i]), int(l[i]), int(b[i])) for i in range(nnet)]


def masks_to_csc(masks, neuron, val=0.0625):
    masks = np.ascontiguousarray(masks, np.int32)
    k = len(masks)
    cp = np.empty(neuron + 1, np.int32)
    ri = np.empty(neuron * k, np.int32)
    vv = np.empty(neuron * k, np.float32)
    lib().orc_masks_to_csc(_p(masks, i32p), k, neuron, val, _p(cp, i32p), _p(ri, i32p),
                           _p(vv, f32p))
    return cp, ri, vv


def csc_to_coo(cp, ri, vv):
    """(row = input, col = output) triplets of a CSC matrix."""
    n = len(cp) - 1
    col = np.repeat(np.arange(n, dtype=np.int32), np.diff(cp))
    return ri.astype(np.int32), col, vv.astype(np.float32)


def coo_to_csr(row, col, val, n):
    order = np.lexsort((col, row))
    r, c, v = row[order], col[order], val[order]
    rp = np.zeros(n + 1, np.int32)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp).astype(np.int32), c.astype(np.int32), v.astype(np.float32)


def coo_to_csc(row, col, val, n):
    order = np.lexsort((row, col))
    r, c, v = row[order], col[order], val[order]
    cp = np.zeros(n + 1, np.int32)
    np.add.at(cp, c + 1, 1)
    return np.cumsum(cp).astype(np.int32), r.astype(np.int32), v.astype(np.float32)


# ------------------------------------------------------------ BCSC builder
def bcsc_greedy(row, col, val, bs=16):
    """Reference greedy BCSC (src/utils/matrix.h:1200-1269).
    Returns (col_ptr, row_index, col_index, values[nblocks*bs*bs])."""
    row = np.ascontiguousarray(row, np.int32)
    col = np.ascontiguousarray(col, np.int32)
    val = np.ascontiguousarray(val, np.float32)
    cp, ri, ci = i32p(), i32p(), i32p()
    vv = f32p()
    ncp, nb = C.c_int32(), C.c_int32()
    L = lib()
    rc = L.orc_bcsc_greedy(len(row), _p(row, i32p), _p(col, i32p), _p(val, f32p), bs, bs,
                           C.byref(cp), C.byref(ncp), C.byref(ri), C.byref(nb), C.byref(ci),
                           C.byref(vv))
    if rc != 0:
        raise RuntimeError("bcsc build failed")
    try:
        out = (np.ctypeslib.as_array(cp, (ncp.value,)).copy(),
               np.ctypeslib.as_array(ri, (nb.value,)).copy(),
               np.ctypeslib.as_array(ci, (ncp.value - 1,)).copy(),
               np.ctypeslib.as_array(vv, (nb.value * bs * bs,)).copy())
    finally:
        for p in (cp, ri, ci, vv):
            L.orc_free(C.cast(p, C.c_void_p))
    return out


# ------------------------------------------------------------------ layers
def ref_layer(a_hilo, values, fuse, idx_ptr, index, bias, batch, neuron):
    """Reference kernel arithmetic (src/kernels/kernel.cu:240-379)."""
    a = np.ascontiguousarray(a_hilo, np.float32)
    v = np.ascontiguousarray(values, np.float32)
    fz = np.ascontiguousarray(fuse, np.int32)
    ip = np.ascontiguousarray(idx_ptr, np.int32)
    ix = np.ascontiguousarray(index, np.int32)
    nbc = neuron // 16
    if np.any(ix[ip[:nbc]] + 15 >= neuron) or np.any(ix[ip[:nbc] + 1] + 15 >= neuron):
        raise ValueError("reference kernel would read fuse[] past its end on this input")
    c = np.empty((neuron, batch), np.float32)
    lib().orc_ref_layer(_p(a, f32p), _p(v, f32p), _p(c, f32p), _p(fz, i32p), _p(ip, i32p),
                        _p(ix, i32p), bias, batch, neuron)
    return c


def bcsc_layer(a, values, fuse, idx_ptr, index, bias, batch, neuron, bs=16):
    """True BCSC product over every block of each block column."""
    a = np.ascontiguousarray(a, np.float32)
    v = np.ascontiguousarray(values, np.float32)
    ip = np.ascontiguousarray(idx_ptr, np.int32)
    ix = np.ascontiguousarray(index, np.int32)
    fz = None if fuse is None else np.ascontiguousarray(fuse, np.int32)
    c = np.empty((neuron, batch), np.float32)
    lib().orc_bcsc_layer(_p(a, f32p), _p(v, f32p), _p(c, f32p),
                         _p(fz, i32p) if fz is not None else None, _p(ip, i32p), _p(ix, i32p),
                         len(ip) - 1, bias, batch, neuron, bs, bs)
    return c


# -------------------------------------------------------------- recurrence
def _layer_ptrs(arrs, t):
    keep = [np.ascontiguousarray(a) for a in arrs]
    return keep, (t * len(keep))(*[a.ctypes.data_as(t) for a in keep])


def infer_fp64(csc_layers, y0, bias, tau=1e-5, threads=0, want_max=False, want_final=False):
    """FP64 recurrence; csc_layers = [(colptr, rowidx, vals)].  Returns
    dict(death=[rows], maxval=[rows, L] | None, final=[rows, N] | None)."""
    rows, neuron = y0.shape
    L = len(csc_layers)
    k1, cps = _layer_ptrs([c[0].astype(np.int32) for c in csc_layers], i32p)
    k2, ris = _layer_ptrs([c[1].astype(np.int32) for c in csc_layers], i32p)
    k3, vvs = _layer_ptrs([c[2].astype(np.float32) for c in csc_layers], f32p)
    y0 = np.ascontiguousarray(y0)
    u8 = _p(y0, u8p) if y0.dtype == np.uint8 else None
    f32 = None
    if y0.dtype != np.uint8:
        y0 = np.ascontiguousarray(y0, np.float32)
        f32 = _p(y0, f32p)
    death = np.empty(rows, np.int32)
    mx = np.empty((rows, L), np.float64) if want_max else None
    fin = np.empty((rows, neuron), np.float64) if want_final else None
    lib().orc_infer_fp64(neuron, L, rows, cps, ris, vvs, u8, f32, bias, tau, threads,
                         _p(death, i32p), _p(mx, f64p) if mx is not None else None,
                         _p(fin, f64p) if fin is not None else None)
    return dict(death=death, maxval=mx, final=fin)


def replay_fp64(csc_layers, y0, bias, row_ids, upto):
    rows, neuron = y0.shape
    k1, cps = _layer_ptrs([c[0].astype(np.int32) for c in csc_layers], i32p)
    k2, ris = _layer_ptrs([c[1].astype(np.int32) for c in csc_layers], i32p)
    k3, vvs = _layer_ptrs([c[2].astype(np.float32) for c in csc_layers], f32p)
    ids = np.ascontiguousarray(row_ids, np.int64)
    y0 = np.ascontiguousarray(y0)
    u8 = _p(y0, u8p) if y0.dtype == np.uint8 else None
    f32 = None
    if y0.dtype != np.uint8:
        y0 = np.ascontiguousarray(y0, np.float32)
        f32 = _p(y0, f32p)
    out = np.empty((len(ids), neuron), np.float64)
    lib().orc_replay_fp64(neuron, upto, len(ids), _p(ids, i64p), cps, ris, vvs, u8, f32, bias,
                          _p(out, f64p))
    return out


def infer_fp32_csr(csr_layers, y0_u8, bias, tau=1e-5, threads=0):
    """Multithreaded FP32 CSR CPU baseline.  Returns (alive_count, death)."""
    rows, neuron = y0_u8.shape
    L = len(csr_layers)
    k1, rps = _layer_ptrs([c[0].astype(np.int32) for c in csr_layers], i32p)
    k2, cis = _layer_ptrs([c[1].astype(np.int32) for c in csr_layers], i32p)
    k3, vvs = _layer_ptrs([c[2].astype(np.float32) for c in csr_layers], f32p)
    y0 = np.ascontiguousarray(y0_u8, np.uint8)
    death = np.empty(rows, np.int32)
    alive = lib().orc_infer_fp32_csr(neuron, L, rows, rps, cis, vvs, _p(y0, u8p), bias, tau,
                                     threads, _p(death, i32p))
    return int(alive), death


def survivors_per_layer(death, layers):
    """alive[l] = rows still alive after layer l (l = 0..L-1)."""
    d = np.asarray(death)
    return np.array([(d > l).sum() for l in range(layers)], np.int64)


# ------------------------------------------------------- reference formats
def write_weight_tsv(path, row, col, val):
    """src/cospdnn.cpp:72-79 + matrix.h:282-289: 'u v val', 1-based, u = input."""
    with open(path, "w") as f:
        for r, c, v in zip(row.tolist(), col.tolist(), val.tolist()):
            f.write(f"{r + 1}\t{c + 1}\t{v:.6g}\n")


def read_bcsc_dump(path, bs=16):
    raw = open(path, "rb").read()
    off = 0
    out = []
    for _ in range(3):
        n = int(np.frombuffer(raw, np.int32, 1, off)[0])
        off += 4
        out.append(np.frombuffer(raw, np.int32, n, off).copy())
        off += 4 * n
    vals = np.frombuffer(raw, np.float32, (len(raw) - off) // 4, off).copy()
    return out[0], out[1], out[2], vals

"""cospdnn_b200 -- B200 (sm_100a) sparse-DNN inference engine, Python host side.

Thin ctypes layer over the C ABI in include/cospdnn_b200.h (libcospdnn_b200.so,
built in-tree by `python -m cospdnn_b200.build`).  There is no CPU fallback:
every entry point raises if the CUDA library is missing or a call fails.

Mirrors of the reference's operator surface (paths relative to CoSpDNN):
  layer()                    <- ftxj::cospdnn_single       src/kernels/kernel.cuh:179-189
  prune_compact()            <- check_active_f_col + host compaction + matrix_reshape
                                src/kernels/kernel.cu:129-172, src/cospdnn.cu:236-276
  test_graph_challenge_tc()  <- host layer loop           src/cospdnn.cuh:14-21
  test_graph_challenge_tc_co() <- two-network loop        src/cospdnn.cuh:22-35
  Engine                     <- both loops, any number of networks in one graph
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcospdnn_b200.so")

# status codes (include/cospdnn_b200.h)
OK, ERR_INVALID, ERR_CUDA, ERR_NOMEM, ERR_STATE, ERR_DEVICE, ERR_UNSUPPORTED = range(7)
LAYER_A_FLOAT, LAYER_B_FLOAT, LAYER_REFERENCE_ARITH = 0x1, 0x2, 0x4
PRUNE_OUT_HALF_HILO = 0x1
PREC_FP32, PREC_FP16, PREC_BF16 = 0, 1, 2
KERNEL_AUTO, KERNEL_CUDA_CORE, KERNEL_TCGEN05 = 0, 1, 2
INPUT_U8, INPUT_F32, INPUT_BITS = 0, 1, 2
# bias table of the reference CLI (src/cospdnn.cpp:97-102)
BIAS = {65536: -0.45, 16384: -0.4, 4096: -0.35, 1024: -0.3}
THRESHOLD = 1e-5  # src/kernels/kernel.cu:133

_lib = None


class CospdnnError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cospdnn error {code}: {msg}")
        self.code = code


class NetDesc(C.Structure):
    _fields_ = [("neuron", C.c_int), ("layers", C.c_int), ("rows", C.c_int), ("bias", C.c_float),
                ("threshold", C.c_float), ("precision", C.c_int), ("kernel", C.c_int)]


def lib():
    """Loads the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: build it with `python -m cospdnn_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, ip, i32p, i64p, f32p = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int32), \
            C.POINTER(C.c_int64), C.POINTER(C.c_float)
        L.cospdnn_last_error.restype = C.c_char_p
        L.cospdnn_last_error.argtypes = []
        L.cospdnn_version.restype = C.c_int
        L.cospdnn_layer.argtypes = [vp, vp, vp, vp, vp, vp, C.c_float, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_uint, vp]
        L.cospdnn_prune_workspace_bytes.restype = C.c_size_t
        L.cospdnn_prune_workspace_bytes.argtypes = [C.c_int]
        L.cospdnn_prune_compact.argtypes = [vp, C.c_int, C.c_int, C.c_float, vp, vp, vp, vp, vp,
                                            C.c_uint, vp, C.c_size_t, vp]
        L.cospdnn_engine_create.argtypes = [C.POINTER(vp), C.c_int]
        L.cospdnn_engine_destroy.argtypes = [vp]
        L.cospdnn_engine_destroy.restype = None
        L.cospdnn_engine_add_net.argtypes = [vp, C.POINTER(NetDesc), ip]
        L.cospdnn_engine_set_layer_csc.argtypes = [vp, C.c_int, C.c_int, i32p, i32p, f32p]
        L.cospdnn_engine_set_layer_bcsc.argtypes = [vp, C.c_int, C.c_int, i32p, C.c_int, i32p,
                                                    C.c_int, f32p, C.c_int, i32p]
        L.cospdnn_engine_build.argtypes = [vp]
        L.cospdnn_engine_set_input.argtypes = [vp, C.c_int, vp, C.c_int, C.c_int, vp]
        L.cospdnn_engine_run.argtypes = [vp, vp]
        L.cospdnn_engine_result.argtypes = [vp, C.c_int, i32p, i64p, i64p, i64p, vp]
        L.cospdnn_engine_final_values.argtypes = [vp, C.c_int, f32p, C.c_int64, vp]
        L.cospdnn_engine_launch_count.argtypes = [vp, i64p, vp]
        # declared for every entry point: an undeclared size_t or pointer would
        # be passed as a C int
        L.cospdnn_version.argtypes = []
        L.cospdnn_device_count.argtypes = []
        L.cospdnn_device_count.restype = C.c_int
        L.cospdnn_prune_compact_noalloc.argtypes = [vp, C.c_int, C.c_int, C.c_float, vp, vp, vp, vp, vp,
                                                    C.c_uint, vp]
        L.cospdnn_engine_run_timed.argtypes = [vp, vp, f32p]
        L.cospdnn_engine_result_async.argtypes = [vp, C.c_int, vp, C.c_size_t, vp]
        L.cospdnn_engine_profile_layers.argtypes = [vp, vp, C.c_int, f32p, ip]
        L.cospdnn_engine_set_test_limits.argtypes = [vp, C.c_longlong, C.c_int, C.c_int]
        L.cospdnn_engine_final_bound.argtypes = [vp, C.c_int, f32p, vp]
        L.cospdnn_engine_net_info.argtypes = [vp, C.c_int, ip, ip, ip, vp]
        L.cospdnn_engine_layer_values.argtypes = [vp, C.c_int, C.c_int, f32p, i32p, f32p, C.c_int64, i64p, vp]
        L.cospdnn_run_networks.argtypes = [vp, C.c_int, C.c_int, f32p]
        L.cospdnn_synth_input.argtypes = [vp, C.c_int64, C.c_int, C.c_uint64, C.c_int, C.c_int64, C.c_double,
                                          C.c_double, C.c_int, vp]
        _lib = L
    return _lib


def _check(rc):
    if rc != OK:
        raise CospdnnError(rc, lib().cospdnn_last_error().decode())


def _ptr(t):
    """Device address of a torch tensor (or None)."""
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream(stream):
    if stream is None:
        return None
    return C.c_void_p(stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream))


def _np(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


# ------------------------------------------------------------ layer entries
def layer(A, B, C_out, fuse, idx_ptr, index, bias, batch, neuron, blocksize_c=16, blocksize_r=16,
          nblockcols=None, flags=0, stream=None):
    """cospdnn_single with the reference's argument meaning; torch CUDA tensors."""
    if nblockcols is None:
        nblockcols = idx_ptr.numel() - 1
    _check(lib().cospdnn_layer(_ptr(A), _ptr(B), _ptr(C_out), _ptr(fuse), _ptr(idx_ptr),
                               _ptr(index), float(bias), int(batch), int(neuron),
                               int(blocksize_c), int(blocksize_r), int(nblockcols), int(flags),
                               _stream(stream)))


def prune_workspace_bytes(batch):
    return int(lib().cospdnn_prune_workspace_bytes(int(batch)))


def prune_compact(C_in, neuron, batch, threshold, A_out, category, map_in, map_out, count,
                  workspace, flags=0, stream=None):
    _check(lib().cospdnn_prune_compact(_ptr(C_in), int(neuron), int(batch), float(threshold),
                                       _ptr(A_out), _ptr(category), _ptr(map_in), _ptr(map_out),
                                       _ptr(count), int(flags), _ptr(workspace),
                                       workspace.numel() * workspace.element_size(),
                                       _stream(stream)))


# ------------------------------------------------------------------ engine
class Engine:
    """Whole-network engine: add networks, set weights, build, then
    set_input / run / result as often as needed."""

    def __init__(self, device=0):
        self._h = C.c_void_p()
        _check(lib().cospdnn_engine_create(C.byref(self._h), int(device)))
        self.nets = []

    def close(self):
        if self._h:
            lib().cospdnn_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_net(self, neuron, layers, rows, bias=None, threshold=THRESHOLD, precision=PREC_FP16,
                kernel=KERNEL_AUTO):
        if bias is None:
            bias = BIAS[neuron]
        d = NetDesc(int(neuron), int(layers), int(rows), float(bias), float(threshold),
                    int(precision), int(kernel))
        nid = C.c_int()
        _check(lib().cospdnn_engine_add_net(self._h, C.byref(d), C.byref(nid)))
        self.nets.append(dict(neuron=neuron, layers=layers, rows=rows, bias=bias))
        return nid.value

    def set_layer_csc(self, net, layer, colptr, rowidx, vals):
        cp, ri, vv = _np(colptr, np.int32), _np(rowidx, np.int32), _np(vals, np.float32)
        _check(lib().cospdnn_engine_set_layer_csc(
            self._h, net, layer, cp.ctypes.data_as(C.POINTER(C.c_int32)),
            ri.ctypes.data_as(C.POINTER(C.c_int32)), vv.ctypes.data_as(C.POINTER(C.c_float))))

    def set_layer_bcsc(self, net, layer, col_ptr, row_index, values, blocksize=16, fuse=None):
        cp, ri, vv = _np(col_ptr, np.int32), _np(row_index, np.int32), _np(values, np.float32)
        fz = None if fuse is None else _np(fuse, np.int32)
        _check(lib().cospdnn_engine_set_layer_bcsc(
            self._h, net, layer, cp.ctypes.data_as(C.POINTER(C.c_int32)), len(cp),
            ri.ctypes.data_as(C.POINTER(C.c_int32)), len(ri),
            vv.ctypes.data_as(C.POINTER(C.c_float)), int(blocksize),
            None if fz is None else fz.ctypes.data_as(C.POINTER(C.c_int32))))

    def build(self):
        _check(lib().cospdnn_engine_build(self._h))

    def set_input(self, net, y0, fmt=None, stream=None):
        """y0: numpy array (host; pinned memory not required) or torch CUDA
        tensor; uint8 -> INPUT_U8, float32 -> INPUT_F32 unless fmt given."""
        on_device = hasattr(y0, "data_ptr") and getattr(y0, "is_cuda", False)
        if on_device:
            ptr = C.c_void_p(y0.data_ptr())
            dt = str(y0.dtype)
        else:
            if not hasattr(y0, "ctypes"):
                y0 = np.asarray(y0)
            if not y0.flags["C_CONTIGUOUS"]:
                y0 = np.ascontiguousarray(y0)
            self._keep = y0
            ptr = C.c_void_p(y0.ctypes.data)
            dt = str(y0.dtype)
        if fmt is None:
            fmt = INPUT_U8 if "uint8" in dt else INPUT_F32
        _check(lib().cospdnn_engine_set_input(self._h, net, ptr, int(fmt), int(on_device),
                                              _stream(stream)))

    def run(self, stream=None):
        _check(lib().cospdnn_engine_run(self._h, _stream(stream)))

    def result(self, net, stream=None):
        info = self.nets[net]
        cats = np.empty(max(1, info["rows"]), np.int32)
        alive = np.zeros(info["layers"], np.int64)
        rech = np.zeros(info["layers"], np.int64)
        cnt = C.c_int64()
        _check(lib().cospdnn_engine_result(
            self._h, net, cats.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(cnt),
            alive.ctypes.data_as(C.POINTER(C.c_int64)), rech.ctypes.data_as(C.POINTER(C.c_int64)),
            _stream(stream)))
        return dict(categories=cats[:cnt.value].copy(), alive=alive, rechecked=rech)

    def final_values(self, net, max_rows, stream=None):
        out = np.empty((max(1, max_rows), self.nets[net]["neuron"]), np.float32)
        _check(lib().cospdnn_engine_final_values(self._h, net,
                                                 out.ctypes.data_as(C.POINTER(C.c_float)),
                                                 int(max_rows), _stream(stream)))
        return out[:max_rows]

    def layer_values(self, net, layer, max_rows=None, stream=None, bounds=False):
        """Outputs of `layer` for the rows kept after it (ascending original
        row order) and their original ids: (values [k][neuron], ids [k]),
        plus each row's proven error bound [k] when bounds=True."""
        info = self.nets[net]
        if max_rows is None:
            max_rows = info["rows"]
        out = np.empty((max(1, max_rows), info["neuron"]), np.float32)
        ids = np.empty(max(1, max_rows), np.int32)
        bnd = np.empty(max(1, max_rows), np.float32)
        cnt = C.c_int64()
        _check(lib().cospdnn_engine_layer_values(self._h, net, int(layer),
                                                 out.ctypes.data_as(C.POINTER(C.c_float)),
                                                 ids.ctypes.data_as(C.POINTER(C.c_int32)),
                                                 bnd.ctypes.data_as(C.POINTER(C.c_float)),
                                                 int(max_rows), C.byref(cnt), _stream(stream)))
        k = cnt.value
        return (out[:k], ids[:k], bnd[:k]) if bounds else (out[:k], ids[:k])

    def profile_layers(self, max_iters=None, stream=None):
        """The layer loop run eagerly with each iteration's layer kernels
        timed by CUDA events: per-iteration milliseconds (numpy array)."""
        if max_iters is None:
            max_iters = max(n["layers"] for n in self.nets) + 1
        ms = np.zeros(max_iters, np.float32)
        it = C.c_int()
        _check(lib().cospdnn_engine_profile_layers(self._h, _stream(stream), int(max_iters),
                                                   ms.ctypes.data_as(C.POINTER(C.c_float)), C.byref(it)))
        return ms[:it.value]

    def set_test_limits(self, wait_cycles=0, max_iters=0, withhold_stage=0):
        """Test hooks of the device-side failure paths (see the C header):
        bounded-wait limit in cycles, layer-loop guard, withheld tcgen05
        stage; all 0 restores the defaults."""
        _check(lib().cospdnn_engine_set_test_limits(self._h, int(wait_cycles), int(max_iters),
                                                    int(withhold_stage)))

    def final_bound(self, net, stream=None):
        """Max over the surviving rows of the proven bound on |final value -
        FP64 recurrence value| after the last run."""
        v = C.c_float()
        _check(lib().cospdnn_engine_final_bound(self._h, net, C.byref(v), _stream(stream)))
        return v.value

    def net_info(self, net, stream=None):
        """dict(kernel=KERNEL_CUDA_CORE | KERNEL_TCGEN05, row_tile=rows per
        row tile (0: MMA tiles or row-major), layer0_counted=bool (last run))."""
        k, t, c = C.c_int(), C.c_int(), C.c_int()
        _check(lib().cospdnn_engine_net_info(self._h, net, C.byref(k), C.byref(t), C.byref(c),
                                             _stream(stream)))
        return dict(kernel=k.value, row_tile=t.value, layer0_counted=bool(c.value))

    def launch_count(self, stream=None):
        v = C.c_int64()
        _check(lib().cospdnn_engine_launch_count(self._h, C.byref(v), _stream(stream)))
        return v.value


# ------------------------------------------------- reference host API mirror
class NetworkC(C.Structure):
    """cospdnn_network (include/cospdnn_b200.h)."""
    _fields_ = [("desc", NetDesc), ("colptr", C.c_void_p), ("rowidx", C.c_void_p), ("vals", C.c_void_p),
                ("y0", C.c_void_p), ("format", C.c_int), ("categories", C.c_void_p), ("count", C.c_void_p),
                ("alive_per_layer", C.c_void_p)]


def run_networks(networks, device=0):
    """One call for any number of networks (cospdnn_run_networks).  Each item:
    dict(neuron, layers (list of CSC (colptr, rowidx, vals)), y0 (uint8 or
    float32 [rows][neuron]), bias, threshold=THRESHOLD, precision=PREC_FP16,
    kernel=KERNEL_AUTO).  Returns ([dict(categories, alive)], device ms)."""
    keep, structs, outs = [], [], []
    for w in networks:
        L = len(w["layers"])
        y0 = np.ascontiguousarray(w["y0"])
        fmt = INPUT_U8 if y0.dtype == np.uint8 else INPUT_F32
        if fmt == INPUT_F32:
            y0 = np.ascontiguousarray(y0, np.float32)
        cps = [np.ascontiguousarray(cp, np.int32) for cp, _, _ in w["layers"]]
        ris = [np.ascontiguousarray(ri, np.int32) for _, ri, _ in w["layers"]]
        vvs = [np.ascontiguousarray(vv, np.float32) for _, _, vv in w["layers"]]
        P32, PF = C.POINTER(C.c_int32), C.POINTER(C.c_float)
        acp = (P32 * L)(*[a.ctypes.data_as(P32) for a in cps])
        ari = (P32 * L)(*[a.ctypes.data_as(P32) for a in ris])
        avv = (PF * L)(*[a.ctypes.data_as(PF) for a in vvs])
        rows = y0.shape[0]
        cats = np.zeros(max(1, rows), np.int32)
        cnt = np.zeros(1, np.int64)
        alive = np.zeros(max(1, L), np.int64)
        d = NetDesc(int(w["neuron"]), L, rows, float(w["bias"]), float(w.get("threshold", THRESHOLD)),
                    int(w.get("precision", PREC_FP16)), int(w.get("kernel", KERNEL_AUTO)))
        structs.append(NetworkC(d, C.cast(acp, C.c_void_p), C.cast(ari, C.c_void_p), C.cast(avv, C.c_void_p),
                                y0.ctypes.data, fmt, cats.ctypes.data, cnt.ctypes.data, alive.ctypes.data))
        keep += [y0, cps, ris, vvs, acp, ari, avv]
        outs.append((cats, cnt, alive, L))
    arr = (NetworkC * len(structs))(*structs)
    ms = C.c_float()
    _check(lib().cospdnn_run_networks(C.addressof(arr), len(structs), int(device), C.byref(ms)))
    res = [{"categories": cats[:int(cnt[0])].copy(), "alive": alive[:L].copy()} for cats, cnt, alive, L in outs]
    return res, ms.value


def test_graph_challenge_tc(input, weight, row_idx, ptr, fuse_list, batch, neuron, bias,
                            blocksize_c=16, blocksize_r=16, gpu_id=0, gpu_num=1,
                            precision=PREC_FP16, threshold=THRESHOLD, verbose=True):
    """Mirror of the reference's test_graph_challenge_tc (src/cospdnn.cu:3-369).

    input      [batch][neuron] values (numpy; binary images in the Graph Challenge)
    weight     per layer: BCSC block values (bcsc_values_)
    row_idx    per layer: block start rows (bcsc_row_index_)
    ptr        per layer: block-column pointer (bcsc_len_)
    fuse_list  per layer: activation row of each weight row (or None)
    Runs every layer on GPU `gpu_id` (rows split over gpu_num slices as in
    src/cospdnn.cu:23,35-44, this call computing slice gpu_id).  Prints the
    reference's per-layer "layer l, feature = n" lines when verbose and
    returns dict(categories, alive).  Raises on error instead of exiting.
    """
    rows_per = (batch + gpu_num - 1) // gpu_num
    lo, hi = gpu_id * rows_per, min((gpu_id + 1) * rows_per, batch)
    x = np.asarray(input)[lo:hi]
    L = len(weight)
    eng = Engine(gpu_id if gpu_num > 1 else 0)
    try:
        net = eng.add_net(neuron, L, hi - lo, bias, threshold, precision)
        for l in range(L):
            if blocksize_c != blocksize_r:
                raise CospdnnError(ERR_UNSUPPORTED, "square blocks only")
            fz = None if fuse_list is None else fuse_list[l]
            eng.set_layer_bcsc(net, l, ptr[l], row_idx[l], weight[l], blocksize_c, fz)
        eng.build()
        eng.set_input(net, x.astype(np.uint8) if np.all((x == 0) | (x == 1)) else
                      x.astype(np.float32))
        eng.run()
        res = eng.result(net)
    finally:
        eng.close()
    if verbose:
        for l, n in enumerate(res["alive"]):
            print(f"layer {l}, feature = {n}")
    res["categories"] = res["categories"] + lo
    return res


def test_graph_challenge_tc_co(input1, weight1, row_idx1, ptr1, fuse_list1, batch1, neuron1, bias1,
                               input2, weight2, row_idx2, ptr2, fuse_list2, batch2, neuron2, bias2,
                               blocksize_c=16, blocksize_r=16, gpu_id=0, gpu_num=1,
                               precision=PREC_FP16, threshold=THRESHOLD, verbose=True):
    """Mirror of the reference's test_graph_challenge_tc_co
    (src/cospdnn_double.cu:208-1214): two networks, each given as in
    test_graph_challenge_tc, run in one engine and one graph launch.  They may
    differ in width, depth and batch (the reference needs equal depth).  Each
    network's rows are split over gpu_num slices and slice gpu_id is computed,
    as in src/cospdnn_double.cu:236-274.  Prints "SpDNN k layer l, feature = n"
    for network k = 1, 2 when verbose and returns one dict(categories, alive)
    per network.  Raises on error instead of exiting."""
    if blocksize_c != blocksize_r:
        raise CospdnnError(ERR_UNSUPPORTED, "square blocks only")
    nets = ((input1, weight1, row_idx1, ptr1, fuse_list1, batch1, neuron1, bias1),
            (input2, weight2, row_idx2, ptr2, fuse_list2, batch2, neuron2, bias2))
    eng = Engine(gpu_id if gpu_num > 1 else 0)
    ids, los, xs = [], [], []
    try:
        for inp, weight, row_idx, ptr, fuse_list, batch, neuron, bias in nets:
            rows_per = (batch + gpu_num - 1) // gpu_num
            lo, hi = gpu_id * rows_per, min((gpu_id + 1) * rows_per, batch)
            nid = eng.add_net(neuron, len(weight), hi - lo, bias, threshold, precision)
            for l in range(len(weight)):
                fz = None if fuse_list is None else fuse_list[l]
                eng.set_layer_bcsc(nid, l, ptr[l], row_idx[l], weight[l], blocksize_c, fz)
            ids.append(nid)
            los.append(lo)
            xs.append(np.asarray(inp)[lo:hi])
        eng.build()
        for nid, x in zip(ids, xs):
            eng.set_input(nid, x.astype(np.uint8) if np.all((x == 0) | (x == 1)) else x.astype(np.float32))
        eng.run()
        res = [eng.result(nid) for nid in ids]
    finally:
        eng.close()
    for k, (r, lo) in enumerate(zip(res, los)):
        if verbose:
            for l, n in enumerate(r["alive"]):
                print(f"SpDNN {k + 1} layer {l}, feature = {n}")
        r["categories"] = r["categories"] + lo
    return res[0], res[1]


# mirrors of the reference's host functions, not tests (pytest collects names
# that start with "test" from a module that imports them)
test_graph_challenge_tc.__test__ = False
test_graph_challenge_tc_co.__test__ = False


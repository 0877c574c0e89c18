"""KBSRC on B200: DFT-domain rational resampling with the overlap-save block engine on the GPU (sm_100a).

Python access to the in-tree native libraries through ctypes:
  lib/libkbsrc.so      kbsrc::resample and its C form (include/kbsrc/kbsrc_c.h)
  lib/libkbsrc_gpu.so  the engine's C ABI (include/kbsrc_gpu.h)
The GPU path is the only path: loading fails loudly when the libraries are missing or not built.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# KBSRC_B200_LIB selects another build of the same libraries (a directory holding lib/ and bin/)
LIB_DIR = os.path.join(os.environ.get("KBSRC_B200_LIB", HERE), "lib")
HOST_SO = os.path.join(LIB_DIR, "libkbsrc.so")
GPU_SO = os.path.join(LIB_DIR, "libkbsrc_gpu.so")
CLI = os.path.join(os.path.dirname(LIB_DIR), "bin", "kbsrc")

FAST, EXACT = 0, 1
_P = ctypes.POINTER
_dp = _P(ctypes.c_double)
_lp = _P(ctypes.c_longlong)

# status codes of include/kbsrc_gpu.h
GPU_OK, GPU_E_ARG, GPU_E_NOMEM, GPU_E_CUDA, GPU_E_UNSUPPORTED, GPU_E_NODEVICE = 0, -1, -2, -3, -4, -5


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("length", ctypes.c_double), ("beta", ctypes.c_double),
                ("threads", ctypes.c_int), ("block", ctypes.c_int), ("lpc_edges", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("p", ctypes.c_longlong), ("q", ctypes.c_longlong), ("taps", ctypes.c_longlong),
                ("block", ctypes.c_int), ("threads", ctypes.c_int), ("general_fold", ctypes.c_int),
                ("design_seconds", ctypes.c_double), ("process_seconds", ctypes.c_double),
                ("passband", ctypes.c_double), ("stopband", ctypes.c_double), ("isa", ctypes.c_char_p)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["isa"] = (d["isa"] or b"").decode()
        return d


class BatchItem(ctypes.Structure):
    """kbsrc_batch_item_c (include/kbsrc/kbsrc_c.h)."""
    _fields_ = [("in_", _dp), ("frames", ctypes.c_longlong), ("channels", ctypes.c_int), ("rate_in", ctypes.c_int),
                ("rate_out", ctypes.c_int)]


class GpuShard(ctypes.Structure):
    """kbsrc_gpu_shard (include/kbsrc_gpu.h): one device's share of a conversion."""
    _fields_ = [("blk0", ctypes.c_longlong), ("blk1", ctypes.c_longlong), ("frame0", ctypes.c_longlong),
                ("frames", ctypes.c_longlong), ("out0", ctypes.c_longlong), ("nout", ctypes.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GpuDesc(ctypes.Structure):
    """kbsrc_gpu_desc (include/kbsrc_gpu.h)."""
    _fields_ = [("precision", ctypes.c_int), ("channels", ctypes.c_int), ("P", ctypes.c_longlong),
                ("Q", ctypes.c_longlong), ("nb", ctypes.c_int), ("marg", ctypes.c_int), ("nblk", ctypes.c_longlong),
                ("lead", ctypes.c_longlong), ("o", ctypes.c_longlong), ("frames", ctypes.c_longlong),
                ("nout", ctypes.c_longlong), ("up", ctypes.c_int), ("Jg", ctypes.c_int),
                ("edge_len", ctypes.c_longlong), ("H", _dp), ("H_len", ctypes.c_longlong),
                ("in_format", ctypes.c_int), ("shard", GpuShard)]


# Every symbol the C headers declare: (library, name, restype, argtypes)
GPU_SYMBOLS = {
    "kbsrc_gpu_engine_create": (ctypes.c_int, [_P(GpuDesc), _P(ctypes.c_void_p)]),
    "kbsrc_gpu_engine_run_host": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, _dp]),
    "kbsrc_gpu_engine_run_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "kbsrc_gpu_engine_run_device_timed": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                         ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                         _P(ctypes.c_float), _P(ctypes.c_int)]),
    "kbsrc_gpu_engine_run_host_packed": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                                        ctypes.c_void_p, _lp]),
    "kbsrc_gpu_pack": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_int,
                                      ctypes.c_int, ctypes.c_void_p, _lp, ctypes.c_void_p]),
    "kbsrc_gpu_engine_info": (ctypes.c_int, [ctypes.c_void_p, _lp, _lp, _lp]),
    "kbsrc_gpu_engine_destroy": (None, [ctypes.c_void_p]),
    "kbsrc_gpu_kernel_spectrum": (ctypes.c_int, [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp]),
    "kbsrc_gpu_kernel_spectrum_static": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                        ctypes.c_void_p, ctypes.c_void_p]),
    "kbsrc_gpu_batch_create": (ctypes.c_int, [_P(GpuDesc), ctypes.c_int, _P(ctypes.c_void_p)]),
    "kbsrc_gpu_batch_run_device": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_void_p), _P(ctypes.c_void_p),
                                                  _P(ctypes.c_void_p), _P(ctypes.c_void_p), ctypes.c_void_p]),
    "kbsrc_gpu_batch_run_host": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_void_p), _P(ctypes.c_void_p),
                                                _P(ctypes.c_void_p), _P(ctypes.c_void_p)]),
    "kbsrc_gpu_batch_info": (ctypes.c_int, [ctypes.c_void_p, _lp, _lp, _lp]),
    "kbsrc_gpu_batch_destroy": (None, [ctypes.c_void_p]),
    "kbsrc_gpu_last_error": (ctypes.c_char_p, []),
    "kbsrc_gpu_engine_name": (ctypes.c_char_p, []),
    "kbsrc_gpu_engine_tune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, _P(ctypes.c_int)]),
    "kbsrc_gpu_engine_staging": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_int)]),
    "kbsrc_gpu_init": (ctypes.c_int, []),
    "kbsrc_gpu_shard_plan": (ctypes.c_int, [_P(GpuDesc), ctypes.c_int, _P(GpuShard)]),
    "kbsrc_gpu_use_device": (ctypes.c_int, [ctypes.c_int]),
}
HOST_SYMBOLS = {
    "kbsrc_output_frames": (ctypes.c_longlong, [ctypes.c_longlong, ctypes.c_int, ctypes.c_int]),
    "kbsrc_resample_c": (ctypes.c_longlong, [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             _P(Options), _dp, ctypes.c_longlong, _P(Stats), ctypes.c_char_p,
                                             ctypes.c_int]),
    "kbsrc_version_c": (ctypes.c_char_p, []),
    "kbsrc_prepare_c": (ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       _P(Options), _P(ctypes.c_void_p), ctypes.c_char_p, ctypes.c_int]),
    "kbsrc_conversion_run_c": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_char_p, ctypes.c_int]),
    "kbsrc_conversion_info_c": (ctypes.c_int, [ctypes.c_void_p, _lp, _lp, _P(_dp), _P(_dp),
                                               _P(ctypes.c_void_p), _P(Stats)]),
    "kbsrc_conversion_free_c": (None, [ctypes.c_void_p]),
    "kbsrc_batch_prepare_c": (ctypes.c_int, [_P(BatchItem), ctypes.c_int, _P(Options), _P(ctypes.c_void_p),
                                             ctypes.c_char_p, ctypes.c_int]),
    "kbsrc_batch_run_c": (ctypes.c_int, [ctypes.c_void_p, _P(ctypes.c_void_p), _P(ctypes.c_void_p), ctypes.c_char_p,
                                         ctypes.c_int]),
    "kbsrc_batch_info_c": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _lp, _lp, _P(_dp), _P(_dp),
                                          _P(ctypes.c_int)]),
    "kbsrc_batch_gpu_c": (ctypes.c_void_p, [ctypes.c_void_p]),
    "kbsrc_batch_free_c": (None, [ctypes.c_void_p]),
    "kbsrc_plan_c": (ctypes.c_int, [ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P(Options), _lp,
                                    ctypes.c_char_p, ctypes.c_int]),
    "kbsrc_kernel_taps_c": (ctypes.c_int, [ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_double,
                                           ctypes.c_int, _dp]),
    "kbsrc_burg_c": (ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.c_longlong, _dp]),
    "kbsrc_resample_devices_c": (ctypes.c_longlong, [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                     _P(ctypes.c_int), ctypes.c_int, _P(Options), _dp,
                                                     ctypes.c_longlong, _P(Stats), ctypes.c_char_p, ctypes.c_int]),
    "kbsrc_prepare_share_c": (ctypes.c_int, [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             _P(Options), ctypes.c_int, ctypes.c_int, _P(ctypes.c_void_p),
                                             ctypes.c_char_p, ctypes.c_int]),
    "kbsrc_conversion_share_c": (ctypes.c_int, [ctypes.c_void_p, _lp]),
}
PLAN_KEYS = ["P", "Q", "taps", "nb", "marg", "hop", "nblk", "Nb", "Mb", "pre", "o", "E", "lead", "general", "up",
             "nout"]

_gpu = None
_host = None


def _bind(path, table):
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is not built: run `make -C {HERE}` (or __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    for name, (res, args) in table.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def gpu_lib():
    """libkbsrc_gpu.so with its C ABI bound."""
    global _gpu
    if _gpu is None:
        _gpu = _bind(GPU_SO, GPU_SYMBOLS)
    return _gpu


def host_lib():
    """libkbsrc.so (loads libkbsrc_gpu.so) with its C API bound."""
    global _host
    if _host is None:
        gpu_lib()
        _host = _bind(HOST_SO, HOST_SYMBOLS)
    return _host


def gpu_error():
    return (gpu_lib().kbsrc_gpu_last_error() or b"").decode()


def _ptr(a):
    return a.ctypes.data_as(_dp)


def _options(mode, length, beta, block, lpc, threads):
    prec = {"fast": 0, "exact": 1, "ld": 2, "split": 3, "split16": 4}[mode] if isinstance(mode, str) else int(mode)
    return Options(prec, float(length), float(beta), int(threads), int(block), int(bool(lpc)))


def output_frames(frames, rate_in, rate_out):
    return int(host_lib().kbsrc_output_frames(frames, rate_in, rate_out))


def resample(x, rate_in, rate_out, mode="exact", length=0.2, beta=40.0, block=0, lpc=True, threads=0, stats=None):
    """Converts x (frames, channels) float64 from rate_in to rate_out on the GPU. Returns planar (channels, nout).

    Raises ValueError for rejected arguments (the reference's messages) and RuntimeError for GPU failures.
    """
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
    frames, ch = x.shape
    n = output_frames(frames, rate_in, rate_out)
    if n < 0:
        raise ValueError("sample rates must be positive" if rate_in < 1 or rate_out < 1 else "input too long")
    out = np.zeros((ch, max(n, 1)))
    st = Stats()
    err = ctypes.create_string_buffer(512)
    opt = _options(mode, length, beta, block, lpc, threads)
    r = host_lib().kbsrc_resample_c(_ptr(x), frames, ch, rate_in, rate_out, ctypes.byref(opt), _ptr(out),
                                    out.shape[1], ctypes.byref(st), err, 512)
    if r == -1:
        raise ValueError(err.value.decode())
    if r < 0:
        raise RuntimeError(err.value.decode())
    if stats is not None:
        stats.update(st.as_dict())
    return out[:, :r]


class Conversion:
    """A planned conversion (kbsrc_prepare_c): plan, LPC edges, kernel spectrum and GPU engine, built once for
    input of one shape and run many times.

    share=(index, count): the engine runs only share `index` of the conversion split into `count` contiguous block
    ranges (kbsrc_prepare_share_c, one process per GPU); `self.share` then describes it (blocks, input frames
    [frame0, frame0 + frames) and output samples [out0, out0 + nout)), run() returns that share's output, and the
    device buffers of run_device() hold the share's input span and output range only."""

    def __init__(self, x, rate_in, rate_out, mode="exact", length=0.2, beta=40.0, block=0, lpc=True, threads=0,
                 share=None):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.ndim == 1:
            x = x[:, None]
        self.frames, self.channels = x.shape
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        opt = _options(mode, length, beta, block, lpc, threads)
        if share is None:
            r = host_lib().kbsrc_prepare_c(_ptr(x), self.frames, self.channels, rate_in, rate_out, ctypes.byref(opt),
                                           ctypes.byref(self._h), err, 512)
        else:
            r = host_lib().kbsrc_prepare_share_c(_ptr(x), self.frames, self.channels, rate_in, rate_out,
                                                 ctypes.byref(opt), int(share[0]), int(share[1]),
                                                 ctypes.byref(self._h), err, 512)
        if r == -1:
            raise ValueError(err.value.decode())
        if r < 0:
            raise RuntimeError(err.value.decode())
        nout, elen = ctypes.c_longlong(), ctypes.c_longlong()
        head, tail = _dp(), _dp()
        eng = ctypes.c_void_p()
        st = Stats()
        host_lib().kbsrc_conversion_info_c(self._h, ctypes.byref(nout), ctypes.byref(elen), ctypes.byref(head),
                                           ctypes.byref(tail), ctypes.byref(eng), ctypes.byref(st))
        self.nout, self.edge_len, self.engine = nout.value, elen.value, eng.value
        n = self.edge_len * self.channels
        self.head = np.ctypeslib.as_array(head, (n,)).copy() if n else np.zeros(0)
        self.tail = np.ctypeslib.as_array(tail, (n,)).copy() if n else np.zeros(0)
        self.stats = st.as_dict()
        self.share = None
        if share is not None:
            v = np.zeros(6, dtype=np.int64)
            host_lib().kbsrc_conversion_share_c(self._h, v.ctypes.data_as(_lp))
            self.share = dict(zip(["blk0", "blk1", "frame0", "frames", "out0", "nout"], v.tolist()))

    @property
    def out_len(self):
        """Output samples per channel that run() returns: nout, or the share's."""
        return self.share["nout"] if self.share and self.share["blk1"] else self.nout

    def run(self, x, out=None):
        """Runs on interleaved input x (frames, channels) host memory (the whole input, also for a share); returns
        planar (channels, out_len)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        n = self.out_len
        if out is None:
            out = np.zeros((self.channels, max(n, 1)))
        err = ctypes.create_string_buffer(512)
        if host_lib().kbsrc_conversion_run_c(self._h, _ptr(x), _ptr(out), err, 512):
            raise RuntimeError(err.value.decode())
        return out[:, :n]

    def engine_info(self):
        t, l, b = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        gpu_lib().kbsrc_gpu_engine_info(self.engine, ctypes.byref(t), ctypes.byref(l), ctypes.byref(b))
        return {"tasks": t.value, "launches": l.value, "device_bytes": b.value}

    def run_device(self, d_in, d_head, d_tail, d_out, stream=0):
        """Engine run on device pointers (ints), asynchronous on `stream` (a cudaStream_t as int, 0 = engine's)."""
        rc = gpu_lib().kbsrc_gpu_engine_run_device(self.engine, d_in, d_head, d_tail, d_out, stream or None)
        if rc:
            raise RuntimeError(f"kbsrc_gpu_engine_run_device: {rc} {gpu_error()}")

    PASSES = ["fwd_column", "fwd_row", "split", "merge", "inv_column", "inv_row"]

    def run_device_timed(self, d_in, d_head, d_tail, d_out, stream=0):
        """run_device with an event after every launch; returns {pass: (ms, launches)} (synchronises)."""
        ms = (ctypes.c_float * 6)()
        n = (ctypes.c_int * 6)()
        rc = gpu_lib().kbsrc_gpu_engine_run_device_timed(self.engine, d_in, d_head, d_tail, d_out, stream or None,
                                                         ms, n)
        if rc:
            raise RuntimeError(f"kbsrc_gpu_engine_run_device_timed: {rc} {gpu_error()}")
        return {k: (ms[i], n[i]) for i, k in enumerate(self.PASSES)}

    def tune(self, d_in, d_head, d_tail, d_out, stream=0):
        """Autotuner (kbsrc_gpu_engine_tune): times launch shapes on these device buffers and keeps the fastest
        per four-step pass; returns {pass: (sequences per CTA, threads)} for the passes it tuned."""
        sh = (ctypes.c_int * 8)()
        rc = gpu_lib().kbsrc_gpu_engine_tune(self.engine, d_in, d_head, d_tail, d_out, stream or None, sh)
        if rc:
            raise RuntimeError(f"kbsrc_gpu_engine_tune: {rc} {gpu_error()}")
        names = ["fwd_column", "fwd_row", "inv_column", "inv_row"]
        return {names[i]: (sh[2 * i], sh[2 * i + 1]) for i in range(4) if sh[2 * i]}

    def staging(self):
        """kbsrc_gpu_engine_staging: {pass: True when its stage twiddles are staged in shared memory, False when
        read from the global table} for the four-step passes."""
        st = (ctypes.c_int * 4)()
        rc = gpu_lib().kbsrc_gpu_engine_staging(self.engine, st)
        if rc:
            raise RuntimeError(f"kbsrc_gpu_engine_staging: {rc} {gpu_error()}")
        names = ["fwd_column", "fwd_row", "inv_column", "inv_row"]
        return {names[i]: bool(st[i]) for i in range(4) if st[i] >= 0}

    def run_host_raw(self, x_ptr, head_ptr, tail_ptr, out_ptr):
        """Engine run on host pointers (ints), e.g. pinned buffers; synchronous."""
        rc = gpu_lib().kbsrc_gpu_engine_run_host(self.engine, ctypes.cast(x_ptr, _dp), ctypes.cast(head_ptr, _dp),
                                                 ctypes.cast(tail_ptr, _dp), ctypes.cast(out_ptr, _dp))
        if rc:
            raise RuntimeError(f"kbsrc_gpu_engine_run_host: {rc} {gpu_error()}")

    def close(self):
        if self._h:
            host_lib().kbsrc_conversion_free_c(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many conversions at once (kbsrc_batch_prepare_c): items are (x, rate_in, rate_out) with x (frames, channels)
    float64. Conversions with equal plans share kernel design and GPU launches; the GPU run is one recorded launch
    sequence (CUDA graph) replayed on every run."""

    def __init__(self, items, mode="exact", length=0.2, beta=40.0, block=0, lpc=True, threads=0):
        self.xs = [np.ascontiguousarray(x if np.ndim(x) == 2 else np.asarray(x)[:, None], dtype=np.float64)
                   for x, _, _ in items]
        arr = (BatchItem * len(items))()
        for i, ((_, fi, fo), x) in enumerate(zip(items, self.xs)):
            arr[i] = BatchItem(_ptr(x), x.shape[0], x.shape[1], fi, fo)
        self._h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        opt = _options(mode, length, beta, block, lpc, threads)
        r = host_lib().kbsrc_batch_prepare_c(arr, len(items), ctypes.byref(opt), ctypes.byref(self._h), err, 512)
        if r == -1:
            raise ValueError(err.value.decode())
        if r < 0:
            raise RuntimeError(err.value.decode())
        self.nout, self.edge_len, self.gpu_index, self.head, self.tail = [], [], [], [], []
        for i, x in enumerate(self.xs):
            n, e, gi = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
            hp, tp = _dp(), _dp()
            host_lib().kbsrc_batch_info_c(self._h, i, ctypes.byref(n), ctypes.byref(e), ctypes.byref(hp),
                                          ctypes.byref(tp), ctypes.byref(gi))
            self.nout.append(n.value)
            self.edge_len.append(e.value)
            self.gpu_index.append(gi.value)
            m = e.value * x.shape[1]
            self.head.append(np.ctypeslib.as_array(hp, (m,)).copy() if m else np.zeros(1))
            self.tail.append(np.ctypeslib.as_array(tp, (m,)).copy() if m else np.zeros(1))
        self.gpu = host_lib().kbsrc_batch_gpu_c(self._h)

    def run(self, xs=None):
        """Host buffers in and out; returns a list of planar (channels, nout) arrays."""
        xs = self.xs if xs is None else [np.ascontiguousarray(x, dtype=np.float64) for x in xs]
        outs = [np.zeros((x.shape[1], max(n, 1))) for x, n in zip(xs, self.nout)]
        pin = (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
        pout = (ctypes.c_void_p * len(xs))(*[o.ctypes.data for o in outs])
        err = ctypes.create_string_buffer(512)
        if host_lib().kbsrc_batch_run_c(self._h, pin, pout, err, 512):
            raise RuntimeError(err.value.decode())
        return [o[:, :n] for o, n in zip(outs, self.nout)]

    def gpu_info(self):
        g, t, l = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
        gpu_lib().kbsrc_gpu_batch_info(self.gpu, ctypes.byref(g), ctypes.byref(t), ctypes.byref(l))
        return {"groups": g.value, "tasks": t.value, "launches": l.value}

    def run_device(self, d_in, d_head, d_tail, d_out, stream=0):
        """GPU items only (gpu_index order): lists of device pointers; asynchronous on `stream`."""
        n = len(d_in)
        arrs = [(ctypes.c_void_p * n)(*v) for v in (d_in, d_head, d_tail, d_out)]
        rc = gpu_lib().kbsrc_gpu_batch_run_device(self.gpu, *arrs, stream or None)
        if rc:
            raise RuntimeError(f"kbsrc_gpu_batch_run_device: {rc} {gpu_error()}")

    def close(self):
        if self._h:
            host_lib().kbsrc_batch_free_c(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def resample_devices(x, rate_in, rate_out, devices, mode="exact", length=0.2, beta=40.0, block=0, lpc=True, threads=0,
                     stats=None):
    """resample() with the block loop split across CUDA devices (kbsrc_resample_devices_c): contiguous block ranges,
    one engine per device, nothing exchanged between devices; the same output as resample()."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
    frames, ch = x.shape
    n = output_frames(frames, rate_in, rate_out)
    if n < 0:
        raise ValueError("sample rates must be positive" if rate_in < 1 or rate_out < 1 else "input too long")
    out = np.zeros((ch, max(n, 1)))
    devs = (ctypes.c_int * len(devices))(*devices)
    st = Stats()
    err = ctypes.create_string_buffer(512)
    opt = _options(mode, length, beta, block, lpc, threads)
    r = host_lib().kbsrc_resample_devices_c(_ptr(x), frames, ch, rate_in, rate_out, devs, len(devices),
                                            ctypes.byref(opt), _ptr(out), out.shape[1], ctypes.byref(st), err, 512)
    if r == -1:
        raise ValueError(err.value.decode())
    if r < 0:
        raise RuntimeError(err.value.decode())
    if stats is not None:
        stats.update(st.as_dict())
    return out[:, :r]


def shard_plan(frames, channels, rate_in, rate_out, count, mode="exact", length=0.2, beta=40.0, block=0):
    """The shares of a conversion split into `count` contiguous block ranges (kbsrc_gpu_shard_plan), from the host
    plan alone: a list of dicts blk0, blk1, frame0, frames, out0, nout. No GPU needed."""
    p = plan(frames, channels, rate_in, rate_out, mode, length, beta, block)
    if p["copy"]:
        raise ValueError("equal rates: no block loop to split")
    d = GpuDesc()
    d.precision = {"fast": 0, "exact": 1, "ld": 2, "split": 3, "split16": 4}[mode]
    d.channels, d.P, d.Q, d.nb, d.marg, d.nblk = channels, p["P"], p["Q"], p["nb"], p["marg"], p["nblk"]
    d.lead, d.o, d.frames, d.nout, d.up = p["lead"], p["o"], frames, p["nout"], p["up"]
    n_spec = (p["Mb"] if p["up"] else p["Nb"]) // 2 + 1
    H = np.zeros((n_spec, 2))  # the shares do not depend on the spectrum's values
    d.H, d.H_len = _ptr(H), n_spec
    if p["general"]:
        d.Jg = 1
        H = np.zeros((max(p["Nb"], p["Mb"]) * 2, 2))
        d.H, d.H_len = _ptr(H), H.shape[0]
    out = (GpuShard * count)()
    rc = gpu_lib().kbsrc_gpu_shard_plan(ctypes.byref(d), count, out)
    if rc:
        raise ValueError(gpu_error())
    return [s.as_dict() for s in out]


def plan(frames, channels, rate_in, rate_out, mode="exact", length=0.2, beta=40.0, block=0):
    """The host block plan as a dict (PLAN_KEYS; "copy" True for equal rates). ValueError on rejection."""
    info = np.zeros(16, dtype=np.int64)
    err = ctypes.create_string_buffer(512)
    opt = _options(mode, length, beta, block, True, 0)
    r = host_lib().kbsrc_plan_c(frames, channels, rate_in, rate_out, ctypes.byref(opt), info.ctypes.data_as(_lp),
                                err, 512)
    if r < 0:
        raise ValueError(err.value.decode())
    d = dict(zip(PLAN_KEYS, info.tolist()))
    d["copy"] = r == 1
    return d


def kernel_taps(L, a, b, beta, threads=1):
    out = np.zeros((L + 1, 2))
    if host_lib().kbsrc_kernel_taps_c(L, a, b, beta, threads, _ptr(out)):
        raise ValueError("bad tap arguments")
    return out


def burg(x, n):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(n)
    if host_lib().kbsrc_burg_c(_ptr(x), len(x), n, _ptr(out)):
        raise ValueError("bad arguments")
    return out


FORMATS = {"f64": (0, 8), "f32": (1, 4), "s32": (2, 4), "s24": (3, 3), "s16": (4, 2)}


def pack(planar, fmt, dither=False):
    """The GPU output step (kbsrc_gpu_pack): planar (channels, frames) float64 -> (WAV data bytes, clipped)."""
    import torch
    code, bps = FORMATS[fmt]
    planar = np.ascontiguousarray(planar, dtype=np.float64)
    ch, n = planar.shape
    d_y = torch.from_numpy(planar).cuda()
    d_o = torch.empty(max(1, ch * n * bps), dtype=torch.uint8, device="cuda")
    clipped = ctypes.c_longlong()
    rc = gpu_lib().kbsrc_gpu_pack(d_y.data_ptr(), ch, n, n, code, int(dither), d_o.data_ptr(), ctypes.byref(clipped),
                                  None)
    if rc:
        raise RuntimeError(f"kbsrc_gpu_pack: {rc} {gpu_error()}")
    torch.cuda.synchronize()
    return d_o[:ch * n * bps].cpu().numpy().tobytes(), clipped.value


def kernel_spectrum(taps, n, scale):
    """GPU kernel design (kbsrc_gpu_kernel_spectrum): taps (L+1, 2) (hi, lo) -> H (n/2+1, 2)."""
    taps = np.ascontiguousarray(taps, dtype=np.float64)
    H = np.zeros((n // 2 + 1, 2))
    rc = gpu_lib().kbsrc_gpu_kernel_spectrum(_ptr(taps), taps.shape[0] - 1, n, scale, _ptr(H))
    if rc:
        raise RuntimeError(f"kbsrc_gpu_kernel_spectrum: {rc} {gpu_error()}")
    return H


def build(verbose=False):
    """Compiles the native libraries in place (make -C kbsrc_b200)."""
    import subprocess
    r = subprocess.run(["make", "-C", HERE, "-j4"], capture_output=not verbose, text=True)
    if r.returncode:
        raise RuntimeError(f"build failed:\n{r.stdout}\n{r.stderr}")

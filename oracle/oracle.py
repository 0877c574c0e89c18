"""TEST INFRASTRUCTURE ONLY: ctypes access to the oracle (liboracle.so, the C restatement in kbsrc_oracle.c)
and to the reference built from source (_ref/libkbsrc_ref.so). Only tests/, __graft_entry__.smoke() and
bench.py (cpu_baseline and the reference arm) import this module, always as the checker or the baseline.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libkbsrc_ref.so")
REF_CLI = os.path.join(HERE, "_ref", "kbsrc")
REF_DRIVER = os.path.join(HERE, "_ref", "kbsrc_fenv_driver")

_P = ctypes.POINTER
_dp = _P(ctypes.c_double)
_lp = _P(ctypes.c_longlong)

# Error codes of oracle_resample mapped to the reference's messages (src/resampler.cpp:94-155)
ORACLE_ERRORS = {
    -1: "bad input buffer",
    -2: "sample rates must be positive",
    -3: "option out of range",
    -4: "input too long",
    -5: "length too short for these sample rates",
    -6: "block, rates or length too large",
}
INFO_KEYS = ["P", "Q", "taps", "nb", "marg", "hop", "nblk", "Nb", "Mb", "pre", "o", "E", "tot", "gen", "Jg", "up"]

_oracle = None
_ref = None


def _ptr(a):
    return a.ctypes.data_as(_dp)


def oracle_lib():
    """The oracle shared library (built by `make -C oracle liboracle.so`)."""
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(ORACLE_SO)
        lib.oracle_resample.restype = ctypes.c_longlong
        lib.oracle_resample.argtypes = [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        _dp, ctypes.c_longlong, _lp]
        lib.oracle_resample_blocks.restype = ctypes.c_longlong
        lib.oracle_resample_blocks.argtypes = [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, _dp,
                                               ctypes.c_longlong, _lp]
        lib.oracle_plan.restype = ctypes.c_longlong
        lib.oracle_plan.argtypes = [ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, _lp]
        for name in ("oracle_rfft_forward", "oracle_rfft_inverse", "oracle_cfft"):
            f = getattr(lib, name)
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp]
        lib.oracle_kernel.restype = ctypes.c_longlong
        lib.oracle_kernel.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_longlong, ctypes.c_int, _dp, ctypes.c_longlong]
        lib.oracle_burg.restype = ctypes.c_int
        lib.oracle_burg.argtypes = [_dp, ctypes.c_longlong, ctypes.c_longlong, _dp]
        _oracle = lib
    return _oracle


def nout_of(frames, rate_in, rate_out):
    import math
    g = math.gcd(rate_in, rate_out)
    P, Q = rate_out // g, rate_in // g
    return -(-frames * P // Q)


def plan(frames, channels, rate_in, rate_out, fast=False, length=0.2, beta=40.0, block=0):
    """The oracle's block plan as a dict (keys INFO_KEYS plus nout)."""
    info = np.zeros(16, dtype=np.int64)
    n = oracle_lib().oracle_plan(frames, channels, rate_in, rate_out, int(fast), length, beta, block,
                                 info.ctypes.data_as(_lp))
    if n < 0:
        raise ValueError(ORACLE_ERRORS.get(n, f"error {n}"))
    d = dict(zip(INFO_KEYS, info.tolist()))
    d["nout"] = int(n)
    return d


MODES = {"exact": 0, "fast": 1, "ld": 2}


def resample(x, rate_in, rate_out, fast=False, length=0.2, beta=40.0, block=0, lpc=True, info=None, mode=None):
    """Oracle conversion. x: (frames, channels) float64; mode "exact", "fast" or "ld" (else `fast` decides).
    Returns planar (channels, nout) float64."""
    code = MODES[mode] if mode else int(bool(fast))
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
    frames, ch = x.shape
    cap = max(1, nout_of(frames, rate_in, rate_out))
    out = np.zeros((ch, cap), dtype=np.float64)
    inf = np.zeros(16, dtype=np.int64)
    n = oracle_lib().oracle_resample(_ptr(x), frames, ch, rate_in, rate_out, code, length, beta, block,
                                     int(lpc), _ptr(out), cap, inf.ctypes.data_as(_lp))
    if n < 0:
        raise ValueError(ORACLE_ERRORS.get(n, f"error {n}"))
    if info is not None:
        info.update(zip(INFO_KEYS, inf.tolist()))
    return out[:, :n]


def resample_blocks(x, rate_in, rate_out, blk0, blk1, mode="exact", length=0.2, beta=40.0, block=0, lpc=True):
    """The oracle conversion restricted to blocks [blk0, blk1) of every channel: planar (channels, nout) with the
    samples no block of the range writes left at zero."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
    frames, ch = x.shape
    cap = max(1, nout_of(frames, rate_in, rate_out))
    out = np.zeros((ch, cap), dtype=np.float64)
    inf = np.zeros(16, dtype=np.int64)
    n = oracle_lib().oracle_resample_blocks(_ptr(x), frames, ch, rate_in, rate_out, MODES[mode], length, beta,
                                            block, int(lpc), blk0, blk1, _ptr(out), cap, inf.ctypes.data_as(_lp))
    if n < 0:
        raise ValueError(ORACLE_ERRORS.get(n, f"error {n}"))
    return out[:, :n]


def rfft_forward(mode, r):
    """mode 0 fast, 1 exact, 2 dd. r: (N, 2) float64 (hi, lo). Returns (N/2+1, 4)."""
    r = np.ascontiguousarray(r, dtype=np.float64)
    N = r.shape[0]
    out = np.zeros((N // 2 + 1, 4))
    if oracle_lib().oracle_rfft_forward(mode, N, _ptr(r), _ptr(out)):
        raise ValueError("bad length")
    return out


def rfft_inverse(mode, X, N):
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros((N, 2))
    if oracle_lib().oracle_rfft_inverse(mode, N, _ptr(X), _ptr(out)):
        raise ValueError("bad length")
    return out


def cfft(mode, x):
    """x: (n, 4) complex dd. Returns (n, 4)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    if oracle_lib().oracle_cfft(mode, x.shape[0], _ptr(x), _ptr(out)):
        raise ValueError("bad length")
    return out


def kernel_spectrum(frames, channels, rate_in, rate_out, fast=False, length=0.2, beta=40.0, block=0):
    """The designed kernel spectrum H as (n/2+1, 2) (hi, lo)."""
    p = plan(frames, channels, rate_in, rate_out, fast, length, beta, block)
    n = p["Mb"] if p["up"] else p["Nb"]
    H = np.zeros((n // 2 + 1, 2))
    r = oracle_lib().oracle_kernel(rate_in, rate_out, int(fast), length, beta, block, frames, channels, _ptr(H),
                                   H.shape[0])
    if r < 0:
        raise ValueError(f"error {r}")
    return H


def burg(x, n):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(n)
    oracle_lib().oracle_burg(_ptr(x), len(x), n, _ptr(out))
    return out


# ---- the reference built from source ----------------------------------------------------------------------

def ref_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_SO)
        f = lib.kbsrc_ref_resample
        f.restype = ctypes.c_longlong
        f.argtypes = [_dp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                      ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                      ctypes.c_longlong, _lp, _dp, ctypes.c_char_p, ctypes.c_int]
        _ref = lib
    return _ref


def ref_resample(x, rate_in, rate_out, fast=False, length=0.2, beta=40.0, block=0, lpc=True, threads=0,
                 stats=None, mode=None):
    """The reference library's kbsrc::resample; mode "exact", "fast" or "ld" (else `fast` decides). Returns
    planar (ch, nout)."""
    prec = {"fast": 0, "exact": 1, "ld": 2}[mode] if mode else (0 if fast else 1)
    x = np.ascontiguousarray(x, dtype=np.float64)
    if x.ndim == 1:
        x = x[:, None]
    frames, ch = x.shape
    cap = max(1, nout_of(frames, rate_in, rate_out))
    out = np.zeros((ch, cap))
    plan_ = np.zeros(5, dtype=np.int64)
    secs = np.zeros(2)
    err = ctypes.create_string_buffer(256)
    n = ref_lib().kbsrc_ref_resample(_ptr(x), frames, ch, rate_in, rate_out, prec, length, beta,
                                     threads, block, int(lpc), _ptr(out), cap, plan_.ctypes.data_as(_lp),
                                     _ptr(secs), err, 256)
    if n < 0:
        raise ValueError(err.value.decode() or f"error {n}")
    if stats is not None:
        stats.update(zip(["p", "q", "taps", "block", "threads"], plan_.tolist()))
        stats["design_seconds"], stats["process_seconds"] = secs.tolist()
    return out[:, :n]

"""The kernel-spectrum entry for callers that cannot let a library allocate GPU memory.

An application that has reserved the device's memory for its own pool, or whose other streams must not stall at
cudaFree's device-wide wait, can call kbsrc_gpu_kernel_spectrum_static: it takes the taps and the output in device
memory and keeps its scratch, twiddle tables included, in one device array inside the library. These tests call it
through the C ABI and hold it to the oracle (the reference's kernel design restated in C) and to the allocating
entry, bit for bit, on two calls in a row that share the array, on the caller's own stream, and check its refusals.
This file is collected last so that, on a failure, every other test has already run.
"""
import math

import numpy as np
import pytest

import kbsrc_b200
from oracle import oracle

pytestmark = pytest.mark.gpu


def design(fi, fo, frames, mode="exact", length=0.2, beta=40.0, block=0):
    p = kbsrc_b200.plan(frames, 2, fi, fo, mode, length, beta, block)
    fk = fo if p["up"] else fi
    fml = math.sqrt(beta * beta + 9.8696044010893586) / (2 * 3.14159265358979323846 * length)
    c2 = min(fi, fo) - int(math.ceil(2 * fml))
    g = math.gcd(c2, fk)
    L = int(math.floor(length * fk))
    taps = kbsrc_b200.kernel_taps(L, c2 // g, fk // g, beta, threads=4)
    n = p["Mb"] if p["up"] else p["Nb"]
    return taps, n, float(p["Nb"])


def static_spectrum(taps, n, scale, calls=2, stream=None):
    """Runs the entry `calls` times in a row on `stream` (a torch stream, None: the default stream) and returns
    each result as an (n/2+1, 2) array of (hi, lo) pairs."""
    import torch
    d_taps = torch.from_numpy(np.ascontiguousarray(taps).ravel().copy()).cuda()
    lib = kbsrc_b200.gpu_lib()
    outs = []
    for _ in range(calls):
        d_H = torch.full(((n // 2 + 1) * 2,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        handle = stream.cuda_stream if stream is not None else None
        rc = lib.kbsrc_gpu_kernel_spectrum_static(d_taps.data_ptr(), taps.shape[0] - 1, n, scale, d_H.data_ptr(),
                                                  handle)
        assert rc == 0, kbsrc_b200.gpu_error()
        if stream is not None:
            stream.synchronize()  # the call's work is on that stream alone
        else:
            torch.cuda.synchronize()
        outs.append(d_H.cpu().numpy().reshape(-1, 2))
    return outs


# the oracle cases of the allocating entry (frames, rates, mode, block, --len): four-step forward, upsampling,
# a short kernel and the fast plan's block size
ORACLE_CASES = [(96000, 44100, False, 0, 0.2), (44100, 48000, True, 0, 0.2), (48000, 96000, False, 0, 0.01),
                (96000, 44100, True, 0, 0.2)]


@pytest.mark.parametrize("fi,fo,fast,block,length", ORACLE_CASES)
def test_static_scratch_matches_oracle(fi, fo, fast, block, length):
    frames = 200000
    want = oracle.kernel_spectrum(frames, 2, fi, fo, fast=fast, length=length, block=block)
    taps, n, scale = design(fi, fo, frames, "fast" if fast else "exact", length, 40.0, block)
    for got in static_spectrum(taps, n, scale):
        assert got.shape == want.shape
        assert got.tobytes() == want.tobytes()


# (rate_in, rate_out, frames): a four-step forward size, an upsampling size, and a direct (<= 2048-point) one
CASES = [(96000, 44100, 960000), (44100, 48000, 300000), (8000, 16000, 3000)]


@pytest.mark.parametrize("fi,fo,frames", CASES)
def test_static_scratch_matches_allocating_entry(fi, fo, frames):
    taps, n, scale = design(fi, fo, frames)
    want = kbsrc_b200.kernel_spectrum(taps, n, scale)
    for got in static_spectrum(taps, n, scale):  # consecutive calls share the scratch array
        assert got.tobytes() == want.tobytes()


def test_static_scratch_on_a_side_stream():
    import torch
    taps, n, scale = design(96000, 44100, 200000)
    want = kbsrc_b200.kernel_spectrum(taps, n, scale)
    side = torch.cuda.Stream()
    for got in static_spectrum(taps, n, scale, stream=side):
        assert got.tobytes() == want.tobytes()


def test_static_scratch_rejects_oversized_transform():
    import torch
    taps = np.zeros((11, 2))
    taps[0, 0] = 1.0
    d_taps = torch.from_numpy(taps.ravel().copy()).cuda()
    n = 1 << 20
    d_H = torch.zeros((n // 2 + 1) * 2, dtype=torch.float64, device="cuda")
    rc = kbsrc_b200.gpu_lib().kbsrc_gpu_kernel_spectrum_static(d_taps.data_ptr(), 10, n, 1.0, d_H.data_ptr(), None)
    assert rc == kbsrc_b200.GPU_E_ARG
    assert "static scratch" in kbsrc_b200.gpu_error()


def test_static_scratch_rejects_bluestein_lengths():
    """n/2 = 1013 is prime: its transform needs Bluestein's chirp-z, which this entry does not run."""
    import torch
    taps = np.zeros((11, 2))
    taps[0, 0] = 1.0
    d_taps = torch.from_numpy(taps.ravel().copy()).cuda()
    n = 2 * 1013
    d_H = torch.zeros((n // 2 + 1) * 2, dtype=torch.float64, device="cuda")
    rc = kbsrc_b200.gpu_lib().kbsrc_gpu_kernel_spectrum_static(d_taps.data_ptr(), 10, n, 1.0, d_H.data_ptr(), None)
    assert rc == kbsrc_b200.GPU_E_UNSUPPORTED
    # the allocating entry takes the same n
    assert np.isfinite(kbsrc_b200.kernel_spectrum(taps, n, 1.0)).all()

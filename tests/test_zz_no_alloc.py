"""The kernel-spectrum entry for callers that cannot allocate device memory.

kbsrc_gpu_kernel_spectrum_static keeps its scratch in a device array inside the library, so a caller that owns
all device memory (a fixed pool, a real-time thread, a graph-capture region where allocation is forbidden) passes
only its input taps and output buffer. Its output must equal the allocating entry's, bit for bit, on consecutive
calls that share the array. This file is collected last so that, on a failure, every other test has already run.
"""
import ctypes

import numpy as np
import pytest

import kbsrc_b200

pytestmark = pytest.mark.gpu

# (rate_in, rate_out, frames): a four-step forward size, an upsampling size, and a direct (<= 2048-point) one
CASES = [(96000, 44100, 960000), (44100, 48000, 300000), (8000, 16000, 3000)]


def design(fi, fo, frames, length=0.2, beta=40.0):
    import math
    p = kbsrc_b200.plan(frames, 2, fi, fo, "exact", length, beta, 0)
    fk = fo if p["up"] else fi
    fml = math.sqrt(beta * beta + 9.8696044010893586) / (2 * 3.14159265358979323846 * length)
    c2 = min(fi, fo) - int(math.ceil(2 * fml))
    g = math.gcd(c2, fk)
    L = int(math.floor(length * fk))
    taps = kbsrc_b200.kernel_taps(L, c2 // g, fk // g, beta, threads=4)
    n = p["Mb"] if p["up"] else p["Nb"]
    return taps, n, float(p["Nb"])


@pytest.mark.parametrize("fi,fo,frames", CASES)
def test_static_scratch_matches_allocating_entry(fi, fo, frames):
    import torch
    taps, n, scale = design(fi, fo, frames)
    want = kbsrc_b200.kernel_spectrum(taps, n, scale)
    d_taps = torch.from_numpy(taps.ravel().copy()).cuda()
    lib = kbsrc_b200.gpu_lib()
    for _ in range(2):  # consecutive calls share the scratch array
        d_H = torch.full(((n // 2 + 1) * 2,), float("nan"), dtype=torch.float64, device="cuda")
        rc = lib.kbsrc_gpu_kernel_spectrum_static(d_taps.data_ptr(), taps.shape[0] - 1, n, scale, d_H.data_ptr(),
                                                  None)
        assert rc == 0, kbsrc_b200.gpu_error()
        torch.cuda.synchronize()
        got = d_H.cpu().numpy().reshape(-1, 2)
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

"""Signal properties of GPU conversions at many rate pairs: sine accuracy, no aliasing or imaging, flat passband,
exact equal-rate copies. These hold for any input length, so they check paths the golden cases do not pin
(other ratios, the general fold, Bluestein lengths) against the mathematics rather than against bytes."""
import math

import numpy as np
import pytest

import kbsrc_b200

pytestmark = pytest.mark.gpu

# common, odd, upsampling, downsampling and near-unity pairs
PAIRS = [(96000, 44100), (44100, 48000), (48000, 44100), (44100, 96000), (192000, 44100), (8000, 44100),
         (44100, 8000), (48000, 192000), (44100, 44101), (44101, 44100), (96000, 32001), (22050, 48001),
         (48000, 48001)]


def sines(t, freqs, phases, sign=1.0):
    return sign * sum(0.3 * np.sin(2 * np.pi * f * t + p) for f, p in zip(freqs, phases))


@pytest.mark.parametrize("fi,fo", PAIRS)
@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_sine_accuracy(fi, fo, mode):
    rng = np.random.default_rng(fi * 7 + fo)
    n = fi * 2
    freqs, phases = [100.0, 1000.0, 0.4 * min(fi, fo)], rng.uniform(0, 6, 3)
    t = np.arange(n) / fi
    x = np.stack([sines(t, freqs, phases), sines(t, freqs, phases, -1.0)], 1)
    y = kbsrc_b200.resample(x, fi, fo, mode=mode)
    assert y.shape == (2, -(-n * fo // fi))
    want = sines(np.arange(y.shape[1]) / fo, freqs, phases)
    mid = slice(y.shape[1] // 4, 3 * y.shape[1] // 4)
    err = max(np.abs(y[0, mid] - want[mid]).max(), np.abs(y[1, mid] + want[mid]).max())
    assert 20 * np.log10(err + 1e-300) < -200.0


@pytest.mark.parametrize("fi,fo", [(96000, 44100), (44100, 96000), (1001, 1000), (1000, 1001)])
@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_no_aliasing_or_imaging(fi, fo, mode):
    """The continuous impulse response, sampled at lcm(fi, fo) by interleaving the responses to Q impulses (one
    at each input phase), is flat to 1e-12 in the passband and below -280 dB from the lower Nyquist frequency."""
    length = 0.2
    g = math.gcd(fi, fo)
    P, Q = fo // g, fi // g
    reach = math.ceil(length * fi) + 1
    spacing = Q * math.ceil((2 * reach + 64) / Q)
    pos = spacing * np.arange(1, Q + 1) + np.arange(Q)
    x = np.zeros(spacing * (Q + 2))
    x[pos] = 1.0
    st = {}
    y = kbsrc_b200.resample(x[:, None], fi, fo, mode=mode, length=length, lpc=False, stats=st)[0]
    half = reach * P
    resp = np.zeros(2 * half + 1)
    for m in pos:
        k = np.arange(-(-(m * P - half) // Q), (m * P + half) // Q + 1)
        resp[k * Q - m * P + half] += y[k]
    H = np.abs(np.fft.rfft(resp))
    H /= H[0]
    f = np.arange(len(H)) * (fi * P) / len(resp)
    assert 0 < st["passband"] < st["stopband"] <= min(fi, fo) / 2
    stop_db = 20 * np.log10(H[f >= min(fi, fo) / 2].max() + 1e-300)
    assert stop_db < -280.0
    assert np.abs(H[f <= st["passband"]] - 1).max() < 1e-12


def test_equal_rates_copy_exactly():
    x = np.random.default_rng(5).standard_normal((4410, 3)) * 0.1
    st = {}
    y = kbsrc_b200.resample(x, 44100, 44100, stats=st)
    assert np.array_equal(y, x.T) and st["isa"] == "generic"


@pytest.mark.parametrize("n", [0, 1, 10, 97])
def test_tiny_inputs(n):
    x = np.random.default_rng(n).uniform(-0.5, 0.5, (n, 2))
    y = kbsrc_b200.resample(x, 48000, 44100)
    assert y.shape == (2, -(-n * 44100 // 48000))
    assert np.all(np.isfinite(y))


@pytest.mark.parametrize("fi,fo", [(96000, 44100), (44100, 48000), (44100, 44101)])
def test_ld_agrees_with_exact(fi, fo):
    """x87 extended (64-bit significand) and double-double (~106 bits) differ only by the extended rounding:
    well below 1e-15 of full scale at any length."""
    x = np.random.default_rng(abs(fi - fo)).uniform(-0.5, 0.5, (fi * 3, 2))
    st = {}
    a = kbsrc_b200.resample(x, fi, fo, mode="ld", stats=st)
    b = kbsrc_b200.resample(x, fi, fo, mode="exact")
    assert st["isa"] == "sm_100a" and a.shape == b.shape
    assert np.abs(a - b).max() < 1e-15
    assert not np.array_equal(a, b)  # a different arithmetic really ran

"""The split-precision tensor-core form (mode "split") against the byte-exact engines.

The split form runs the Exact plan with every FFT stage as an int8-sliced DFT-matrix contraction on the tensor
cores and float64 everywhere else, so it is not byte-identical to any reference engine. Its promise is accuracy:
its error against the exact (double-double) output is no worse than that of the reference's fast (float64)
engine on the same input. These tests hold it to that, at small sizes and at the full 180 s benchmark size."""
import numpy as np
import pytest

import kbsrc_b200
from cases import noise, sweep
from kbsrc_b200.roofline import error_stats

pytestmark = pytest.mark.gpu


def errors(x, fi, fo, **kw):
    st = {}
    s = kbsrc_b200.resample(x, fi, fo, mode="split", stats=st, **kw)
    e = kbsrc_b200.resample(x, fi, fo, mode="exact", **kw)
    f = kbsrc_b200.resample(x, fi, fo, mode="fast", **kw)
    assert s.shape == e.shape == f.shape
    assert st["isa"] == "sm_100a"
    return np.abs(s - e).max(initial=0.0), np.abs(f - e).max(initial=0.0), np.abs(e).max(initial=0.0)


CASES = [(96000, 44100, 20000, 2), (44100, 48000, 30000, 1), (48000, 96000, 97, 2), (192000, 44100, 40000, 2),
         (44100, 96000, 10000, 2), (48000, 44100, 10, 1)]


@pytest.mark.parametrize("fi,fo,n,ch", CASES)
def test_split_error_within_fast_error(fi, fo, n, ch):
    x = np.random.default_rng(fi + n).uniform(-0.5, 0.5, (n, ch))
    es, ef, peak = errors(x, fi, fo)
    print(f"split {es:.3e} fast {ef:.3e} peak {peak:.3e}")
    assert es <= max(ef, 4e-17 * peak)


def test_split_full_size_c2():
    """180 s stereo 96 kHz -> 44.1 kHz uniform noise: the headline conversion."""
    x = noise(2, 180, 96000, 2)
    es, ef, peak = errors(x, 96000, 44100)
    print(f"split {es:.3e} fast {ef:.3e} peak {peak:.3e}")
    assert es <= ef


def test_split_c3_sweep_error_stated():
    """60 s stereo 44.1 kHz -> 48 kHz log sine sweep 20 Hz - 20 kHz at amplitude 0.5: the upsampling path, whose
    spectrum is extended periodically (the reference's src/resampler.cpp:72-78) instead of folded. The split form's
    max and RMS error against the exact output, in dB and float64 ULPs, beside the fast engine's; the split form's
    maximum may not exceed the fast engine's."""
    x = sweep(60, 44100, 2)
    st = {}
    s = kbsrc_b200.resample(x, 44100, 48000, mode="split", stats=st)
    e = kbsrc_b200.resample(x, 44100, 48000, mode="exact")
    f = kbsrc_b200.resample(x, 44100, 48000, mode="fast")
    assert st["isa"] == "sm_100a" and s.shape == e.shape == f.shape
    es, ef = error_stats(s, e), error_stats(f, e)
    print(f"split {es}\nfast  {ef}")
    assert es["max_abs"] <= ef["max_abs"]


def test_split_three_radix_sub_fft():
    """192 kHz -> 44.1 kHz with --len 1.0 --beta 60 and block 3024 (the large multichannel plan): the forward
    transform 967,680 = 960 x 1008 has no sub-FFTs of two radices <= 32, so 1008 runs as 8 x 9 x 14."""
    x = np.random.default_rng(5).uniform(-0.5, 0.5, (192000 * 3, 1))
    es, ef, peak = errors(x, 192000, 44100, length=1.0, beta=60.0, block=3024)
    print(f"split {es:.3e} fast {ef:.3e} peak {peak:.3e}")
    assert es <= ef


@pytest.mark.parametrize("fi,fo,n,ch", CASES[:4])
def test_f16_slices_give_the_int8_bytes(fi, fo, n, ch):
    """The f16 form feeds the same 8-bit digits to kind::f16 MMAs with f32 accumulation; every digit product and
    every accumulator is an integer below 2^24, so the sums are exact there too and the output is the same."""
    x = np.random.default_rng(fi + n).uniform(-0.5, 0.5, (n, ch))
    st = {}
    a = kbsrc_b200.resample(x, fi, fo, mode="split")
    b = kbsrc_b200.resample(x, fi, fo, mode="split16", stats=st)
    assert st["isa"] == "sm_100a"
    assert a.tobytes() == b.tobytes()


def test_f16_slices_full_size_c2():
    x = noise(2, 180, 96000, 2)
    b = kbsrc_b200.resample(x, 96000, 44100, mode="split16")
    e = kbsrc_b200.resample(x, 96000, 44100, mode="exact")
    f = kbsrc_b200.resample(x, 96000, 44100, mode="fast")
    eb, ef = error_stats(b, e), error_stats(f, e)
    print(f"split16 {eb}\nfast    {ef}")
    assert eb["max_abs"] <= ef["max_abs"]


def test_split_runs_twice_the_same():
    x = np.random.default_rng(3).uniform(-0.5, 0.5, (30000, 2))
    cv = kbsrc_b200.Conversion(x, 96000, 44100, mode="split")
    a, b = cv.run(x), cv.run(x)
    assert np.array_equal(a, b)


def test_split_rejects_lengths_without_radix_32_factorisation():
    """22050 -> 48001 needs Bluestein transforms: the split form refuses it with a clear error, no fallback."""
    x = np.random.default_rng(1).uniform(-0.5, 0.5, (3000, 1))
    with pytest.raises(RuntimeError, match="split-precision form"):
        kbsrc_b200.resample(x, 22050, 48001, mode="split")

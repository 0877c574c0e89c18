"""The oracle (oracle/kbsrc_oracle.c) pinned against the reference: its own test pins and the golden fixtures
generated from the reference built from source."""
import hashlib

import numpy as np
import pytest

from oracle import oracle
from cases import CASES, make_input, is_small
import refinputs


def test_input_wavs_match_reference_pins(pins):
    assert refinputs.sha(refinputs.wav_f64(refinputs.primary97())) == pins["primary_wav_sha256"]
    assert refinputs.sha(refinputs.wav_f64(refinputs.subnormal97())) == pins["subnormal_wav_sha256"]


@pytest.mark.parametrize("idx", range(6))
def test_oracle_cli_pins(pins, idx):
    name, rate, mode, want = pins["cli"][idx]
    samples = refinputs.primary97() if name == "primary" else refinputs.subnormal97()
    x = np.array(samples).reshape(-1, 2)
    y = oracle.resample(x, 48000, rate, mode=mode)
    assert refinputs.sha(refinputs.wav_f64_planar(y, rate)) == want


def test_oracle_subnormal_planar_pin(pins):
    a = pins["subnormal_96k_planar_args"]
    x = np.array(refinputs.subnormal97()).reshape(-1, 2)
    y = oracle.resample(x, a["rate_in"], a["rate_out"], length=a["length"], beta=a["beta"])
    assert hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() == pins["subnormal_96k_planar_sha256"]


def test_oracle_frame1_pin(pins):
    a = pins["frame1_args"]
    x = np.array(pins["frame1_in"]).reshape(1, 2)
    y = oracle.resample(x, a["rate_in"], a["rate_out"], length=a["length"], beta=a["beta"])
    got = [v.tobytes()[::-1].hex() for v in y.astype("<f8").ravel()]
    assert got == pins["frame1_out_hex"]


@pytest.mark.parametrize("name", [n for n in CASES if is_small(n)])
def test_oracle_matches_golden(golden, name):
    recipe, fi, fo, opts = CASES[name]
    x = make_input(recipe)
    y = oracle.resample(x, fi, fo, mode=opts.get("mode", "exact"), length=opts.get("length", 0.2),
                        beta=opts.get("beta", 40.0), block=opts.get("block", 0), lpc=opts.get("lpc", True))
    assert list(y.shape) == golden[name]["shape"]
    assert hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() == golden[name]["sha256"]


# paths the benchmark configurations do not reach: Bluestein (non-7-smooth), the general fold (near unity)
EXTRA = [(44100, 44101, False, 3000), (96000, 32001, True, 4000), (1001, 1000, False, 2500), (1000, 1001, True, 2500),
         (48000, 48001, False, 3000)]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built here (oracle/_ref)")
@pytest.mark.parametrize("fi,fo,fast,n", EXTRA)
def test_oracle_matches_reference_build(fi, fo, fast, n):
    x = np.random.default_rng(fi + fo).uniform(-0.5, 0.5, (n, 1))
    a = oracle.resample(x, fi, fo, fast=fast)
    b = oracle.ref_resample(x, fi, fo, fast=fast)
    assert a.tobytes() == b.tobytes()

"""GPU parity: the product (C API -> GPU engine) against the reference's outputs, bit for bit.

Golden fixtures (tests/golden/golden.json) hold SHA-256 hashes of the reference's own output for every case in
cases.py, full benchmark sizes included; small cases are also compared with the oracle directly so a mismatch
reports where and by how much."""
import hashlib

import numpy as np
import pytest

import kbsrc_b200
from oracle import oracle
from cases import CASES, make_input, is_small
import refinputs

pytestmark = pytest.mark.gpu

ORDER = sorted(CASES, key=lambda n: (not is_small(n), n))


def run_case(name):
    recipe, fi, fo, opts = CASES[name]
    x = make_input(recipe)
    st = {}
    y = kbsrc_b200.resample(x, fi, fo, mode=opts.get("mode", "exact"), length=opts.get("length", 0.2),
                            beta=opts.get("beta", 40.0), block=opts.get("block", 0), lpc=opts.get("lpc", True),
                            stats=st)
    return x, y, st


@pytest.mark.parametrize("name", ORDER)
def test_matches_reference_bytes(golden, name):
    x, y, st = run_case(name)
    recipe, fi, fo, opts = CASES[name]
    assert list(y.shape) == golden[name]["shape"]
    if fi != fo and y.size:
        assert st["isa"] == "sm_100a"
    got = hashlib.sha256(y.astype("<f8").tobytes()).hexdigest()
    if got != golden[name]["sha256"] and is_small(name):
        want = oracle.resample(x, fi, fo, mode=opts.get("mode", "exact"), length=opts.get("length", 0.2),
                               beta=opts.get("beta", 40.0), block=opts.get("block", 0), lpc=opts.get("lpc", True))
        bad = np.argwhere(y != want)
        pytest.fail(f"{len(bad)} samples differ, first {bad[:3].tolist()}, max diff {np.abs(y - want).max():.3e}")
    assert got == golden[name]["sha256"]


@pytest.mark.parametrize("idx", range(6))
def test_reference_cli_pins_through_api(pins, idx):
    name, rate, mode, want = pins["cli"][idx]
    samples = refinputs.primary97() if name == "primary" else refinputs.subnormal97()
    y = kbsrc_b200.resample(np.array(samples).reshape(-1, 2), 48000, rate, mode=mode)
    assert refinputs.sha(refinputs.wav_f64_planar(y, rate)) == want


def test_reference_subnormal_planar_pin(pins):
    a = pins["subnormal_96k_planar_args"]
    y = kbsrc_b200.resample(np.array(refinputs.subnormal97()).reshape(-1, 2), a["rate_in"], a["rate_out"],
                            length=a["length"], beta=a["beta"])
    assert hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() == pins["subnormal_96k_planar_sha256"]


def test_reference_frame1_pin(pins):
    a = pins["frame1_args"]
    y = kbsrc_b200.resample(np.array(pins["frame1_in"]).reshape(1, 2), a["rate_in"], a["rate_out"],
                            length=a["length"], beta=a["beta"])
    assert [v.tobytes()[::-1].hex() for v in y.astype("<f8").ravel()] == pins["frame1_out_hex"]


@pytest.mark.parametrize("fi,fo,fast,block,length", [(96000, 44100, False, 0, 0.2), (44100, 48000, True, 0, 0.2),
                                                      (48000, 96000, False, 0, 0.01), (96000, 44100, True, 0, 0.2)])
def test_kernel_spectrum_matches_oracle(fi, fo, fast, block, length):
    frames = 200000
    H = oracle.kernel_spectrum(frames, 2, fi, fo, fast=fast, length=length, block=block)
    p = kbsrc_b200.plan(frames, 2, fi, fo, "fast" if fast else "exact", length, 40.0, block)
    import math
    fk = fo if p["up"] else fi
    mn = min(fi, fo)
    fml = math.sqrt(40.0 ** 2 + 9.8696044010893586) / (2 * 3.14159265358979323846 * length)
    c2 = mn - int(math.ceil(2 * fml))
    g = math.gcd(c2, fk)
    L = int(math.floor(length * fk))
    taps = kbsrc_b200.kernel_taps(L, c2 // g, fk // g, 40.0, threads=4)
    n = p["Mb"] if p["up"] else p["Nb"]
    got = kbsrc_b200.kernel_spectrum(taps, n, float(p["Nb"]))
    assert got.tobytes() == H.tobytes()


def test_conversion_reuse_is_deterministic():
    x = np.random.default_rng(3).uniform(-0.5, 0.5, (50000, 2))
    cv = kbsrc_b200.Conversion(x, 96000, 44100, mode="exact")
    a = cv.run(x).copy()
    b = cv.run(x).copy()
    c = kbsrc_b200.resample(x, 96000, 44100, mode="exact")
    assert a.tobytes() == b.tobytes() == c.tobytes()
    info = cv.engine_info()
    assert info["tasks"] > 0 and info["launches"] > 0
    cv.close()

"""The large multichannel configuration at full size (600 s, 8 channels, 192 kHz -> 44.1 kHz, 24-bit PCM input,
--len 1.0 --beta 60): the CLI's dithered s24 output file and the library's planar output are byte-identical to
the reference's (tests/golden/golden_c5.json, made by make_golden_c5.py from the reference built from source),
and the split-precision form's error against exact is within that of fast."""
import hashlib
import json
import os
import subprocess

import pytest

import kbsrc_b200
from cases import C5, pcm24_ints, pcm24_as_f64, write_pcm24_wav

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden_c5.json")))


def sha_file(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for b in iter(lambda: f.read(1 << 24), b""):
            h.update(b)
    return h.hexdigest()


def test_c5_cli_s24_dither_file(tmp_path):
    src, dst = tmp_path / "in.wav", tmp_path / "out.wav"
    write_pcm24_wav(str(src), pcm24_ints(C5["seed"], C5["seconds"], C5["rate_in"], C5["channels"]), C5["rate_in"])
    assert sha_file(src) == GOLD["input_wav_sha256"]
    r = subprocess.run([kbsrc_b200.CLI, "--rate", str(C5["rate_out"]), "--len", str(C5["length"]), "--beta",
                        str(C5["beta"]), "--format", "s24", "--dither", "-v", str(src), str(dst)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "engine=sm_100a" in r.stderr
    assert sha_file(dst) == GOLD["cli_s24_dither_sha256"]


def test_c5_planar_output():
    x = pcm24_as_f64(pcm24_ints(C5["seed"], C5["seconds"], C5["rate_in"], C5["channels"]))
    st = {}
    y = kbsrc_b200.resample(x, C5["rate_in"], C5["rate_out"], length=C5["length"], beta=C5["beta"], stats=st)
    assert list(y.shape) == GOLD["planar_shape"] and st["isa"] == "sm_100a"
    assert hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() == GOLD["planar_sha256"]


def test_c5_split_error_within_fast_error():
    """The split-precision form on the full configuration: its error against exact is no worse than fast's."""
    import numpy as np
    x = pcm24_as_f64(pcm24_ints(C5["seed"], C5["seconds"], C5["rate_in"], C5["channels"]))
    kw = dict(length=C5["length"], beta=C5["beta"])
    e = kbsrc_b200.resample(x, C5["rate_in"], C5["rate_out"], mode="exact", **kw)
    s = kbsrc_b200.resample(x, C5["rate_in"], C5["rate_out"], mode="split", **kw)
    es = np.abs(s - e).max()
    del s
    f = kbsrc_b200.resample(x, C5["rate_in"], C5["rate_out"], mode="fast", **kw)
    ef = np.abs(f - e).max()
    print(f"split {es:.3e} fast {ef:.3e}")
    assert es <= ef

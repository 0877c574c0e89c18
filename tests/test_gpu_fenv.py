"""The caller's floating-point rounding mode, through the library API (kbsrc::resample) on the GPU engine.

Restates the rounding-mode checks of the reference's own suite (HongYue1/KBSRC tests/test_engines.py:154-216)
with a check program of this repository (tests/fenv_check.cpp, linked against libkbsrc.so): an Exact conversion
gives the round-to-nearest bytes in every caller mode (up, down, toward zero), with 1 and 8 host threads; every
call, a rejected one included, hands the caller's mode back unchanged; Fast and LongDouble leave it alone. The
expected bytes are the reference suite's pins (golden/reference_pins.json) where it pins them, else this build's
own round-to-nearest result."""
import hashlib
import os
import platform
import shutil
import struct
import subprocess

import pytest

import kbsrc_b200
import refinputs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++ to build the check program")]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MODES = ["nearest", "up", "down", "zero"]


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    d = tmp_path_factory.mktemp("fenv")
    exe = d / "fenv_check"
    lib = os.path.dirname(kbsrc_b200.HOST_SO)
    subprocess.run(["g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                    os.path.join(ROOT, "tests", "fenv_check.cpp"), "-L", lib, "-lkbsrc", "-lkbsrc_gpu",
                    f"-Wl,-rpath,{lib}"], check=True)
    return exe, d


def run(checker, name, samples, prec, rate_in, rate_out, length, beta=40, threads=1, ch=2):
    exe, d = checker
    src = d / f"{name}.f64"
    src.write_bytes(struct.pack("<%dd" % len(samples), *samples))
    prefix = d / f"{name}_{prec}_{rate_in}_{rate_out}_{threads}"
    r = subprocess.run([str(exe), prec, str(rate_in), str(rate_out), str(ch), str(length), str(beta), str(threads),
                        str(src), str(prefix)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [dict(kv.split("=", 1) for kv in ln.split()) for ln in r.stdout.split("\n") if ln.startswith("mode=")]
    assert [ln["mode"] for ln in lines] == MODES
    out = {}
    for ln in lines:
        p = f"{prefix}.{ln['mode']}.f64"
        out[ln["mode"]] = (ln, open(p, "rb").read() if ln["threw"] == "0" else None)
    return out


@pytest.mark.skipif(platform.machine().lower() not in ("x86_64", "amd64"), reason="pins are x86-64's")
def test_one_frame_in_every_mode_equals_pin(checker, pins):
    a = pins["frame1_args"]
    res = run(checker, "frame1", pins["frame1_in"], "exact", a["rate_in"], a["rate_out"], a["length"], a["beta"])
    for mode, (info, data) in res.items():
        assert info["kept"] == "1" and info["threw"] == "0", (mode, info)
        assert info["engine"] == "sm_100a"
        got = [data[i:i + 8][::-1].hex() for i in range(0, len(data), 8)]
        assert got == pins["frame1_out_hex"], mode


def test_subnormal_input_in_every_mode_equals_pin(checker, pins):
    a = pins["subnormal_96k_planar_args"]
    res = run(checker, "subnormal", refinputs.subnormal97(), "exact", a["rate_in"], a["rate_out"], a["length"],
              a["beta"])
    for mode, (info, data) in res.items():
        assert info["kept"] == "1", (mode, info)
        assert hashlib.sha256(data).hexdigest() == pins["subnormal_96k_planar_sha256"], mode


@pytest.mark.parametrize("rate_out", [96000, 44100])
def test_normal_input_in_every_mode_equals_nearest(checker, rate_out):
    res = run(checker, "primary", refinputs.primary97(), "exact", 48000, rate_out, 0.1)
    ref = res["nearest"][1]
    assert ref and len(ref) > 0
    for mode, (info, data) in res.items():
        assert info["kept"] == "1", (mode, info)
        assert data == ref, mode


@pytest.mark.parametrize("threads", [1, 8])
def test_worker_threads_in_every_mode_equal_nearest(checker, threads):
    res = run(checker, "primary", refinputs.primary97(), "exact", 48000, 96000, 0.1, threads=threads)
    one = run(checker, "primary", refinputs.primary97(), "exact", 48000, 96000, 0.1, threads=1)["nearest"][1]
    for mode, (info, data) in res.items():
        assert info["kept"] == "1" and data == one, (mode, threads)


def test_rejected_call_keeps_the_callers_mode(checker, pins):
    res = run(checker, "frame1", pins["frame1_in"], "exact", 0, 16000, 0.01)
    for mode, (info, _) in res.items():
        assert info["threw"] == "1" and info["kept"] == "1", (mode, info)


@pytest.mark.parametrize("prec", ["fast", "ld"])
def test_fast_and_long_double_keep_the_callers_mode(checker, pins, prec):
    res = run(checker, "frame1", pins["frame1_in"], prec, 8000, 16000, 0.01)
    for mode, (info, _) in res.items():
        assert info["kept"] == "1" and info["threw"] == "0", (mode, info)

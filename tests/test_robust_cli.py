"""Rejected options and malformed WAV headers fail cleanly; their valid neighbours still convert (on the GPU).

Restates, case for case, the reference suite's robustness checks (HongYue1/KBSRC tests/test_robust.py:136-236)
against this repository's `kbsrc` tool: a rejection exits with status 1, prints "kbsrc: <reason>" with the
reference's reason and writes no output file; an accepted neighbour exits 0 with finite samples and the -v plan line
the reference prints (block, taps, P/Q, threads, engine). Rejections happen before any GPU work and run without a
GPU; conversions are marked gpu."""
import math
import os
import random
import re
import struct
import subprocess

import pytest

import kbsrc_b200

OUT_OF_RANGE = "option out of range"
TOO_LARGE = "block, rates or length too large"
TOO_SHORT = "length too short for these sample rates"
PCM_WIDTH = "unsupported PCM width"
FLOAT_SIZE = "IEEE float sample size does not match the block alignment"
NO_CHUNK = "missing fmt/data chunk"
BAD_CHANNELS = "invalid WAV channel count"
BAD_RATE = "invalid WAV sample rate"
WIDE_FRAME = "too many channels for a WAV file in this format"
FAST_BYTES = "sample rate too high for a WAV file with this many channels"
INPUT_RATE = "input sample rate above 10000000 Hz"
MODES = ["exact", "fast", "ld"]


def wav(tag, ch, rate, bits, align, data):
    """RIFF/WAVE bytes with a 16-byte fmt chunk, header fields written as given (valid or not)."""
    fmt = struct.pack("<HHIIHH", tag, ch, rate, rate * align & 0xFFFFFFFF, align, bits)
    body = b"WAVE" + b"fmt " + struct.pack("<I", len(fmt)) + fmt + b"data" + struct.pack("<I", len(data)) + data
    return b"RIFF" + struct.pack("<I", len(body)) + body


def pcm(width, values):
    if width == 1:
        return bytes(v + 128 for v in values)
    return b"".join((v & (1 << 8 * width) - 1).to_bytes(width, "little") for v in values)


def samples_of(path):
    blob = open(path, "rb").read()
    pos = 12
    while pos + 8 <= len(blob):
        tag, size = blob[pos:pos + 4], struct.unpack("<I", blob[pos + 4:pos + 8])[0]
        if tag == b"data":
            data = blob[pos + 8:pos + 8 + size]
            return struct.unpack("<%dd" % (len(data) // 8), data)
        pos += 8 + size + (size & 1)
    return None


RNG = random.Random(0x524F42)
X = [RNG.uniform(-0.5, 0.5) for _ in range(2 * 64)]
INTS = [RNG.randint(-(1 << 31), (1 << 31) - 1) for _ in range(2 * 64)]
F64 = struct.pack("<%dd" % len(X), *X)


def tool(tmp_path, blob, *opts, env=None, timeout=300):
    src, out = tmp_path / "in.wav", tmp_path / "out.wav"
    src.write_bytes(blob)
    if out.exists():
        out.unlink()
    e = dict(os.environ)
    e.pop("KBSRC_CPU", None)
    e.update(env or {})
    r = subprocess.run([kbsrc_b200.CLI, *map(str, opts), str(src), str(out)], capture_output=True, text=True,
                       env=e, timeout=timeout)
    return r, out


def rejected(tmp_path, reason, blob, *opts):
    r, out = tool(tmp_path, blob, *opts)
    assert r.returncode == 1 and r.stderr.startswith("kbsrc: ") and reason in r.stderr, r.stderr
    assert not out.exists()


def converts(tmp_path, blob, *opts, plan=(), env=None):
    r, out = tool(tmp_path, blob, "-v", *opts, env=env)
    assert r.returncode == 0, r.stderr
    y = samples_of(out)
    assert y and all(map(math.isfinite, y))
    for p in plan:
        assert re.search(r"(^|\s)" + re.escape(p) + r"(\s|$)", r.stderr), (p, r.stderr)
    return y


SRC = wav(3, 2, 48000, 64, 16, F64)


# --block at 48 kHz -> 96 kHz, --len 0.1: the kernel margin is 4802 frames, so blocks up to 9604 leave no hop
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("block", [1, 1000, 9604])
def test_block_without_hop_rejected(tmp_path, mode, block):
    rejected(tmp_path, OUT_OF_RANGE, SRC, "--rate", 96000, "--mode", mode, "--len", "0.1", "--block", block)


@pytest.mark.parametrize("block", [536870912, 2147483647])
def test_block_overflowing_transforms_rejected(tmp_path, block):
    rejected(tmp_path, TOO_LARGE, SRC, "--rate", 96000, "--block", block)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("length,reason", [("1e-5", OUT_OF_RANGE), ("5.3e-4", TOO_SHORT)])
def test_kernel_length_rejected(tmp_path, mode, length, reason):
    rejected(tmp_path, reason, SRC, "--rate", 96000, "--mode", mode, "--len", length)


@pytest.mark.parametrize("length", ["1e-8", "0", "-0.1", "10.5"])
def test_kernel_length_out_of_range(tmp_path, length):
    rejected(tmp_path, OUT_OF_RANGE, SRC, "--rate", 96000, "--len", length)


@pytest.mark.parametrize("opts,reason", [(("--len", "2e-5"), OUT_OF_RANGE), (("--len", "5.79e-4"), TOO_SHORT),
                                         (("--len", "5.8e-4", "--beta", 80), TOO_SHORT)])
def test_downsampling_kernel_length_rejected(tmp_path, opts, reason):
    rejected(tmp_path, reason, SRC, "--rate", 44100, *opts)


@pytest.mark.parametrize("rate", [10000001, 2000000000, 2147483647])
def test_input_rate_above_limit_rejected(tmp_path, rate):
    rejected(tmp_path, INPUT_RATE, wav(3, 2, rate, 64, 16, F64), "--rate", 48000)


@pytest.mark.parametrize("tag,bits,align,reason", [
    (1, 0, 2, PCM_WIDTH), (1, 8, 2, PCM_WIDTH), (1, 17, 2, PCM_WIDTH), (1, 33, 4, PCM_WIDTH), (1, 40, 5, PCM_WIDTH),
    (3, 64, 4, FLOAT_SIZE), (3, 32, 8, FLOAT_SIZE), (3, 32, 2, FLOAT_SIZE), (3, 16, 2, "unsupported WAV format")])
def test_bad_sample_layout_rejected(tmp_path, tag, bits, align, reason):
    rejected(tmp_path, reason, wav(tag, 1, 48000, bits, align, bytes(align * 4096)), "--rate", 96000)


@pytest.mark.parametrize("blob,reason", [
    (wav(3, 0, 48000, 64, 16, F64), BAD_CHANNELS), (wav(3, 2, 0, 64, 16, F64), BAD_RATE),
    (wav(3, 2, 1 << 31, 64, 16, F64), BAD_RATE), (wav(3, 2, (1 << 32) - 1, 64, 16, F64), BAD_RATE),
    (SRC[:12] + SRC[36:], NO_CHUNK)])
def test_bad_header_rejected(tmp_path, blob, reason):
    rejected(tmp_path, reason, blob, "--rate", 96000)


WIDE = wav(1, 8192, 192000, 16, 2 * 8192, bytes(2 * 8192 * 4))


@pytest.mark.parametrize("fmt,reason", [("f64", WIDE_FRAME), ("f32", FAST_BYTES)])
def test_output_header_limits_rejected(tmp_path, fmt, reason):
    rejected(tmp_path, reason, WIDE, "--rate", 192000, "--format", fmt)


def test_wide_s16_output_header(tmp_path):
    """8192 channels of s16 at 192 kHz fit: 16384 bytes per frame (equal rates: the host copy, no GPU)."""
    r, out = tool(tmp_path, WIDE, "--rate", 192000, "--format", "s16")
    assert r.returncode == 0, r.stderr
    assert struct.unpack("<HIIH", out.read_bytes()[22:34]) == (8192, 192000, 192000 * 16384, 16384)


def test_equal_rates_plan_line(tmp_path):
    converts(tmp_path, SRC, "--rate", 48000, plan=["P/Q=1/1", "threads=1", "engine=generic"],
             env={"KBSRC_CPU": "generic"})


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
def test_smallest_block_with_a_hop_converts(tmp_path, mode):
    converts(tmp_path, SRC, "--rate", 96000, "--mode", mode, "--len", "0.1", "--block", 9605,
             plan=["block=9720", "engine=sm_100a"])


@pytest.mark.gpu
@pytest.mark.parametrize("opts,plan", [(("--rate", 96000), ()), (("--rate", 96000, "--len", "0.1", "--block", 20000),
                                                                   ("block=20000",)),
                                       (("--rate", 44100, "--len", "5.8e-4"), ("taps=55",)),
                                       (("--rate", 16000, "--len", 10), ("taps=960001",))])
def test_neighbours_convert(tmp_path, opts, plan):
    converts(tmp_path, SRC, *opts, plan=plan)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
def test_shortest_kernel_converts(tmp_path, mode):
    converts(tmp_path, SRC, "--rate", 96000, "--mode", mode, "--len", "5.33e-4", plan=["taps=103"])


@pytest.mark.gpu
def test_ten_megahertz_input_converts(tmp_path):
    converts(tmp_path, wav(3, 2, 10000000, 64, 16, F64), "--rate", 48000, "--len", "0.001", "--mode", "fast")


@pytest.mark.gpu
@pytest.mark.parametrize("name,tag,bits,width", [("u8", 1, 8, 1), ("s16", 1, 16, 2), ("s24", 1, 24, 3),
                                                 ("s32", 1, 32, 4), ("f32", 3, 32, 4), ("f64", 3, 64, 8)])
def test_every_input_format_converts(tmp_path, name, tag, bits, width):
    if tag == 3:
        data = struct.pack("<%d%s" % (len(X), "f" if width == 4 else "d"), *X)
    else:
        data = pcm(width, [v >> 32 - bits for v in INTS])
    converts(tmp_path, wav(tag, 2, 48000, bits, 2 * width, data), "--rate", 96000)


@pytest.mark.gpu
@pytest.mark.parametrize("bits,width", [(12, 2), (20, 3)])
def test_short_pcm_decodes_like_its_container(tmp_path, bits, width):
    data = pcm(width, [(v >> 32 - bits) << 8 * width - bits for v in INTS])
    full = converts(tmp_path, wav(1, 2, 48000, 8 * width, 2 * width, data), "--rate", 96000)
    part = converts(tmp_path, wav(1, 2, 48000, bits, 2 * width, data), "--rate", 96000)
    assert part == full

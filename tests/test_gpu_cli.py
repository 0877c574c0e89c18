"""The kbsrc command-line tool on the GPU engine: the reference test suite's pinned output files, the -v plan
line, output formats, and byte parity with the reference CLI where it is built (oracle/_ref)."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import kbsrc_b200
from oracle import oracle
import refinputs

pytestmark = pytest.mark.gpu


def cli(*args, binary=None):
    return subprocess.run([binary or kbsrc_b200.CLI, *map(str, args)], capture_output=True, text=True)


@pytest.mark.parametrize("idx", range(6))
def test_cli_reproduces_reference_pins(tmp_path, pins, idx):
    name, rate, mode, want = pins["cli"][idx]
    src = tmp_path / "in.wav"
    src.write_bytes(refinputs.wav_f64(refinputs.primary97() if name == "primary" else refinputs.subnormal97()))
    out = tmp_path / "out.wav"
    r = cli("--rate", rate, "--mode", mode, "-v", src, out)
    assert r.returncode == 0, r.stderr
    assert "engine=sm_100a" in r.stderr
    assert refinputs.sha(out.read_bytes()) == want


def test_verbose_plan_line(tmp_path):
    x = np.random.default_rng(1).uniform(-0.5, 0.5, 2 * 64)
    src = tmp_path / "in.wav"
    src.write_bytes(refinputs.wav_f64(x.tolist()))
    r = cli("--rate", 96000, "--len", "0.1", "--block", 9605, "-v", src, tmp_path / "o.wav")
    assert r.returncode == 0, r.stderr
    assert re.search(r"P/Q=2/1 taps=\d+ block=9720 threads=1 engine=sm_100a", r.stderr)
    assert re.search(r"passband 0-[0-9.]+ Hz, stopband from [0-9.]+ Hz", r.stderr)
    r = cli("--rate", 96000, "--len", "5.33e-4", "-v", src, tmp_path / "o.wav")
    assert r.returncode == 0 and "taps=103" in r.stderr


def read_wav_samples(path):
    blob = open(path, "rb").read()
    pos, fmt = 12, None
    while pos + 8 <= len(blob):
        tag, size = blob[pos:pos + 4], struct.unpack("<I", blob[pos + 4:pos + 8])[0]
        if tag == b"fmt ":
            fmt = struct.unpack("<HHIIHH", blob[pos + 8:pos + 24])
        if tag == b"data":
            return fmt, blob[pos + 8:pos + 8 + size]
        pos += 8 + size + (size & 1)
    raise ValueError("no data chunk")


@pytest.mark.parametrize("fmt,tol", [("f32", 2 ** -24), ("s32", 2 ** -31), ("s24", 2 ** -23), ("s16", 2 ** -15)])
def test_output_formats(tmp_path, fmt, tol):
    t = np.arange(48000) / 48000
    s = 0.5 * np.sin(2 * np.pi * 440 * t)
    src = tmp_path / "in.wav"
    src.write_bytes(refinputs.wav_f64(s.tolist(), ch=1))
    assert cli("--rate", 44100, src, tmp_path / "ref.wav").returncode == 0
    ref = np.frombuffer(read_wav_samples(tmp_path / "ref.wav")[1], "<f8")
    r = cli("--rate", 44100, "--format", fmt, src, tmp_path / "o.wav")
    assert r.returncode == 0, r.stderr
    _, data = read_wav_samples(tmp_path / "o.wav")
    if fmt == "f32":
        y = np.frombuffer(data, "<f4").astype(float)
    else:
        w = {"s32": 4, "s24": 3, "s16": 2}[fmt]
        raw = np.frombuffer(data, np.uint8).reshape(-1, w).astype(np.int64)
        v = sum(raw[:, i] << (8 * i) for i in range(w))
        v = np.where(v >= 1 << (8 * w - 1), v - (1 << (8 * w)), v)
        y = v / 2.0 ** (8 * w - 1)
    assert np.abs(y - ref).max() <= tol


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
@pytest.mark.parametrize("args", [["--rate", 44100, "--format", "s24", "--dither"],
                                  ["--rate", 44100, "--format", "s16"],
                                  ["--rate", 96000, "--format", "f32", "--mode", "fast"],
                                  ["--rate", 22050, "--format", "s32", "--dither", "--no-lpc"]])
def test_cli_bytes_equal_reference_cli(tmp_path, args):
    x = np.random.default_rng(9).uniform(-0.9, 0.9, (20000, 2))
    src = tmp_path / "in.wav"
    src.write_bytes(refinputs.wav_f64(x.ravel().tolist(), ch=2, rate=48000))
    a, b = tmp_path / "a.wav", tmp_path / "b.wav"
    ra = cli(*args, src, a)
    rb = cli(*args, src, b, binary=oracle.REF_CLI)
    assert ra.returncode == rb.returncode == 0, (ra.stderr, rb.stderr)
    assert a.read_bytes() == b.read_bytes()


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
@pytest.mark.parametrize("fmt", ["s16", "s24", "s32", "f32", "f64"])
@pytest.mark.parametrize("dither", [False, True])
def test_gpu_pack_equals_reference_writer(tmp_path, fmt, dither):
    """The GPU output step against the reference's writer: equal rates make the reference CLI write the input
    samples themselves, so its data section is the packing of exactly these samples (values beyond +-1 clip)."""
    x = np.random.default_rng(4).uniform(-1.2, 1.2, (7001, 3))
    x[5, 1] = np.nan
    src = tmp_path / "in.wav"
    from test_host import wav
    src.write_bytes(wav(3, 3, 48000, 64, 24, x.astype("<f8").tobytes()))
    ref = tmp_path / "ref.wav"
    r = subprocess.run([oracle.REF_CLI, str(src), str(ref), "--rate", "48000", "--format", fmt] +
                       (["--dither"] if dither else []), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    _, want = read_wav_samples(ref)
    got, clipped = kbsrc_b200.pack(x.T, fmt, dither)
    assert got == want
    m = re.search(r"warning: (\d+) samples clipped", r.stderr)
    assert clipped == (int(m.group(1)) if m else 0)


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
@pytest.mark.parametrize("frames,ch", [(524288, 2), (524289, 1), (700001, 3)])
def test_gpu_dither_across_chunks_equals_reference_writer(tmp_path, frames, ch):
    """The dither stream is generated in chunks of 2^20 draws (2^19 samples) whose start states come from a
    jump-ahead tree; samples on both sides of every chunk boundary match the reference's sequential generator.
    The sizes end exactly on a boundary, one sample past it, and inside a fifth chunk."""
    x = np.random.default_rng(frames).uniform(-0.99, 0.99, (frames, ch))
    src = tmp_path / "in.wav"
    from test_host import wav
    src.write_bytes(wav(3, ch, 48000, 64, 8 * ch, x.astype("<f8").tobytes()))
    ref = tmp_path / "ref.wav"
    r = subprocess.run([oracle.REF_CLI, str(src), str(ref), "--rate", "48000", "--format", "s24", "--dither"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    _, want = read_wav_samples(ref)
    got, _ = kbsrc_b200.pack(x.T, "s24", True)
    assert got == want


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
def test_cli_dither_across_chunks_equals_reference_cli(tmp_path):
    """A conversion whose dithered output spans several generator chunks (2.65 M samples): the CLI's file equals
    the reference CLI's byte for byte."""
    x = np.random.default_rng(17).uniform(-0.9, 0.9, (48000 * 30, 2))
    src = tmp_path / "in.wav"
    src.write_bytes(refinputs.wav_f64(x.ravel().tolist(), ch=2, rate=48000))
    a, b = tmp_path / "a.wav", tmp_path / "b.wav"
    args = ["--rate", 44100, "--format", "s16", "--dither"]
    ra = cli(*args, src, a)
    rb = cli(*args, src, b, binary=oracle.REF_CLI)
    assert ra.returncode == rb.returncode == 0, (ra.stderr, rb.stderr)
    assert a.read_bytes() == b.read_bytes()


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
@pytest.mark.parametrize("tag,bits,width", [(1, 8, 1), (1, 16, 2), (1, 20, 3), (1, 24, 3), (1, 32, 4), (3, 32, 4),
                                            (3, 64, 8)])
def test_cli_input_formats_equal_reference_cli(tmp_path, tag, bits, width):
    """The GPU decodes the WAV data section itself (the CLI hands it over as stored): every input sample format
    gives the reference CLI's output bytes."""
    from test_host import wav
    rng = np.random.default_rng(bits + width)
    n, ch = 30000, 3
    if tag == 3:
        data = rng.uniform(-0.9, 0.9, n * ch).astype("<f4" if width == 4 else "<f8").tobytes()
    else:
        v = rng.integers(0, 256, (n * ch, width), dtype=np.uint8)
        data = v.tobytes()
    src = tmp_path / "in.wav"
    src.write_bytes(wav(tag, ch, 48000, bits, ch * width, data))
    a, b = tmp_path / "a.wav", tmp_path / "b.wav"
    args = ["--rate", 44100, "--format", "s24", "--dither"]
    ra = cli(*args, src, a)
    rb = cli(*args, src, b, binary=oracle.REF_CLI)
    assert ra.returncode == rb.returncode == 0, (ra.stderr, rb.stderr)
    assert a.read_bytes() == b.read_bytes()


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
@pytest.mark.parametrize("frames", [0, 1, 2, 97])
@pytest.mark.parametrize("tag,bits,width", [(1, 24, 3), (1, 16, 2), (3, 64, 8)])
def test_cli_tiny_files_equal_reference_cli(tmp_path, frames, tag, bits, width):
    """Empty and tiny data sections through the raw-input path give the reference CLI's bytes."""
    from test_host import wav
    rng = np.random.default_rng(frames + bits)
    ch = 2
    if tag == 3:
        data = rng.uniform(-0.9, 0.9, frames * ch).astype("<f8").tobytes()
    else:
        data = rng.integers(0, 256, (frames * ch, width), dtype=np.uint8).tobytes()
    src = tmp_path / "in.wav"
    src.write_bytes(wav(tag, ch, 48000, bits, ch * width, data))
    a, b = tmp_path / "a.wav", tmp_path / "b.wav"
    args = ["--rate", 44100, "--format", "s16", "--dither"]
    ra = cli(*args, src, a)
    rb = cli(*args, src, b, binary=oracle.REF_CLI)
    assert ra.returncode == rb.returncode, (ra.stderr, rb.stderr)
    if rb.returncode == 0:
        assert a.read_bytes() == b.read_bytes()

"""Host-side logic of the product without a GPU: libraries load and export the C ABI, planning, Kaiser taps and
Burg LPC match the oracle bit for bit, and the command-line tool rejects bad usage and arguments like the
reference (exit status, message, no output file)."""
import os
import re
import struct
import subprocess

import numpy as np
import pytest

import kbsrc_b200
from oracle import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(kbsrc_\w+)\s*\(", text))


def test_gpu_library_exports_every_declared_symbol():
    lib = kbsrc_b200.gpu_lib()
    names = declared_functions("kbsrc_gpu.h")
    assert names and names <= set(kbsrc_b200.GPU_SYMBOLS)
    for n in names:
        assert hasattr(lib, n), n


def test_host_library_exports_every_declared_symbol():
    lib = kbsrc_b200.host_lib()
    names = declared_functions(os.path.join("kbsrc", "kbsrc_c.h"))
    assert names and names <= set(kbsrc_b200.HOST_SYMBOLS)
    for n in names:
        assert hasattr(lib, n), n


def test_engine_name_and_version():
    assert kbsrc_b200.gpu_lib().kbsrc_gpu_engine_name() == b"sm_100a"
    assert kbsrc_b200.host_lib().kbsrc_version_c().startswith(b"1.3.0")


PLANS = [(960000, 2, 96000, 44100, "exact", 0.2, 40, 0), (17280000, 2, 96000, 44100, "exact", 0.2, 40, 0),
         (17280000, 2, 96000, 44100, "fast", 0.2, 40, 0), (97, 2, 48000, 96000, "exact", 0.2, 40, 0),
         (1, 2, 8000, 16000, "exact", 0.01, 40, 0), (30000, 3, 44100, 48000, "fast", 0.2, 40, 0),
         (115200000, 8, 192000, 44100, "exact", 1.0, 60, 0), (20000, 1, 44100, 48000, "exact", 0.2, 40, 700),
         (64, 2, 48000, 96000, "exact", 0.1, 40, 9605), (0, 1, 48000, 44100, "exact", 0.2, 40, 0),
         (5000, 1, 44100, 44101, "exact", 0.2, 40, 0), (3000, 6, 22050, 48000, "fast", 0.02, 40, 0)]


@pytest.mark.parametrize("frames,ch,fi,fo,mode,length,beta,block", PLANS)
def test_plan_matches_oracle(frames, ch, fi, fo, mode, length, beta, block):
    p = kbsrc_b200.plan(frames, ch, fi, fo, mode, length, beta, block)
    q = oracle.plan(frames, ch, fi, fo, fast=mode == "fast", length=length, beta=beta, block=block)
    for k in ("P", "Q", "taps", "nb", "marg", "hop", "nblk", "Nb", "Mb", "pre", "o", "E", "up", "nout"):
        assert p[k] == q[k], k
    assert p["general"] == q["gen"]


@pytest.mark.parametrize("args,msg", [
    ((100, 2, 0, 44100, "exact", 0.2, 40, 0), "sample rates must be positive"),
    ((100, 2, 48000, 96000, "exact", 0.1, 40, 9604), "option out of range"),
    ((100, 2, 48000, 96000, "exact", 1e-5, 40, 0), "option out of range"),
    ((100, 2, 48000, 96000, "exact", 5.3e-4, 40, 0), "length too short for these sample rates"),
    ((100, 2, 48000, 96000, "exact", 0.2, 40, 536870912), "block, rates or length too large"),
    ((100, 2, 48000, 96000, "exact", 10.5, 40, 0), "option out of range"),
    ((100, 0, 48000, 96000, "exact", 0.2, 40, 0), "bad input buffer"),
])
def test_plan_rejections(args, msg):
    with pytest.raises(ValueError, match=msg):
        kbsrc_b200.plan(*args)


def test_kernel_taps_match_oracle_pieces():
    # taps enter the spectrum; compare through the oracle's design of the same plan: H = rfft(taps) / Nb, so
    # equal taps are checked via the GPU test; here the tap values against a direct dd restatement
    h = kbsrc_b200.kernel_taps(200, 21, 40, 40.0, threads=3)
    h1 = kbsrc_b200.kernel_taps(200, 21, 40, 40.0, threads=1)
    assert h.tobytes() == h1.tobytes()  # independent of the thread count
    assert h[0, 0] == pytest.approx(21 / 40, rel=1e-15)


@pytest.mark.parametrize("seed,n", [(1, 5000), (2, 4096), (3, 100), (4, 60)])
def test_burg_matches_oracle(seed, n):
    x = np.random.default_rng(seed).standard_normal(n).cumsum() * 1e-3
    a = kbsrc_b200.burg(x, 1000)
    b = oracle.burg(x, 1000)
    assert a.tobytes() == b.tobytes()


def cli(*args):
    return subprocess.run([kbsrc_b200.CLI, *map(str, args)], capture_output=True, text=True)


def wav(tag, ch, rate, bits, align, data):
    fmt = struct.pack("<HHIIHH", tag, ch, rate, rate * align & 0xFFFFFFFF, align, bits)
    body = b"WAVE" + b"fmt " + struct.pack("<I", len(fmt)) + fmt + b"data" + struct.pack("<I", len(data)) + data
    return b"RIFF" + struct.pack("<I", len(body)) + body


@pytest.fixture
def src(tmp_path):
    x = np.random.default_rng(0).uniform(-0.5, 0.5, 128)
    p = tmp_path / "in.wav"
    p.write_bytes(wav(3, 2, 48000, 64, 16, x.astype("<f8").tobytes()))
    return p


@pytest.mark.parametrize("extra,code,msg", [
    (["--rate", "0"], 2, "--rate must be between"), (["--rate", "abc"], 2, "invalid value for --rate"),
    (["--mode", "nope"], 2, "mode must be"), (["--format", "x"], 2, "format must be"),
    (["--len", "-1"], 1, "option out of range"), (["--block", "9604", "--len", "0.1", "--rate", "96000"], 1,
                                                 "option out of range"),
    (["--len", "5.3e-4", "--rate", "96000"], 1, "length too short"),
    (["--block", "2147483647", "--rate", "96000"], 1, "block, rates or length too large"),
])
def test_cli_rejections(tmp_path, src, extra, code, msg):
    out = tmp_path / "o.wav"
    r = cli(src, out, *extra)
    assert r.returncode == code and r.stderr.startswith("kbsrc: ") and msg in r.stderr, r.stderr
    assert not out.exists()


def test_cli_missing_and_bad_files(tmp_path):
    r = cli(tmp_path / "missing.wav", tmp_path / "o.wav")
    assert r.returncode == 1 and "cannot open input" in r.stderr
    bad = tmp_path / "bad.wav"
    bad.write_bytes(wav(1, 1, 48000, 0, 2, bytes(64)))
    r = cli(bad, tmp_path / "o.wav", "--rate", 96000)
    assert r.returncode == 1 and "unsupported PCM width" in r.stderr
    r = cli(tmp_path / "only_one.wav")
    assert r.returncode == 2


def test_cli_equal_rates_copy_without_gpu(tmp_path, src):
    out = tmp_path / "o.wav"
    r = cli(src, out, "--rate", 48000, "-v")
    assert r.returncode == 0, r.stderr
    assert "P/Q=1/1" in r.stderr and "threads=1" in r.stderr and "engine=generic" in r.stderr
    data = out.read_bytes()
    x = np.frombuffer(src.read_bytes()[-1024:], "<f8")
    assert np.frombuffer(data[-1024:], "<f8").tobytes() == x.tobytes()


@pytest.mark.skipif(not os.path.exists(oracle.REF_CLI), reason="reference CLI not built (oracle/_ref)")
@pytest.mark.parametrize("fmt", ["s16", "s24", "s32", "f32", "f64"])
@pytest.mark.parametrize("dither", [False, True])
def test_wav_writer_bytes_equal_reference_cli(tmp_path, fmt, dither):
    """Equal rates take the host copy path, so the writer (scaling, TPDF dither from mt19937_64(12345), rounding,
    clipping, header) is compared with the reference CLI without a GPU."""
    x = np.random.default_rng(3).uniform(-1.2, 1.2, (5000, 3))
    src = tmp_path / "in.wav"
    src.write_bytes(wav(3, 3, 48000, 64, 24, x.astype("<f8").tobytes()))
    extra = ["--dither"] if dither else []
    a, b = tmp_path / "a.wav", tmp_path / "b.wav"
    ra = cli(src, a, "--rate", 48000, "--format", fmt, *extra)
    rb = subprocess.run([oracle.REF_CLI, str(src), str(b), "--rate", "48000", "--format", fmt, *extra],
                        capture_output=True, text=True)
    assert ra.returncode == rb.returncode == 0, (ra.stderr, rb.stderr)
    assert ra.stderr == rb.stderr  # the clipped-samples warning
    assert a.read_bytes() == b.read_bytes()


def test_gpu_path_fails_loudly_without_a_device():
    """No silent CPU fallback: with no usable CUDA device a conversion raises with the runtime's reason."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        kbsrc_b200.resample(np.zeros((1000, 1)), 48000, 44100)
    rc = kbsrc_b200.gpu_lib().kbsrc_gpu_kernel_spectrum(np.zeros(4).ctypes.data_as(kbsrc_b200._dp), 1, 8, 1.0,
                                                        np.zeros(10).ctypes.data_as(kbsrc_b200._dp))
    assert rc == kbsrc_b200.GPU_E_NODEVICE


def test_c_abi_rejects_bad_descriptors():
    d = kbsrc_b200.GpuDesc()
    e = ctypes_void_p()
    assert kbsrc_b200.gpu_lib().kbsrc_gpu_engine_create(None, e) == kbsrc_b200.GPU_E_ARG
    d.precision, d.channels, d.P, d.Q, d.nb, d.marg = 7, 1, 1, 2, 10, 2
    assert kbsrc_b200.gpu_lib().kbsrc_gpu_engine_create(d, e) == kbsrc_b200.GPU_E_ARG
    assert "precision" in kbsrc_b200.gpu_error()
    d.precision, d.nb = 1, 3  # odd block
    assert kbsrc_b200.gpu_lib().kbsrc_gpu_engine_create(d, e) == kbsrc_b200.GPU_E_ARG


def ctypes_void_p():
    import ctypes
    return ctypes.c_void_p()


def test_two_rank_reference_bench_on_cpu():
    """bench.py under torchrun with 2 gloo ranks: rank 0 alone runs the reference arm and prints one JSON line,
    the other rank exits cleanly (the launch the driver uses for N > 1)."""
    from oracle import oracle
    if not oracle.ref_available():
        pytest.skip("reference not built (oracle/_ref)")
    import json
    import sys
    r = subprocess.run([sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
                        "--master-addr", "127.0.0.1", "--master-port", "29517", os.path.join(ROOT, "bench.py"),
                        "--impl", "reference", "--gpus", "2", "--workload", "c1_exact", "--steps", "1", "--warmup",
                        "0"], capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["n_gpus"] == 2


@pytest.mark.parametrize("n,split,radices", [
    (100800, (315, 320), [(15, 21), (16, 20)]),   # C2 forward: two radices per sub-FFT
    (46305, (147, 315), [(7, 21), (15, 21)]),     # C2 inverse
    (222264, (441, 504), [(21, 21), (21, 24)]),   # C5 inverse
    (967680, (960, 1008), [(30, 32), (8, 9, 14)]),  # C5 forward: no four-radix split, so 1008 takes three
])
def test_split_form_plans(n, split, radices):
    """The split form's transform plans (the Python model of make_tc_fft, which bench.py uses to count the
    tensor-core work): four radices <= 32 where any split allows them, else a three-radix sub-FFT whose every
    stage has at most 128 rows."""
    from kbsrc_b200 import roofline
    assert roofline.tc_split(n) == split
    got = [roofline.tc_radices(N) for N in split]
    assert got == radices
    for N, rads in zip(split, got):
        assert all(r <= 32 for r in rads) and N // min(rads) <= 128


def test_split_form_rejects_large_prime_factors():
    from kbsrc_b200 import roofline
    assert roofline.tc_split(2 * 2087 * 9) is None

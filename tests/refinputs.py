"""The reference test suite's seeded inputs (HongYue1/KBSRC tests/test_engines.py:93-115), rebuilt here so the
pinned hashes in golden/reference_pins.json can be checked: 97 stereo frames of dyadic values and of subnormal
values, written as 64-bit float WAV files with an 18-byte fmt chunk and a fact chunk."""
import hashlib
import math
import random
import struct


def primary97():
    rng = random.Random(0x4B42535243)
    return [rng.randint(-1048576, 1048576) / 1048576 for _ in range(194)]


def subnormal97():
    rng = random.Random(12345)
    return [math.ldexp(rng.randint(-1024, 1024) / 1024, -1024) for _ in range(194)]


def wav_f64(samples, ch=2, rate=48000):
    data = struct.pack("<%dd" % len(samples), *samples)
    fmt = struct.pack("<HHIIHHH", 3, ch, rate, rate * 8 * ch, 8 * ch, 64, 0)
    body = (b"WAVE" + b"fmt " + struct.pack("<I", len(fmt)) + fmt + b"fact" +
            struct.pack("<II", 4, len(samples) // ch) + b"data" + struct.pack("<I", len(data)) + data)
    return b"RIFF" + struct.pack("<I", len(body)) + body


def wav_f64_planar(planar, rate):
    """The kbsrc CLI's f64 output file (1 or 2 channels) for planar samples (channels, frames)."""
    import numpy as np
    ch = planar.shape[0]
    inter = np.ascontiguousarray(planar.T).astype("<f8").ravel().tolist()
    return wav_f64(inter, ch=ch, rate=rate)


def sha(b):
    return hashlib.sha256(b).hexdigest()

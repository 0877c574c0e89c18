"""Seeded synthetic inputs and the parity case list shared by the golden-fixture generator and the tests.

The workloads stand in for the configurations the engine is measured on (uniform noise in [-0.5, 0.5) from
numpy's default_rng, a log sine sweep); no external data is involved.
"""
import numpy as np


def noise(seed, seconds, rate, channels):
    """i.i.d. uniform [-0.5, 0.5) f64 samples, (frames, channels), from default_rng(seed)."""
    return np.random.default_rng(seed).uniform(-0.5, 0.5, (int(round(seconds * rate)), channels))


def sweep(seconds, rate, channels=2, f0=20.0, f1=20000.0, amp=0.5):
    """Log sine sweep f0 -> f1 Hz over `seconds`, the same on every channel."""
    T = float(seconds)
    t = np.arange(int(round(seconds * rate))) / rate
    k = np.log(f1 / f0)
    x = amp * np.sin(2 * np.pi * f0 * T / k * (np.exp(t / T * k) - 1))
    return np.repeat(x[:, None], channels, axis=1)


# name -> (input recipe, rate_in, rate_out, options). Recipes: ("noise", seed, seconds, rate, ch),
# ("sweep", seconds, rate, ch), ("frames", seed, frames, ch).
CASES = {
    # configurations of the benchmark
    "c1_96k_44k1_exact": (("noise", 1, 10, 96000, 2), 96000, 44100, {"mode": "exact"}),
    "c2_96k_44k1_exact": (("noise", 2, 180, 96000, 2), 96000, 44100, {"mode": "exact"}),
    "c2_96k_44k1_fast": (("noise", 2, 180, 96000, 2), 96000, 44100, {"mode": "fast"}),
    "c3_sweep_44k1_48k_exact": (("sweep", 60, 44100, 2), 44100, 48000, {"mode": "exact"}),
    "c3_sweep_44k1_48k_fast": (("sweep", 60, 44100, 2), 44100, 48000, {"mode": "fast"}),
    # small cases: down/up, both modes, direct and four-step transforms, options, channel counts, edges
    "s_48k_96k_exact_97": (("frames", 11, 97, 2), 48000, 96000, {"mode": "exact"}),
    "s_48k_96k_fast_97": (("frames", 11, 97, 2), 48000, 96000, {"mode": "fast"}),
    "s_48k_44k1_exact_97": (("frames", 12, 97, 2), 48000, 44100, {"mode": "exact"}),
    "s_48k_44k1_fast_97": (("frames", 12, 97, 2), 48000, 44100, {"mode": "fast"}),
    "s_8k_16k_exact_1_len001": (("frames", 13, 1, 2), 8000, 16000, {"mode": "exact", "length": 0.01}),
    "s_8k_16k_fast_50_len001": (("frames", 13, 50, 1), 8000, 16000, {"mode": "fast", "length": 0.01}),
    "s_16k_8k_exact_300_len001": (("frames", 14, 300, 1), 16000, 8000, {"mode": "exact", "length": 0.01}),
    "s_96k_44k1_exact_20000": (("frames", 15, 20000, 2), 96000, 44100, {"mode": "exact"}),
    "s_96k_44k1_fast_20000": (("frames", 15, 20000, 2), 96000, 44100, {"mode": "fast"}),
    "s_44k1_48k_exact_30000": (("frames", 16, 30000, 1), 44100, 48000, {"mode": "exact"}),
    "s_44k1_48k_fast_30000": (("frames", 16, 30000, 3), 44100, 48000, {"mode": "fast"}),
    "s_192k_44k1_exact_40000": (("frames", 17, 40000, 2), 192000, 44100, {"mode": "exact"}),
    "s_44k1_96k_exact_10000": (("frames", 18, 10000, 2), 44100, 96000, {"mode": "exact"}),
    "s_44k1_8k_fast_20000": (("frames", 19, 20000, 1), 44100, 8000, {"mode": "fast"}),
    "s_8k_44k1_exact_3000": (("frames", 20, 3000, 1), 8000, 44100, {"mode": "exact"}),
    "s_48k_192k_fast_5000": (("frames", 21, 5000, 2), 48000, 192000, {"mode": "fast"}),
    "s_96k_48k_exact_nolpc": (("frames", 22, 15000, 2), 96000, 48000, {"mode": "exact", "lpc": False}),
    "s_44k1_48k_exact_block": (("frames", 23, 20000, 1), 44100, 48000, {"mode": "exact", "block": 700}),
    "s_96k_44k1_exact_len05_beta60": (("frames", 24, 30000, 1), 96000, 44100,
                                      {"mode": "exact", "length": 0.05, "beta": 60.0}),
    "s_48k_96k_exact_6ch": (("frames", 25, 4000, 6), 48000, 96000, {"mode": "exact"}),
    "s_48k_44k1_exact_10frames": (("frames", 26, 10, 1), 48000, 44100, {"mode": "exact"}),
    "s_48k_44k1_exact_empty": (("frames", 27, 0, 1), 48000, 44100, {"mode": "exact"}),
    "s_22k05_48k_fast_len002": (("frames", 28, 3000, 1), 22050, 48000, {"mode": "fast", "length": 0.02}),
    # near-unity ratios (general fold) and transform lengths that are not 7-smooth (Bluestein)
    "s_44k1_44k101_exact": (("frames", 29, 3000, 1), 44100, 44101, {"mode": "exact"}),
    "s_44k101_44k1_fast": (("frames", 30, 3000, 2), 44101, 44100, {"mode": "fast"}),
    "s_1001_1000_exact": (("frames", 31, 2500, 1), 1001, 1000, {"mode": "exact"}),
    "s_1000_1001_fast": (("frames", 32, 2500, 1), 1000, 1001, {"mode": "fast"}),
    "s_48k_48k001_exact": (("frames", 33, 3000, 1), 48000, 48001, {"mode": "exact"}),
    "s_96k_32k001_exact": (("frames", 34, 4000, 1), 96000, 32001, {"mode": "exact"}),
    "s_96k_32k001_fast": (("frames", 35, 4000, 2), 96000, 32001, {"mode": "fast"}),
    "s_22k05_48k001_exact": (("frames", 36, 3000, 1), 22050, 48001, {"mode": "exact"}),
    # Precision::LongDouble (x87 extended): the same paths in the third arithmetic
    "s_48k_96k_ld_97": (("frames", 11, 97, 2), 48000, 96000, {"mode": "ld"}),
    "s_48k_44k1_ld_97": (("frames", 12, 97, 2), 48000, 44100, {"mode": "ld"}),
    "s_8k_16k_ld_1_len001": (("frames", 13, 1, 2), 8000, 16000, {"mode": "ld", "length": 0.01}),
    "s_96k_44k1_ld_20000": (("frames", 15, 20000, 2), 96000, 44100, {"mode": "ld"}),
    "s_44k1_48k_ld_30000": (("frames", 16, 30000, 1), 44100, 48000, {"mode": "ld"}),
    "s_96k_48k_ld_nolpc": (("frames", 22, 15000, 2), 96000, 48000, {"mode": "ld", "lpc": False}),
    "s_48k_44k1_ld_empty": (("frames", 27, 0, 1), 48000, 44100, {"mode": "ld"}),
    "s_44k1_44k101_ld": (("frames", 29, 3000, 1), 44100, 44101, {"mode": "ld"}),
    "s_22k05_48k001_ld": (("frames", 36, 3000, 1), 22050, 48001, {"mode": "ld"}),
    "c1_96k_44k1_ld": (("noise", 1, 10, 96000, 2), 96000, 44100, {"mode": "ld"}),
}


def make_input(recipe):
    kind = recipe[0]
    if kind == "noise":
        _, seed, seconds, rate, ch = recipe
        return noise(seed, seconds, rate, ch)
    if kind == "sweep":
        _, seconds, rate, ch = recipe
        return sweep(seconds, rate, ch)
    _, seed, frames, ch = recipe
    return np.random.default_rng(seed).uniform(-0.5, 0.5, (frames, ch))


def is_small(name):
    return name.startswith("s_")


# The uneven multi-file queue: for file i of `count`, length uniform in [min_s, max_s] seconds (whole frames),
# 1-8 channels, an input rate from C4_RATES_IN and an output rate from C4_RATES_OUT, all drawn from
# default_rng(seed); samples normal(0, 0.2) from default_rng([seed, i]), clipped to +-1 and rounded to float32
# (the files are 32-bit float WAVs).
C4_RATES_IN = [44100, 48000, 88200, 96000, 192000]
C4_RATES_OUT = [44100, 48000, 96000]


def c4_specs(seed=3, count=256, min_s=1.0, max_s=60.0):
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(count):
        sec = rng.uniform(min_s, max_s)
        ch = int(rng.integers(1, 9))
        fi = int(rng.choice(C4_RATES_IN))
        fo = int(rng.choice(C4_RATES_OUT))
        specs.append((int(round(sec * fi)), ch, fi, fo))
    return specs


def c4_samples(seed, i, frames, ch):
    x = np.random.default_rng([seed, i]).normal(0.0, 0.2, (frames, ch))
    return np.clip(x, -1.0, 1.0).astype(np.float32).astype(np.float64)


# the scaled-down queue of the parity tests: 48 files of 0.2-3 s
C4_SMALL = dict(seed=3, count=48, min_s=0.2, max_s=3.0)


# The large multichannel configuration: 600 s of 8-channel 192 kHz 24-bit PCM, uniform integers in
# [-2^23, 2^23) from default_rng(4), converted to 44.1 kHz with --len 1.0 --beta 60, s24 output with TPDF dither.
C5 = dict(seed=4, seconds=600, rate_in=192000, rate_out=44100, channels=8, length=1.0, beta=60.0)


def pcm24_ints(seed, seconds, rate, ch):
    """The 24-bit sample values (frames x channels, int32)."""
    return np.random.default_rng(seed).integers(-2 ** 23, 2 ** 23, (int(seconds * rate), ch)).astype(np.int32)


def write_pcm24_wav(path, ints, rate):
    """A 24-bit PCM WAV file (16-byte fmt chunk) of the int32 samples, written in slices of frames."""
    import struct
    frames, ch = ints.shape
    data_len = frames * ch * 3
    with open(path, "wb") as f:
        f.write(b"RIFF" + struct.pack("<I", 36 + data_len) + b"WAVE" + b"fmt " + struct.pack("<I", 16) +
                struct.pack("<HHIIHH", 1, ch, rate, rate * ch * 3, ch * 3, 24) + b"data" + struct.pack("<I", data_len))
        step = 1 << 20
        for f0 in range(0, frames, step):
            b = ints[f0:f0 + step].astype("<i4").view(np.uint8).reshape(-1, 4)[:, :3]
            f.write(np.ascontiguousarray(b).tobytes())


def pcm24_as_f64(ints):
    """The values the WAV reader delivers: v / 2^23."""
    return ints.astype(np.float64) / 8388608.0

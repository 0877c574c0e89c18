"""Writes tests/golden/golden_c5.json: the reference's output for the large multichannel configuration (600 s,
8 channels, 192 kHz -> 44.1 kHz, 24-bit PCM input, --len 1.0 --beta 60, exact).

  * cli_s24_dither_sha256: the output WAV of the reference tool, `kbsrc --rate 44100 --len 1.0 --beta 60
    --format s24 --dither in.wav out.wav` (oracle/_ref/kbsrc, built from the reference's sources);
  * planar_sha256: the planar float64 output of the reference library's kbsrc::resample (exact).

Run here, where the reference tree exists (about 20 GB of memory and 4 GB of scratch disk):
    make -C oracle && python tests/golden/make_golden_c5.py
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import C5, pcm24_ints, write_pcm24_wav, pcm24_as_f64  # noqa: E402
from oracle import oracle  # noqa: E402


def sha_file(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for b in iter(lambda: f.read(1 << 24), b""):
            h.update(b)
    return h.hexdigest()


def main():
    c = C5
    ints = pcm24_ints(c["seed"], c["seconds"], c["rate_in"], c["channels"])
    out = {"config": c}
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "in.wav"), os.path.join(d, "out.wav")
        write_pcm24_wav(src, ints, c["rate_in"])
        out["input_wav_sha256"] = sha_file(src)
        t = time.time()
        r = subprocess.run([oracle.REF_CLI, "--rate", str(c["rate_out"]), "--len", str(c["length"]), "--beta",
                            str(c["beta"]), "--format", "s24", "--dither", "-v", src, dst], capture_output=True,
                           text=True)
        assert r.returncode == 0, r.stderr
        out["cli_s24_dither_sha256"] = sha_file(dst)
        out["cli_seconds"] = round(time.time() - t, 1)
        out["cli_verbose"] = r.stderr.strip().splitlines()
        print(out["cli_verbose"], flush=True)
    x = pcm24_as_f64(ints)
    del ints
    y = oracle.ref_resample(x, c["rate_in"], c["rate_out"], length=c["length"], beta=c["beta"])
    out["planar_sha256"] = hashlib.sha256(y.astype("<f8").tobytes()).hexdigest()
    out["planar_shape"] = list(y.shape)
    with open(os.path.join(HERE, "golden_c5.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(out["planar_shape"], out["cli_s24_dither_sha256"][:16], out["planar_sha256"][:16])


if __name__ == "__main__":
    main()

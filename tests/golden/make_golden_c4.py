"""Writes tests/golden/golden_c4.json: SHA-256 of the reference's exact output for each of the 256 files of the
full uneven queue (cases.c4_specs() with the default arguments), one file at a time.

The outputs come from HongYue1/KBSRC built from source (oracle/_ref). Run here, where the reference tree exists:
    make -C oracle && python tests/golden/make_golden_c4.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import c4_samples, c4_specs  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    files = []
    for i, (frames, ch, fi, fo) in enumerate(c4_specs()):
        x = c4_samples(3, i, frames, ch)
        y = oracle.ref_resample(x, fi, fo).astype("<f8", copy=False)
        files.append({"spec": [frames, ch, fi, fo], "sha256": hashlib.sha256(y.tobytes()).hexdigest(),
                      "shape": list(y.shape)})
        print(i, frames, ch, fi, fo, files[-1]["sha256"][:16], flush=True)
    with open(os.path.join(HERE, "golden_c4.json"), "w") as f:
        json.dump({"generator": "HongYue1/KBSRC 1.3.0 built from source (oracle/_ref), kbsrc::resample, exact",
                   "files": files}, f, indent=0)


if __name__ == "__main__":
    main()

"""Writes tests/golden/golden.json: SHA-256 of the reference's output for every case in cases.py.

The outputs come from HongYue1/KBSRC built from its own sources (oracle/Makefile -> oracle/_ref), called through
its public kbsrc::resample. Run here, where the reference tree exists:
    make -C oracle && python tests/golden/make_golden.py
The hash covers the planar float64 output, channel after channel, little-endian.
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES, make_input  # noqa: E402
from oracle import oracle  # noqa: E402


def main():
    out = {}
    for name, (recipe, fi, fo, opts) in CASES.items():
        x = make_input(recipe)
        y = oracle.ref_resample(x, fi, fo, mode=opts.get("mode", "exact"), length=opts.get("length", 0.2),
                                beta=opts.get("beta", 40.0), block=opts.get("block", 0), lpc=opts.get("lpc", True))
        y = y.astype("<f8", copy=False)
        out[name] = {"sha256": hashlib.sha256(y.tobytes()).hexdigest(), "shape": list(y.shape),
                     "input_sha256": hashlib.sha256(x.astype("<f8").tobytes()).hexdigest()}
        print(name, y.shape, out[name]["sha256"][:16], flush=True)
    # the scaled-down uneven queue, exact mode, one reference conversion per file
    from cases import C4_SMALL, c4_specs, c4_samples
    c4 = []
    for i, (frames, ch, fi, fo) in enumerate(c4_specs(**C4_SMALL)):
        x = c4_samples(C4_SMALL["seed"], i, frames, ch)
        y = oracle.ref_resample(x, fi, fo).astype("<f8", copy=False)
        c4.append({"spec": [frames, ch, fi, fo], "sha256": hashlib.sha256(y.tobytes()).hexdigest(),
                   "shape": list(y.shape)})
    print("c4_small", len(c4), "files", flush=True)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "HongYue1/KBSRC 1.3.0 built from source (oracle/_ref), kbsrc::resample",
                   "cases": out, "c4_small": c4}, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()

"""The full uneven queue at its benchmark size: 256 files of 1-60 s, 1-8 channels, input rates from {44.1, 48, 88.2,
96, 192} kHz and output rates from {44.1, 48, 96} kHz (cases.c4_specs, seed 3), exact mode, run as GPU batches.

Every file's planar output must hash to the reference's own output for that file converted alone
(tests/golden/golden_c4.json, from the reference built from source), and every file whose rates differ must have
run on the GPU. The queue runs as four batches of 64 files to bound host memory (each batch is one recorded launch
sequence of its plan groups)."""
import hashlib
import json
import os

import pytest

import kbsrc_b200
from cases import c4_samples, c4_specs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PER_BATCH = 64


def test_full_queue_matches_reference_per_file():
    with open(os.path.join(ROOT, "tests", "golden", "golden_c4.json")) as f:
        golden = json.load(f)["files"]
    specs = c4_specs(seed=3, count=256)
    assert [g["spec"] for g in golden] == [list(s) for s in specs]
    bad, gpu_files, groups = [], 0, 0
    for lo in range(0, len(specs), PER_BATCH):
        idx = list(range(lo, min(lo + PER_BATCH, len(specs))))
        xs = [c4_samples(3, i, specs[i][0], specs[i][1]) for i in idx]
        b = kbsrc_b200.Batch([(x, specs[i][2], specs[i][3]) for x, i in zip(xs, idx)])
        for k, i in enumerate(idx):
            fi, fo = specs[i][2], specs[i][3]
            assert (b.gpu_index[k] >= 0) == (fi != fo), f"file {i}: resampled off the GPU or copied on it"
        gpu_files += sum(g >= 0 for g in b.gpu_index)
        groups += b.gpu_info()["groups"]
        ys = b.run()
        for k, i in enumerate(idx):
            y = ys[k]
            if list(y.shape) != golden[i]["shape"] or \
                    hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() != golden[i]["sha256"]:
                bad.append(i)
        b.close()
        del xs, ys, b
    print(f"{gpu_files} files on the GPU in {groups} plan groups")
    assert gpu_files == sum(s[2] != s[3] for s in specs)
    assert not bad, f"{len(bad)} files differ from the reference: {bad[:10]}"

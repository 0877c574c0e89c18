"""The uneven multi-file queue on the GPU: one batch of files with mixed lengths, channel counts and rate pairs
(equal rates included), each output byte-identical to the reference's conversion of that file alone."""
import hashlib
import json
import os

import numpy as np
import pytest

import kbsrc_b200
from cases import C4_SMALL, c4_samples, c4_specs

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_batch_matches_per_file_reference():
    with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
        want = json.load(f)["c4_small"]
    specs = c4_specs(**C4_SMALL)
    xs = [c4_samples(C4_SMALL["seed"], i, n, ch) for i, (n, ch, _, _) in enumerate(specs)]
    b = kbsrc_b200.Batch([(x, fi, fo) for x, (_, _, fi, fo) in zip(xs, specs)])
    info = b.gpu_info()
    assert info["groups"] >= 1 and info["tasks"] > 0
    for rep in range(2):  # the second run replays the recorded launch sequence
        ys = b.run()
        bad = [i for i, (y, w) in enumerate(zip(ys, want))
               if list(y.shape) != w["shape"] or hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() != w["sha256"]]
        assert not bad, f"run {rep}: files {bad[:5]} differ from the reference"
    b.close()


def test_batch_equals_single_conversions():
    rng = np.random.default_rng(11)
    items = [(rng.uniform(-0.5, 0.5, (n, ch)), fi, fo) for n, ch, fi, fo in
             [(30000, 2, 96000, 44100), (20000, 1, 96000, 44100), (5000, 3, 44100, 48000), (7000, 2, 48000, 48000),
              (1, 2, 8000, 16000), (9000, 1, 44100, 44101)]]
    for mode in ("exact", "fast"):
        ys = kbsrc_b200.Batch(items, mode=mode).run()
        for (x, fi, fo), y in zip(items, ys):
            assert y.tobytes() == kbsrc_b200.resample(x, fi, fo, mode=mode).tobytes()


def test_batch_device_run_with_new_buffers():
    import torch
    rng = np.random.default_rng(12)
    items = [(rng.uniform(-0.5, 0.5, (n, ch)), fi, fo) for n, ch, fi, fo in
             [(40000, 2, 96000, 44100), (15000, 1, 48000, 96000)]]
    b = kbsrc_b200.Batch(items)
    want = b.run()
    for rep in range(2):  # fresh device buffers each time: the recorded run reads them from the item table
        d_in = [torch.from_numpy(x).cuda() for x, _, _ in items]
        d_h = [torch.from_numpy(h).cuda() for h in b.head]
        d_t = [torch.from_numpy(t).cuda() for t in b.tail]
        d_o = [torch.full((x.shape[1] * n,), float("nan"), dtype=torch.float64, device="cuda")
               for (x, _, _), n in zip(items, b.nout)]
        b.run_device([t.data_ptr() for t in d_in], [t.data_ptr() for t in d_h], [t.data_ptr() for t in d_t],
                     [t.data_ptr() for t in d_o])
        torch.cuda.synchronize()
        for o, w, n in zip(d_o, want, b.nout):
            assert o.cpu().numpy().reshape(-1, n).tobytes() == w.tobytes()


@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_queue_equals_group_launches(mode, monkeypatch):
    """The batch queue (one persistent launch per pass and wave over all groups' tasks) against each group run on
    its own launches (KBSRC_GPU_QUEUE=0): the same bytes per file, in fewer launches. The queue holds the groups
    with four-step 7-smooth transforms; the short files' direct transforms run on their own launches after it."""
    rng = np.random.default_rng(21)
    items = [(rng.uniform(-0.5, 0.5, (n, ch)), fi, fo) for n, ch, fi, fo in
             [(400000, 2, 96000, 44100), (300000, 1, 48000, 96000), (250000, 3, 44100, 48000),
              (500000, 1, 192000, 44100), (120000, 2, 88200, 48000), (2000, 1, 48000, 44100),
              (60000, 2, 48000, 48000), (350000, 2, 96000, 44100)]]
    queued = kbsrc_b200.Batch(items, mode=mode)
    monkeypatch.setenv("KBSRC_GPU_QUEUE", "0")
    grouped = kbsrc_b200.Batch(items, mode=mode)
    a, b = queued.run(), grouped.run()
    assert all(x.tobytes() == y.tobytes() for x, y in zip(a, b))
    assert queued.gpu_info()["launches"] < grouped.gpu_info()["launches"]
    for (x, fi, fo), y in zip(items[:2], a[:2]):
        assert y.tobytes() == kbsrc_b200.resample(x, fi, fo, mode=mode).tobytes()
    queued.close()
    grouped.close()

"""Multi-GPU shares of one conversion, run on one GPU: every share through its own engine, output ranges
concatenated, against the reference's bytes.

A share (kbsrc_gpu_shard) is a contiguous block range with only the input frames its blocks read and the output
samples they write; engines of different shares exchange nothing. With one GPU here, the shares of a conversion
run one after another on it (and resample_devices runs them on device 0 listed twice), which exercises everything
a multi-GPU run does except the second device."""
import hashlib

import numpy as np
import pytest

import kbsrc_b200
from cases import CASES, make_input

pytestmark = pytest.mark.gpu


def sha(y):
    return hashlib.sha256(np.ascontiguousarray(y).astype("<f8").tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["c2_96k_44k1_exact", "c2_96k_44k1_fast", "c3_sweep_44k1_48k_exact"])
@pytest.mark.parametrize("count", [2, 3])
def test_shares_back_to_back_equal_reference(golden, name, count):
    """Full benchmark sizes: each share's engine holds only its input span and output range."""
    recipe, fi, fo, opts = CASES[name]
    x = make_input(recipe)
    parts = []
    for k in range(count):
        cv = kbsrc_b200.Conversion(x, fi, fo, mode=opts["mode"], share=(k, count))
        s = cv.share
        assert s["blk1"] > s["blk0"] and cv.engine_info()["tasks"] == (s["blk1"] - s["blk0"]) * x.shape[1]
        parts.append(cv.run(x).copy())
        cv.close()
    y = np.concatenate(parts, axis=1)
    assert list(y.shape) == golden[name]["shape"]
    assert sha(y) == golden[name]["sha256"]


@pytest.mark.parametrize("name", ["c1_96k_44k1_exact", "s_96k_44k1_exact_20000", "s_44k1_48k_fast_30000",
                                  "s_48k_96k_exact_6ch", "s_96k_32k001_exact", "s_44k1_44k101_exact",
                                  "s_96k_44k1_ld_20000"])
def test_resample_devices_equals_reference(golden, name):
    recipe, fi, fo, opts = CASES[name]
    x = make_input(recipe)
    st = {}
    y = kbsrc_b200.resample_devices(x, fi, fo, [0, 0], mode=opts.get("mode", "exact"),
                                    length=opts.get("length", 0.2), beta=opts.get("beta", 40.0),
                                    block=opts.get("block", 0), lpc=opts.get("lpc", True), stats=st)
    assert st["isa"] == "sm_100a"
    assert list(y.shape) == golden[name]["shape"]
    assert sha(y) == golden[name]["sha256"]


def test_device_resident_shares():
    """run_device on a share: the device input buffer is the share's span, the output buffer its range."""
    import torch
    x = np.random.default_rng(9).uniform(-0.5, 0.5, (600000, 2))
    want = kbsrc_b200.resample(x, 96000, 44100)
    got = []
    for k in range(3):
        cv = kbsrc_b200.Conversion(x, 96000, 44100, share=(k, 3))
        s = cv.share
        d_in = torch.from_numpy(x[s["frame0"]:s["frame0"] + s["frames"]].copy()).cuda()
        d_h = torch.from_numpy(cv.head).cuda()
        d_t = torch.from_numpy(cv.tail).cuda()
        d_o = torch.full((2 * s["nout"],), float("nan"), dtype=torch.float64, device="cuda")
        cv.run_device(d_in.data_ptr(), d_h.data_ptr(), d_t.data_ptr(), d_o.data_ptr())
        torch.cuda.synchronize()
        got.append(d_o.cpu().numpy().reshape(2, s["nout"]))
        cv.close()
    assert np.concatenate(got, axis=1).tobytes() == want.tobytes()


def test_split_form_shares_equal_whole():
    """The split-precision form is deterministic, so its shares concatenate to its own whole output."""
    x = np.random.default_rng(10).uniform(-0.5, 0.5, (400000, 2))
    want = kbsrc_b200.resample(x, 96000, 44100, mode="split")
    parts = [kbsrc_b200.Conversion(x, 96000, 44100, mode="split", share=(k, 2)).run(x).copy() for k in range(2)]
    assert np.concatenate(parts, axis=1).tobytes() == want.tobytes()

"""The autotuner (kbsrc_gpu_engine_tune) changes only launch shapes: after tuning, the conversion still writes
the reference's bytes, and every four-step pass has a shape."""
import hashlib

import numpy as np
import pytest
import torch

import kbsrc_b200
from cases import CASES, make_input

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1_96k_44k1_exact", "s_96k_44k1_fast_20000", "s_44k1_48k_exact_30000"])
def test_tuned_engine_keeps_reference_bytes(golden, name):
    recipe, fi, fo, opts = CASES[name]
    x = make_input(recipe)
    cv = kbsrc_b200.Conversion(x, fi, fo, mode=opts.get("mode", "exact"))
    dev = torch.device("cuda")
    d_in = torch.from_numpy(x).to(dev)
    d_h = torch.from_numpy(cv.head if cv.head.size else np.zeros(1)).to(dev)
    d_t = torch.from_numpy(cv.tail if cv.tail.size else np.zeros(1)).to(dev)
    d_out = torch.empty(x.shape[1] * cv.nout, dtype=torch.float64, device=dev)
    p = (d_in.data_ptr(), d_h.data_ptr(), d_t.data_ptr(), d_out.data_ptr())
    shapes = cv.tune(*p)
    assert set(shapes) == {"fwd_column", "fwd_row", "inv_column", "inv_row"}
    assert all(f >= 1 and t >= 64 for f, t in shapes.values())
    cv.run_device(*p)
    torch.cuda.synchronize()
    y = d_out.cpu().numpy().reshape(x.shape[1], cv.nout)
    assert hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() == golden[name]["sha256"]
    z = cv.run(x)  # the host path with the tuned shapes
    assert hashlib.sha256(z.astype("<f8").tobytes()).hexdigest() == golden[name]["sha256"]


@pytest.mark.parametrize("name", ["c1_96k_44k1_exact", "s_44k1_48k_exact_30000", "c1_96k_44k1_ld"])
def test_twiddles_from_global_memory_keep_reference_bytes(golden, monkeypatch, name):
    """KBSRC_GPU_TW_GLOBAL=1: the double-double and extended passes read their stage twiddles from the global table
    instead of a shared-memory copy (a choice the autotuner also makes per pass); the bytes do not change."""
    if name not in CASES:
        pytest.skip(f"no case {name}")
    recipe, fi, fo, opts = CASES[name]
    monkeypatch.setenv("KBSRC_GPU_TW_GLOBAL", "1")
    x = make_input(recipe)
    cv = kbsrc_b200.Conversion(x, fi, fo, mode=opts.get("mode", "exact"))
    try:
        assert cv.staging() and not any(cv.staging().values())
        y = cv.run(x)
    finally:
        cv.close()
    assert hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() == golden[name]["sha256"]


def test_one_sequence_ctas_read_global_twiddles(monkeypatch):
    """With one sequence per CTA (forced here by a 60 KB shared-memory budget on 625- and 640-point sub-FFTs) the
    double-double passes read their stage twiddles from the global table by default; the bytes equal the staged
    form and the default shapes."""
    x = np.random.default_rng(41).uniform(-0.5, 0.5, (10 * 192000, 1))
    args = dict(mode="exact", length=1.0, beta=60.0)
    want = kbsrc_b200.resample(x, 192000, 44100, **args)
    monkeypatch.setenv("KBSRC_GPU_SMEM_KB", "60")
    cv = kbsrc_b200.Conversion(x, 192000, 44100, **args)
    try:
        st = cv.staging()
        assert st["fwd_column"] is False and st["fwd_row"] is False
        one = cv.run(x).copy()
    finally:
        cv.close()
    monkeypatch.setenv("KBSRC_GPU_TW_GLOBAL", "0")
    cv = kbsrc_b200.Conversion(x, 192000, 44100, **args)
    try:
        assert cv.staging() and all(cv.staging().values())
        staged = cv.run(x).copy()
    finally:
        cv.close()
    assert one.tobytes() == want.tobytes()
    assert staged.tobytes() == want.tobytes()

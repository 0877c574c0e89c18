"""Multi-GPU shares of one conversion, on the CPU: the host planner (kbsrc_gpu_shard_plan) and the data path it
implies, checked with the oracle in two gloo ranks.

A conversion's tasks are independent: block b of channel c reads its own input span and writes a disjoint output
range (the reference's src/resampler.cpp:48-50,80-84). A share is a contiguous block range with the input frames
those blocks read and the output samples they write. Run share k on rank k, gather the output ranges in order,
and the concatenation must be the whole conversion, byte for byte; no data moves between ranks before the gather."""
import os

import numpy as np
import pytest

import kbsrc_b200
from oracle import oracle

# the first three have 5-7 blocks per channel; the others are the short, near-unity and non-7-smooth plans
CASES = [(200000, 2, 96000, 44100, "exact"), (100000, 1, 44100, 48000, "fast"), (60000, 3, 48000, 96000, "exact"),
         (40000, 2, 96000, 44100, "exact"), (3000, 1, 44100, 44101, "exact"), (5000, 2, 96000, 32001, "fast")]


@pytest.mark.parametrize("frames,ch,fi,fo,mode", CASES)
@pytest.mark.parametrize("count", [1, 2, 3, 7])
def test_shares_partition_blocks_and_output(frames, ch, fi, fo, mode, count):
    p = kbsrc_b200.plan(frames, ch, fi, fo, mode)
    count = min(count, p["nblk"])
    sh = kbsrc_b200.shard_plan(frames, ch, fi, fo, count, mode)
    assert [s["blk0"] for s in sh] == [p["nblk"] * k // count for k in range(count)]
    assert [s["blk1"] for s in sh] == [p["nblk"] * (k + 1) // count for k in range(count)]
    assert sh[0]["out0"] == 0 and sum(s["nout"] for s in sh) == p["nout"]
    for a, b in zip(sh, sh[1:]):
        assert a["out0"] + a["nout"] == b["out0"]
    hopQ, hopP, Nb = p["hop"] * p["Q"], p["hop"] * p["P"], p["Nb"]
    for s in sh:
        # the input span is exactly what the share's blocks read, clipped to the signal
        lo = max(0, s["blk0"] * hopQ - p["lead"])
        hi = min(frames, (s["blk1"] - 1) * hopQ + Nb - p["lead"])
        assert (s["frame0"], s["frame0"] + s["frames"]) == (min(lo, frames), max(min(lo, frames), hi))
        # every sample the share's blocks write lies in its output range
        w0, w1 = max(0, s["blk0"] * hopP - p["o"]), min(p["nout"], s["blk1"] * hopP - p["o"])
        assert w1 <= w0 or (s["out0"] <= w0 and w1 <= s["out0"] + s["nout"])


@pytest.mark.parametrize("frames,ch,fi,fo,mode", CASES[:3])
def test_oracle_shares_concatenate_to_whole(frames, ch, fi, fo, mode):
    x = np.random.default_rng(frames + ch).uniform(-0.5, 0.5, (frames, ch))
    whole = oracle.resample(x, fi, fo, mode=mode)
    sh = kbsrc_b200.shard_plan(frames, ch, fi, fo, 3, mode)
    parts = []
    for s in sh:
        y = oracle.resample_blocks(x, fi, fo, s["blk0"], s["blk1"], mode=mode)
        parts.append(y[:, s["out0"]:s["out0"] + s["nout"]])
    assert np.concatenate(parts, axis=1).tobytes() == whole.tobytes()


def _rank(rank, world, port, result_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    frames, ch, fi, fo, mode = CASES[0]
    x = np.random.default_rng(frames + ch).uniform(-0.5, 0.5, (frames, ch))
    s = kbsrc_b200.shard_plan(frames, ch, fi, fo, world, mode)[rank]
    # this rank holds only its input span: every frame outside it is zeroed, so its output cannot depend on them
    # (the LPC edges, computed from the signal's ends, are read only by the first and last shares, which hold
    # those ends)
    span = np.zeros_like(x)
    span[s["frame0"]:s["frame0"] + s["frames"]] = x[s["frame0"]:s["frame0"] + s["frames"]]
    y = oracle.resample_blocks(span, fi, fo, s["blk0"], s["blk1"], mode=mode)
    mine = y[:, s["out0"]:s["out0"] + s["nout"]]
    parts = [None] * world
    dist.all_gather_object(parts, mine)
    if rank == 0:
        np.save(result_path, np.concatenate(parts, axis=1))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_each_convert_their_share(tmp_path):
    """Two ranks, one share each: rank k converts only its block range (with LPC edges from the whole signal's
    ends) and the gathered output ranges equal the whole conversion."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    out = str(tmp_path / "gathered.npy")
    mp.spawn(_rank, args=(2, port, out), nprocs=2, join=True)
    frames, ch, fi, fo, mode = CASES[0]
    x = np.random.default_rng(frames + ch).uniform(-0.5, 0.5, (frames, ch))
    assert np.load(out).tobytes() == oracle.resample(x, fi, fo, mode=mode).tobytes()


def test_engine_refuses_a_share_that_misses_its_span():
    """The C ABI checks a share against its blocks before anything else: a share whose input span is one frame
    short is an argument error (no device needed to see it)."""
    import ctypes
    frames, ch, fi, fo, mode = CASES[0]
    p = kbsrc_b200.plan(frames, ch, fi, fo, mode)
    sh = kbsrc_b200.shard_plan(frames, ch, fi, fo, 2, mode)
    d = kbsrc_b200.GpuDesc()
    d.precision, d.channels, d.P, d.Q, d.nb, d.marg, d.nblk = 1, ch, p["P"], p["Q"], p["nb"], p["marg"], p["nblk"]
    d.lead, d.o, d.frames, d.nout, d.up = p["lead"], p["o"], frames, p["nout"], p["up"]
    H = np.zeros((p["Nb"] // 2 + 1, 2))
    d.H, d.H_len = H.ctypes.data_as(kbsrc_b200._dp), H.shape[0]
    s = sh[1]
    d.shard = kbsrc_b200.GpuShard(s["blk0"], s["blk1"], s["frame0"] + 1, s["frames"] - 1, s["out0"], s["nout"])
    e = ctypes.c_void_p()
    assert kbsrc_b200.gpu_lib().kbsrc_gpu_engine_create(ctypes.byref(d), ctypes.byref(e)) == kbsrc_b200.GPU_E_ARG
    assert "shard" in kbsrc_b200.gpu_error()

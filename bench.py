#!/usr/bin/env python
"""Throughput of the DFT-domain resampling block engine on B200: output Msamples/s.

Workload (default): 180 s of stereo 96 kHz float64 noise (uniform [-0.5, 0.5), numpy default_rng(2)) converted
to 44.1 kHz in exact (double-double) mode with the defaults (--len 0.2, --beta 40, LPC edges, automatic block):
107 blocks x 2 channels of a 201600-point forward and 92610-point inverse real FFT. One step = the whole
block loop of that conversion (every (channel, block) task), output byte-identical to the reference.

  value  device-resident: input, LPC edges and output in HBM; the engine's launches only (CUDA events)
  e2e    the same through the C ABI with host buffers: kbsrc_gpu_engine_run_host on pinned memory, the H2D copy
         of the input and edges and the D2H copy of the output inside the timed region
  --impl reference: the reference's own engine (HongYue1/KBSRC built from source, oracle/_ref) on the host
         cores, its Stats::process_seconds (the block loop run_engine) per conversion

Multi-GPU (torchrun, N ranks): one conversion of N times the workload's length, split into N contiguous block
ranges (kbsrc_gpu_shard_plan); rank k holds only share k's input span (its blocks' inputs, halo included) and output
range on its GPU. No collective on the data path (the only one is the timing max); weak scaling.
"""
import argparse
import json
import math
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

WORKLOADS = {
    "c2_exact": dict(seed=2, seconds=180, rate_in=96000, rate_out=44100, channels=2, mode="exact"),
    "c2_fast": dict(seed=2, seconds=180, rate_in=96000, rate_out=44100, channels=2, mode="fast"),
    # the split-precision tensor-core form of the same conversion (not byte-identical; error against exact stated)
    "c2_split": dict(seed=2, seconds=180, rate_in=96000, rate_out=44100, channels=2, mode="split"),
    "c1_exact": dict(seed=1, seconds=10, rate_in=96000, rate_out=44100, channels=2, mode="exact"),
    "c3_exact": dict(sweep=True, seconds=60, rate_in=44100, rate_out=48000, channels=2, mode="exact"),
    # the split-precision form on the 60 s stereo 44.1k -> 48k log sweep (upsampling: periodic spectrum extension)
    "c3_split": dict(sweep=True, seconds=60, rate_in=44100, rate_out=48000, channels=2, mode="split"),
    # large multichannel, long kernel: 600 s 8 ch 192k -> 44.1k from 24-bit PCM, --len 1.0 --beta 60
    "c5_exact": dict(pcm24=True, seed=4, seconds=600, rate_in=192000, rate_out=44100, channels=8, mode="exact",
                     length=1.0, beta=60.0),
    # its split-precision form (the 967,680-point forward transform has three-radix sub-FFTs)
    "c5_split": dict(pcm24=True, seed=4, seconds=600, rate_in=192000, rate_out=44100, channels=8, mode="split",
                     length=1.0, beta=60.0),
    # the uneven queue: 256 files, 1-60 s, 1-8 channels, mixed rate pairs, one GPU batch (exact)
    "c4_exact": dict(batch=True, seed=3, files=256, mode="exact"),
}
METRIC = "out Msamples/s 96k->44.1k exact (180 s stereo f64, byte-identical to the reference)"
METRIC_SPLIT = ("out Msamples/s 96k->44.1k split-precision tensor-core form (180 s stereo f64; error against the "
                "exact output and throughput against the plain exact GPU engine stated)")
METRIC_OF = {
    "c3_split": "out Msamples/s 44.1k->48k split-precision tensor-core form (60 s stereo log sweep 20 Hz-20 kHz at "
                "0.5; error against the exact output and throughput against the plain exact GPU engine stated)",
    "c5_exact": "out Msamples/s 192k->44.1k exact (600 s 8-channel 24-bit PCM, --len 1.0 --beta 60, byte-identical "
                "to the reference)",
    "c5_split": "out Msamples/s 192k->44.1k split-precision tensor-core form (600 s 8-channel 24-bit PCM, --len 1.0 "
                "--beta 60; error against the exact output and throughput against the plain exact GPU engine stated)",
}
TENSOR_INT8_PEAK_TOPS = 4500.0  # nominal dense int8 of B200; no measured int8 figure exists for this pool


def make_input(w):
    from cases import noise, sweep, pcm24_ints, pcm24_as_f64
    if w.get("pcm24"):
        return pcm24_as_f64(pcm24_ints(w["seed"], w["seconds"], w["rate_in"], w["channels"]))
    if w.get("sweep"):
        return sweep(w["seconds"], w["rate_in"], w["channels"])
    return noise(w["seed"], w["seconds"], w["rate_in"], w["channels"])


class ClockSampler:
    """Samples SM clock and clock-event reasons through NVML every 20 ms while running."""

    REASONS = {"gpu_idle": 0x1, "applications_clocks_setting": 0x2, "sw_power_cap": 0x4, "hw_slowdown": 0x8,
               "sync_boost": 0x10, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "hw_power_brake_slowdown": 0x80, "display_clock_setting": 0x100}

    def __init__(self, index):
        self.samples, self.reasons, self.ok = [], set(), False
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            pass
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                mhz = self.nv.nvmlDeviceGetClockInfo(self.h, self.nv.NVML_CLOCK_SM)
                r = self.nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                util = self.nv.nvmlDeviceGetUtilizationRates(self.h).gpu
                self.samples.append((mhz, util))
                for k, bit in self.REASONS.items():
                    if r & bit and k != "gpu_idle":
                        self.reasons.add(k)
            except Exception:
                pass
            time.sleep(0.02)

    def __enter__(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        loaded = [m for m, u in self.samples if u > 50] or [m for m, _ in self.samples]
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def fp64_peak():
    """Measured FP64 instruction rate of this GPU (ops/s, one DFMA/DADD/DMUL = 1), max over the three kinds."""
    import ctypes
    lib = ctypes.CDLL(os.path.join(ROOT, "kbsrc_b200", "lib", "libkbsrc_probe.so"))
    lib.kbsrc_probe_fp64.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    rates = {}
    for kind, name in ((0, "dfma"), (1, "dadd"), (2, "dmul")):
        v = ctypes.c_double()
        if lib.kbsrc_probe_fp64(kind, ctypes.byref(v)) == 0:
            rates[name] = v.value
    return rates


def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_bf16_tflops():
    """The measured dense bf16 GEMM rate of this pool's B200 (burst), else the fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"])
    except Exception:
        return 1590.0


def load_traffic():
    """dram bytes per launch from the committed ncu summary, if any: {workload: {pass: bytes}}."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def cpu_reference(x, w, threads, runs=1):
    """The reference engine on the host (oracle/_ref): output Msamples/s from its process_seconds."""
    from oracle import oracle
    if not oracle.ref_available():
        return None
    n_out, secs, walls = 0, 0.0, 0.0
    for _ in range(runs):
        st = {}
        t = time.perf_counter()
        y = oracle.ref_resample(x, w["rate_in"], w["rate_out"], fast=w["mode"] == "fast", threads=threads, stats=st,
                                length=w.get("length", 0.2), beta=w.get("beta", 40.0))
        walls += time.perf_counter() - t
        n_out += y.size
        secs += st["process_seconds"]
    return {"engine_msps": n_out / secs / 1e6, "wall_msps": n_out / walls / 1e6, "threads": st["threads"],
            "process_seconds": secs / runs, "wall_seconds": walls / runs, "samples": n_out // runs}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def reference_arm(args, w, world, rank, pg):
    if rank != 0:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    x = make_input(w)
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_reference(x, w, threads)
    n_out, secs, walls = 0, 0.0, 0.0
    for _ in range(args.steps):
        r = cpu_reference(x, w, threads)
        n_out += r["samples"]
        secs += r["process_seconds"]
        walls += r["wall_seconds"]
    value = n_out / secs / 1e6
    line = {"impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Msamples/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(secs / args.steps * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if w["mode"] == "fast" else "dd (double-double f64 pairs)",
            "data": "synthetic", "config": {"workload": args.workload, **{k: v for k, v in w.items()}},
            "whole_call_msps": round(n_out / walls / 1e6, 3),
            "cpu_baseline": {"value": round(value, 3), "unit": "Msamples/s", "cores": threads, "kind": "reference",
                             "sample": f"{args.steps} full conversions of the workload, engine time "
                                       "(Stats::process_seconds) with all host threads"},
            "e2e": {"value": round(value, 3), "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def write_f64_wav(path, x, rate):
    """A float64 WAV file (18-byte fmt chunk, fact chunk) of interleaved samples x (frames x channels)."""
    import struct
    frames, ch = x.shape
    n = frames * ch * 8
    fmt = struct.pack("<HHIIHHH", 3, ch, rate, rate * 8 * ch, 8 * ch, 64, 0)
    with open(path, "wb") as f:
        f.write(b"RIFF" + struct.pack("<I", 4 + 8 + len(fmt) + 12 + 8 + n) + b"WAVE" + b"fmt " +
                struct.pack("<I", len(fmt)) + fmt + b"fact" + struct.pack("<II", 4, frames) + b"data" +
                struct.pack("<I", n))
        f.write(np.ascontiguousarray(x, dtype="<f8").tobytes())


def cli_e2e(w, x):
    """Wall time of the kbsrc command line on the workload as a WAV file (read, decode, kernel design, LPC,
    conversion, output step, write), ours and the reference tool built from source: the 24-bit file with s24
    dithered output for PCM workloads, else the float64 file with float64 output."""
    import subprocess
    import tempfile
    import kbsrc_b200
    from cases import pcm24_ints, write_pcm24_wav
    from oracle import oracle
    out = {}
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "in.wav")
        args = ["--rate", str(w["rate_out"]), "--len", str(w.get("length", 0.2)), "--beta", str(w.get("beta", 40.0)),
                "--mode", w["mode"]]
        if w.get("pcm24"):
            write_pcm24_wav(src, pcm24_ints(w["seed"], w["seconds"], w["rate_in"], w["channels"]), w["rate_in"])
            args += ["--format", "s24", "--dither", src]
        else:
            write_f64_wav(src, x, w["rate_in"])
            args += ["--format", "f64", src]
        tools = [("ours", kbsrc_b200.CLI)] + ([("reference", oracle.REF_CLI)] if os.path.exists(oracle.REF_CLI) else [])
        for name, exe in tools:
            dst = os.path.join(d, name + ".wav")
            t = time.perf_counter()
            r = subprocess.run([exe] + args + [dst], capture_output=True, text=True)
            out[name + "_seconds"] = round(time.perf_counter() - t, 3)
            out[name + "_ok"] = r.returncode == 0
            if os.path.exists(dst):
                os.remove(dst)
        out["input_bytes"] = os.path.getsize(src)
    return out


def companion_form(mode, x, w, kw, dev, stream, args, ref_out, tune):
    """Another precision of the same conversion, measured in the same process on the same resident input: device
    ms per step over args.steps block loops, its output's error against the exact output `ref_out` (the reference's
    bytes), and its roofline. Used to put the split-precision form and the fast engine beside plain exact."""
    import torch
    import kbsrc_b200
    from kbsrc_b200 import roofline
    frames, ch = x.shape
    cv = kbsrc_b200.Conversion(x, w["rate_in"], w["rate_out"], mode=mode, **kw)
    plan = kbsrc_b200.plan(frames, ch, w["rate_in"], w["rate_out"], mode, **kw)
    d_in = torch.from_numpy(x).to(dev)
    d_head = torch.from_numpy(cv.head).to(dev) if cv.head.size else torch.zeros(1, dtype=torch.float64, device=dev)
    d_tail = torch.from_numpy(cv.tail).to(dev) if cv.tail.size else torch.zeros(1, dtype=torch.float64, device=dev)
    d_out = torch.empty(ch * max(cv.nout, 1), dtype=torch.float64, device=dev)
    ptrs = (d_in.data_ptr(), d_head.data_ptr(), d_tail.data_ptr(), d_out.data_ptr())
    for _ in range(args.warmup):
        cv.run_device(*ptrs, stream=stream)
    torch.cuda.synchronize()
    shapes = cv.tune(*ptrs, stream=stream) if tune and not mode.startswith("split") else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        cv.run_device(*ptrs, stream=stream)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    y = d_out[:ch * cv.nout].cpu().numpy().reshape(ch, cv.nout)
    out = {"ms_per_step": round(ms, 4), "value": round(ch * cv.nout / (ms * 1e-3) / 1e6, 3), "unit": "Msamples/s",
           "error_vs_exact": roofline.error_stats(y, ref_out), "gpu_launches_per_step": cv.engine_info()["launches"]}
    if shapes is not None:
        out["tuned_shapes"] = shapes
    if mode == "fast":
        work = roofline.conversion_work(plan, ch, False)
        peaks = fp64_peak()
        hbm, how = measured_hbm_gbs()
        t_fp64 = work["ops_total"] / max(peaks.values()) if peaks else None
        t_hbm = work["compulsory_bytes"] / (hbm * 1e9)
        roof_ms = max(t_fp64 or 0.0, t_hbm) * 1e3
        out["roofline"] = {"bound": "max(fp64, hbm)", "roofline_ms_per_step": round(roof_ms, 4),
                           "fp64_ms": round(t_fp64 * 1e3, 4) if t_fp64 else None, "hbm_ms": round(t_hbm * 1e3, 4),
                           "frac": round(roof_ms / ms, 4), "fp64_ops_per_step": work["ops_total"],
                           "compulsory_bytes_per_step": work["compulsory_bytes"],
                           "note": "roofline time = max(FP64 instructions / measured FP64 issue rate, compulsory "
                                   "bytes (each block's input span and kept output) / HBM peak (" + how + ")); "
                                   "frac = roofline time / measured time"}
    else:
        eb = 2 if mode == "split16" else 1
        tw = roofline.split_work(plan, ch, eb)
        peak = TENSOR_INT8_PEAK_TOPS if eb == 1 else measured_bf16_tflops()  # f16 runs at the bf16 rate
        out["tensor_ops_per_step"] = tw["ops_total"]
        out["tensor_kind"] = "int8" if eb == 1 else "f16"
        out["tensor_frac_of_nominal"] = round(tw["ops_total"] / (ms * 1e-3) / 1e12 / peak, 4)
    cv.close()
    return out


def product_arm(args, w, world, rank, local, pg):
    import torch
    import kbsrc_b200
    from kbsrc_b200 import roofline

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    exact = w["mode"] == "exact"
    split = w["mode"] == "split"
    # N ranks: one conversion of N times the workload's length, split into N contiguous block ranges (shares); each
    # rank holds only its share's input span and output range on its GPU, and no data moves between GPUs
    x_all = make_input(w if world == 1 else dict(w, seconds=w["seconds"] * world))
    frames, ch = x_all.shape
    kw = dict(length=w.get("length", 0.2), beta=w.get("beta", 40.0))
    cv = kbsrc_b200.Conversion(x_all, w["rate_in"], w["rate_out"], mode=w["mode"], share=(rank, world) if world > 1
                               else None, **kw)
    plan = kbsrc_b200.plan(frames, ch, w["rate_in"], w["rate_out"], w["mode"], **kw)
    work = roofline.conversion_work(plan, ch, exact or split)
    twork = roofline.split_work(plan, ch) if split else None
    info = cv.engine_info()
    nout_all, nout = cv.nout, cv.out_len  # output samples per channel: the whole conversion's, this rank's
    x = x_all[cv.share["frame0"]:cv.share["frame0"] + cv.share["frames"]] if cv.share else x_all
    d_in = torch.from_numpy(x).to(dev)
    d_head = torch.from_numpy(cv.head).to(dev) if cv.head.size else torch.zeros(1, dtype=torch.float64, device=dev)
    d_tail = torch.from_numpy(cv.tail).to(dev) if cv.tail.size else torch.zeros(1, dtype=torch.float64, device=dev)
    d_out = torch.empty(ch * max(nout, 1), dtype=torch.float64, device=dev)
    # a dedicated stream: the engine runs and the CUDA events are recorded on it (handle 0 would mean the
    # engine's own stream in the C ABI)
    side = torch.cuda.Stream(dev)
    torch.cuda.set_stream(side)
    stream = side.cuda_stream
    ptrs = (d_in.data_ptr(), d_head.data_ptr(), d_tail.data_ptr(), d_out.data_ptr())

    def step():
        cv.run_device(*ptrs, stream=stream)

    L2_BYTES = 126 << 20
    resident = x.nbytes + 8 * ch * nout
    flush = torch.empty((256 << 20) // 8, dtype=torch.float64, device=dev) if resident < 2 * L2_BYTES else None

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    tuned = cv.tune(*ptrs, stream=stream) if args.tune else None
    if pg:
        pg.barrier()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    phys = vis[local] if local < len(vis) and vis[local].strip().isdigit() else str(local)
    sampler = ClockSampler(int(phys))
    with sampler:
        # value: K block loops on resident data. Inputs larger than L2 run back to back; a smaller input is timed
        # step by step with a 256 MB write between steps (untimed), so no step starts with its data in L2.
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if flush is None:
            e0.record()
            for _ in range(args.steps):
                step()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
        else:
            ms = 0.0
            for _ in range(args.steps):
                flush.fill_(1.0)
                e0.record()
                step()
                e1.record()
                torch.cuda.synchronize()
                ms += e0.elapsed_time(e1)
        # per-pass device time over K more steps (an event after every launch, same stream)
        pass_ms = {}
        for _ in range(args.steps):
            for k, (t, n) in cv.run_device_timed(*ptrs, stream=stream).items():
                a = pass_ms.setdefault(k, [0.0, 0])
                a[0] += t
                a[1] += n
        # e2e: through the C ABI with pinned host buffers, copies inside the timed region
        hx = torch.from_numpy(x).pin_memory()
        hh = torch.from_numpy(cv.head.copy() if cv.head.size else np.zeros(1)).pin_memory()
        ht = torch.from_numpy(cv.tail.copy() if cv.tail.size else np.zeros(1)).pin_memory()
        ho = torch.empty(ch * max(nout, 1), dtype=torch.float64).pin_memory()
        cv.run_host_raw(hx.data_ptr(), hh.data_ptr(), ht.data_ptr(), ho.data_ptr())
        e2e_steps = max(3, args.steps // 2)
        if pg:
            pg.barrier()
        t = time.perf_counter()
        for _ in range(e2e_steps):
            cv.run_host_raw(hx.data_ptr(), hh.data_ptr(), ht.data_ptr(), ho.data_ptr())
        e2e_s = time.perf_counter() - t
        # the copy floor of that path: the same bytes up (pinned -> device) and down (device -> pinned) on two
        # streams at once, no compute
        up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
        d_x2 = torch.empty_like(d_in)
        torch.cuda.synchronize()
        t = time.perf_counter()
        for _ in range(e2e_steps):
            with torch.cuda.stream(up):
                d_x2.copy_(hx, non_blocking=True)
            with torch.cuda.stream(down):
                ho.copy_(d_out, non_blocking=True)
            torch.cuda.synchronize()
        copy_s = time.perf_counter() - t
        del d_x2
    h2d_all = int(8 * (x.size + cv.head.size + cv.tail.size))  # this rank's copies per step, summed below
    d2h_all = int(8 * ch * nout)
    if pg:
        import torch.distributed as dist
        tt = torch.tensor([ms, e2e_s, copy_s], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, e2e_s, copy_s = tt.tolist()
        bb = torch.tensor([h2d_all, d2h_all], dtype=torch.float64, device=dev)
        dist.all_reduce(bb, op=dist.ReduceOp.SUM)
        h2d_all, d2h_all = (int(v) for v in bb.tolist())
    # byte-identity of what was timed, against the reference's hash for this workload
    got = ho[:ch * nout].numpy().reshape(ch, nout)
    import hashlib
    digest = hashlib.sha256(got.astype("<f8").tobytes()).hexdigest()
    golden_sha = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as f:
            gold = json.load(f)["cases"]
        key = {"c2_exact": "c2_96k_44k1_exact", "c2_fast": "c2_96k_44k1_fast", "c1_exact": "c1_96k_44k1_exact",
               "c3_exact": "c3_sweep_44k1_48k_exact"}.get(args.workload) if not args.seconds and world == 1 else None
        golden_sha = gold.get(key, {}).get("sha256")
        if args.workload == "c5_exact" and not args.seconds and world == 1:
            with open(os.path.join(ROOT, "tests", "golden", "golden_c5.json")) as f:
                golden_sha = json.load(f)["planar_sha256"]
    except Exception:
        pass
    if rank != 0:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    samples = ch * nout_all  # the whole job's output, summed over the ranks' shares
    value = samples * args.steps / (ms * 1e-3) / 1e6
    e2e = samples * e2e_steps / e2e_s / 1e6
    # roofline of the dominant kernel
    launches_per_step = {k: v[1] / args.steps for k, v in pass_ms.items()}
    avg_ms = {k: v[0] / v[1] for k, v in pass_ms.items() if v[1]}
    share = {k: v[0] / sum(a[0] for a in pass_ms.values()) for k, v in pass_ms.items() if v[1]}
    top = max(avg_ms, key=lambda k: pass_ms[k][0])
    waves = max(1, int(round(launches_per_step[top])))
    tasks_per_launch = info["tasks"] / waves
    traffic = load_traffic().get(args.workload, {}).get(top)
    if split:
        achieved = twork["int8_ops_per_task"][top] * tasks_per_launch / (avg_ms[top] * 1e-3)
        roof = {"bound": "tensor", "achieved": round(achieved / 1e12, 3), "peak": TENSOR_INT8_PEAK_TOPS,
                "unit": "TOPS (int8)", "frac": round(achieved / 1e12 / TENSOR_INT8_PEAK_TOPS, 4), "traffic": traffic,
                "kernel": top, "peak_source": "nominal dense int8 (of nominal; no measured int8 peak on this pool)",
                "note": "issued int8 MMA operations (M x N x K x 2, padding included) of the top pass per second; "
                        "the pass is bound by the slicing and recombination on the CUDA cores, not the tensor pipe"}
    elif exact:
        peaks = fp64_peak()
        peak = max(peaks.values()) if peaks else None
        achieved = work["ops_per_task"][top] * tasks_per_launch / (avg_ms[top] * 1e-3)
        roof = {"bound": "fp64", "achieved": round(achieved / 1e12, 3), "peak": round(peak / 1e12, 3) if peak else None,
                "unit": "TFLOP/s", "frac": round(achieved / peak, 4) if peak else None,
                "traffic": traffic, "kernel": top,
                "note": "FP64 instructions/s (add, mul, fma each 1) of the reference operation sequence; peak = "
                        "measured DFMA/DADD/DMUL issue rate of this GPU (of measured)",
                "peak_by_kind_tflops": {k: round(v / 1e12, 3) for k, v in peaks.items()}}
    else:
        peak, how = measured_hbm_gbs()
        b = roofline.pass_bytes(plan, exact)[top] * tasks_per_launch
        achieved = b / (avg_ms[top] * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "traffic": traffic, "kernel": top, "peak_source": how}
    whole_ops = work["ops_total"] / (ms * 1e-3 / args.steps)
    cpu = None
    if world == 1 and not args.no_cpu:
        c_all = cpu_reference(x, w, os.cpu_count() or 1)
        c_8 = cpu_reference(x, w, 8)
        if c_all:
            cpu = {"value": round(c_all["engine_msps"], 3), "unit": "Msamples/s", "cores": c_all["threads"],
                   "kind": "reference",
                   "sample": "one full conversion of the workload by the reference built from source, engine "
                             "time (Stats::process_seconds), all host threads",
                   "value_t8": round(c_8["engine_msps"], 3), "whole_call_msps": round(c_all["wall_msps"], 3)}
    extra = {}
    if tuned is not None:
        extra["tuned_shapes"] = tuned
        extra["twiddles_in_shared_memory"] = cv.staging()
    if (w.get("pcm24") or not args.no_cpu) and not args.seconds and world == 1 and not split:
        extra["cli_e2e"] = cli_e2e(w, x)  # the tool a user runs, on the workload's file, ours and the reference's
    if args.workload in ("c2_exact", "c5_exact") and world == 1 and not args.seconds and not args.no_forms:
        # the metric's other half: the split-precision form (and the fast engine) beside plain exact, same process,
        # same resident input, errors against the exact output just timed
        ref_y = got.copy()
        for mode in ("split", "split16", "fast"):
            try:
                f = companion_form(mode, x, w, kw, dev, stream, args, ref_y, args.tune)
            except RuntimeError as e:  # a form without a plan for this workload's transform lengths
                extra[mode] = {"unsupported": str(e)}
                continue
            f["vs_plain_exact"] = round((ms / args.steps) / f["ms_per_step"], 4)
            extra[mode] = f
    if split:  # the comparison the form exists for: accuracy against exact, throughput against plain exact
        ref = kbsrc_b200.Conversion(x, w["rate_in"], w["rate_out"], mode="exact", **kw)
        fast = kbsrc_b200.Conversion(x, w["rate_in"], w["rate_out"], mode="fast", **kw)
        y_exact, y_fast = ref.run(x), fast.run(x)
        extra["error_vs_exact"] = {"split": roofline.error_stats(got, y_exact),
                                   "fast": roofline.error_stats(y_fast, y_exact)}
        d_out2 = torch.empty_like(d_out)
        p2 = (d_in.data_ptr(), d_head.data_ptr(), d_tail.data_ptr(), d_out2.data_ptr())
        for _ in range(args.warmup):
            ref.run_device(*p2, stream=stream)
        e0.record()
        for _ in range(args.steps):
            ref.run_device(*p2, stream=stream)
        e1.record()
        torch.cuda.synchronize()
        ms_exact = e0.elapsed_time(e1)
        extra["plain_exact_ms_per_step"] = round(ms_exact / args.steps, 4)
        extra["vs_plain_exact"] = round(ms_exact / ms, 4)
        extra["int8_ops_per_step"] = twork["int8_ops_total"]
        ref.close()
        fast.close()
    line = {
        "metric": METRIC_OF.get(args.workload, METRIC_SPLIT if split else METRIC), "value": round(value, 3), "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "dd (double-double f64 pairs)" if exact else ("int8 tensor-core slices, f64" if split else "f64"),
        "data": "synthetic",
        "config": {"workload": args.workload, **w, "tasks": work["tasks"], "block": plan["nb"],
                   "fft_points": [plan["Nb"], plan["Mb"]],
                   "l2": (f"inputs larger than L2 ({x.nbytes / 1e6:.0f} MB)" if flush is None else
                          f"input {x.nbytes / 1e6:.0f} MB: L2 flushed (256 MB write) before each step, steps timed "
                          "one by one"),
                   "parallelism": ("one GPU" if world == 1 else
                                   f"{world} block-range shares of one {w['seconds'] * world:g} s conversion, one per "
                                   "GPU, no inter-GPU data")},
        "e2e": {"value": round(e2e, 3), "unit": "Msamples/s", "h2d_bytes_per_step": h2d_all,
                "d2h_bytes_per_step": d2h_all, "path": "kbsrc_gpu_engine_run_host (C ABI), pinned",
                "copy_floor_ms_per_step": round(copy_s / e2e_steps * 1e3, 3),
                "frac_of_copy_floor": round(copy_s / e2e_s, 4)},
        "gpu_launches": int(info["launches"] * args.steps),
        "roofline": roof,
        "passes": {k: {"ms": round(avg_ms[k], 4), "share": round(share[k], 4),
                       "launches_per_step": launches_per_step[k]} for k in avg_ms},
        "fp64_ops_per_step": work["ops_total"], "whole_step_tflops": round(whole_ops / 1e12, 3),
        "cpu_baseline": cpu,
        "clocks": sampler.summary(),
        "output_sha256_matches_reference": golden_sha == digest if golden_sha else None,
        **extra,
    }
    print(json.dumps(line), flush=True)
    cv.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def batch_arm(args, w, world, rank, local, pg):
    """The uneven multi-file queue as one GPU batch (kbsrc_b200.Batch): value on device-resident buffers, e2e
    through the C batch entry with host buffers registered as pinned memory."""
    import ctypes
    import hashlib
    import torch
    import kbsrc_b200
    from kbsrc_b200 import roofline
    from cases import c4_samples, c4_specs

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    specs = c4_specs(seed=w["seed"], count=w["files"])
    xs = [c4_samples(w["seed"], i, n, ch) for i, (n, ch, _, _) in enumerate(specs)]
    t = time.perf_counter()
    b = kbsrc_b200.Batch([(x, fi, fo) for x, (_, _, fi, fo) in zip(xs, specs)], mode=w["mode"])
    prepare_s = time.perf_counter() - t
    info = b.gpu_info()
    gpu_items = [i for i, g in enumerate(b.gpu_index) if g >= 0]
    samples = sum(specs[i][1] * b.nout[i] for i in range(len(specs)))
    gpu_samples = sum(specs[i][1] * b.nout[i] for i in gpu_items)
    ops = 0
    for i in gpu_items:
        n, ch, fi, fo = specs[i]
        p = kbsrc_b200.plan(n, ch, fi, fo, w["mode"])
        ops += roofline.conversion_work(p, ch, w["mode"] == "exact")["ops_total"]
    side = torch.cuda.Stream(dev)
    torch.cuda.set_stream(side)
    d_in = [torch.from_numpy(xs[i]).to(dev) for i in gpu_items]
    d_h = [torch.from_numpy(b.head[i]).to(dev) for i in gpu_items]
    d_t = [torch.from_numpy(b.tail[i]).to(dev) for i in gpu_items]
    d_o = [torch.empty(specs[i][1] * max(b.nout[i], 1), dtype=torch.float64, device=dev) for i in gpu_items]
    ptrs = [[t.data_ptr() for t in v] for v in (d_in, d_h, d_t, d_o)]
    for _ in range(args.warmup):
        b.run_device(*ptrs, stream=side.cuda_stream)
    torch.cuda.synchronize()
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
    phys = vis[local] if local < len(vis) and vis[local].strip().isdigit() else str(local)
    sampler = ClockSampler(int(phys))
    with sampler:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            b.run_device(*ptrs, stream=side.cuda_stream)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
    # byte identity of the timed outputs against the reference, file by file
    golden = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "golden_c4.json")) as f:
            golden = json.load(f)["files"]
    except Exception:
        pass
    mism = None
    if golden and w["files"] == len(golden):
        mism = 0
        for k, i in enumerate(gpu_items):
            y = d_o[k][:specs[i][1] * b.nout[i]].cpu().numpy()
            if hashlib.sha256(y.astype("<f8").tobytes()).hexdigest() != golden[i]["sha256"]:
                mism += 1
    del d_in, d_h, d_t, d_o, ptrs
    torch.cuda.empty_cache()
    # e2e: host buffers (registered pinned) through the batch C entry, copies inside the timed region
    outs = [np.zeros((x.shape[1], max(n, 1))) for x, n in zip(xs, b.nout)]
    cudart = torch.cuda.cudart()
    regs = []
    for a in xs + outs:
        if a.nbytes and int(cudart.cudaHostRegister(a.ctypes.data, a.nbytes, 0)) == 0:
            regs.append(a)
    pin = (ctypes.c_void_p * len(xs))(*[x.ctypes.data for x in xs])
    pout = (ctypes.c_void_p * len(xs))(*[o.ctypes.data for o in outs])
    err = ctypes.create_string_buffer(512)
    kbsrc_b200.host_lib().kbsrc_batch_run_c(b._h, pin, pout, err, 512)  # first call allocates
    e2e_steps = max(2, args.steps // 3)
    t = time.perf_counter()
    for _ in range(e2e_steps):
        if kbsrc_b200.host_lib().kbsrc_batch_run_c(b._h, pin, pout, err, 512):
            raise RuntimeError(err.value.decode())
    e2e_s = time.perf_counter() - t
    for a in regs:
        cudart.cudaHostUnregister(a.ctypes.data)
    value = gpu_samples * args.steps / (ms * 1e-3) / 1e6  # the timed loop runs the GPU files
    peaks = fp64_peak()
    peak = max(peaks.values()) if peaks else None
    achieved = ops / (ms * 1e-3 / args.steps)
    cpu = None
    if not args.no_cpu:
        from oracle import oracle
        if oracle.ref_available():
            n_out, secs = 0, 0.0
            for i in range(8):  # bounded sample: the first 8 files, engine time, all host threads
                st = {}
                y = oracle.ref_resample(xs[i], specs[i][2], specs[i][3], threads=os.cpu_count() or 1, stats=st)
                n_out += y.size
                secs += st["process_seconds"]
            cpu = {"value": round(n_out / secs / 1e6, 3), "unit": "Msamples/s", "cores": os.cpu_count(),
                   "kind": "reference", "sample": "the first 8 files of the queue, each converted alone by the "
                   "reference built from source, engine time (Stats::process_seconds), all host threads"}
    line = {
        "metric": "out Msamples/s, uneven 256-file queue, exact (byte-identical per file)", "value": round(value, 3),
        "unit": "Msamples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "dd (double-double f64 pairs)", "data": "synthetic",
        "config": {"workload": args.workload, "files": w["files"], "gpu_files": len(gpu_items),
                   "output_samples": samples, "gpu_output_samples": gpu_samples, "groups": info["groups"],
                   "tasks": info["tasks"], "l2": "inputs larger than L2"},
        "e2e": {"value": round(samples * e2e_steps / e2e_s / 1e6, 3), "unit": "Msamples/s",
                "h2d_bytes_per_step": int(sum(8 * x.size for x in xs) + sum(8 * (h.size + t.size) for h, t in
                                                                            zip(b.head, b.tail))),
                "d2h_bytes_per_step": int(8 * samples), "path": "kbsrc_batch_run_c (C API), pinned"},
        "gpu_launches": int(info["launches"] * args.steps),
        "roofline": {"bound": "fp64", "achieved": round(achieved / 1e12, 3),
                     "peak": round(peak / 1e12, 3) if peak else None, "unit": "TFLOP/s",
                     "frac": round(achieved / peak, 4) if peak else None, "traffic": None, "kernel": "whole batch",
                     "note": "FP64 instructions of all groups per step / step time; the batch runs as one graph"},
        "prepare_seconds": round(prepare_s, 3),
        "cpu_baseline": cpu, "clocks": sampler.summary(),
        "files_differing_from_reference": mism,
    }
    print(json.dumps(line), flush=True)
    b.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--workload", default="c2_exact", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the split-precision and fast companions of the exact workloads")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="skip the autotuner (launch shapes per pass, chosen after warm-up, before timing)")
    ap.add_argument("--seconds", type=float, default=None,
                    help="shorter input of the same workload (profiling captures of a small case)")
    args = ap.parse_args()
    w = dict(WORKLOADS[args.workload])
    if args.seconds and "seconds" in w:
        w["seconds"] = args.seconds
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        reference_arm(args, w, world, rank, pg)
    elif w.get("batch"):
        batch_arm(args, w, world, rank, local, pg)
    else:
        product_arm(args, w, world, rank, local, pg)


if __name__ == "__main__":
    main()

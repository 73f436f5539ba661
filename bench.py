#!/usr/bin/env python
"""Benchmark of the TDD hot path on B200: DM-trials x samples per second.

Workload (one step = one dedispersion of the whole series): nchan 4096,
f_top 1500 MHz, channel width -0.078125 MHz, dt 64 us, 2^21 samples of 8-bit
input, DM list generate_dm_list(0, 2000, 40 us, 1.25) = 3643 DMs, max delay
35500, float32 output (3643 x 2061652 samples, 30 GB). Seeded synthetic input
(noise + 8 dispersed pulses) generated on the device; it is larger than L2,
so no flush is needed between steps.

  value  device-resident input and output (DEDISP_DEVICE_POINTERS), timed
         with CUDA events on the plan's stream: K1 transpose + K2 kernels.
  e2e    the C-ABI call dedisp_execute with pinned HOST buffers (H2D of the
         input and D2H of the 30 GB output inside the timed region), in gulps
         of --e2e-gulp output samples (set through dedisp_set_gulp_size).

N > 1 GPUs (torchrun): each rank runs its own replica of the workload (no
collective on the data path); value = all ranks' units / max-over-ranks time.

--impl reference times the reference's CPU implementation of this path (the
CPU oracle port: brute-force integer TDD, all host threads) on bounded samples
of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DM-trials x samples/s (TDD, 1 B200)"
UNIT = "DM-trials*samples/s"


def workload_name(nbits):
    return f"tdd 4096ch 2^21 samples {nbits}-bit, 3643 DMs (0-2000, 40us, tol 1.25), f32 out"


def workload_config(nbits, nsamps, ndm, md, world):
    """The `config` object of both arms' JSON lines."""
    return {"workload": workload_name(nbits), "nchans": 4096, "nsamps": nsamps, "ndm": ndm,
            "max_delay": md, "in_nbits": nbits, "out_nbits": 32,
            "l2": "inputs (8.6 GB) larger than L2; no flush", "parallelism": f"replicas x{world}"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nbits", type=int, default=8, choices=[2, 4, 8])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-gulp", type=int, default=1 << 18,
                    help="gulp size (dedisp_set_gulp_size) of the e2e call: with several gulps the "
                         "host copies of neighbouring gulps overlap each gulp's kernels")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fdd", action="store_true")
    ap.add_argument("--tile-variant", type=int, default=-1,
                    help="tiled-kernel tile shape for 8-bit input (-1: time all, use the fastest)")
    ap.add_argument("--fdd-only", action="store_true",
                    help="run only the FDD forms (config 2) and print their JSON object")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the streaming server (config 4) and print its JSON object")
    ap.add_argument("--batched-fdd-only", action="store_true",
                    help="run only the batched multi-beam FDD (config 3) and print its JSON object")
    ap.add_argument("--batched-only", action="store_true",
                    help="run only the batched multi-beam TDD (config 3) and print its JSON object")
    ap.add_argument("--profile-case", default="",
                    help="run one small case for ncu and exit: tdd (the TDD workload with "
                         "2^17 samples), fdd / fdd-tc (config-2 geometry with 2^18 samples, FP32 "
                         "or tensor-core MAC), fdd-tc-n80 (the tensor-core MAC's config-2 shape "
                         "per bin, 80 columns, on a few GB), fdd-series (config-2 geometry with "
                         "2^18 samples, whole-series spectrum, one-segment FP32 MAC)")
    return ap.parse_args()


def profile_case(args):
    """One execution of a reduced workload, sized for ncu captures: the same
    kernels and DM list as the benchmark, fewer samples."""
    import torch
    import dedisp_tests_b200 as dd
    from dedisp_tests_b200 import synthetic as sy
    if args.profile_case == "tdd":
        cfg = sy.config1(nbits=args.nbits, nsamps=1 << 17)
        p = dd.TDDPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
        p.generate_dm_list(*cfg.dm_gen)
        if args.tile_variant >= 0:
            p.set_tile_variant(args.tile_variant)
        nbits = args.nbits
    elif args.profile_case == "fdd-tc-n80":
        # the MAC's per-bin shape at config 2 (1024 channels = 16 chunks,
        # 2048 DMs = 16 tiles, 39 segments = 80 columns) on a few GB: DMs
        # 0-250 (max delay 1311), 8192-point segments, 39 x 6881 samples
        import dataclasses
        cfg = dataclasses.replace(sy.config2(), nsamps=39 * 6881,
                                  dm_list=(250.0 * np.arange(2048) / 2047.0).astype(np.float32))
        p = dd.FDDGPUPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
        p.set_dm_list(cfg.dm_list)
        p.set_options(segmented=1, precision=1, segment_nfft=8192)
        nbits = 32
    elif args.profile_case == "fdd-series":
        # whole-series spectrum, FP32 one-segment MAC: config 2 at 2^18
        # samples (N = 16384 x 17, 139264 bins)
        cfg = sy.config2(nsamps=1 << 18)
        p = dd.FDDGPUPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
        p.set_dm_list(cfg.dm_list)
        p.set_options(segmented=0, precision=0)
        nbits = 32
    else:
        cfg = sy.config2(nsamps=1 << 18)
        p = dd.FDDGPUPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
        p.set_dm_list(cfg.dm_list)
        p.set_options(segmented=1, precision=1 if args.profile_case == "fdd-tc" else 0)
        nbits = 32
    d_in = sy.make_input_torch(cfg)
    rows = p.output_row_length(cfg.nsamps)
    d_out = torch.empty((p.get_dm_count(), rows), dtype=torch.float32, device="cuda")
    for _ in range(2):
        p.execute(cfg.nsamps, d_in, nbits, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
    torch.cuda.synchronize()
    print("profile case done:", args.profile_case, cfg.nsamps, p.get_dm_count())


# ---------------------------------------------------------------------------
# CPU baseline (oracle port)
# ---------------------------------------------------------------------------

def cpu_sample(cfg, dms_all, md, n_dm=16, n_t=65536, seed=99):
    """A bounded sample of the workload: n_dm DMs spread over the list and
    n_t output samples (input rows n_t + max_delay, numpy generated)."""
    from dedisp_tests_b200 import synthetic as sy
    sub = sy.Config(cfg.name, cfg.nchans, cfg.f_top, cfg.df, cfg.dt, n_t + md, cfg.nbits,
                    cfg.mean, cfg.sigma, [], seed=seed)
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((sub.nsamps, sub.nchans), dtype=np.float32) * sub.sigma + sub.mean
    packed = sy.pack(sy.quantise(x, cfg.nbits), cfg.nbits)
    pick = np.linspace(0, len(dms_all) - 1, n_dm).astype(int)
    return packed, dms_all[pick], n_t


def time_cpu_oracle(cfg, dms_all, md, steps=1, warmup=0, n_dm=16, n_t=65536):
    from oracle import pyoracle as po
    packed, dms, n_t = cpu_sample(cfg, dms_all, md, n_dm, n_t)
    delays = po.delay_table(cfg.nchans, np.float32(cfg.dt), np.float32(cfg.f_top),
                            np.float32(cfg.df))
    km = np.ones(cfg.nchans, np.int32)
    cores = os.cpu_count() or 1
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        po.tdd(packed, packed.shape[0], packed.shape[1], cfg.nbits, cfg.nchans, delays, km, dms,
               32, n_t, nthreads=cores)
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    t = sum(times) / len(times)
    return {"value": len(dms) * n_t / t, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{len(dms)} DMs spread over the 3643-DM list x {n_t} output samples "
                      f"x 4096 channels ({cfg.nbits}-bit), oracle brute force, "
                      f"{len(times)} timed runs of {t:.2f} s"}, t


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


# ---------------------------------------------------------------------------
# FDD forms (plain FP32 CUDA-core MAC vs 3xBF16 tensor-core MAC)
# ---------------------------------------------------------------------------

def delay_table_f32(nchans, dt, f0, df):
    """The plan's per-channel delay table, in the same float32 operation order
    (df forced negative; a = 1/(f0 + c df); (float)(4.15e3/dt * (a^2 - b^2)))."""
    f0 = np.float32(f0)
    df = -np.abs(np.float32(df))
    c = np.arange(nchans, dtype=np.float32)
    a = np.float32(1.0) / (f0 + c * df)
    b = np.float32(1.0) / f0
    diff = a * a - b * b
    return (4.15e3 / np.float64(np.float32(dt)) * diff.astype(np.float64)).astype(np.float32)


def fdd_fp64_rows(x_tc, delays, dms, nout):
    """Dedispersed time series in float64 for a few DMs: sum_c x[c][t + d],
    d = trunc(float32(dm * delay[c])) (the FDD plan's delay rule); x_tc is
    the unpacked input [nsamps][nchans] (float32, already scaled)."""
    out = np.zeros((len(dms), nout), np.float64)
    for i, dm in enumerate(dms):
        d = np.trunc(np.float32(dm) * delays).astype(np.int64)
        for c in range(x_tc.shape[1]):
            out[i] += x_tc[d[c]:d[c] + nout, c]
    return out


def _time_cufft(shape_in, inverse, n, dev, stream, reps=3):
    """cuFFT (torch.fft) comparator: ms per batched real transform of the
    given input shape (real rows of n points, or complex rows of n/2 + 1
    bins for the inverse), CUDA events on the bench stream."""
    import torch
    if inverse:
        x = torch.randn(shape_in, dtype=torch.complex64, device=dev)
        f = lambda: torch.fft.irfft(x, n=n)  # noqa: E731
    else:
        x = torch.randn(shape_in, dtype=torch.float32, device=dev)
        f = lambda: torch.fft.rfft(x)  # noqa: E731
    y = f()
    del y
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    ts = []
    for _ in range(reps):
        e0.record(stream)
        y = f()
        e1.record(stream)
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
        del y
    del x
    torch.cuda.empty_cache()
    return min(ts)


def _fdd_run(dd, cfg, d_in, in_nbits, dm_list, local, stream, steps, warm, **opts):
    """One FDD plan on device buffers: mean device ms per execute over
    `steps` timed executes, the MAC and stage times of the last, the plan
    and its output."""
    import torch
    p = dd.FDDGPUPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df, local)
    p.set_dm_list(dm_list)
    p.set_options(**opts)
    p.set_stream(stream.cuda_stream)
    p.set_timing(True)
    nout = p.output_row_length(cfg.nsamps)
    d_out = torch.empty((len(dm_list), nout), dtype=torch.float32, device=f"cuda:{local}")
    for _ in range(warm):
        p.execute(cfg.nsamps, d_in, in_nbits, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kms, launches = [], 0
    e0.record(stream)
    for _ in range(steps):
        p.execute(cfg.nsamps, d_in, in_nbits, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
        t = p.get_timing()
        kms.append(t["kernel_ms"])
        launches += t["launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    return p, d_out, e0.elapsed_time(e1) / steps, sum(kms) / len(kms), launches / steps, p.get_stage_times()


def run_fdd(args, local, world, stream, max_over_ranks):
    """Config 2: 1024 ch, 2^20 float32 samples, 2048 DMs over 0-1000,
    device-resident. (a) Segmented with 2^15-sample FFTs (39 segments), both
    MAC forms, error against float64 on a DM subset; (b) the same geometry
    with 8-bit samples and TDD's round-half-even delays against the TDD
    plan's output; (c) the whole-series spectrum (the fork's default output,
    N = round_up(2^20 + 5243, 16384) = 1064960 = 16384 x 65) on tensor cores,
    error against float64 on two DMs; (d) cuFFT (torch.fft) on the same
    transform shapes beside this library's FFT stage times."""
    import dataclasses
    import torch
    import dedisp_tests_b200 as dd
    from dedisp_tests_b200 import synthetic as sy
    from oracle import pyoracle as po
    dev = f"cuda:{local}"
    cfg = sy.config2()
    d_in = sy.make_input_torch(cfg, device=dev)
    # float64 check on 4 DMs over the first 2^17 output samples
    h_in = d_in.cpu().numpy().view(np.float32).reshape(cfg.nsamps, cfg.nchans)
    scale = np.float32(1.0 / cfg.nchans)
    delays = delay_table_f32(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
    dm_list = np.asarray(cfg.dm_list, np.float32)
    rows = np.array([1, 700, 1400, 2047])
    n_chk = 1 << 17
    x_tc = None
    out = {}
    steps = max(1, min(args.steps, 3))
    for name, prec in (("fdd_fp32_plain", 0), ("fdd_bf16x3_tc", 1)):
        p, d_out, ms, mac_ms, launches, stages = _fdd_run(
            dd, cfg, d_in, 32, dm_list, local, stream, steps, max(1, min(args.warmup, 2)),
            segmented=1, precision=prec, segment_nfft=1 << 15)
        ms = max_over_ranks(ms)
        ndm, md = p.get_dm_count(), p.get_max_delay()
        nout = p.output_row_length(cfg.nsamps)
        units = ndm * nout
        nseg = -(-cfg.nsamps // ((1 << 15) - md))
        nbins = (1 << 15) // 2 + 1
        cmac = float(ndm) * cfg.nchans * nseg * nbins
        if x_tc is None:
            x_tc = h_in[: n_chk + md] * scale
            ref = fdd_fp64_rows(x_tc, delays, dm_list[rows], n_chk)
        got = d_out[torch.as_tensor(rows, device=d_out.device), :n_chk].double().cpu().numpy()
        rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        mx = float(np.abs(got - ref).max() / np.abs(ref).max())
        if prec == 0:
            roof = {"bound": "fp32-fma", "flop": 8 * cmac,
                    "achieved_TFLOPs": round(8 * cmac / (mac_ms * 1e-3) / 1e12, 2),
                    "note": "8 real flops per complex MAC on CUDA cores"}
        else:
            # the burst figure: the MAC is timed alone (fallback: the earlier
            # measurement on this pool when the peaks file is absent)
            peak = measured_peaks().get("bf16_tflops")
            src = "MEASURED_PEAKS.json bf16_tflops (cuBLAS bf16 GEMM, burst), of measured"
            if not peak:
                peak, src = 1590.0, "fallback 1590 TFLOP/s (earlier measurement), of fallback"
            ach = 24 * cmac / (mac_ms * 1e-3) / 1e12
            roof = {"bound": "tensor", "flop": 24 * cmac, "achieved_TFLOPs": round(ach, 2),
                    "peak_TFLOPs": peak, "frac": round(ach / peak, 4), "peak_source": src,
                    "note": "3 bf16 real GEMMs [ndm x 2nact] x [2nact x 2nseg] per bin"}
        out[name] = {"value": units * world / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                     "mac_ms": mac_ms, "launches_per_step": launches,
                     "stage_ms": {k: round(v, 3) for k, v in stages.items()},
                     "rel_l2_vs_fp64": rel, "max_abs_vs_fp64": mx,
                     "error_sample": f"DMs {rows.tolist()} x first {n_chk} samples",
                     "roofline": roof, "ndm": ndm, "nseg": nseg, "nfft": 1 << 15,
                     "max_delay": md}
        del d_out, p
        torch.cuda.empty_cache()
    # (d) cuFFT on the segmented shapes: 1024 x 39 real rows of 32768 forward,
    # 2048 x 39 rows of 16385 bins inverse
    nseg = out["fdd_bf16x3_tc"]["nseg"]
    out["cufft_comparator"] = {
        "segmented_r2c_ms": _time_cufft((cfg.nchans * nseg, 1 << 15), False, 1 << 15, dev, stream),
        "segmented_c2r_ms": _time_cufft((2048 * nseg, (1 << 14) + 1), True, 1 << 15, dev, stream),
        "ours_segmented_r2c_ms": out["fdd_bf16x3_tc"]["stage_ms"]["fft_fwd"],
        "ours_segmented_c2r_ms": out["fdd_bf16x3_tc"]["stage_ms"]["fft_inv"],
        "note": "torch.fft (cuFFT) batched real transforms of the same lengths and row counts, "
                "contiguous rows; ours read overlapping segments (r2c) and write the stitched "
                "series (c2r)"}

    # (c) whole-series spectrum (N = 1064960; the fork's default output): the
    # default FP32 form (one-segment MAC) and the tensor-core form
    wrows = np.array([3, 1500])
    x_full = np.ascontiguousarray((h_in * scale).T)
    spec_ref = None
    for name, prec in (("fdd_fp32_whole_series_spectrum", 0), ("fdd_bf16x3_tc_whole_series_spectrum", 1)):
        p, d_out, ms, mac_ms, launches, stages = _fdd_run(
            dd, cfg, d_in, 32, dm_list, local, stream, steps, 1, segmented=0, precision=prec)
        ms = max_over_ranks(ms)
        md = p.get_max_delay()
        nfft = p.output_row_length(cfg.nsamps)
        units = 2048 * (cfg.nsamps - md)
        if spec_ref is None:
            spec_ref = po.fdd_spectrum(x_full, delays, np.ones(cfg.nchans, np.int32), dm_list[wrows], nfft)
        got = d_out[torch.as_tensor(wrows, device=d_out.device)].double().cpu().numpy()
        cmac = 2048.0 * cfg.nchans * (nfft // 2 + 1)
        out[name] = {
            "value": units * world / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "mac_ms": mac_ms,
            "stage_ms": {k: round(v, 3) for k, v in stages.items()}, "nfft": nfft,
            "rel_l2_vs_fp64": float(np.linalg.norm(got - spec_ref) / np.linalg.norm(spec_ref)),
            "max_abs_vs_fp64": float(np.abs(got - spec_ref).max() / np.abs(spec_ref).max()),
            "error_sample": f"DMs {wrows.tolist()}, all {nfft // 2} bins"}
        if prec == 1:
            out[name]["mac_TFLOPs"] = round(24 * cmac / (mac_ms * 1e-3) / 1e12, 2)
            out[name]["note"] = ("one series: 2 of the MMA's 16 columns carry data, so the MAC is "
                                 "bound by phasor generation, not the tensor pipe")
            out[name]["cufft_r2c_ms"] = _time_cufft((cfg.nchans, nfft), False, nfft, dev, stream)
        else:
            out[name]["mac_TFLOPs"] = round(8 * cmac / (mac_ms * 1e-3) / 1e12, 2)
            out[name]["note"] = ("one-segment FP32 MAC: per-bin phasor table, 8 real flops per "
                                 "complex MAC on CUDA cores")
        del d_out, p
        torch.cuda.empty_cache()
    del x_full

    # (b) against the TDD plan: config-2 geometry with 8-bit samples
    cfg8 = dataclasses.replace(cfg, nbits=8, mean=127.5, sigma=24.0, float_input=False,
                               pulses=[dataclasses.replace(q, amp=q.amp * 24.0) for q in cfg.pulses])
    del d_in
    d8 = sy.make_input_torch(cfg8, device=dev)
    t = dd.TDDPlan(cfg8.nchans, cfg8.dt, cfg8.f_top, cfg8.df, local)
    t.set_dm_list(dm_list)
    nout = cfg8.nsamps - t.get_max_delay()
    trows = torch.arange(0, 2048, 64, device=dev)
    tdd_out = torch.empty((2048, nout), dtype=torch.float32, device=dev)
    t.execute(cfg8.nsamps, d8, 8, tdd_out, 32, dd.DEDISP_DEVICE_POINTERS)
    den = float(np.float32(255.0) * np.float32(cfg8.nchans))
    factor = float(np.float32(3.0 * 1024.0 / 255.0 / 16.0))
    want = ((torch.round(tdd_out[trows].double() * den / factor) - 127.5 * cfg8.nchans) / cfg8.nchans)
    del tdd_out, t
    torch.cuda.empty_cache()
    vs = {}
    for name, prec in (("fp32_plain", 0), ("bf16x3_tc", 1)):
        p, d_out, _, _, _, _ = _fdd_run(dd, cfg8, d8, 8, dm_list, local, stream, 1, 0, segmented=1,
                                        precision=prec, segment_nfft=1 << 15, round_delays=True)
        got = d_out[trows].double()
        vs[name] = {"rel_l2": float(torch.linalg.norm(got - want) / torch.linalg.norm(want)),
                    "max_abs": float((got - want).abs().max() / want.abs().max())}
        del d_out, p, got
        torch.cuda.empty_cache()
    out["vs_tdd_plan"] = dict(vs, sample=f"config-2 geometry with 8-bit samples (24 levels per sigma), "
                                         f"round-half-even delays, 32 DMs (every 64th) x all "
                                         f"{nout} samples; TDD sums decoded exactly from the "
                                         f"plan's float output")
    del d8, want
    torch.cuda.empty_cache()
    return out


def run_batched(args, local, world, stream, max_over_ranks):
    """Config 3: 96 beams of 1536 ch (8-bit), each with its own sample count,
    DM range and trial count, dedispersed by the batch engine (one persistent
    launch per wave of beams, each wave a replayed CUDA graph, tile shape
    from the autotuner). Outputs of a wave go to a device pool that the next
    wave reuses (all outputs together, 577 GB, exceed HBM; a consumer would
    take each wave's rows before the next). The plain single-beam form and
    per-beam tiled plans are timed on the first four beams."""
    import torch
    import dedisp_tests_b200 as dd
    from dedisp_tests_b200 import synthetic as sy
    beams = sy.config3()
    c0 = beams[0]
    dev = f"cuda:{local}"
    mds = []
    for c in beams:
        p = dd.TDDPlan(c.nchans, c.dt, c.f_top, c.df)
        p.set_dm_list(c.dm_list)
        mds.append(p.get_max_delay())
        p.close()
    nouts = [c.nsamps - m for c, m in zip(beams, mds)]
    units = [len(c.dm_list) * n for c, n in zip(beams, nouts)]
    out_bytes = [u * 4 for u in units]
    d_in = [sy.make_input_torch(c, device=dev) for c in beams]
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info(local)
    budget = free - 12e9  # output pool + transposed-input workspace
    # workspace per beam: channel-major packed rows (1x the input) plus the
    # quad-strided rows of the quad variants (4x), with padding
    in_bytes = [x.numel() * 5.3 for x in d_in]

    def partition(cap):
        waves, cur, acc = [], [], 0.0
        for i in range(len(beams)):
            cost = out_bytes[i] + in_bytes[i]
            if cur and acc + cost > cap:
                waves.append(cur)
                cur, acc = [], 0.0
            cur.append(i)
            acc += cost
        waves.append(cur)
        return waves

    cap = budget
    while True:
        waves = partition(cap)
        need = (max(sum(out_bytes[i] for i in w) for w in waves) +
                max(sum(in_bytes[i] for i in w) for w in waves))
        if need <= budget or cap < 1e9:
            break
        cap *= 0.9
    pool = torch.empty(max(sum(out_bytes[i] for i in w) for w in waves), dtype=torch.uint8, device=dev)
    batches = []
    for w in waves:
        b = dd.Batch(c0.nchans, c0.dt, c0.f_top, c0.df, in_nbits=8, out_nbits=32, device=local)
        spec, off = [], 0
        for i in w:
            c = beams[i]
            y = pool[off:off + out_bytes[i]]
            off += out_bytes[i]
            spec.append((d_in[i], c.nchans, c.nsamps, c.dm_list, y, nouts[i] * 4))
        b.set_beams(spec)
        batches.append(b)
    ws_bytes = max(b.workspace_size() for b in batches)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    for b in batches:
        b.set_workspace(ws, ws_bytes)
    shape = batches[0].autotune(stream.cuda_stream)
    for b in batches:
        b.set_shape(*shape)

    def batched_step():
        for b in batches:
            b.execute(stream.cuda_stream, use_graph=True)

    batched_step()  # warm-up: captures each wave's graph
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    steps = 1
    e0.record(stream)
    for _ in range(steps):
        batched_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1)) / steps
    total_units = float(sum(units))
    # kernels per graph: K1d (quad-strided rows) or K1 per beam + 1
    launches_per_step = sum(b.get_timing()["launches"] for b in batches)
    res = {"workload": "96 beams x 1536 ch 8-bit, nsamp U[2^17,2^20], DM max U[500,3000], "
                       "ndm U[1024,4096] linear (seeded), f32 out",
           "units": total_units, "waves": len(waves), "beams_per_wave": [len(w) for w in waves],
           "shape": {"variant": shape[0], "chan_per_stage": shape[1]},
           "batched": {"value": total_units * world / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
                       "launches_per_step": launches_per_step}}
    for b in batches:
        b.close()
    del pool, ws, batches, spec, y
    torch.cuda.empty_cache()

    # single-beam comparators: tiled plans on the first 24 beams, the plain
    # (reference-decomposition) kernel on the first 8 (about 10x slower)
    for name, kernel, nsub in (("plain_single_beam", 1, 8), ("tiled_single_beam", 2, 24)):
        sub = list(range(nsub))
        sub_units = float(sum(units[i] for i in sub))
        # one output buffer, overwritten beam after beam (a consumer would
        # take each beam's rows in between)
        ybuf = torch.empty(max(units[i] for i in sub), dtype=torch.float32, device=dev)
        outs = [ybuf[:units[i]].view(len(beams[i].dm_list), nouts[i]) for i in sub]
        # one plan at a time (each holds its own rows workspace), timed
        # after its own warm-up; the times add up
        t = 0.0
        for i in sub:
            c = beams[i]
            p = dd.TDDPlan(c.nchans, c.dt, c.f_top, c.df, local)
            p.set_dm_list(c.dm_list)
            p.set_kernel(kernel)
            p.set_stream(stream.cuda_stream)
            y = outs[sub.index(i)]
            if kernel == 2:
                p.execute(c.nsamps, d_in[i], 8, y, 32, dd.DEDISP_DEVICE_POINTERS)  # warm-up
            torch.cuda.synchronize()
            e0.record(stream)
            p.execute(c.nsamps, d_in[i], 8, y, 32, dd.DEDISP_DEVICE_POINTERS)
            e1.record(stream)
            torch.cuda.synchronize()
            t += max_over_ranks(e0.elapsed_time(e1))
            p.close()
            del p
        res[name] = {"value": sub_units * world / (t * 1e-3), "unit": UNIT, "ms": t,
                     "sample": f"beams 0-{nsub - 1} ({sub_units:.3e} DM-trials x samples), one plan "
                               f"execute per beam"}
        del outs, ybuf
        torch.cuda.empty_cache()
    res["batched_vs_plain"] = res["batched"]["value"] / res["plain_single_beam"]["value"]
    res["batched_vs_tiled_single_beam"] = res["batched"]["value"] / res["tiled_single_beam"]["value"]
    del d_in
    torch.cuda.empty_cache()
    return res


def run_batched_fdd(args, local, world, stream, max_over_ranks, nbeams=12, nplain=4):
    """Config 3, Fourier domain: the first `nbeams` of the 96 seeded beams
    (1536 ch, 8-bit, nsamp U[2^17, 2^20], DM max U[500, 3000], 1024-4096
    linear trials), segmented time series. Batched: FddBatch objects in waves
    sized to the free memory, each one replayed CUDA graph with one persistent
    tensor-core MAC launch over all its beams per MMA-form class (segment
    groups of at most 32 MMA columns and wider ones). Compared with one FDD plan
    execute per beam on the same beams: tensor-core plans, and plain FP32
    plans on the first `nplain`. Both tensor-core forms run with the reference
    segment rule and with the automatic one (the segment length with the least
    modelled device time; the same series, other rounding)."""
    import torch
    import dedisp_tests_b200 as dd
    from dedisp_tests_b200 import synthetic as sy
    dev = f"cuda:{local}"
    beams = sy.config3()[:nbeams]
    c0 = beams[0]
    mds = []
    for c in beams:
        p = dd.TDDPlan(c.nchans, c.dt, c.f_top, c.df)
        p.set_dm_list(c.dm_list)
        mds.append(p.get_max_delay())
        p.close()
    nouts = [c.nsamps - m for c, m in zip(beams, mds)]
    units = [len(c.dm_list) * n for c, n in zip(beams, nouts)]
    out_bytes = [u * 4 for u in units]
    d_in = [sy.make_input_torch(c, device=dev) for c in beams]
    torch.cuda.synchronize()
    total = float(sum(units))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def spec(i, y):
        c = beams[i]
        return (d_in[i], c.nchans, c.nsamps, c.dm_list, y, nouts[i] * 4)

    def batched(seg):
        free, _ = torch.cuda.mem_get_info(local)
        budget = free - 8e9
        # waves: add beams while workspace + outputs fit the budget
        probe = torch.empty(16, dtype=torch.uint8, device=dev)  # stand-in output (sizing only)
        waves, cur = [], []
        for i in range(nbeams):
            trial = cur + [i]
            b = dd.FddBatch(c0.nchans, c0.dt, c0.f_top, c0.df, in_nbits=8, device=local)
            b.set_segment_nfft(seg)
            b.set_beams([spec(j, probe) for j in trial])
            need = b.workspace_size() + sum(out_bytes[j] for j in trial)
            b.close()
            if cur and need > budget / 1.05:
                waves.append(cur)
                cur = [i]
            else:
                cur = trial
        waves.append(cur)
        pool = torch.empty(max(sum(out_bytes[j] for j in w) for w in waves), dtype=torch.uint8, device=dev)
        batches, bsources = [], {}
        for w in waves:
            b = dd.FddBatch(c0.nchans, c0.dt, c0.f_top, c0.df, in_nbits=8, device=local)
            b.set_segment_nfft(seg)
            sp, off = [], 0
            for j in w:
                sp.append(spec(j, pool[off:off + out_bytes[j]]))
                off += out_bytes[j]
            b.set_beams(sp)
            for j in range(len(w)):
                src = b.phasor_source(j)
                bsources[src] = bsources.get(src, 0) + 1
            batches.append(b)
        ws_bytes = max(b.workspace_size() for b in batches)
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        for b in batches:
            b.set_workspace(ws, ws_bytes)

        def batched_step():
            for b in batches:
                b.execute(stream.cuda_stream, use_graph=True)

        batched_step()  # warm-up: captures each wave's graph
        for b in batches:
            b.sync(stream.cuda_stream)
        e0.record(stream)
        batched_step()
        e1.record(stream)
        for b in batches:
            b.sync(stream.cuda_stream)
        ms = max_over_ranks(e0.elapsed_time(e1))
        r = {"value": total * world / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
             "waves": len(waves), "beams_per_wave": [len(w) for w in waves]}
        # error of the last wave's first beam (the pool holds the last wave's
        # rows) against float64 on two DMs x 2^16 samples
        bi = waves[-1][0]
        y0 = pool[:out_bytes[bi]].view(torch.float32).view(len(beams[bi].dm_list), -1)
        c = beams[bi]
        nchk = min(1 << 16, nouts[bi])
        h = d_in[bi][:nchk + mds[bi]].cpu().numpy()
        x = (h.astype(np.float32) - np.float32(127.5)) * np.float32(1.0 / c.nchans)
        delays = delay_table_f32(c.nchans, c.dt, c.f_top, c.df)
        drows = np.array([len(c.dm_list) // 3, len(c.dm_list) - 1])
        ref = fdd_fp64_rows(x, delays, np.asarray(c.dm_list, np.float32)[drows], nchk)
        got = y0[torch.as_tensor(drows, device=dev), :nchk].double().cpu().numpy()
        r["rel_l2_vs_fp64"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        r["max_abs_vs_fp64"] = float(np.abs(got - ref).max() / np.abs(ref).max())
        r["error_sample"] = f"beam {bi}, DMs {drows.tolist()} x first {nchk} samples"
        # stage split of one more step (direct launches with events, untimed above)
        split = {"prep_ms": 0.0, "mac_ms": 0.0, "post_ms": 0.0}
        balance = []
        nlaunch = 0
        for b in batches:
            b.set_timing(True)
            b.execute(stream.cuda_stream, use_graph=False)
            t = b.get_timing()
            bal = b.get_mac_balance()
            b.set_timing(False)
            for k in split:
                split[k] += t[k]
            nlaunch += t["launches"]
            balance.append([round(bal["cta_max_ms"], 1), round(bal["cta_mean_ms"], 1)])
        r["launches_per_step"] = nlaunch
        r["stage_ms"] = {k: round(v, 2) for k, v in split.items()}
        r["mac_cta_max_mean_ms"] = balance
        r["phasor_sources"] = bsources
        for b in batches:
            b.close()
        del pool, ws, batches
        torch.cuda.empty_cache()
        return r

    def single(prec, sub, seg):
        """One plan execute per beam (each timed after its own warm-up)."""
        tms, su, stage_sum, sources = 0.0, 0.0, {"prep_ms": 0.0, "mac_ms": 0.0, "post_ms": 0.0}, {}
        for i in sub:
            c = beams[i]
            p = dd.FDDGPUPlan(c.nchans, c.dt, c.f_top, c.df, local)
            p.set_dm_list(c.dm_list)
            p.set_options(segmented=1, precision=prec, segment_nfft=seg)
            p.set_stream(stream.cuda_stream)
            y = torch.empty((len(c.dm_list), nouts[i]), dtype=torch.float32, device=dev)
            p.execute(c.nsamps, d_in[i], 8, y, 32, dd.DEDISP_DEVICE_POINTERS)  # warm-up (allocation)
            torch.cuda.synchronize()
            e0.record(stream)
            p.execute(c.nsamps, d_in[i], 8, y, 32, dd.DEDISP_DEVICE_POINTERS)
            e1.record(stream)
            torch.cuda.synchronize()
            tms += max_over_ranks(e0.elapsed_time(e1))
            su += units[i]
            # stage split and phasor source from one more (timed-stage) execute
            p.set_timing(True)
            p.execute(c.nsamps, d_in[i], 8, y, 32, dd.DEDISP_DEVICE_POINTERS)
            st_ms = p.get_stage_times()
            stage_sum["mac_ms"] += st_ms["mac"]
            stage_sum["prep_ms"] += st_ms["unpack"] + st_ms["fft_fwd"] + st_ms["layout"]
            stage_sum["post_ms"] += st_ms["transpose"] + st_ms["fft_inv"]
            if prec == 1:
                src = p.get_phasor_source()
                sources[src] = sources.get(src, 0) + 1
            p.close()
            del y
            torch.cuda.empty_cache()
        r = {"value": su * world / (tms * 1e-3), "unit": UNIT, "ms": tms,
             "sample": f"beams {sub[0]}-{sub[-1]} ({su:.3e} DM-trials x samples), one plan "
                       f"execute per beam (each plan timed after its own warm-up)",
             "stage_ms": {k: round(v, 2) for k, v in stage_sum.items()}}
        if prec == 1:
            r["phasor_sources"] = sources
        return r

    res = {"workload": f"first {nbeams} of the 96 config-3 beams (1536 ch 8-bit, seeded), segmented "
                       f"FDD, f32 time-series out", "units": total}
    res["batched_bf16x3_tc"] = batched(0)
    res["batched_bf16x3_tc"]["segments"] = "reference rule"
    _log("batched fdd (reference segments) done")
    res["batched_bf16x3_tc_auto_segments"] = batched("auto")
    res["batched_bf16x3_tc_auto_segments"]["segments"] = "automatic (least modelled time)"
    _log("batched fdd (automatic segments) done")
    res["tc_single_beam"] = single(1, list(range(nbeams)), 0)
    res["tc_single_beam_auto_segments"] = single(1, list(range(nbeams)), "auto")
    res["plain_fp32_single_beam"] = single(0, list(range(nplain)), 0)
    _log("per-beam fdd plans done")
    res["batched_vs_plain_fp32"] = res["batched_bf16x3_tc"]["value"] / res["plain_fp32_single_beam"]["value"]
    res["batched_vs_tc_single_beam"] = res["batched_bf16x3_tc"]["value"] / res["tc_single_beam"]["value"]
    res["batched_auto_vs_plain_fp32"] = (res["batched_bf16x3_tc_auto_segments"]["value"] /
                                         res["plain_fp32_single_beam"]["value"])
    res["batched_auto_vs_tc_single_beam_auto"] = (res["batched_bf16x3_tc_auto_segments"]["value"] /
                                                  res["tc_single_beam_auto_segments"]["value"])
    del d_in
    torch.cuda.empty_cache()
    return res


def run_serving(args, local, world):
    """Config 4: 32 beams of 4096 ch 2-bit (f_top 1500 MHz, df -0.078125 MHz,
    dt 64 us), 2048 DM trials over 0-1500, through the streaming server: 28
    TDD beams (gulps of 16384, 65536 or 262144 samples) and 4 FDD beams (3xBF16
    tensor-core MAC, gulps of 16384 or 65536). FDD segments are 32768 points,
    the shortest above the 26616-sample overlap tail: the MAC's cost is set by
    its phasors, one per (DM, channel, bin) and shared by all segments, so it
    grows with the bins of a segment (nfft / 2), not with the segment count
    (65536-point segments measured 2x slower per gulp). Gulps arrive as a Poisson process at 1x, 2x, 4x
    and 8x the aggregate real-time sample rate (32 x 15625 samples/s) for a
    fixed window each (20 s: at least 100 gulps per rate, so p99 is not the
    maximum); outputs stay on the device (a GPU consumer reads each worker's
    buffer). All beams read the same pinned host gulp (its contents do not
    affect the work). Per worker: the fraction of the window it was busy
    (host clock, start to done) and its device time."""
    import torch
    import dedisp_tests_b200 as dd
    from dedisp_tests_b200 import synthetic as sy
    nch, f0, df, dt, nbits = 4096, 1500.0, -0.078125, 64e-6, 2
    dms = (1500.0 * np.arange(2048) / 2047.0).astype(np.float32)
    nbeams, n_fdd = 32, 4
    sizes_tdd, sizes_fdd = [16384, 65536, 262144], [16384, 65536]
    srv = dd.StreamServer(nch, dt, f0, df, in_nbits=nbits, device=local, hbm_budget=int(120e9),
                          max_gulp=max(sizes_tdd), tdd_workers=4, fdd_workers=1, fdd_precision=1,
                          fdd_segment=32768, fdd_max_gulp=max(sizes_fdd))
    kinds = [0] * (nbeams - n_fdd) + [1] * n_fdd
    for k in kinds:
        srv.add_beam(dms, k)
    held = srv.start()
    cfg = sy.Config("serve-gulp", nch, f0, df, dt, max(sizes_tdd), nbits, 1.5, 1.0,
                    [sy.Pulse(700.0, 8.0, 1e-3, 3.0)], seed=20261207)
    host = torch.empty((cfg.nsamps, nch * nbits // 8), dtype=torch.uint8, pin_memory=True)
    host.copy_(sy.make_input_torch(cfg, device=f"cuda:{local}").cpu())
    rt_rate = nbeams * 15625.0
    rng = np.random.default_rng(7)
    window = float(os.environ.get("DEDISP_SERVE_WINDOW_S", "20"))
    out = {"workload": "32 beams x 4096 ch 2-bit, 2048 DMs 0-1500, 28 TDD + 4 FDD beams",
           "hbm_budget_bytes": int(120e9), "device_bytes_held": held, "workers": "4 TDD (ids 0-3) + 1 FDD (id 4)",
           "window_s": window, "rates": {}}
    mean_n = ((nbeams - n_fdd) * np.mean(sizes_tdd) + n_fdd * np.mean(sizes_fdd)) / nbeams
    for rate in (1, 2, 4, 8):
        lam = rate * rt_rate / mean_n
        n0 = len(srv.records())
        t0 = time.perf_counter()
        t_next = t0
        while True:
            t_next += rng.exponential(1.0 / lam)
            if t_next - t0 > window:
                break
            b = int(rng.integers(0, nbeams))
            n = int(rng.choice(sizes_tdd if kinds[b] == 0 else sizes_fdd))
            dly = t_next - time.perf_counter()
            if dly > 0:
                time.sleep(dly)
            srv.submit(b, host, n)
        srv.drain()
        recs = srv.records()[n0:]
        lat = np.array([r["t_done"] - r["t_submit"] for r in recs])
        samples = float(sum(r["nsamps"] for r in recs))
        wall = max(r["t_done"] for r in recs) - min(r["t_submit"] for r in recs)
        out["rates"][f"{rate}x"] = {
            "gulps": len(recs), "samples": samples,
            "latency_p50_ms": float(np.percentile(lat, 50) * 1e3),
            "latency_p99_ms": float(np.percentile(lat, 99) * 1e3),
            "throughput": samples * len(dms) / wall, "unit": UNIT,
            "real_time_factor": samples / wall / rt_rate,
            "offered_real_time_factor": float(rate),
            "worker_busy_fraction": {
                str(w): round(sum(r["t_done"] - r["t_start"] for r in recs if r["worker"] == w) / wall, 3)
                for w in sorted({r["worker"] for r in recs})},
            "worker_device_fraction": {
                str(w): round(sum(r["device_ms"] for r in recs if r["worker"] == w) * 1e-3 / wall, 3)
                for w in sorted({r["worker"] for r in recs})}}
    srv.close()
    del host
    torch.cuda.empty_cache()
    return out


def _log(msg):
    """Progress on stderr (the JSON line is the only stdout)."""
    print(f"[bench {time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------

def run_ours(args):
    import torch
    import dedisp_tests_b200 as dd
    from dedisp_tests_b200 import synthetic as sy

    from dedisp_tests_b200.replicas import Replicas
    reps = Replicas.from_env("nccl")
    world, rank, local = reps.world, reps.rank, reps.local
    barrier, max_over_ranks = reps.barrier, reps.max_over_ranks
    if world > 1 and not (args.serve_only or args.batched_fdd_only or args.batched_only or args.fdd_only):
        # several GPUs: the headline workload (replicas) only; the one-GPU
        # sections (FDD forms, batches, serving, input widths) would hold
        # every GPU for minutes without adding to the scaling figure
        args.no_fdd = args.no_batched = args.no_serve = args.no_variants = True

    stream = torch.cuda.current_stream()
    if args.serve_only:
        res = run_serving(args, local, world)
        if rank == 0:
            print(json.dumps({"serving": res}), flush=True)
        reps.close()
        return
    if args.batched_fdd_only:
        resf = run_batched_fdd(args, local, world, stream, max_over_ranks)
        if rank == 0:
            print(json.dumps({"batched_fdd": resf}), flush=True)
        reps.close()
        return
    if args.batched_only:
        res = run_batched(args, local, world, stream, max_over_ranks)
        resf = run_batched_fdd(args, local, world, stream, max_over_ranks)
        if rank == 0:
            print(json.dumps({"batched": res, "batched_fdd": resf}), flush=True)
        reps.close()
        return
    if args.fdd_only:
        fdd = run_fdd(args, local, world, stream, max_over_ranks)
        if rank == 0:
            print(json.dumps({"fdd": fdd}), flush=True)
        reps.close()
        return

    cfg = sy.config1(nbits=args.nbits)

    def make_plan(kernel=0):
        p = dd.TDDPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df, local)
        p.generate_dm_list(*cfg.dm_gen)
        p.set_stream(stream.cuda_stream)
        if kernel:
            p.set_kernel(kernel)
        return p

    plan = make_plan()
    ndm, md = plan.get_dm_count(), plan.get_max_delay()
    nout = cfg.nsamps - md
    units = ndm * nout
    d_in = sy.make_input_torch(cfg, device=f"cuda:{local}")
    d_out = torch.empty((ndm, nout), dtype=torch.float32, device=f"cuda:{local}")
    flags = dd.DEDISP_DEVICE_POINTERS

    def step(p, nbits=args.nbits, inp=d_in):
        p.execute(cfg.nsamps, inp, nbits, d_out, 32, flags)

    # --- tile shape: pick the fastest tiled-kernel variant on this workload ---
    tune = {}
    if args.nbits == 8 and args.tile_variant < 0:
        plan.set_timing(True)
        for v in range(dd.tdd_variant_count(8)):
            plan.set_tile_variant(v)
            step(plan)
            step(plan)
            t = plan.get_timing()
            # whole device step: K1d (quad-strided variants) or K1, then K2
            tune[v] = t["kernel_ms"] + t["prep_ms"]
        best = min(tune, key=tune.get)
    else:
        best = max(args.tile_variant, 0)
    plan.set_tile_variant(best)

    # --- value: device-resident ---------------------------------------------
    plan.set_timing(True)
    for _ in range(args.warmup):
        step(plan)
    torch.cuda.synchronize()
    barrier()
    kms, pms, launches = [], [], 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            step(plan)
            t = plan.get_timing()
            kms.append(t["kernel_ms"])
            pms.append(t["prep_ms"])
            launches += t["launches"]  # K1 transposes and K2 launches
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    clocks = clk.summary()
    ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    value = units * world / (ms * 1e-3)

    # --- roofline of the dominant kernel (K2) --------------------------------
    import ctypes as C
    peak = C.c_double()
    probe = C.CDLL(os.path.join(os.path.dirname(dd.LIB_PATH), "libdedisp_probe.so"))
    probe.dedisp_probe_alu.restype = C.c_int
    probe.dedisp_probe_alu.argtypes = [C.c_int, C.POINTER(C.c_double)]
    if probe.dedisp_probe_alu(local, C.byref(peak)) != 0:
        raise RuntimeError("integer-pipe probe failed")
    k2_ms = sum(kms) / len(kms)
    adds = float(units) * cfg.nchans
    # DRAM bytes per K2 launch: ncu captures (2026-12-03, --clock-control none)
    # of each quad-strided shape on the same workload cut to 2^17 samples
    # (dram__bytes_read.sum + dram__bytes_write.sum of one launch), scaled by
    # the time tiles of the full launch (every tile streams its own delay
    # band, so the traffic grows with the tiles).
    # variant ({J, NW} of the library's quad shapes): (bytes in the capture,
    # time tiles in the capture, samples per tile = 128 J)
    captured = {5: (10798106368 + 1397426944, 38, 2560),   # {20, 12}
                6: (9808037376 + 1385468928, 34, 2816),    # {22, 12}
                7: (11724679936 + 1397582848, 42, 2304),   # {18, 12}
                8: (12990360064 + 1396900352, 47, 2048)}   # {16, 12}
    traffic, traffic_note = None, "no capture for this variant"
    if args.nbits == 8 and best in captured and cfg.nchans == 4096 and ndm == 3643:
        b, tiles_cap, bt = captured[best]
        tiles = -(-nout // bt)
        traffic = round(b / tiles_cap * tiles)
        traffic_note = (f"ncu capture 2026-12-03 of variant {best} on the workload cut to 2^17 samples "
                        f"({tiles_cap} tiles), scaled to this launch's {tiles} tiles; not measured "
                        f"in this run")
    achieved = adds / (k2_ms * 1e-3) / 1e12
    roofline = {"bound": "int-alu", "achieved": round(achieved, 3), "peak": round(peak.value / 1e12, 3),
                "unit": "Tadd/s", "frac": round(achieved * 1e12 / peak.value, 4),
                "traffic": traffic,
                "traffic_source": traffic_note,
                "peak_source": "measured in this run: dedisp_probe_alu (lib/libdedisp_probe.so; 32-bit add "
                               "lane-ops/s, all SMs)",
                "k2_ms": round(k2_ms, 3), "k1_ms": round(sum(pms) / len(pms), 3),
                "algorithmic": "nchan=4096 integer adds per DM-trial x sample; "
                               f"{adds:.3e} adds per step",
                "hbm_view": {"algorithmic_bytes": int(cfg.nsamps * 4096 * args.nbits // 8 +
                                                      units * 4),
                             "achieved_GBs": round((cfg.nsamps * 4096 * args.nbits // 8 +
                                                    units * 4) / (k2_ms * 1e-3) / 1e9, 1)}}

    # --- variants: plain form, other input widths -----------------------------
    variants = {}
    if not args.no_variants:
        plain = make_plan(kernel=1)
        plain.set_timing(True)
        step(plain)
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        step(plain)
        ev1.record(stream)
        torch.cuda.synchronize()
        pm = max_over_ranks(ev0.elapsed_time(ev1))
        variants["plain_8bit"] = {"value": units * world / (pm * 1e-3), "ms_per_step": pm,
                                  "kernel_ms": plain.get_timing()["kernel_ms"]}
        del plain
        for nb in (2, 4, 8):
            if nb == args.nbits:
                continue
            c2 = sy.config1(nbits=nb)
            inp = sy.make_input_torch(c2, device=f"cuda:{local}")
            p2 = make_plan()
            p2.set_timing(True)
            step(p2, nb, inp)
            torch.cuda.synchronize()
            ev0.record(stream)
            for _ in range(2):
                step(p2, nb, inp)
            ev1.record(stream)
            torch.cuda.synchronize()
            vm = max_over_ranks(ev0.elapsed_time(ev1)) / 2
            t = p2.get_timing()
            variants[f"tiled_{nb}bit"] = {"value": units * world / (vm * 1e-3),
                                          "ms_per_step": vm, "kernel_ms": t["kernel_ms"],
                                          "frac_int_alu": round(adds / (t["kernel_ms"] * 1e-3)
                                                                / peak.value, 4)}
            del inp, p2
        variants[f"tiled_{args.nbits}bit"] = {"value": value, "ms_per_step": ms,
                                              "kernel_ms": k2_ms}
        torch.cuda.empty_cache()

    # --- e2e: host buffers through the C ABI ----------------------------------
    e2e = None
    if not args.no_e2e:
        try:
            import psutil
            # every rank on this node pins its own buffers, so the node must
            # hold them all; the ranks take the same branch (their barriers
            # and reductions below must match)
            local_world = int(os.environ.get("LOCAL_WORLD_SIZE", "1"))
            need = (d_in.numel() + ndm * nout * 4) * local_world
            avail = psutil.virtual_memory().available
            if max_over_ranks(0.0 if avail >= need * 1.25 else 1.0) > 0.0:
                e2e = {"value": None, "unit": UNIT, "skipped": f"host RAM {avail/1e9:.0f} GB < "
                                                               f"{need*1.25/1e9:.0f} GB needed"}
            else:
                h_in = torch.empty(d_in.shape, dtype=torch.uint8, pin_memory=True)
                h_in.copy_(d_in)
                h_out = torch.empty((ndm, nout), dtype=torch.float32, pin_memory=True)
                del d_out
                torch.cuda.empty_cache()
                hp = dd.TDDPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df, local)
                hp.generate_dm_list(*cfg.dm_gen)
                hp.set_tile_variant(best)
                hp.set_gulp_size(args.e2e_gulp)
                hp.execute(cfg.nsamps, h_in, args.nbits, h_out, 32)  # warm-up
                torch.cuda.synchronize()
                barrier()
                ksteps = max(1, min(args.steps, 2))
                t0 = time.perf_counter()
                for _ in range(ksteps):
                    hp.execute(cfg.nsamps, h_in, args.nbits, h_out, 32)
                torch.cuda.synchronize()
                dt_e2e = max_over_ranks(time.perf_counter() - t0) / ksteps
                e2e = {"value": units * world / dt_e2e, "unit": UNIT,
                       "h2d_bytes_per_step": int(h_in.numel()),
                       "d2h_bytes_per_step": int(ndm * nout * 4), "ms_per_step": dt_e2e * 1e3,
                       "steps": ksteps, "gulp": args.e2e_gulp}
                del h_in, h_out, hp
        except Exception as ex:  # report, do not hide
            e2e = {"value": None, "unit": UNIT, "error": repr(ex)}

    # --- CPU baseline (rank 0 at N=1) -------------------------------------------
    cpu = None
    if not args.no_cpu and world == 1:
        cpu, _ = time_cpu_oracle(cfg, plan.get_dm_list(), md)

    # --- FDD forms (config 2) -------------------------------------------------------
    fdd = None
    _log("tdd sections done")
    if not args.no_fdd:
        del plan, d_in
        d_out = None
        torch.cuda.empty_cache()
        fdd = run_fdd(args, local, world, stream, max_over_ranks)
        _log("fdd done")

    # --- batched multi-beam TDD (config 3) ----------------------------------------
    batched = None
    if not args.no_batched:
        if args.no_fdd:
            del plan, d_in
            d_out = None
            torch.cuda.empty_cache()
        batched = run_batched(args, local, world, stream, max_over_ranks)
        _log("batched tdd done")

    # --- batched multi-beam FDD (config 3) -----------------------------------------
    batched_fdd = None
    if not args.no_batched:
        batched_fdd = run_batched_fdd(args, local, world, stream, max_over_ranks)
        _log("batched fdd done")

    # --- streaming server (config 4) -----------------------------------------------
    serving = None
    if not args.no_serve:
        serving = run_serving(args, local, world)
        _log("serving done")

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"u{args.nbits}->u32 sums->f32", "data": "synthetic (seeded, on device)",
            "config": workload_config(args.nbits, cfg.nsamps, ndm, md, world),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches * world, "clocks": clocks, "variants": variants,
            "tile_variant": {"chosen": best, "step_ms_by_variant": tune},
            "fdd": fdd, "batched": batched, "batched_fdd": batched_fdd, "serving": serving,
        }
        print(json.dumps(line), flush=True)
    reps.close()


def run_reference(args):
    """The reference's CPU implementation of the path: the oracle port (the
    reference's own CPU code for this path needs FFTW, absent here)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from dedisp_tests_b200 import synthetic as sy
    from oracle import pyoracle as po
    cfg = sy.config1(nbits=args.nbits)
    dms = po.generate_dm_list(cfg.nchans, cfg.dt, cfg.f_top, cfg.df, *cfg.dm_gen)
    delays = po.delay_table(cfg.nchans, np.float32(cfg.dt), np.float32(cfg.f_top),
                            np.float32(cfg.df))
    md = po.max_delay(dms, delays)
    cpu, t = time_cpu_oracle(cfg, dms, md, steps=args.steps, warmup=min(args.warmup, 1))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    line = {"metric": METRIC, "value": cpu["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"u{args.nbits}->u32 sums->f32", "data": "synthetic (seeded)",
            "config": workload_config(args.nbits, cfg.nsamps, len(dms), md, world),
            "impl": "reference", "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    a = parse()
    if a.profile_case:
        profile_case(a)
    elif a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)

"""Generates the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py host   # no GPU: plan setup + epilogue
    python tests/golden/make_golden.py gpu    # on a GPU box: reference plans

Both modes run the reference's own code compiled from its sources by
oracle/ref/Makefile into oracle/_ref/ (run `make -C oracle/ref` first where
the reference tree is available; the built libraries travel with the tree).

host: delay tables, DM lists and max delays from the reference dedisp::Plan
      (src/Plan.cpp) and the TDD epilogue from scale_output
      (src/tdd/dedisperse/dedisperse_kernel.cuh:45-64) over a sweep of sums.
gpu:  outputs of the reference TDDPlan, DedispPlan and FDDGPUPlan on small
      seeded inputs (inputs are regenerated from the stored recipe; their
      SHA-256 is stored to detect drift).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from dedisp_tests_b200 import synthetic as sy  # noqa: E402

# (nchans, dt, f0, df): the benchmark configurations and the reference's
# own test/benchmark recipes (bin/test/test.hpp:103-121,
# bin/test/ctestdedisp.c:166-186, bin/benchmark/bench.hpp:143-161).
PLAN_PARAMS = [
    (1024, 250e-6, 1581.8, -0.390625),
    (4096, 64e-6, 1500.0, -0.078125),
    (1536, 81.92e-6, 1670.0, -0.25),
    (3072, 100e-6, 169.589996337891, -30.7199914522957 / 3072),
    (1024, 250e-6, 1581.0, -100.0 / 1024),
    (1024, 64e-6, 1581.0, -400.0 / 1024),
    (64, 1e-3, 400.0, 1.0),
]
DM_GEN = [
    (1, 0.0, 2000.0, 40.0, 1.25),    # config 1
    (3, 20.0, 60.0, 4.0, 1.25),      # bin/test/test.hpp
    (4, 2.0, 100.0, 4.0, 1.25),      # bin/test/ctestdedisp.c
    (5, 0.0, 1000.0, 64.0, 1.1),
]


def host() -> None:
    out = {}
    for i, (n, dt, f0, df) in enumerate(PLAN_PARAMS):
        out[f"params_{i}"] = np.array([n, dt, f0, df], np.float64)
        out[f"delay_{i}"] = po.ref_delay_table(n, dt, f0, df)
    for j, (pi, s, e, ti, tol) in enumerate(DM_GEN):
        n, dt, f0, df = PLAN_PARAMS[pi]
        dms, md = po.ref_generate_dm_list(n, dt, f0, df, s, e, ti, tol)
        out[f"dmgen_{j}"] = np.array([pi, s, e, ti, tol], np.float64)
        out[f"dmlist_{j}"] = dms
        out[f"dmmax_{j}"] = np.array([md], np.int64)
    np.savez_compressed(os.path.join(HERE, "plan_setup.npz"), **out)

    rng = np.random.default_rng(7)
    rows = []
    for in_nb in (1, 2, 4, 8, 16, 32):
        for out_nb in (8, 16, 32):
            for nch in (1, 7, 64, 1024, 3072, 4096, 8192):
                mx = nch * ((1 << in_nb) - 1)
                sums = list(rng.integers(0, mx + 1, 40)) + [0, 1, mx, mx // 2]
                for s in sums:
                    v = po.ref_scale_output(int(s), in_nb, out_nb, nch)
                    bits = int(np.asarray(v, np.float32).view(np.uint32)) if out_nb == 32 \
                        else int(v)
                    rows.append((in_nb, out_nb, nch, int(s), bits))
    np.savez_compressed(os.path.join(HERE, "epilogue.npz"),
                        table=np.array(rows, dtype=np.uint64))
    print("host fixtures written")


# Reference GPU cases: (plan, nchans, f0, df, dt, nsamps, nbits, out_nbits,
# ndm, dm_max, killmask_every, seed)
GPU_CASES = [
    ("tdd", 128, 1581.8, -1.5625, 250e-6, 8192, 8, 32, 32, 200.0, 0, 11),
    ("tdd", 256, 1500.0, -0.5, 64e-6, 6001, 2, 8, 20, 150.0, 0, 12),
    ("tdd", 64, 1400.0, -2.0, 100e-6, 5000, 4, 16, 24, 300.0, 5, 13),
    ("tdd", 32, 1581.8, -3.125, 250e-6, 4096, 16, 32, 16, 100.0, 0, 14),
    ("tdd", 96, 1670.0, -1.0, 81.92e-6, 4000, 1, 32, 12, 120.0, 0, 15),
    ("tdd", 16, 1581.8, -6.25, 250e-6, 3000, 32, 32, 8, 80.0, 0, 16),
    ("dedisp", 128, 1581.8, -1.5625, 250e-6, 8192, 8, 32, 32, 200.0, 7, 17),
    ("dedisp", 256, 1500.0, -0.5, 64e-6, 6000, 2, 16, 20, 150.0, 0, 18),
]
# The reference whole-series FDD runs its forward FFT nchan_batch/64 times
# (FDDGPUPlan.cpp:114-115,486-494, batch = min(nchans/4, 64)), i.e. never for
# fewer than 256 channels; its phasor kernel is only launched for channel
# batches of 1/16/32/64/128/256 (FDDKernel.cu:79-87); and it touches a popped
# DM job when ndm is a multiple of its DM batch (FDDGPUPlan.cpp:352-368). The
# cases therefore use 256 channels (whole series), 128 (segmented, fixed batch
# of 32) and ndm 18 / 14.
FDD_CASES = [
    # (nchans, f0, df, dt, nsamps, ndm, dm_max, segmented, seed)
    ("fdd", 256, 1581.8, -0.78125, 250e-6, 12000, 18, 60.0, 0, 21),
    ("fdd", 128, 1581.8, -1.5625, 250e-6, 40000, 14, 80.0, 1, 22),
]


def gpu_case_input(nchans, f0, df, dt, nsamps, nbits, seed):
    rng = np.random.default_rng(seed)
    if nbits == 32:
        vals = rng.integers(0, 1 << 32, (nsamps, nchans), dtype=np.uint64).astype(np.uint32)
        return sy.pack(vals, 32)
    cfg = sy.Config("golden", nchans, f0, df, dt, nsamps, nbits, (2 ** nbits - 1) / 2.0,
                    max(1.0, (2 ** nbits) / 6.0),
                    [sy.Pulse(dm=0.5 * 100.0, t0=0.3, width=2 * dt, amp=(2 ** nbits) / 3.0)],
                    seed=seed)
    return sy.make_input(cfg)


def gpu() -> None:
    out = {}
    for k, (plan, nch, f0, df, dt, ns, nb, onb, ndm, dmax, kme, seed) in enumerate(GPU_CASES):
        inp = gpu_case_input(nch, f0, df, dt, ns, nb, seed)
        dms = np.linspace(0, dmax, ndm, dtype=np.float32)
        km = np.ones(nch, np.int32)
        if kme:
            km[::kme] = 0
        delays = po.ref_delay_table(nch, dt, f0, df)
        md = po.max_delay(dms, delays)
        nout = ns - md
        res, md_ref = po.ref_execute(plan, nch, dt, f0, df, dms, km, ns, inp, nb, onb,
                                     ndm * nout, gulp_size=1 << 30)
        assert md_ref == md
        out[f"case_{k}"] = np.array([k, nch, f0, df, dt, ns, nb, onb, ndm, dmax, kme, seed],
                                    np.float64)
        out[f"plan_{k}"] = np.array([plan])
        out[f"sha_{k}"] = np.array([hashlib.sha256(inp.tobytes()).hexdigest()])
        out[f"out_{k}"] = res
        print("tdd case", k, plan, nb, onb, "ok")
    for k, (plan, nch, f0, df, dt, ns, ndm, dmax, seg, seed) in enumerate(FDD_CASES):
        cfg = sy.Config("golden-fdd", nch, f0, df, dt, ns, 8, 127.5, 20.0,
                        [sy.Pulse(dm=dmax / 2, t0=0.5, width=1e-3, amp=30.0)], seed=seed)
        inp = sy.make_input(cfg)
        dms = np.linspace(0, dmax, ndm, dtype=np.float32)
        delays = po.ref_delay_table(nch, dt, f0, df)
        md = po.max_delay(dms, delays)
        if seg:
            row = ns - md
        else:
            row = po.fdd_nfft_spectrum(ns, md)
        res, _ = po.ref_execute("fdd", nch, dt, f0, df, dms, None, ns, inp, 8, 32, ndm * row,
                                segmented=bool(seg))
        out[f"fcase_{k}"] = np.array([k, nch, f0, df, dt, ns, ndm, dmax, seg, seed], np.float64)
        out[f"fsha_{k}"] = np.array([hashlib.sha256(inp.tobytes()).hexdigest()])
        # three DM rows (first, middle, last) keep the fixture small
        rows = [0, ndm // 2, ndm - 1]
        out[f"fout_{k}"] = res.view(np.float32).reshape(ndm, row)[rows].copy()
        out[f"frows_{k}"] = np.array(rows)
        print("fdd case", k, "segmented" if seg else "spectrum", "ok")
    dest = os.environ.get("GOLDEN_OUT", HERE)
    os.makedirs(dest, exist_ok=True)
    np.savez_compressed(os.path.join(dest, "ref_gpu_outputs.npz"), **out)
    print("gpu fixtures written to", dest)


if __name__ == "__main__":
    mode = sys.argv[1] if len(sys.argv) > 1 else "host"
    {"host": host, "gpu": gpu}[mode]()

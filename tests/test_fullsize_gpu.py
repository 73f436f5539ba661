"""Parity at the full sizes the benchmark reports, through the C ABI.

* Config 2 (FDD): 1024 channels, 2^20 float32 samples, 2048 DMs over
  0-1000, segmented with 32768-point FFTs (39 segments of 27525 good samples,
  max delay 5243), in both MAC forms: against the FP64 oracle on a DM subset
  over all output samples, and -- on the same geometry with 8-bit samples,
  the reference FDD's own input format -- against the TDD plan's output on
  every DM and sample.
* Config 1 (TDD) at 2 and 4 bits: 4096 channels, 2^21 samples, 3643 DMs, the
  default quad-strided kernel with samples widened to bytes, bit-exact against
  the oracle on 6 DMs x 3 windows of 65536 samples.

Tolerances (relative L2 over the compared rows, and max-abs relative to max
|ref|): FP32 MAC 2e-6 / 2e-5; 3xBF16 tensor-core MAC 1e-5 / 1e-4.
"""
import dataclasses

import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL = {0: (2e-6, 2e-5), 1: (1e-5, 1e-4)}
PICK = np.array([0, 1, 700, 1024, 1400, 2047])


def _errs(ours, ref):
    ours = np.asarray(ours, np.float64)
    ref = np.asarray(ref, np.float64)
    return (np.linalg.norm(ours - ref) / np.linalg.norm(ref),
            np.abs(ours - ref).max() / np.abs(ref).max())


def _fdd_plan(cfg, precision, round_delays=False):
    p = dd.FDDGPUPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
    p.set_dm_list(np.asarray(cfg.dm_list, np.float32))
    p.set_options(segmented=1, precision=precision, segment_nfft=1 << 15, round_delays=round_delays)
    p.set_timing(True)
    return p


@pytest.fixture(scope="module")
def config2_fp64():
    """Config-2 input on the device and the FP64 oracle rows of PICK."""
    import torch
    cfg = sy.config2()
    d_in = sy.make_input_torch(cfg)
    h_in = d_in.cpu().numpy()
    md = 5243
    nout = cfg.nsamps - md
    x = po.fdd_unpack(h_in, cfg.nsamps, h_in.shape[1], 32, cfg.nchans)
    del h_in
    delays = po.delay_table(cfg.nchans, np.float32(cfg.dt), np.float32(cfg.f_top), np.float32(cfg.df))
    dms = np.asarray(cfg.dm_list, np.float32)
    ref = po.fdd_timeseries(x, delays, np.ones(cfg.nchans, np.int32), dms[PICK], nout)
    del x
    yield cfg, d_in, ref, nout
    del d_in
    torch.cuda.empty_cache()


@pytest.mark.parametrize("precision", [0, 1])
def test_config2_full_geometry_vs_fp64(config2_fp64, precision):
    import torch
    cfg, d_in, ref, nout = config2_fp64
    p = _fdd_plan(cfg, precision)
    assert (p.get_dm_count(), p.get_max_delay()) == (2048, 5243)
    assert p.output_row_length(cfg.nsamps) == nout
    d_out = torch.empty((2048, nout), dtype=torch.float32, device="cuda")
    p.execute(cfg.nsamps, d_in, 32, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
    assert p.get_timing()["variant"] == precision
    got = d_out[torch.as_tensor(PICK, device="cuda")].cpu().numpy()
    rel, mx = _errs(got, ref)
    print(f"config 2 precision {precision}: rel-L2 {rel:.3e} max-abs {mx:.3e} vs FP64")
    assert rel < TOL[precision][0] and mx < TOL[precision][1], (rel, mx)
    del d_out, p
    torch.cuda.empty_cache()


def test_config2_geometry_vs_tdd_plan():
    """8-bit samples (config 2's noise and pulses quantised at 24 levels per
    sigma around 127.5): the FDD time series with TDD's round-half-even
    delays equals (S - 127.5 nchans) / nchans, S the TDD integer sum. S is
    recovered exactly from the TDD plan's float output (S < 2^24, so
    rint(out * den / factor) undoes the two FP32 roundings of the epilogue).
    Compared on all 2048 DMs x 1043333 samples, on the device."""
    import torch
    base = sy.config2()
    cfg = dataclasses.replace(base, nbits=8, mean=127.5, sigma=24.0, float_input=False,
                              pulses=[dataclasses.replace(q, amp=q.amp * 24.0) for q in base.pulses])
    d_in = sy.make_input_torch(cfg)
    dms = np.asarray(cfg.dm_list, np.float32)
    t = dd.TDDPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
    t.set_dm_list(dms)
    nout = cfg.nsamps - t.get_max_delay()
    tdd_out = torch.empty((2048, nout), dtype=torch.float32, device="cuda")
    t.execute(cfg.nsamps, d_in, 8, tdd_out, 32, dd.DEDISP_DEVICE_POINTERS)
    den = float(np.float32(255.0) * np.float32(cfg.nchans))
    factor = float(np.float32(3.0 * 1024.0 / 255.0 / 16.0))
    want = torch.empty((2048, nout), dtype=torch.float32, device="cuda")
    for r0 in range(0, 2048, 256):  # FP64 on the device, 256 rows at a time
        s = torch.round(tdd_out[r0:r0 + 256].double() * den / factor)
        want[r0:r0 + 256] = ((s - 127.5 * cfg.nchans) / cfg.nchans).float()
    del tdd_out, t
    torch.cuda.empty_cache()
    for precision in (0, 1):
        p = _fdd_plan(cfg, precision, round_delays=True)
        got = torch.empty((2048, nout), dtype=torch.float32, device="cuda")
        p.execute(cfg.nsamps, d_in, 8, got, 32, dd.DEDISP_DEVICE_POINTERS)
        assert p.get_timing()["variant"] == precision
        num = sum(float(((got[r0:r0 + 256].double() - want[r0:r0 + 256].double()) ** 2).sum())
                  for r0 in range(0, 2048, 256))
        rel = (num / float((want.double() ** 2).sum())) ** 0.5
        mx = float((got - want).abs().max()) / float(want.abs().max())
        print(f"config 2 geometry, 8-bit, precision {precision}: rel-L2 {rel:.3e} "
              f"max-abs {mx:.3e} vs the TDD plan")
        assert rel < TOL[precision][0] and mx < TOL[precision][1], (precision, rel, mx)
        del got, p
        torch.cuda.empty_cache()


@pytest.mark.parametrize("nbits", [2, 4])
def test_config1_full_size_narrow_inputs(nbits):
    import torch
    cfg = sy.config1(nbits=nbits)
    d_in = sy.make_input_torch(cfg)
    p = dd.TDDPlan(cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
    p.generate_dm_list(*cfg.dm_gen)
    ndm, md = p.get_dm_count(), p.get_max_delay()
    assert (ndm, md) == (3643, 35500)
    nout = cfg.nsamps - md
    out = torch.empty((ndm, nout), dtype=torch.float32, device="cuda")
    p.execute(cfg.nsamps, d_in, nbits, out, 32, dd.DEDISP_DEVICE_POINTERS)
    pick = np.array([0, 1, 911, 1822, 2700, ndm - 1])
    dms = p.get_dm_list()
    delays = po.delay_table(cfg.nchans, np.float32(cfg.dt), np.float32(cfg.f_top), np.float32(cfg.df))
    L = 65536
    for ta in (0, nout // 2, nout - L):
        win = d_in[ta:ta + L + md].cpu().numpy()
        ref = po.tdd(win, L + md, win.shape[1], nbits, cfg.nchans, delays,
                     np.ones(cfg.nchans, np.int32), dms[pick], 32, L)
        got = out[torch.as_tensor(pick, device="cuda"), ta:ta + L].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (nbits, ta)
    del out, d_in, p
    torch.cuda.empty_cache()

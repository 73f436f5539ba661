"""FDD on the GPU against the FP64 oracle, through the C ABI.

Tolerances are stated per test as relative L2 error (||ours - ref|| /
||ref||) and max-abs error relative to max |ref|. The FP32 form computes
exact integer phase indices and table phasors, so its error is FP32 FFT and
summation rounding only.
"""
import os

import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

FP32_REL_L2 = 2e-6
FP32_MAX_ABS = 2e-5


def _errs(ours, ref):
    ours = np.asarray(ours, np.float64)
    ref = np.asarray(ref, np.float64)
    rel = np.linalg.norm(ours - ref) / max(np.linalg.norm(ref), 1e-300)
    mx = np.abs(ours - ref).max() / max(np.abs(ref).max(), 1e-300)
    return rel, mx


def _input(nchans, nsamps, seed, float_input=False, f0=1581.8, df=-1.5625, dt=250e-6):
    cfg = sy.Config("t", nchans, f0, df, dt, nsamps, 8, 0.0 if float_input else 127.5,
                    1.0 if float_input else 20.0,
                    [sy.Pulse(dm=40.0, t0=0.4 * nsamps * dt, width=1e-3,
                              amp=0.5 if float_input else 30.0)],
                    seed=seed, float_input=float_input)
    return sy.make_input(cfg), (nchans, dt, f0, df)


def _plan(params, dms, km=None, **opts):
    p = dd.FDDGPUPlan(*params)
    p.set_dm_list(dms)
    if km is not None:
        p.set_killmask(km)
    p.set_options(**opts)
    return p


def _oracle_x(inp, nsamps, params, in_nbits):
    nchans = params[0]
    return po.fdd_unpack(inp, nsamps, inp.shape[1], in_nbits, nchans)


def _delays(params):
    nchans, dt, f0, df = params
    return po.delay_table(nchans, np.float32(dt), np.float32(f0), np.float32(df))


@pytest.mark.parametrize("in_nbits", [8, 32])
def test_segmented_timeseries(in_nbits):
    nchans, nsamps = 128, 90000
    inp, params = _input(nchans, nsamps, 3, float_input=(in_nbits == 32))
    dms = np.linspace(0, 120, 37, dtype=np.float32)
    p = _plan(params, dms, segmented=1)
    md = p.get_max_delay()
    nout = nsamps - md
    assert p.output_row_length(nsamps) == nout
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, in_nbits, out, 32)
    x = _oracle_x(inp, nsamps, params, in_nbits)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (rel, mx)


def test_whole_series_spectrum_default():
    """The fork's default output: the first nfft/2 dedispersed bins."""
    nchans, nsamps = 64, 12000
    inp, params = _input(nchans, nsamps, 5)
    dms = np.linspace(0, 60, 18, dtype=np.float32)
    p = _plan(params, dms, segmented=0)
    md = p.get_max_delay()
    nfft = po.fdd_nfft_spectrum(nsamps, md)
    assert p.output_row_length(nsamps) == nfft
    out = np.zeros((len(dms), nfft), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, nfft)
    rel, mx = _errs(out, ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (rel, mx)


def test_whole_series_timeseries_and_killmask_and_rounding():
    nchans, nsamps = 128, 20000
    inp, params = _input(nchans, nsamps, 7)
    dms = np.linspace(0, 90, 25, dtype=np.float32)
    km = np.ones(nchans, np.int32)
    km[3::7] = 0
    for rnd in (False, True):
        p = _plan(params, dms, km=km, segmented=0, timeseries=True, round_delays=rnd)
        nout = nsamps - p.get_max_delay()
        out = np.zeros((len(dms), nout), np.float32)
        p.execute(nsamps, inp, 8, out, 32)
        x = _oracle_x(inp, nsamps, params, 8)
        ref = po.fdd_timeseries(x, _delays(params), km, dms, nout, round_delays=rnd)
        rel, mx = _errs(out, ref)
        assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (rnd, rel, mx)


def test_round_delays_matches_tdd_pulse():
    """With round-half-even delays the FDD time series is the TDD sum of the
    unpacked samples (same integer delays, dedisperse_kernel.cuh:165)."""
    nchans, nsamps = 64, 30000
    inp, params = _input(nchans, nsamps, 9)
    dms = np.linspace(0, 50, 11, dtype=np.float32)
    p = _plan(params, dms, segmented=1, round_delays=True)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    sums = po.tdd_sums(inp, nsamps, nchans, 8, nchans, _delays(params), np.ones(nchans, np.int32),
                       dms, nout).astype(np.float64)
    # x = (v - 127.5) / nchans  ->  sum_c x = (sum_c v - 127.5 nchans) / nchans
    ref = (sums - 127.5 * nchans) / nchans
    rel, mx = _errs(out, ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (rel, mx)


def test_device_pointers():
    import torch
    nchans, nsamps = 64, 40000
    inp, params = _input(nchans, nsamps, 11)
    dms = np.linspace(0, 80, 16, dtype=np.float32)
    p = _plan(params, dms, segmented=1)
    nout = nsamps - p.get_max_delay()
    d_in = torch.from_numpy(inp).cuda()
    d_out = torch.zeros((len(dms), nout), dtype=torch.float32, device="cuda")
    p.execute(nsamps, d_in, 8, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(d_out.cpu().numpy(), ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS


@pytest.mark.parametrize("precision", [0, 1])
def test_spectrum_output_on_device_pointers(precision):
    """The whole-series spectrum (the fork's default output,
    src/fdd/FDDGPUPlan.hpp:6) kept on the device: device input and output
    rows, both MAC forms, against the FP64 spectrum."""
    import torch
    nchans, nsamps = 128, 30000
    inp, params = _input(nchans, nsamps, 17)
    dms = np.linspace(0, 90, 40, dtype=np.float32)
    p = _plan(params, dms, segmented=0, precision=precision)
    p.set_timing(True)
    row = p.output_row_length(nsamps)
    assert row == po.fdd_nfft_spectrum(nsamps, p.get_max_delay())
    d_in = torch.from_numpy(inp).cuda()
    d_out = torch.full((len(dms), row), 3.0, dtype=torch.float32, device="cuda")
    p.execute(nsamps, d_in, 8, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
    torch.cuda.synchronize()
    assert p.get_timing()["variant"] == precision
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, row)
    rel, mx = _errs(d_out.cpu().numpy(), ref)
    lim = (FP32_REL_L2, FP32_MAX_ABS) if precision == 0 else (1e-5, 1e-4)
    assert rel < lim[0] and mx < lim[1], (precision, rel, mx)


def test_use_segmented_environment(monkeypatch):
    nchans, nsamps = 64, 40000
    inp, params = _input(nchans, nsamps, 13)
    dms = np.linspace(0, 40, 8, dtype=np.float32)
    p = _plan(params, dms)  # segmented=-1: follow USE_SEGMENTED
    monkeypatch.setenv("USE_SEGMENTED", "1")
    assert p.output_row_length(nsamps) == nsamps - p.get_max_delay()
    monkeypatch.setenv("USE_SEGMENTED", "0")
    assert p.output_row_length(nsamps) == po.fdd_nfft_spectrum(nsamps, p.get_max_delay())


GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_gpu_outputs.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="no reference GPU golden outputs")
def test_against_reference_fdd_outputs():
    """Outputs of the reference FDDGPUPlan (same inputs) against ours and the
    FP64 oracle. The reference evaluates phases in FP32 with sin/cos.approx
    and no range reduction (fdd_kernel.cuh:61-74,229-232), so it is only
    close to FP64; ours must be at least 5x closer. In segmented mode the
    reference runs its phasor kernel over nsamp/2+1 flattened bins
    (FDDGPUPlan.cpp:740,1103-1116) instead of all nchunk segments, so its
    later segments are not dedispersed; only the fully covered first
    segment is compared."""
    from tests.golden.make_golden import FDD_CASES
    g = np.load(GOLDEN)
    for k, (_, nch, f0, df, dt, ns, ndm, dmax, seg, seed) in enumerate(FDD_CASES):
        cfg = sy.Config("golden-fdd", nch, f0, df, dt, ns, 8, 127.5, 20.0,
                        [sy.Pulse(dm=dmax / 2, t0=0.5, width=1e-3, amp=30.0)], seed=seed)
        inp = sy.make_input(cfg)
        params = (nch, dt, f0, df)
        dms = np.linspace(0, dmax, ndm, dtype=np.float32)
        rows = g[f"frows_{k}"]
        refgpu = g[f"fout_{k}"].astype(np.float64)
        p = _plan(params, dms, segmented=int(seg))
        row = p.output_row_length(ns)
        out = np.zeros((ndm, row), np.float32)
        p.execute(ns, inp, 8, out, 32)
        x = _oracle_x(inp, ns, params, 8)
        if seg:
            nout = ns - p.get_max_delay()
            f64 = po.fdd_timeseries(x, _delays(params), np.ones(nch, np.int32), dms, nout)
            nfft, good, _ = po.fdd_segment_geometry(ns, p.get_max_delay())
            sl = slice(0, good)
        else:
            f64 = po.fdd_spectrum(x, _delays(params), np.ones(nch, np.int32), dms, row)
            sl = slice(0, row)
        ref_err = _errs(refgpu[:, sl], f64[rows][:, sl])[0]
        our_err = _errs(out[rows][:, sl], f64[rows][:, sl])[0]
        assert ref_err < 5e-2, ref_err
        assert our_err < FP32_REL_L2 and our_err * 5 < ref_err, (our_err, ref_err)


@pytest.mark.parametrize("nbits,precision", [(1, 0), (2, 0), (4, 0), (2, 1), (16, 0)])
def test_packed_input_widths(nbits, precision):
    """1/2/4/16-bit packed input (an extension; samples centred at
    (2^nbits - 1) / 2), both MAC forms."""
    nchans, nsamps = 128, 40000
    rng = np.random.default_rng(40 + nbits)
    vals = rng.integers(0, 1 << nbits, (nsamps, nchans), dtype=np.uint32)
    inp = sy.pack(vals, nbits)
    params = (nchans, 250e-6, 1581.8, -1.5625)
    dms = np.linspace(0, 90, 21, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=precision)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, nbits, out, 32)
    x = _oracle_x(inp, nsamps, params, nbits)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    tol = (FP32_REL_L2, FP32_MAX_ABS) if precision == 0 else (1e-5, 1e-4)
    assert rel < tol[0] and mx < tol[1], (rel, mx)


@pytest.mark.parametrize("segment_nfft,nchans,nsamps,dm_max", [
    (65536, 64, 200000, 100.0),
    (131072, 32, 300000, 100.0),
    (262144, 32, 600000, 100.0),
    (1 << 20, 32, 1100000, 50.0),
    (0, 64, 400000, 2500.0),     # the reference rule picks 131072-point segments here
])
def test_four_step_fft_segments(segment_nfft, nchans, nsamps, dm_max):
    """Segments longer than 32768 samples use the four-step FFT (column and
    row passes through a scratch buffer)."""
    inp, params = _input(nchans, nsamps, 17, float_input=True, f0=1400.0, df=-2.0, dt=64e-6)
    dms = np.linspace(0, dm_max, 12, dtype=np.float32)
    p = _plan(params, dms, segmented=1, segment_nfft=segment_nfft)
    md = p.get_max_delay()
    nfft, good, nchunk = po.fdd_segment_geometry(nsamps, md) if segment_nfft == 0 else (segment_nfft, segment_nfft - md, 0)
    assert nfft > 32768
    nout = nsamps - md
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, 32, out, 32)
    x = _oracle_x(inp, nsamps, params, 32)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (rel, mx)


@pytest.mark.parametrize("segment_nfft,nchans,nsamps,dm_max", [
    (512, 40, 30000, 50.0),
    (1024, 48, 60000, 150.0),
    (2048, 37, 60000, 300.0),
    (4096, 33, 80000, 600.0),
    (8192, 40, 100000, 1000.0),
    (16384, 64, 150000, 1500.0),
    (32768, 64, 200000, 2000.0),
])
def test_single_cta_fft_lengths(segment_nfft, nchans, nsamps, dm_max):
    """Every single-CTA transform length: row counts below, at and above
    one wave of the persistent FFT kernels, and segments that start on odd
    sample offsets (nsamp_good odd)."""
    inp, params = _input(nchans, nsamps, 23, float_input=True, f0=1400.0, df=-2.0, dt=64e-6)
    dms = np.linspace(0, dm_max, 7, dtype=np.float32)
    p = _plan(params, dms, segmented=1, segment_nfft=segment_nfft)
    md = p.get_max_delay()
    assert md < segment_nfft
    nout = nsamps - md
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, 32, out, 32)
    x = _oracle_x(inp, nsamps, params, 32)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (rel, mx)


@pytest.mark.parametrize("dm_max", [4000.0, 9000.0])
def test_whole_series_large_delays(dm_max):
    """The FP32 whole-series MAC with max delays of about 14000 samples (the
    one-segment kernel's per-bin table) and about 31000 (its table would not
    fit shared memory: the tiled kernel), spectrum output, round-half-even
    delays; FP32 tolerance against FP64."""
    nchans, nsamps = 64, 60000
    inp, params = _input(nchans, nsamps, 13, dt=64e-6)
    dms = np.linspace(0, dm_max, 24, dtype=np.float32)
    p = _plan(params, dms, segmented=0, round_delays=True)
    md = p.get_max_delay()
    assert (md > 25000) == (dm_max > 5000), md
    nfft = po.fdd_nfft_spectrum(nsamps, md)
    out = np.zeros((len(dms), nfft), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, nfft, round_delays=True)
    rel, mx = _errs(out, ref)
    assert rel < FP32_REL_L2 and mx < FP32_MAX_ABS, (md, rel, mx)

"""FDD with the tensor-core (tcgen05, 3xBF16) phasor MAC against the FP64
oracle, through the C ABI.

The 3xBF16 form splits phasors and spectra into BF16 hi + lo parts and
accumulates hi*hi + hi*lo + lo*hi in FP32. Its representation error is about
2^-16 of each operand, so the stated bound on the dedispersed output is
rel-L2 <= 1e-5 against FP64 (max-abs, relative to max |ref|, <= 1e-4).
"""
import numpy as np
import pytest

import dedisp_tests_b200 as dd

from tests.test_fdd_gpu import _delays, _errs, _input, _oracle_x, _plan
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TC_REL_L2 = 1e-5
TC_MAX_ABS = 1e-4


def _run(p, nsamps, inp, in_nbits, ndm):
    p.set_timing(True)
    row = p.output_row_length(nsamps)
    out = np.zeros((ndm, row), np.float32)
    p.execute(nsamps, inp, in_nbits, out, 32)
    assert p.get_timing()["variant"] == 1, "tensor-core MAC did not run"
    return out


def test_tc_whole_series_spectrum_small():
    """One DM tile, one segment: N = 16384, 64 channels (one K chunk)."""
    nchans, nsamps = 64, 12000
    inp, params = _input(nchans, nsamps, 5)
    dms = np.linspace(0, 60, 18, dtype=np.float32)
    p = _plan(params, dms, segmented=0, precision=1)
    out = _run(p, nsamps, inp, 8, len(dms))
    nfft = out.shape[1]
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, nfft)
    rel, mx = _errs(out, ref)
    print("tc spectrum", rel, mx)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


@pytest.mark.parametrize("in_nbits", [8, 32])
def test_tc_segmented_timeseries(in_nbits):
    """Several segments, padded channel count (96 -> 128), 200 DMs (two tiles)."""
    nchans, nsamps = 96, 90000
    inp, params = _input(nchans, nsamps, 3, float_input=(in_nbits == 32))
    dms = np.linspace(0, 120, 200, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=1)
    nout = nsamps - p.get_max_delay()
    out = _run(p, nsamps, inp, in_nbits, len(dms))
    assert out.shape[1] == nout
    x = _oracle_x(inp, nsamps, params, in_nbits)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    print("tc segmented", in_nbits, rel, mx)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


def test_tc_killmask_rounding_matches_plain():
    """Killmask and round-half-even delays; the tensor-core and FP32 forms
    agree with each other and with the oracle."""
    nchans, nsamps = 128, 14000
    inp, params = _input(nchans, nsamps, 7)
    dms = np.linspace(0, 90, 131, dtype=np.float32)
    km = np.ones(nchans, np.int32)
    km[3::7] = 0
    x = _oracle_x(inp, nsamps, params, 8)
    for rnd in (False, True):
        p = _plan(params, dms, km=km, segmented=0, timeseries=True, round_delays=rnd, precision=1)
        out = _run(p, nsamps, inp, 8, len(dms))
        nout = nsamps - p.get_max_delay()
        ref = po.fdd_timeseries(x, _delays(params), km, dms, nout, round_delays=rnd)
        rel, mx = _errs(out[:, :nout], ref)
        print("tc killmask", rnd, rel, mx)
        assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rnd, rel, mx)
        q = _plan(params, dms, km=km, segmented=0, timeseries=True, round_delays=rnd, precision=0)
        plain = np.zeros_like(out)
        q.execute(nsamps, inp, 8, plain, 32)
        rel2, _ = _errs(out, plain)
        assert rel2 < TC_REL_L2, rel2


def test_tc_repeat_is_deterministic():
    nchans, nsamps = 64, 30000
    inp, params = _input(nchans, nsamps, 9)
    dms = np.linspace(0, 50, 140, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=1)
    a = _run(p, nsamps, inp, 8, len(dms))
    b = _run(p, nsamps, inp, 8, len(dms))
    assert np.array_equal(a, b)


def test_tc_negative_dms_use_quarter_wave_phasors():
    """Negative DMs (negative delays) take the kernel's quarter-wave phasor
    path instead of the per-bin delay table; spectrum output, circular shifts."""
    nchans, nsamps = 64, 12000
    inp, params = _input(nchans, nsamps, 6)
    dms = np.linspace(-30, 60, 45, dtype=np.float32)
    p = _plan(params, dms, segmented=0, precision=1)
    out = _run(p, nsamps, inp, 8, len(dms))
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, out.shape[1])
    rel, mx = _errs(out, ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


@pytest.mark.parametrize("nsamps", [72000, 102000])
def test_tc_many_segments(nsamps):
    """2048-point segments: 36 segments (80 accumulator columns) and 51
    segments (112 columns, close to the 128-column limit); killmask,
    rounded delays."""
    nchans = 64
    inp, params = _input(nchans, nsamps, 11)
    dms = np.linspace(0, 20, 37, dtype=np.float32)
    km = np.ones(nchans, np.int32)
    km[9::13] = 0
    p = _plan(params, dms, km=km, segmented=1, precision=1, round_delays=True, segment_nfft=2048)
    md = p.get_max_delay()
    nout = nsamps - md
    nseg = -(-nsamps // (2048 - md))  # segments of the reference rule (FDDGPUPlan.cpp:762-777)
    assert (2 * nseg <= 80) == (nsamps == 72000)
    out = _run(p, nsamps, inp, 8, len(dms))
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), km, dms, nout, round_delays=True)
    rel, mx = _errs(out[:, :nout], ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (nseg, rel, mx)


@pytest.mark.parametrize("form", ["1", "2", "3"])
def test_tc_selectable_mma_forms(form, monkeypatch):
    """The MMA forms chosen by DEDISP_TC_FORM (read at each launch): 1 the
    fused A_hi x [B_hi | B_lo] form, 2 the three-MMA form with two A buffers
    (the default takes three when the accumulators fit 64 columns), 3 the
    fused form at 64-channel chunks (npad <= 32; this shape has more segments,
    so it takes the default form). Same tolerance against FP64."""
    monkeypatch.setenv("DEDISP_TC_FORM", form)
    nchans, nsamps = 96, 90000
    inp, params = _input(nchans, nsamps, 7)
    dms = np.linspace(0, 120, 200, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=1)
    nout = nsamps - p.get_max_delay()
    out = _run(p, nsamps, inp, 8, len(dms))
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (form, rel, mx)


@pytest.mark.parametrize("cap,source", [(None, "table"), ("1024", "hybrid"), ("0", "direct")])
def test_tc_phasor_sources(cap, source, monkeypatch):
    """The three phasor sources of a non-power-of-two transform (whole series,
    N = 16384 x 3), chosen through the table-extent cap DEDISP_TC_TABLE_CAP:
    the per-bin table over every delay (max delay ~2700), the table over
    delays 0..1024 with the larger ones computed from the twiddle tables, and
    every phasor computed. Same tolerance against FP64."""
    if cap is None:
        monkeypatch.delenv("DEDISP_TC_TABLE_CAP", raising=False)
    else:
        monkeypatch.setenv("DEDISP_TC_TABLE_CAP", cap)
    nchans, nsamps = 64, 40000
    inp, params = _input(nchans, nsamps, 12)
    dms = np.linspace(0, 3300, 40, dtype=np.float32)
    p = _plan(params, dms, segmented=0, precision=1)
    assert p.get_max_delay() > 2000
    out = _run(p, nsamps, inp, 8, len(dms))
    assert p.get_phasor_source() == source
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, out.shape[1])
    rel, mx = _errs(out, ref)
    print("tc phasor source", source, rel, mx)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (source, rel, mx)


def test_tc_quarter_wave_for_power_of_two_when_table_capped(monkeypatch):
    """Power-of-two segments with the table capped at 0: the quarter-wave
    table (cheaper than computing every phasor) serves the MAC."""
    monkeypatch.setenv("DEDISP_TC_TABLE_CAP", "0")
    nchans, nsamps = 96, 90000
    inp, params = _input(nchans, nsamps, 3)
    dms = np.linspace(0, 120, 200, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=1)
    nout = nsamps - p.get_max_delay()
    out = _run(p, nsamps, inp, 8, len(dms))
    assert p.get_phasor_source() == "quarter"
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


def test_tc_automatic_segment_length():
    """segment_nfft="auto": the segment length with the least modelled time
    (16384 points here, against 65536 by the reference rule); the same series
    within the same tolerance against FP64."""
    params = (128, 128e-6, 1500.0, -1.0)
    nchans, nsamps = params[0], 123457
    inp, _ = _input(nchans, nsamps, 21, f0=params[2], df=params[3], dt=params[1])
    dms = np.linspace(0, 3000, 300, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=1, segment_nfft="auto")
    md = p.get_max_delay()
    assert dd.fdd_segment_length(nsamps, md, len(dms), nchans, 1, "auto") == 16384
    assert dd.fdd_segment_length(nsamps, md, len(dms), nchans, 1, 0) == 65536
    nout = nsamps - md
    out = _run(p, nsamps, inp, 8, len(dms))
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    rel, mx = _errs(out, ref)
    print("tc auto segments", rel, mx)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


def test_tc_fft_rows_beyond_one_launch():
    """3900 DMs x 17 segments of 65536 points: more inverse-transform rows
    than one launch's grid takes (65535), so the four-step transforms run in
    launches of whole DMs. Rows at the start, middle and end of the DM list
    against FP64 (device output; about 70 GB on the device)."""
    import torch
    nchans, nsamps = 64, 1_100_000
    inp, params = _input(nchans, nsamps, 4)
    dms = np.linspace(0, 10, 3900, dtype=np.float32)
    p = _plan(params, dms, segmented=1, precision=1, segment_nfft=65536)
    md = p.get_max_delay()
    nout = nsamps - md
    assert len(dms) * -(-nsamps // (65536 - md)) > 65535
    d_in = torch.from_numpy(inp).cuda()
    y = torch.empty((len(dms), nout), dtype=torch.float32, device="cuda")
    p.set_timing(True)
    p.execute(nsamps, d_in, 8, y, 32, dd.DEDISP_DEVICE_POINTERS)
    torch.cuda.synchronize()
    assert p.get_timing()["variant"] == 1
    rows = np.array([0, 1950, 3899])
    got = y[torch.as_tensor(rows, device="cuda")].double().cpu().numpy()
    del y
    torch.cuda.empty_cache()
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms[rows], nout)
    rel, mx = _errs(got, ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


@pytest.mark.parametrize("case", ["segmented", "many-segments", "whole-series", "table-capped"])
def test_tc_cta_pairs(case, monkeypatch):
    """DEDISP_TC_PAIR=1: the MAC on CTA pairs (tcgen05 cta_group::2, M = 256:
    each CTA produces the phasors of its 128 DMs and loads half of every B
    chunk; the leader issues the MMAs over both). Shapes: 200 DMs in one
    256-DM tile (rows past the DM list masked), 36 segments (N = 72 -> 96),
    one segment (N = 32, three A buffers), and the hybrid phasor source. Same
    tolerance against FP64."""
    monkeypatch.setenv("DEDISP_TC_PAIR", "1")
    if case == "segmented":
        nchans, nsamps = 96, 90000
        inp, params = _input(nchans, nsamps, 3)
        dms = np.linspace(0, 120, 200, dtype=np.float32)
        p = _plan(params, dms, segmented=1, precision=1)
    elif case == "many-segments":
        nchans, nsamps = 64, 72000
        inp, params = _input(nchans, nsamps, 11)
        dms = np.linspace(0, 20, 300, dtype=np.float32)
        p = _plan(params, dms, segmented=1, precision=1, segment_nfft=2048)
    elif case == "whole-series":
        nchans, nsamps = 64, 12000
        inp, params = _input(nchans, nsamps, 5)
        dms = np.linspace(0, 60, 18, dtype=np.float32)
        p = _plan(params, dms, segmented=0, precision=1)
    else:
        monkeypatch.setenv("DEDISP_TC_TABLE_CAP", "1024")
        nchans, nsamps = 64, 40000
        inp, params = _input(nchans, nsamps, 12)
        dms = np.linspace(0, 3300, 40, dtype=np.float32)
        p = _plan(params, dms, segmented=0, precision=1)
    out = _run(p, nsamps, inp, 8, len(dms))
    assert p.get_tc_form() in ("pair", "pair-deep"), p.get_tc_form()
    x = _oracle_x(inp, nsamps, params, 8)
    if case in ("whole-series", "table-capped"):
        ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, out.shape[1])
        rel, mx = _errs(out, ref)
    else:
        nout = nsamps - p.get_max_delay()
        ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
        rel, mx = _errs(out[:, :nout], ref)
    print("tc pairs", case, p.get_tc_form(), rel, mx)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (case, rel, mx)


@pytest.mark.parametrize("case", ["whole-series", "segmented"])
def test_tc_fused_wide_form(case, monkeypatch):
    """The fused MMAs (A_hi x [B_hi | B_lo], A_lo x B_hi) at 64-channel
    chunks with three A buffers, the default for npad <= 32 (also selected by
    DEDISP_TC_FORM=3): one segment
    (whole series, spectrum) and 16 segments (time series, killmask). Same
    tolerance against FP64."""
    monkeypatch.setenv("DEDISP_TC_FORM", "3")
    if case == "whole-series":
        nchans, nsamps = 128, 30000
        inp, params = _input(nchans, nsamps, 17)
        dms = np.linspace(0, 80, 150, dtype=np.float32)
        p = _plan(params, dms, segmented=0, precision=1)
        km = np.ones(nchans, np.int32)
    else:
        nchans, nsamps = 96, 30000
        inp, params = _input(nchans, nsamps, 19)
        dms = np.linspace(0, 40, 140, dtype=np.float32)
        km = np.ones(nchans, np.int32)
        km[5::11] = 0
        p = _plan(params, dms, km=km, segmented=1, precision=1, segment_nfft=2048)
    out = _run(p, nsamps, inp, 8, len(dms))
    assert p.get_tc_form() == "fused-wide", p.get_tc_form()
    x = _oracle_x(inp, nsamps, params, 8)
    if case == "whole-series":
        ref = po.fdd_spectrum(x, _delays(params), km, dms, out.shape[1])
        rel, mx = _errs(out, ref)
    else:
        nout = nsamps - p.get_max_delay()
        ref = po.fdd_timeseries(x, _delays(params), km, dms, nout)
        rel, mx = _errs(out[:, :nout], ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (case, rel, mx)

"""FDD transform lengths of every kind, through the C ABI, against the FP64
oracle, in both MAC forms.

The whole-series length rule round_up(nsamps + max_delay, 16384)
(src/fdd/FDDGPUPlan.cpp:85-93; time series: round_up(nsamps + 1, 16384)) gives
N = 16384 Q for any Q, rarely a power of two: Q = 3, 5 and 13 (a prime radix
above 8, summed directly), 65 (config 2's 1064960), and Q = 128 (N = 2^21,
above the power-of-two four-step range). Segmented plans with more than 64
segments run the tensor-core MAC in segment groups.

Tolerances (relative L2 and max-abs relative to max |ref|): FP32 MAC 2e-6 /
2e-5; 3xBF16 tensor-core MAC 1e-5 / 1e-4.
"""
import numpy as np
import pytest

import dedisp_tests_b200 as dd
from oracle import pyoracle as po
from tests.test_fdd_gpu import _delays, _errs, _input, _oracle_x, _plan

pytestmark = pytest.mark.gpu

TOL = {0: (2e-6, 2e-5), 1: (1e-5, 1e-4)}


def _check(out, ref, precision, what):
    rel, mx = _errs(out, ref)
    print(f"{what} precision {precision}: rel-L2 {rel:.3e} max-abs {mx:.3e}")
    assert rel < TOL[precision][0] and mx < TOL[precision][1], (what, precision, rel, mx)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("q", [3, 5, 13, 65, 128])
def test_whole_series_spectrum_any_length(q, precision):
    nchans = 64
    dms = np.linspace(0, 30, 9, dtype=np.float32)
    probe = _plan(_input(nchans, 1000, 1)[1], dms)
    md = probe.get_max_delay()
    nsamps = 16384 * q - md - 1000  # nsamps + max_delay rounds up to 16384 q
    inp, params = _input(nchans, nsamps, 40 + q)
    p = _plan(params, dms, segmented=0, precision=precision)
    p.set_timing(True)
    row = p.output_row_length(nsamps)
    assert row == 16384 * q
    out = np.zeros((len(dms), row), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    assert p.get_timing()["variant"] == precision
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, row)
    _check(out, ref, precision, f"spectrum N = 16384 x {q}")


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("nsamps", [70000, 200000])
def test_whole_series_timeseries_any_length(nsamps, precision):
    """N = round_up(nsamps + 1, 16384): 81920 (Q = 5) and 212992 (Q = 13)."""
    nchans = 64
    inp, params = _input(nchans, nsamps, 60)
    dms = np.linspace(0, 45, 12, dtype=np.float32)
    p = _plan(params, dms, segmented=0, timeseries=True, precision=precision)
    p.set_timing(True)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    assert p.get_timing()["variant"] == precision
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    _check(out, ref, precision, f"time series nsamps {nsamps}")


@pytest.mark.parametrize("precision", [0, 1])
def test_segmented_more_than_64_segments(precision):
    """70 segments of 16384-point FFTs: the tensor-core MAC runs two segment
    groups (64 + 6) into one output."""
    nchans = 64
    dms = np.linspace(0, 60, 20, dtype=np.float32)
    probe = _plan(_input(nchans, 1000, 1)[1], dms)
    good = 16384 - probe.get_max_delay()
    nsamps = 69 * good + good // 2
    inp, params = _input(nchans, nsamps, 71)
    p = _plan(params, dms, segmented=1, segment_nfft=16384, precision=precision)
    p.set_timing(True)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    t = p.get_timing()
    assert t["variant"] == precision
    if precision == 1:
        assert t["launches"] == 2, t
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    _check(out, ref, precision, "70 segments")


@pytest.mark.parametrize("precision", [0, 1])
def test_segmented_long_segments_large_delays(precision):
    """Max delay ~30000 samples: the reference doubling rule picks 262144-point
    segments. Neither the per-bin delay table (30001 phasors) nor the
    quarter-wave table (65537) fits shared memory, so the tensor-core MAC
    computes every phasor from the two-level twiddle tables."""
    nchans = 128
    dms = np.linspace(0, 64, 10, dtype=np.float32)
    kw = dict(f0=400.0, df=-1.0, dt=64e-6)
    probe = _plan(_input(nchans, 1000, 1, **kw)[1], dms)
    md = probe.get_max_delay()
    assert 26214 < md < 52428, md
    nsamps = 400000
    inp, params = _input(nchans, nsamps, 81, **kw)
    p = _plan(params, dms, segmented=1, precision=precision)
    p.set_timing(True)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, inp, 8, out, 32)
    assert p.get_timing()["variant"] == precision
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_timeseries(x, _delays(params), np.ones(nchans, np.int32), dms, nout)
    _check(out, ref, precision, "262144-point segments")

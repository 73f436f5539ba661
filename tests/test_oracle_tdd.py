"""Known-answer and cross-checks of the CPU oracle itself (CPU only)."""
import numpy as np
import pytest

from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po


def _numpy_tdd_sums(samples, delays, km, dms, nsamps_out):
    """Pure-numpy restatement: sum_c km[c] * x[t + rn(dm*delay[c]), c]."""
    nsamps, nchans = samples.shape
    out = np.zeros((len(dms), nsamps_out), np.uint64)
    for i, dm in enumerate(dms):
        d = np.array([po.delay_rn(float(dm), float(x)) for x in delays], np.int64)
        for c in range(nchans):
            if km[c] == 0:
                continue
            idx = np.arange(nsamps_out) + d[c]
            v = np.where(idx < nsamps, samples[np.minimum(idx, nsamps - 1), c], 0)
            out[i] += (np.uint64(km[c]) * v.astype(np.uint64)) & np.uint64(0xFFFFFFFF)
    return out


@pytest.mark.parametrize("nbits", [1, 2, 4, 8, 16, 32])
def test_oracle_sums_match_numpy(nbits):
    rng = np.random.default_rng(nbits)
    nchans = 64 if nbits < 32 else 8
    nsamps = 700
    vals = rng.integers(0, 1 << min(nbits, 31), (nsamps, nchans), dtype=np.int64).astype(np.uint32)
    packed = sy.pack(vals, nbits)
    delays = po.delay_table(nchans, 1e-3, 400.0, -1.0)
    dms = np.linspace(0, 40, 9, dtype=np.float32)
    km = np.ones(nchans, np.int32)
    km[3::7] = 0
    md = po.max_delay(dms, delays)
    nout = nsamps - md
    ours = po.tdd_sums(packed, nsamps, packed.shape[1], nbits, nchans, delays, km, dms, nout)
    ref = _numpy_tdd_sums(vals, delays, km, dms, nout)
    assert np.array_equal(ours, ref)


def test_impulse_gives_shifted_delta_per_dm():
    nchans, nsamps = 32, 600
    delays = po.delay_table(nchans, 1e-3, 400.0, -1.0)
    vals = np.zeros((nsamps, nchans), np.uint32)
    t_imp = 450
    vals[t_imp, :] = 1
    dms = np.array([0.0, 10.0, 30.0], np.float32)
    md = po.max_delay(dms, delays)
    sums = po.tdd_sums(sy.pack(vals, 8), nsamps, nchans, 8, nchans, delays,
                       np.ones(nchans, np.int32), dms, nsamps - md)
    for i, dm in enumerate(dms):
        for c in range(nchans):
            t = t_imp - po.delay_rn(float(dm), float(delays[c]))
            if 0 <= t < nsamps - md:
                assert sums[i, t] >= 1
        assert sums[i].sum() == sum(1 for c in range(nchans)
                                    if 0 <= t_imp - po.delay_rn(float(dm), float(delays[c]))
                                    < nsamps - md)


def test_constant_input_gives_constant_output():
    nchans, nsamps = 64, 1000
    delays = po.delay_table(nchans, 250e-6, 1500.0, -1.0)
    vals = np.full((nsamps, nchans), 3, np.uint32)
    dms = np.linspace(0, 50, 5, dtype=np.float32)
    md = po.max_delay(dms, delays)
    km = np.ones(nchans, np.int32)
    km[:10] = 0
    out = po.tdd(sy.pack(vals, 2), nsamps, nchans // 4, 2, nchans, delays, km, dms, 32,
                 nsamps - md)
    expect = po.scale_output(3 * 54, 2, 32, nchans)
    assert np.all(out == expect)


def test_killmask_zero_everything():
    nchans, nsamps = 32, 400
    delays = po.delay_table(nchans, 1e-3, 400.0, -1.0)
    vals = np.random.default_rng(0).integers(0, 256, (nsamps, nchans)).astype(np.uint32)
    dms = np.array([0.0, 5.0], np.float32)
    md = po.max_delay(dms, delays)
    out = po.tdd(sy.pack(vals, 8), nsamps, nchans, 8, nchans, delays,
                 np.zeros(nchans, np.int32), dms, 8, nsamps - md)
    assert np.all(out == 0)


def test_fft_matches_numpy():
    rng = np.random.default_rng(1)
    for n in (16, 1024, 48, 16384 * 3, 1000):
        z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        assert np.allclose(po.fft(z), np.fft.fft(z), atol=1e-8 * np.sqrt(n), rtol=0)


def test_fdd_spectrum_is_fft_of_timeseries():
    nchans, nsamps = 16, 3000
    rng = np.random.default_rng(2)
    raw = rng.integers(0, 256, (nsamps, nchans)).astype(np.uint8)
    x = po.fdd_unpack(raw, nsamps, nchans, 8, nchans)
    assert np.array_equal(x, (raw.T.astype(np.float32) - np.float32(127.5)) * np.float32(1 / 16))
    delays = po.delay_table(nchans, 1e-3, 400.0, -2.0)
    dms = np.array([0.0, 7.0, 19.0], np.float32)
    km = np.ones(nchans, np.int32)
    md = po.max_delay(dms, delays)
    nfft = po.fdd_nfft_spectrum(nsamps, md)
    spec = po.fdd_spectrum(x, delays, km, dms, nfft)
    ts = po.fdd_timeseries(x, delays, km, dms, nsamps - md)
    for i in range(len(dms)):
        z = spec[i, 0::2] + 1j * spec[i, 1::2]
        full = np.concatenate([z, [0], np.conj(z[1:][::-1])])
        # the Nyquist bin is not part of the output; rebuild it directly
        d = np.array([po.lib().orc_delay_trunc(float(dms[i]), float(v)) for v in delays])
        zt = np.zeros(nfft)
        for c in range(nchans):
            zt += np.roll(np.concatenate([x[c], np.zeros(nfft - nsamps)]), -d[c])
        ref = np.fft.fft(zt)
        assert np.allclose(z, ref[: nfft // 2], atol=1e-9 * np.abs(ref).max())
        assert np.allclose(zt[: nsamps - md], ts[i], atol=1e-9)
        del full


def test_segment_geometry_matches_reference_rule():
    # config 2: max delay 5243 -> nfft 32768, nsamp_good 27525, 39 chunks
    assert po.fdd_segment_geometry(1 << 20, 5243) == (32768, 27525, 39)
    assert po.fdd_nfft_spectrum(1 << 20, 5243) == 1064960


@pytest.mark.parametrize("nbits", [1, 2, 4, 8, 16])
def test_oracle_fdd_unpack_packed_widths(nbits):
    """Packed samples are centred at (2^nbits - 1) / 2 and scaled by 1/nchans
    (8-bit: the reference's (v - 127.5) / nchan)."""
    rng = np.random.default_rng(nbits)
    nchans, nsamps = 64, 50
    vals = rng.integers(0, 1 << nbits, (nsamps, nchans), dtype=np.uint32)
    packed = sy.pack(vals, nbits)
    x = po.fdd_unpack(packed, nsamps, packed.shape[1], nbits, nchans)
    mid = np.float32(((1 << nbits) - 1) * 0.5)
    want = ((vals.astype(np.float32) - mid) * np.float32(1.0 / nchans)).T
    assert np.array_equal(x, want)

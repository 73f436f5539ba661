"""Batched multi-beam FDD through the C ABI: every beam's output must match an
FDD plan run on that beam alone (segmented time series, tensor-core MAC) and
the FP64 oracle, with and without the captured CUDA graph, for ragged beams
(different sample counts, DM ranges and trial counts, an unsorted DM list,
segment lengths from 16384 to 65536 points, a beam with more than 64
segments), other input widths and a killmask.

Tolerances (relative L2; max-abs relative to max |ref|): against the FP64
oracle 1e-5 / 1e-4 (the 3xBF16 tensor-core form); against the single-beam
plan 1e-5 / 1e-4 as well, since a batch may take its phasors from the
two-level twiddle tables where a lone plan reads its quarter-wave table.
"""
import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = (128, 128e-6, 1500.0, -1.0)
TOL = (1e-5, 1e-4)


def _errs(ours, ref):
    ours = np.asarray(ours, np.float64)
    ref = np.asarray(ref, np.float64)
    return (np.linalg.norm(ours - ref) / np.linalg.norm(ref),
            np.abs(ours - ref).max() / np.abs(ref).max())


def _beam_inputs(nbits, seed, specs):
    """specs: (nsamps, dm list). Noise around mid-scale plus a pulse."""
    rng = np.random.default_rng(seed)
    out = []
    for nsamps, dms in specs:
        hi = (1 << nbits) - 1
        vals = np.clip(np.rint(rng.normal(hi / 2, max(hi / 6, 0.6), (nsamps, PARAMS[0]))), 0, hi)
        out.append((sy.pack(vals.astype(np.uint32), nbits), np.asarray(dms, np.float32)))
    return out


def _run_batch(nbits, host, km=None, graph=True, reps=2, sources=None):
    import torch
    b = dd.FddBatch(*PARAMS, in_nbits=nbits)
    if km is not None:
        b.set_killmask(km)
    probe = dd.TDDPlan(*PARAMS)
    beams, outs = [], []
    for packed, dms in host:
        probe.set_dm_list(dms)
        nout = packed.shape[0] - probe.get_max_delay()
        x = torch.from_numpy(packed).cuda()
        y = torch.full((len(dms), nout + 5), -7.0, dtype=torch.float32, device="cuda")
        beams.append((x, packed.shape[1], packed.shape[0], dms, y, y.shape[1] * 4))
        outs.append((y, nout))
    b.set_beams(beams)
    if sources is not None:
        sources.extend(b.phasor_source(i) for i in range(len(beams)))
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(reps):
        for y, _ in outs:
            y.fill_(-7.0)
        b.execute(stream, use_graph=graph)
        b.sync(stream)
    res = []
    for (y, nout) in outs:
        h = y.cpu().numpy()
        assert np.all(h[:, nout:] == -7.0), "wrote past the row"
        res.append(h[:, :nout])
    b.close()
    return res


def _plan_out(packed, nbits, dms, km=None):
    p = dd.FDDGPUPlan(*PARAMS)
    p.set_dm_list(dms)
    if km is not None:
        p.set_killmask(km)
    p.set_options(segmented=1, precision=1)
    nout = packed.shape[0] - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(packed.shape[0], packed, nbits, out, 32)
    return out


def _oracle(packed, nbits, dms, km=None):
    nchans = PARAMS[0]
    delays = po.delay_table(nchans, np.float32(PARAMS[1]), np.float32(PARAMS[2]), np.float32(PARAMS[3]))
    km = np.ones(nchans, np.int32) if km is None else np.asarray(km, np.int32)
    x = po.fdd_unpack(packed, packed.shape[0], packed.shape[1], nbits, nchans)
    probe = dd.TDDPlan(*PARAMS)
    probe.set_dm_list(dms)
    nout = packed.shape[0] - probe.get_max_delay()
    return po.fdd_timeseries(x, delays, km, dms, nout)


def _specs():
    rng = np.random.default_rng(3)
    unsorted = rng.uniform(0, 90, 41).astype(np.float32)
    unsorted[-1] = 90.0
    return [(40000, np.linspace(0, 60, 150)),        # 16384-point segments
            (123457, np.linspace(0, 3000, 300)),     # 65536-point segments (max delay ~8400)
            (90000, unsorted),                       # unsorted list, last DM sets the max delay
            (1200000, np.linspace(0, 30, 20)),       # more than 64 segments (two groups)
            (30000, np.linspace(0, 10, 129))]        # two DM tiles of 128 + 1


@pytest.mark.parametrize("graph", [True, False])
def test_fdd_batch_matches_plans_and_oracle(graph):
    host = _beam_inputs(8, 11, _specs())
    got = _run_batch(8, host, graph=graph)
    for i, ((packed, dms), g) in enumerate(zip(host, got)):
        want = _plan_out(packed, 8, dms)
        assert g.shape == want.shape
        rel, mx = _errs(g, want)
        assert rel < TOL[0] and mx < TOL[1], ("vs plan", i, rel, mx)
        if packed.shape[0] <= 200000:
            ref = _oracle(packed, 8, dms)
            rel, mx = _errs(g, ref)
            print(f"beam {i}: rel-L2 {rel:.3e} max-abs {mx:.3e} vs FP64")
            assert rel < TOL[0] and mx < TOL[1], ("vs FP64", i, rel, mx)


@pytest.mark.parametrize("nbits", [2, 32])
def test_fdd_batch_other_widths_and_killmask(nbits):
    specs = [(50000, np.linspace(0, 80, 64)), (70000, np.linspace(0, 40, 200))]
    if nbits == 32:
        rng = np.random.default_rng(5)
        host = []
        for nsamps, dms in specs:
            x = rng.standard_normal((nsamps, PARAMS[0])).astype("<f4")
            host.append((np.ascontiguousarray(x).view(np.uint8).reshape(nsamps, -1),
                         np.asarray(dms, np.float32)))
    else:
        host = _beam_inputs(nbits, 17, specs)
    km = np.ones(PARAMS[0], np.int32)
    km[::7] = 0
    got = _run_batch(nbits, host, km=km)
    for i, ((packed, dms), g) in enumerate(zip(host, got)):
        ref = _oracle(packed, nbits, dms, km)
        rel, mx = _errs(g, ref)
        assert rel < TOL[0] and mx < TOL[1], (nbits, i, rel, mx)


def test_fdd_batch_hybrid_phasors(monkeypatch):
    """Every beam's per-bin table capped at delays 0..1024 (the larger delays
    computed from the twiddle tables): the same outputs as the lone plans
    and the FP64 oracle."""
    monkeypatch.setenv("DEDISP_TC_TABLE_CAP", "1024")
    specs = [(123457, np.linspace(0, 3000, 300)), (60000, np.linspace(0, 700, 140))]
    host = _beam_inputs(8, 23, specs)
    sources = []
    got = _run_batch(8, host, sources=sources)
    monkeypatch.delenv("DEDISP_TC_TABLE_CAP")
    # 65536-point segments (max delay ~8400): the quarter-wave table costs
    # less than 12 % table coverage; max delay ~1960: the hybrid source
    assert sources == ["quarter", "hybrid"], sources
    for i, ((packed, dms), g) in enumerate(zip(host, got)):
        want = _plan_out(packed, 8, dms)
        rel, mx = _errs(g, want)
        assert rel < TOL[0] and mx < TOL[1], ("vs plan", i, rel, mx)
        ref = _oracle(packed, 8, dms)
        rel, mx = _errs(g, ref)
        assert rel < TOL[0] and mx < TOL[1], ("vs FP64", i, rel, mx)


def test_fdd_batch_automatic_segment_lengths():
    """set_segment_nfft("auto"): per beam the segment length with the least
    modelled time (2048 to 32768 points for these beams, against 16384 and
    65536 by the reference rule); same tolerance against the FP64 oracle."""
    import torch
    host = _beam_inputs(8, 29, _specs())
    b = dd.FddBatch(*PARAMS, in_nbits=8)
    b.set_segment_nfft("auto")
    probe = dd.TDDPlan(*PARAMS)
    beams, outs = [], []
    for packed, dms in host:
        probe.set_dm_list(dms)
        nout = packed.shape[0] - probe.get_max_delay()
        x = torch.from_numpy(packed).cuda()
        y = torch.full((len(dms), nout), -7.0, dtype=torch.float32, device="cuda")
        beams.append((x, packed.shape[1], packed.shape[0], dms, y, y.shape[1] * 4))
        outs.append(y)
    b.set_beams(beams)
    stream = torch.cuda.current_stream().cuda_stream
    b.execute(stream, use_graph=True)
    b.sync(stream)
    for i, ((packed, dms), y) in enumerate(zip(host, outs)):
        if packed.shape[0] > 200000:
            continue
        ref = _oracle(packed, 8, dms)
        rel, mx = _errs(y.cpu().numpy(), ref)
        assert rel < TOL[0] and mx < TOL[1], ("auto segments vs FP64", i, rel, mx)
    b.close()


def test_fdd_batch_cta_pairs(monkeypatch):
    """The batch's MAC on CTA pairs (DEDISP_TC_PAIR=1): every beam against
    its FP64 oracle."""
    monkeypatch.setenv("DEDISP_TC_PAIR", "1")
    specs = [(40000, np.linspace(0, 60, 150)), (123457, np.linspace(0, 3000, 300)),
             (30000, np.linspace(0, 10, 129))]
    host = _beam_inputs(8, 31, specs)
    got = _run_batch(8, host)
    for i, ((packed, dms), g) in enumerate(zip(host, got)):
        ref = _oracle(packed, 8, dms)
        rel, mx = _errs(g, ref)
        assert rel < TOL[0] and mx < TOL[1], ("pairs vs FP64", i, rel, mx)

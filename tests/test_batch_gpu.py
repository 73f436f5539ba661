"""Batched multi-beam TDD through the C ABI: every beam's output must be bit
identical to a TDD plan run on that beam alone (and to the CPU oracle), with
and without the captured CUDA graph, after autotuning, for ragged beams
(different sample counts, DM lists, an unsorted list, a beam with no output
samples), other input widths and a general killmask."""
import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = (384, 81.92e-6, 1670.0, -0.25)


def _beams(nbits, seed, specs):
    """specs: list of (nsamps, dm list). Returns packed host inputs."""
    rng = np.random.default_rng(seed)
    out = []
    for nsamps, dms in specs:
        vals = rng.integers(0, 1 << nbits, (nsamps, PARAMS[0]), dtype=np.uint32)
        out.append((sy.pack(vals, nbits), np.asarray(dms, np.float32)))
    return out


def _plan_out(packed, nsamps, nbits, dms, km=None):
    p = dd.TDDPlan(*PARAMS)
    p.set_dm_list(dms)
    if km is not None:
        p.set_killmask(km)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    if nout:
        p.execute(nsamps, packed, nbits, out, 32)
    return out


def _run_batch(nbits, host, km=None, tune=False, graph=True, reps=2, shape=None):
    import torch
    b = dd.Batch(*PARAMS, in_nbits=nbits, out_nbits=32)
    if km is not None:
        b.set_killmask(km)
    d_in, d_out, beams = [], [], []
    for packed, dms in host:
        nsamps = packed.shape[0]
        x = torch.from_numpy(packed).cuda()
        d_in.append(x)
        beams.append([x, packed.shape[1], nsamps, dms, None, 0])
    # output rows sized from the plan rule (max delay of the last DM)
    b_probe = dd.TDDPlan(*PARAMS)
    for i, (packed, dms) in enumerate(host):
        b_probe.set_dm_list(dms)
        nout = packed.shape[0] - b_probe.get_max_delay()
        y = torch.full((len(dms), max(nout, 1) + 3), -7.0, dtype=torch.float32, device="cuda")
        d_out.append((y, nout))
        beams[i][4] = y
        beams[i][5] = y.shape[1] * 4
    b.set_beams([tuple(x) for x in beams])
    for i, (_, nout) in enumerate(d_out):
        assert b.max_delay(i) == host[i][0].shape[0] - nout
    if shape is not None:
        b.set_shape(*shape)
    if tune:
        b.autotune()
    b.set_timing(True)
    for _ in range(reps):
        b.execute(0, use_graph=graph)
    torch.cuda.synchronize()
    t = b.get_timing()
    res = []
    for y, nout in d_out:
        a = y.cpu().numpy()
        assert np.all(a[:, max(nout, 0):] == -7.0)  # nothing written past the row
        res.append(a[:, :nout])
    b.close()
    return res, t


def _specs(rng_seed=3):
    rng = np.random.default_rng(rng_seed)
    unsorted = rng.uniform(0, 150, 77).astype(np.float32)
    unsorted[-1] = 150.0  # the max delay follows the last DM
    return [(9000, np.linspace(0, 120, 100)), (14000, np.linspace(0, 300, 61)),
            (6000, unsorted), (12000, np.linspace(5, 200, 130)),
            (2000, np.linspace(0, 100, 20))]


def test_batch_8bit_matches_plans_graph_and_direct():
    specs = _specs()
    # a beam with exactly max_delay samples: no output samples, no work
    p = dd.TDDPlan(*PARAMS)
    p.set_dm_list(np.linspace(0, 80, 9, dtype=np.float32))
    specs.append((p.get_max_delay(), np.linspace(0, 80, 9)))
    host = _beams(8, 11, specs)
    want = [_plan_out(p, p.shape[0], 8, d) for p, d in host]
    assert want[-1].shape[1] == 0
    for graph in (False, True):
        got, t = _run_batch(8, host, graph=graph)
        for g, w in zip(got, want):
            assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
        # per beam with output one K1d (the default shape is quad-strided,
        # built straight from the input), then one persistent launch
        assert t["launches"] == sum(w.shape[1] > 0 for w in want) + 1


def test_batch_oracle_one_beam_and_every_shape():
    host = _beams(8, 12, _specs(4)[:3])
    packed, dms = host[1]
    delays = po.delay_table(PARAMS[0], np.float32(PARAMS[1]), np.float32(PARAMS[2]),
                            np.float32(PARAMS[3]))
    for v in range(dd.batch_variant_count(8)):
        for cs in (0, 8):
            got, _ = _run_batch(8, host, shape=(v, cs), reps=1)
            nout = got[1].shape[1]
            ref = po.tdd(packed, packed.shape[0], packed.shape[1], 8, PARAMS[0], delays,
                         np.ones(PARAMS[0], np.int32), dms, 32, nout)
            assert np.array_equal(got[1].view(np.uint32), ref.view(np.uint32)), (v, cs)


def test_batch_autotune_keeps_results():
    host = _beams(8, 13, _specs(5))
    want = [_plan_out(p, p.shape[0], 8, d) for p, d in host]
    got, _ = _run_batch(8, host, tune=True)
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))


@pytest.mark.parametrize("nbits", [2, 4])
def test_batch_other_widths(nbits):
    host = _beams(nbits, 14, _specs(6)[:3])
    want = [_plan_out(p, p.shape[0], nbits, d) for p, d in host]
    # default: quad-strided rows (samples widened to bytes), persistent launch
    got, t = _run_batch(nbits, host)
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
    assert t["launches"] == len(host) + 1  # K1d per beam, one persistent launch
    # packed-row kernel: one dedispersion launch per beam
    got, t = _run_batch(nbits, host, shape=(0, 0))
    for g, w in zip(got, want):
        assert np.array_equal(g.view(np.uint32), w.view(np.uint32))
    assert t["launches"] == 2 * len(host)


def test_batch_killmask_zero_one_and_general():
    host = _beams(8, 15, _specs(7)[:3])
    km = np.ones(PARAMS[0], np.int32)
    km[3::17] = 0
    for mask in (km, np.where(np.arange(PARAMS[0]) % 5 == 0, 2, km).astype(np.int32)):
        want = [_plan_out(p, p.shape[0], 8, d, km=mask) for p, d in host]
        got, _ = _run_batch(8, host, km=mask)
        for g, w in zip(got, want):
            assert np.array_equal(g.view(np.uint32), w.view(np.uint32))


def test_batches_share_one_workspace():
    import torch
    host_a = _beams(8, 16, _specs(8)[:2])
    host_b = _beams(8, 17, _specs(9)[2:4])
    outs = []
    batches = []
    for host in (host_a, host_b):
        b = dd.Batch(*PARAMS)
        beams, ys = [], []
        for packed, dms in host:
            p = dd.TDDPlan(*PARAMS)
            p.set_dm_list(dms)
            nout = packed.shape[0] - p.get_max_delay()
            x = torch.from_numpy(packed).cuda()
            y = torch.zeros((len(dms), nout), dtype=torch.float32, device="cuda")
            beams.append((x, packed.shape[1], packed.shape[0], dms, y, nout * 4))
            ys.append(y)
        b.set_beams(beams)
        batches.append((b, beams))
        outs.append(ys)
    nbytes = max(b.workspace_size() for b, _ in batches)
    ws = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    for b, _ in batches:
        b.set_workspace(ws, nbytes)
    for _ in range(2):
        for b, _ in batches:
            b.execute(0, use_graph=True)
    torch.cuda.synchronize()
    for host, ys in zip((host_a, host_b), outs):
        for (packed, dms), y in zip(host, ys):
            w = _plan_out(packed, packed.shape[0], 8, dms)
            assert np.array_equal(y.cpu().numpy().view(np.uint32), w.view(np.uint32))
    for b, _ in batches:
        b.close()

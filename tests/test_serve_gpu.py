"""Streaming server through the C ABI: the concatenated per-gulp outputs of a
beam must equal one dedispersion of the whole zero-prefixed series (the tail
starts as max_delay zero rows): bit for bit for TDD beams, within the FDD
tolerance against the FP64 oracle for FDD beams; gulps of one beam stay in
order while several beams and workers run concurrently."""
import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

PARAMS = (256, 64e-6, 1500.0, -0.25)


def _stream(nbits, ngulps, seed, lengths):
    rng = np.random.default_rng(seed)
    gl = [int(rng.choice(lengths)) for _ in range(ngulps)]
    vals = rng.integers(0, 1 << nbits, (sum(gl), PARAMS[0]), dtype=np.uint32)
    return sy.pack(vals, nbits), gl


def _run(server, beams, d_outs):
    """beams: list of (beam id, packed series, gulp lengths); interleaved submits."""
    import torch
    tickets = []
    offs = [0] * len(beams)
    k = 0
    while any(offs[i] < len(b[2]) for i, b in enumerate(beams)):
        i = k % len(beams)
        k += 1
        bid, packed, gl = beams[i]
        if offs[i] >= len(gl):
            continue
        g = offs[i]
        r0 = sum(gl[:g])
        n = gl[g]
        rows = np.ascontiguousarray(packed[r0:r0 + n])
        out = torch.empty((server_dm[bid], n), dtype=torch.float32, device="cuda")
        tickets.append(server.submit(bid, rows, n, out))
        d_outs[bid].append(out)
        offs[i] += 1
    server.drain()
    torch.cuda.synchronize()
    return tickets


server_dm = {}


@pytest.mark.parametrize("fdd_precision", [0, 1])
@pytest.mark.parametrize("nbits", [2, 8])
def test_tdd_and_fdd_beams_match_whole_series(nbits, fdd_precision):
    """fdd_precision 0: FP32 CUDA-core MAC (rel-L2 < 2e-6 against FP64);
    1: 3xBF16 tensor-core MAC (rel-L2 < 1e-5)."""
    import torch
    s = dd.StreamServer(*PARAMS, in_nbits=nbits, max_gulp=12000, tdd_workers=2, fdd_workers=1,
                        fdd_precision=fdd_precision)
    dms_a = np.linspace(0, 150, 37, dtype=np.float32)
    dms_b = np.linspace(0, 220, 53, dtype=np.float32)
    ids = [s.add_beam(dms_a, 0), s.add_beam(dms_b, 0), s.add_beam(dms_a, 0), s.add_beam(dms_b, 1)]
    for i, d in zip(ids, (dms_a, dms_b, dms_a, dms_b)):
        server_dm[i] = len(d)
    held = s.start()
    assert held > 0
    data = [_stream(nbits, 7, 50 + i, [1000, 4096, 12000, 333]) for i in range(4)]
    outs = {i: [] for i in ids}
    _run(s, [(ids[i], data[i][0], data[i][1]) for i in range(4)], outs)
    recs = s.records()
    assert len(recs) == sum(len(d[1]) for d in data)
    for r in recs:
        assert r["t_submit"] <= r["t_start"] <= r["t_done"] and r["device_ms"] > 0
    for bi in range(4):
        bid = ids[bi]
        packed, gl = data[bi]
        dms = (dms_a, dms_b, dms_a, dms_b)[bi]
        md = s.max_delay(bid)
        series = np.concatenate([np.zeros((md, packed.shape[1]), np.uint8), packed])
        got = np.concatenate([o.cpu().numpy() for o in outs[bid]], axis=1)
        assert got.shape == (len(dms), sum(gl))
        if bi < 3:  # TDD beam: bit-exact with one plan over the whole series
            p = dd.TDDPlan(*PARAMS)
            p.set_dm_list(dms)
            want = np.zeros((len(dms), sum(gl)), np.float32)
            p.execute(series.shape[0], series, nbits, want, 32)
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), bi
        else:       # FDD beam: time-domain FP64 oracle of the same series
            delays = po.delay_table(PARAMS[0], np.float32(PARAMS[1]), np.float32(PARAMS[2]),
                                    np.float32(PARAMS[3]))
            x = po.fdd_unpack(series, series.shape[0], series.shape[1], nbits, PARAMS[0])
            ref = po.fdd_timeseries(x, delays, np.ones(PARAMS[0], np.int32), dms, sum(gl))
            rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert rel < (2e-6 if fdd_precision == 0 else 1e-5), rel
    s.close()


def test_budget_is_enforced():
    s = dd.StreamServer(*PARAMS, in_nbits=8, max_gulp=4096, tdd_workers=1, hbm_budget=1 << 20)
    s.add_beam(np.linspace(0, 100, 20, dtype=np.float32), 0)
    with pytest.raises(dd.DedispError) as e:
        s.start()
    assert e.value.code == 1  # DEDISP_MEM_ALLOC_FAILED
    s.close()

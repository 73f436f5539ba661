"""The oracle pinned against the reference itself (CPU only).

Golden fixtures in tests/golden/ were produced by the reference's own code
(tests/golden/make_golden.py); when the reference pieces are built in
oracle/_ref they are also compared live.
"""
import os

import numpy as np
import pytest

from oracle import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _f32bits(a):
    return np.asarray(a, np.float32).view(np.uint32)


def test_delay_tables_match_reference_golden():
    g = np.load(os.path.join(GOLDEN, "plan_setup.npz"))
    i = 0
    while f"params_{i}" in g:
        n, dt, f0, df = g[f"params_{i}"]
        ours = po.delay_table(int(n), float(np.float32(dt)), float(np.float32(f0)),
                              float(np.float32(df)))
        assert np.array_equal(_f32bits(ours), _f32bits(g[f"delay_{i}"])), i
        i += 1
    assert i >= 7


def test_dm_lists_and_max_delay_match_reference_golden():
    g = np.load(os.path.join(GOLDEN, "plan_setup.npz"))
    j = 0
    while f"dmgen_{j}" in g:
        pi, s, e, ti, tol = g[f"dmgen_{j}"]
        n, dt, f0, df = g[f"params_{int(pi)}"]
        dms = po.generate_dm_list(int(n), dt, f0, df, s, e, ti, tol)
        ref = g[f"dmlist_{j}"]
        assert len(dms) == len(ref)
        assert np.array_equal(_f32bits(dms), _f32bits(ref))
        delays = po.delay_table(int(n), float(np.float32(dt)), float(np.float32(f0)),
                                float(np.float32(df)))
        assert po.max_delay(dms, delays) == int(g[f"dmmax_{j}"][0])
        j += 1
    # config 1: 3643 DMs, max delay 35500 samples
    assert len(g["dmlist_0"]) == 3643 and int(g["dmmax_0"][0]) == 35500


def test_epilogue_matches_reference_golden():
    tab = np.load(os.path.join(GOLDEN, "epilogue.npz"))["table"]
    bad = 0
    for in_nb, out_nb, nch, s, bits in tab.tolist():
        v = po.scale_output(int(s), int(in_nb), int(out_nb), int(nch))
        mine = int(np.asarray(v, np.float32).view(np.uint32)) if out_nb == 32 else int(v)
        bad += mine != int(bits)
    assert bad == 0 and len(tab) > 5000


def test_oracle_matches_reference_gpu_tdd_outputs():
    """The whole TDD loop of the oracle against outputs of the reference's own
    TDDPlan / DedispPlan run on a B200 (tests/golden/make_golden.py gpu)."""
    import hashlib
    from tests.golden.make_golden import GPU_CASES, gpu_case_input
    g = np.load(os.path.join(GOLDEN, "ref_gpu_outputs.npz"))
    checked = 0
    for k, (plan, nch, f0, df, dt, ns, nb, onb, ndm, dmax, kme, seed) in enumerate(GPU_CASES):
        inp = gpu_case_input(nch, f0, df, dt, ns, nb, seed)
        assert hashlib.sha256(inp.tobytes()).hexdigest() == str(g[f"sha_{k}"][0])
        dms = np.linspace(0, dmax, ndm, dtype=np.float32)
        km = np.ones(nch, np.int32)
        if kme:
            km[::kme] = 0
        delays = po.delay_table(nch, np.float32(dt), np.float32(f0), np.float32(df))
        nout = ns - po.max_delay(dms, delays)
        ours = po.tdd(inp, ns, inp.shape[1], nb, nch, delays, km, dms, onb, nout)
        ref = g[f"out_{k}"]
        if plan == "tdd" and nb == 32:
            # reference defect: no 32-bit unpack kernel in TDDPlan, zeros out
            assert not ref.any()
            continue
        assert np.array_equal(ours.view(np.uint8).ravel(), ref), (k, plan, nb)
        checked += 1
    assert checked == 7


@pytest.mark.skipif(not po.ref_available("libref_plan.so"), reason="reference not built")
def test_live_reference_plan_sweep():
    rng = np.random.default_rng(3)
    for _ in range(40):
        n = int(rng.choice([16, 64, 333, 1024, 4096]))
        dt = float(np.float32(rng.uniform(20e-6, 1e-3)))
        f0 = float(np.float32(rng.uniform(100.0, 3000.0)))
        df = float(np.float32(-rng.uniform(0.01, 0.8) * f0 / n / 1.5))
        assert np.array_equal(_f32bits(po.delay_table(n, dt, f0, df)),
                              _f32bits(po.ref_delay_table(n, dt, f0, df)))
        dms = np.sort(rng.uniform(0, 3000, int(rng.integers(1, 50)))).astype(np.float32)
        d = po.delay_table(n, dt, f0, df)
        assert po.max_delay(dms, d) == po.ref_set_dm_list_max_delay(n, dt, f0, df, dms)


@pytest.mark.skipif(not po.ref_available("libref_epilogue.so"), reason="reference not built")
def test_live_reference_epilogue_legacy_and_tdd():
    rng = np.random.default_rng(5)
    for in_nb in (1, 2, 4, 8, 16, 32):
        for out_nb in (8, 16, 32):
            nch = int(rng.choice([1, 100, 2048, 8192]))
            mx = nch * ((1 << in_nb) - 1)
            for s in rng.integers(0, mx + 1, 50):
                a = po.scale_output(int(s), in_nb, out_nb, nch)
                for legacy in (False, True):
                    b = po.ref_scale_output(int(s), in_nb, out_nb, nch, legacy=legacy)
                    assert np.asarray(a).tobytes() == np.asarray(b).tobytes()

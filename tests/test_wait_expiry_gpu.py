"""Expiry of the kernels' bounded waits, through the C ABI.

The quad-strided TDD kernels (single plan and persistent batch) and the
tensor-core FDD MAC poll mbarriers for their own bulk copies and MMAs, each
poll bounded by a limit of GPU global time. With the expiry test switched on
(dedisp_b200_set_wait_expiry_test) every such kernel also waits, at the first
wait of its pipeline, on an mbarrier that nothing arrives on: the limit (1 ms
here) runs out, the kernel waits (bounded) for its own copies and MMAs still
in flight, frees its tensor memory and returns, and the call must report
DEDISP_INTERNAL_GPU_ERROR. The same plan, run again with the switch off, must
then give correct results (bit-exact for TDD, the tensor-core tolerance for
FDD): the error path leaves the plan and the context usable.
"""
import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po
from tests.test_fdd_gpu import _delays, _errs, _input, _oracle_x, _plan
from tests.test_fdd_tc_gpu import TC_MAX_ABS, TC_REL_L2

pytestmark = pytest.mark.gpu

INTERNAL = dd.ERROR_NAMES.index("DEDISP_INTERNAL_GPU_ERROR")
LIMIT_NS = 1_000_000


class _Expiry:
    """Switches the expiry test on (with a 1 ms limit) for the block."""

    def __enter__(self):
        dd.set_wait_limit_ns(LIMIT_NS)
        dd.set_wait_expiry_test(True)
        assert dd.get_wait_limit_ns() == LIMIT_NS

    def __exit__(self, *exc):
        dd.set_wait_expiry_test(False)
        dd.set_wait_limit_ns(0)
        assert dd.get_wait_limit_ns() == 2_000_000_000


def _tdd_case(nchans=256, nsamps=20000, seed=5):
    rng = np.random.default_rng(seed)
    vals = rng.integers(0, 256, (nsamps, nchans)).astype(np.uint32)
    packed = sy.pack(vals, 8)
    dms = np.linspace(0, 200, 37, dtype=np.float32)
    params = (nchans, 250e-6, 1500.0, -1.0)
    delays = po.delay_table(nchans, np.float32(params[1]), np.float32(params[2]), np.float32(params[3]))
    return packed, dms, params, delays


def test_tdd_plan_wait_expiry_then_recovers():
    packed, dms, params, delays = _tdd_case()
    nsamps, nchans = packed.shape[0], params[0]
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    with _Expiry():
        with pytest.raises(dd.DedispError) as ei:
            p.execute(nsamps, packed, 8, out, 32)
    assert ei.value.detail == INTERNAL, ei.value
    p.execute(nsamps, packed, 8, out, 32)
    ref = po.tdd(packed, nsamps, nchans, 8, nchans, delays, np.ones(nchans, np.int32), dms, 32, nout)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


def test_tc_fdd_wait_expiry_then_recovers():
    nchans, nsamps = 64, 12000
    inp, params = _input(nchans, nsamps, 5)
    dms = np.linspace(0, 60, 18, dtype=np.float32)
    p = _plan(params, dms, segmented=0, precision=1)
    p.set_timing(True)
    out = np.zeros((len(dms), p.output_row_length(nsamps)), np.float32)
    with _Expiry():
        with pytest.raises(dd.DedispError) as ei:
            p.execute(nsamps, inp, 8, out, 32)
    assert ei.value.detail == INTERNAL, ei.value
    p.execute(nsamps, inp, 8, out, 32)
    assert p.get_timing()["variant"] == 1
    x = _oracle_x(inp, nsamps, params, 8)
    ref = po.fdd_spectrum(x, _delays(params), np.ones(nchans, np.int32), dms, out.shape[1])
    rel, mx = _errs(out, ref)
    assert rel < TC_REL_L2 and mx < TC_MAX_ABS, (rel, mx)


def test_batch_wait_expiry_then_recovers():
    """The persistent batch launch reports the expiry through its own error
    word (dedisp_b200_batch_sync), not through another plan's."""
    import torch
    packed, dms, params, delays = _tdd_case(nchans=384, nsamps=16000, seed=9)
    nsamps = packed.shape[0]
    b = dd.Batch(*params, in_nbits=8, out_nbits=32)
    probe = dd.TDDPlan(*params)
    probe.set_dm_list(dms)
    nout = nsamps - probe.get_max_delay()
    d_in = torch.from_numpy(packed).cuda()
    d_out = torch.zeros((len(dms), nout), dtype=torch.float32, device="cuda")
    b.set_beams([(d_in, packed.shape[1], nsamps, dms, d_out, nout * 4)])
    stream = torch.cuda.current_stream().cuda_stream
    with _Expiry():
        b.execute(stream, use_graph=False)
        with pytest.raises(dd.DedispError) as ei:
            b.sync(stream)
    assert ei.value.code == INTERNAL, ei.value
    # a plan run after the failed batch reports no error of the batch's
    out = np.zeros((len(dms), nout), np.float32)
    probe.execute(nsamps, packed, 8, out, 32)
    b.execute(stream, use_graph=False)
    b.sync(stream)
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), out.view(np.uint32))

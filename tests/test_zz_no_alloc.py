"""The allocation-free TDD entry point, through the C ABI.

dedisp_b200_tdd_execute_noalloc serves callers that cannot call cudaMalloc
(real-time pipelines that forbid allocation after start-up, processes whose
device memory belongs to another allocator). It
must produce exactly what a TDD plan with DEDISP_DEVICE_POINTERS produces
(the TDD tolerance is bit-exactness), on consecutive calls that reuse its
shared scratch with different shapes. This file is collected last so that a
failing run stops only after every other test has run.
"""
import ctypes as C

import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy

pytestmark = pytest.mark.gpu


def _noalloc_fn():
    fn = dd.lib().dedisp_b200_tdd_execute_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_ulong, C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_ulong, C.c_void_p,
                   C.c_ulong, C.c_void_p, C.c_ulong, C.c_ulong, C.c_void_p, C.c_ulong, C.c_ulong,
                   C.c_void_p]
    msg = dd.lib().dedisp_b200_noalloc_last_message
    msg.restype = C.c_char_p
    return fn, msg


def _case(nchans, nbits, nsamps, dms, km, seed, out_nbits):
    import torch
    rng = np.random.default_rng(seed)
    vals = rng.integers(0, 1 << nbits, (nsamps, nchans)).astype(np.uint32)
    packed = sy.pack(vals, nbits)
    params = (nchans, 250e-6, 1581.8, -400.0 / nchans)
    # the existing entry point: a TDD plan on device pointers
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    if km is not None:
        p.set_killmask(km)
    nout = nsamps - p.get_max_delay()
    odt = {8: torch.uint8, 16: torch.int16, 32: torch.float32}[out_nbits]
    d_in = torch.from_numpy(packed).cuda()
    expect = torch.zeros((len(dms), nout), dtype=odt, device="cuda")
    p.execute(nsamps, d_in, nbits, expect, out_nbits, dd.DEDISP_DEVICE_POINTERS)
    # the allocation-free entry point on the same device buffers
    fn, msg = _noalloc_fn()
    got = torch.full((len(dms), nout), 7, dtype=odt, device="cuda")
    dms32 = np.ascontiguousarray(dms, np.float32)
    kmp = None if km is None else np.ascontiguousarray(km, np.int32)
    stream = torch.cuda.current_stream().cuda_stream
    rc = fn(nchans, np.float32(params[1]), np.float32(params[2]), np.float32(params[3]),
            dms32.ctypes.data, len(dms32), None if kmp is None else kmp.ctypes.data, nsamps,
            d_in.data_ptr(), nbits, packed.shape[1], got.data_ptr(), out_nbits,
            nout * out_nbits // 8, stream)
    assert rc == 0, msg()
    assert msg() == b"", "the message must be empty after a successful call"
    torch.cuda.synchronize()
    return got, expect


def test_noalloc_matches_plan_on_two_consecutive_calls():
    import torch
    # call 1: 8-bit, ascending DMs, float output
    got, expect = _case(256, 8, 20000, np.linspace(0, 300, 45, dtype=np.float32), None, 1, 32)
    assert torch.equal(got.view(torch.int32), expect.view(torch.int32))
    # call 2 reuses the shared scratch: 2-bit, unsorted DMs, a killmask with
    # zeros, 16-bit output, a different shape
    rng = np.random.default_rng(2)
    dms = rng.uniform(0, 200, 33).astype(np.float32)
    dms[-1] = 200.0
    km = np.ones(512, np.int32)
    km[::5] = 0
    got, expect = _case(512, 2, 24000, dms, km, 3, 16)
    assert torch.equal(got, expect)


@pytest.mark.parametrize("in_nbits", [1, 4, 16, 32])
def test_noalloc_other_widths_8bit_output(in_nbits):
    """Input widths whose tiled-kernel instances the calls above do not reach,
    with 8-bit (clipped) output, two calls in a row."""
    import torch
    for seed in (11, 12):
        got, expect = _case(256, in_nbits, 12000 + 1000 * seed,
                            np.linspace(0, 150 + seed, 21, dtype=np.float32), None, seed, 8)
        assert torch.equal(got, expect), (in_nbits, seed)


def test_noalloc_all_channels_killed():
    """An all-zero killmask (no active channel) gives the plan's output."""
    import torch
    km = np.zeros(256, np.int32)
    got, expect = _case(256, 8, 15000, np.linspace(0, 100, 17, dtype=np.float32), km, 21, 32)
    assert torch.equal(got.view(torch.int32), expect.view(torch.int32))


def test_noalloc_rejects_oversized_request():
    import torch
    fn, msg = _noalloc_fn()
    nchans, nsamps = 4096, 1 << 16  # 4097 x 16384 words > 16 Mi words of scratch
    d_in = torch.zeros((nsamps, nchans), dtype=torch.uint8, device="cuda")
    d_out = torch.zeros((4, nsamps), dtype=torch.float32, device="cuda")
    dms = np.zeros(4, np.float32)
    rc = fn(nchans, np.float32(64e-6), np.float32(1500.0), np.float32(-0.078125), dms.ctypes.data,
            4, None, nsamps, d_in.data_ptr(), 8, nchans, d_out.data_ptr(), 32, nsamps * 4, None)
    assert rc == 1  # DEDISP_MEM_ALLOC_FAILED
    assert b"64 MiB" in msg()
    # the next successful call clears the message
    got, expect = _case(64, 8, 6000, np.linspace(0, 50, 9, dtype=np.float32), None, 31, 32)
    assert torch.equal(got.view(torch.int32), expect.view(torch.int32))

"""TDD parity on the GPU, through the C ABI (libdedisp.so).

The bar is bit-exact equality with the CPU oracle (integer sums and the
reference FP32 epilogue), for every input width, output width, kernel form,
killmask, stride, DM range and pointer kind; at full production size the
tiled kernel is compared bit for bit with the plain kernel on the whole
output and with the oracle on a subset.
"""
import os

import numpy as np
import pytest

import dedisp_tests_b200 as dd
from dedisp_tests_b200 import synthetic as sy
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

OUT_DTYPE = {8: np.uint8, 16: np.uint16, 32: np.float32}


def _case(nbits, nchans, nsamps, ndm, dm_max, seed, f0=1500.0, df=-1.0, dt=250e-6):
    rng = np.random.default_rng(seed)
    hi = (1 << nbits) if nbits < 32 else (1 << 32)
    vals = rng.integers(0, hi, (nsamps, nchans), dtype=np.uint64).astype(np.uint32)
    packed = sy.pack(vals, nbits)
    dms = np.linspace(0, dm_max, ndm, dtype=np.float32)
    return packed, dms, (nchans, dt, f0, df)


def _oracle(packed, nsamps, nbits, params, dms, km, out_nbits, nout, in_stride=None):
    nchans, dt, f0, df = params
    delays = po.delay_table(nchans, np.float32(dt), np.float32(f0), np.float32(df))
    return po.tdd(packed, nsamps, in_stride or packed.shape[1], nbits, nchans, delays, km, dms,
                  out_nbits, nout)


def _run(cls, packed, nsamps, nbits, params, dms, out_nbits, kernel=0, km=None, gulp=0):
    p = cls(*params)
    p.set_dm_list(dms)
    if km is not None:
        p.set_killmask(km)
    if kernel:
        p.set_kernel(kernel)
    if gulp:
        p.set_gulp_size(gulp)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), OUT_DTYPE[out_nbits])
    p.execute(nsamps, packed, nbits, out, out_nbits)
    return out, nout


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("nbits,nchans", [(1, 96), (2, 128), (4, 64), (8, 128), (16, 32),
                                          (32, 16)])
def test_all_widths_bit_exact(nbits, nchans, kernel):
    nsamps = 9000
    packed, dms, params = _case(nbits, nchans, nsamps, 67, 400.0, 100 + nbits)
    km = np.ones(nchans, np.int32)
    for out_nbits in (8, 16, 32):
        ours, nout = _run(dd.TDDPlan, packed, nsamps, nbits, params, dms, out_nbits, kernel)
        ref = _oracle(packed, nsamps, nbits, params, dms, km, out_nbits, nout)
        assert np.array_equal(ours.view(np.uint8), ref.view(np.uint8)), (nbits, out_nbits)


@pytest.mark.parametrize("variant", range(9))
def test_tiled8_tile_variants_bit_exact(variant):
    """Every tile shape of the 8-bit kernel (packed rows 0-4, quad-strided
    rows 5-8); > 256 channels so the 16-bit lanes are flushed several times,
    with a killmask thinning the list."""
    assert dd.tdd_variant_count(8) == 9
    nchans, nsamps = 1100, 12000
    packed, dms, params = _case(8, nchans, nsamps, 75, 600.0, 900 + variant, df=-0.25)
    km = np.ones(nchans, np.int32)
    km[7::31] = 0
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    p.set_killmask(km)
    p.set_kernel(2)
    p.set_tile_variant(variant)
    nout = nsamps - p.get_max_delay()
    out = np.zeros((len(dms), nout), np.float32)
    p.execute(nsamps, packed, 8, out, 32)
    ref = _oracle(packed, nsamps, 8, params, dms, km, 32, nout)
    assert np.array_equal(out.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("variant", range(5, 9))
def test_quad_variants_gulps_unsorted_out_widths(variant):
    """Quad-strided variants over several gulps (the rows are rebuilt per
    gulp), an unsorted DM list with a repeat (permuted output rows), a
    partial last DM block, and 8/16/32-bit outputs."""
    nchans, nsamps = 320, 26000
    packed, _, params = _case(8, nchans, nsamps, 1, 1.0, 40 + variant, df=-0.5)
    rng = np.random.default_rng(variant)
    dms = rng.uniform(0, 400, 77).astype(np.float32)
    dms[5] = dms[40]
    dms[-1] = 400.0
    km = np.ones(nchans, np.int32)
    for out_nbits, gulp in ((8, 3001), (16, 0), (32, 7777)):
        p = dd.TDDPlan(*params)
        p.set_dm_list(dms)
        p.set_kernel(2)
        p.set_tile_variant(variant)
        if gulp:
            p.set_gulp_size(gulp)
        nout = nsamps - p.get_max_delay()
        out = np.zeros((len(dms), nout), OUT_DTYPE[out_nbits])
        p.execute(nsamps, packed, 8, out, out_nbits)
        ref = _oracle(packed, nsamps, 8, params, dms, km, out_nbits, nout)
        assert np.array_equal(out.view(np.uint8), ref.view(np.uint8)), (out_nbits, gulp)


@pytest.mark.parametrize("nbits", [1, 2, 4])
def test_narrow_widths_every_variant(nbits):
    """1/2/4-bit input through the packed-row kernel (variant 0) and the four
    quad-strided shapes (samples widened to bytes): random and all-maximum
    samples over > 256 channels, a killmask, two gulps."""
    nchans, nsamps = 1056, 9000
    packed, dms, params = _case(nbits, nchans, nsamps, 70, 500.0, 300 + nbits, df=-0.25)
    full = sy.pack(np.full((nsamps, nchans), (1 << nbits) - 1, np.uint32), nbits)
    km = np.ones(nchans, np.int32)
    km[5::37] = 0
    assert dd.tdd_variant_count(nbits) == 5
    for data in (packed, full):
        ref = None
        for variant in range(5):
            p = dd.TDDPlan(*params)
            p.set_dm_list(dms)
            p.set_killmask(km)
            p.set_kernel(2)
            p.set_tile_variant(variant)
            p.set_gulp_size(4000)
            nout = nsamps - p.get_max_delay()
            out = np.zeros((len(dms), nout), np.float32)
            p.execute(nsamps, data, nbits, out, 32)
            if ref is None:
                ref = _oracle(data, nsamps, nbits, params, dms, km, 32, nout)
            assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), (variant, data is full)


def test_tiled8_saturated_bytes():
    """All samples 255: every 16-bit lane reaches 256 * 255 before a flush."""
    nchans, nsamps = 1024, 6000
    packed = np.full((nsamps, nchans), 255, np.uint8)
    params = (nchans, 250e-6, 1500.0, -0.5)
    dms = np.linspace(0, 300, 45, dtype=np.float32)
    for variant in range(dd.tdd_variant_count(8)):
        p = dd.TDDPlan(*params)
        p.set_dm_list(dms)
        p.set_kernel(2)
        p.set_tile_variant(variant)
        nout = nsamps - p.get_max_delay()
        out = np.zeros((len(dms), nout), np.float32)
        p.execute(nsamps, packed, 8, out, 32)
        ref = _oracle(packed, nsamps, 8, params, dms, np.ones(nchans, np.int32), 32, nout)
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), variant


@pytest.mark.parametrize("nbits", [2, 8])
def test_killmask_zero_one_and_general(nbits):
    nchans, nsamps = 256, 6000
    packed, dms, params = _case(nbits, nchans, nsamps, 40, 300.0, 7)
    km = np.ones(nchans, np.int32)
    km[5::9] = 0
    ours, nout = _run(dd.TDDPlan, packed, nsamps, nbits, params, dms, 32, km=km)
    assert np.array_equal(ours, _oracle(packed, nsamps, nbits, params, dms, km, 32, nout))
    km2 = km.copy()
    km2[::11] = 2  # not 0/1: the reference multiplies; the plain form handles it
    ours, nout = _run(dd.TDDPlan, packed, nsamps, nbits, params, dms, 32, km=km2)
    assert np.array_equal(ours, _oracle(packed, nsamps, nbits, params, dms, km2, 32, nout))
    kz = np.zeros(nchans, np.int32)
    ours, nout = _run(dd.DedispPlan, packed, nsamps, nbits, params, dms, 16, km=kz)
    assert np.array_equal(ours, _oracle(packed, nsamps, nbits, params, dms, kz, 16, nout))


def test_strides_guru_and_gulps():
    nbits, nchans, nsamps = 8, 128, 20000
    packed, dms, params = _case(nbits, nchans, nsamps, 50, 500.0, 9)
    km = np.ones(nchans, np.int32)
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    md = p.get_max_delay()
    nout = nsamps - md
    ref = _oracle(packed, nsamps, nbits, params, dms, km, 32, nout)
    # padded input rows (stride 160 bytes) and output rows (nout + 13 floats)
    padded = np.zeros((nsamps, 160), np.uint8)
    padded[:, :nchans] = packed
    out = np.full((len(dms), nout + 13), -1.0, np.float32)
    p.execute_adv(nsamps, padded, 8, 160, out, 32, (nout + 13) * 4)
    assert np.array_equal(out[:, :nout], ref)
    assert np.all(out[:, nout:] == -1.0)
    # a DM sub-range [7, 7 + 20)
    sub = np.zeros((20, nout), np.float32)
    p.execute_guru(nsamps, packed, 8, nchans, sub, 32, nout * 4, 7, 20)
    assert np.array_equal(sub, ref[7:27])
    # many small gulps; 12000 (whole time tiles, a quarter-size first gulp)
    for gulp in (997, 4096, 12000):
        ours, _ = _run(dd.TDDPlan, packed, nsamps, nbits, params, dms, 32, gulp=gulp)
        assert np.array_equal(ours, ref), gulp


@pytest.mark.parametrize("nbits", [2, 8])
def test_host_gulp_schedule(nbits):
    """Host buffers over several gulps: the first a quarter of the gulp
    size, the middle ones whole time tiles, the last split into DM groups
    for the output copies; device buffers with the same gulp size run
    uniform gulps. Both bit-exact against the oracle."""
    import torch
    nchans, nsamps = 256, 70000
    packed, dms, params = _case(nbits, nchans, nsamps, 90, 800.0, 31)
    km = np.ones(nchans, np.int32)
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    nout = nsamps - p.get_max_delay()
    ref = _oracle(packed, nsamps, nbits, params, dms, km, 32, nout)
    for gulp in (16384, 25000):
        ours, _ = _run(dd.TDDPlan, packed, nsamps, nbits, params, dms, 32, gulp=gulp)
        assert np.array_equal(ours, ref), gulp
    d_in = torch.from_numpy(np.ascontiguousarray(packed)).cuda()
    d_out = torch.zeros((len(dms), nout), dtype=torch.float32, device="cuda")
    p.set_gulp_size(16384)
    p.execute(nsamps, d_in, nbits, d_out, 32, dd.DEDISP_DEVICE_POINTERS)
    assert np.array_equal(d_out.cpu().numpy(), ref)


def test_unsorted_and_repeated_dm_list():
    nbits, nchans, nsamps = 4, 64, 7000
    packed, _, params = _case(nbits, nchans, nsamps, 1, 1.0, 11)
    rng = np.random.default_rng(1)
    dms = rng.uniform(0, 250, 45).astype(np.float32)
    dms[10] = dms[3]
    dms[-1] = 250.0  # the reference's max delay is taken from the last DM
    km = np.ones(nchans, np.int32)
    for kernel in (1, 2):
        ours, nout = _run(dd.TDDPlan, packed, nsamps, nbits, params, dms, 32, kernel)
        assert np.array_equal(ours, _oracle(packed, nsamps, nbits, params, dms, km, 32, nout))


def test_device_pointers_and_async():
    import torch
    nbits, nchans, nsamps = 2, 512, 12000
    packed, dms, params = _case(nbits, nchans, nsamps, 64, 300.0, 13)
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    nout = nsamps - p.get_max_delay()
    d_in = torch.from_numpy(packed).cuda()
    d_out = torch.zeros((len(dms), nout), dtype=torch.float32, device="cuda")
    p.execute(nsamps, d_in, nbits, d_out, 32, dd.DEDISP_DEVICE_POINTERS | dd.DEDISP_ASYNC)
    p.sync()
    ref = _oracle(packed, nsamps, nbits, params, dms, np.ones(nchans, np.int32), 32, nout)
    assert np.array_equal(d_out.cpu().numpy(), ref)


def test_nsamps_equal_max_delay_is_empty():
    packed, dms, params = _case(8, 64, 3000, 4, 100.0, 17)
    p = dd.TDDPlan(*params)
    p.set_dm_list(dms)
    md = p.get_max_delay()
    out = np.zeros(16, np.float32)
    p.execute(md, packed, 8, out, 32)  # nothing to compute, no error


def test_config0_full_bit_exact():
    cfg = sy.config0()
    packed = sy.make_input(cfg)
    params = (cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
    for cls, kernel in ((dd.DedispPlan, 0), (dd.TDDPlan, 2)):
        ours, nout = _run(cls, packed, cfg.nsamps, 8, params, cfg.dm_list, 32, kernel)
        assert nout == 65536 - 2622
        ref = _oracle(packed, cfg.nsamps, 8, params, cfg.dm_list, np.ones(1024, np.int32), 32,
                      nout)
        assert np.array_equal(ours, ref)
    # the injected pulse is recovered near DM 250, t = 4.0 s
    i, t = np.unravel_index(np.argmax(ours), ours.shape)
    assert abs(cfg.dm_list[i] - 250.0) < 5.0 and abs(t * cfg.dt - 4.0) < 0.01


REF_TDD = po.ref_available("libref_tdd.so")


@pytest.mark.skipif(not REF_TDD, reason="reference GPU plans not built")
@pytest.mark.parametrize("plan,nbits,nchans,out_nbits", [
    ("tdd", 8, 128, 32), ("tdd", 2, 256, 8), ("tdd", 4, 64, 16), ("tdd", 1, 96, 32),
    ("tdd", 16, 32, 32), ("tdd", 32, 16, 32), ("dedisp", 8, 128, 32), ("dedisp", 2, 128, 16)])
def test_reference_gpu_plan_bit_exact(plan, nbits, nchans, out_nbits):
    """The reference's own TDDPlan / DedispPlan (compiled from its sources)
    against the oracle and against this library, same inputs."""
    nsamps = 8000
    packed, dms, params = _case(nbits, nchans, nsamps, 33, 250.0, 31 + nbits)
    nchans, dt, f0, df = params
    km = np.ones(nchans, np.int32)
    km[::13] = 0
    cls = dd.TDDPlan if plan == "tdd" else dd.DedispPlan
    ours, nout = _run(cls, packed, nsamps, nbits, params, dms, out_nbits, km=km)
    raw, _ = po.ref_execute(plan, nchans, np.float32(dt), np.float32(f0), np.float32(df), dms,
                            km, nsamps, packed, nbits, out_nbits, len(dms) * nout,
                            gulp_size=1 << 30)
    refout = raw.view(OUT_DTYPE[out_nbits]).reshape(len(dms), nout)
    orc = _oracle(packed, nsamps, nbits, params, dms, km, out_nbits, nout)
    assert np.array_equal(ours.view(np.uint8), orc.view(np.uint8))
    if plan == "tdd" and nbits == 32:
        # Reference defect: TDDPlan's transpose_unpack has no 32-bit
        # instantiation (src/tdd/unpack/unpack.cu:187-196), so no unpack
        # kernel runs and the sums are taken over whatever the transposed
        # buffer held (zeros on a fresh device, stale data after earlier
        # plans). Either way they are not the dedispersed input.
        assert not np.array_equal(refout.view(np.uint8), orc.view(np.uint8))
        return
    assert np.array_equal(refout.view(np.uint8), orc.view(np.uint8))


GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ref_gpu_outputs.npz")


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="no reference GPU golden outputs")
def test_golden_reference_outputs():
    import hashlib
    from tests.golden.make_golden import GPU_CASES, gpu_case_input
    g = np.load(GOLDEN)
    for k, (plan, nch, f0, df, dt, ns, nb, onb, ndm, dmax, kme, seed) in enumerate(GPU_CASES):
        inp = gpu_case_input(nch, f0, df, dt, ns, nb, seed)
        assert hashlib.sha256(inp.tobytes()).hexdigest() == str(g[f"sha_{k}"][0])
        dms = np.linspace(0, dmax, ndm, dtype=np.float32)
        km = np.ones(nch, np.int32)
        if kme:
            km[::kme] = 0
        cls = dd.TDDPlan if plan == "tdd" else dd.DedispPlan
        ours, nout = _run(cls, inp, ns, nb, (nch, dt, f0, df), dms, onb, km=km)
        if plan == "tdd" and nb == 32:  # reference defect, see above
            assert not g[f"out_{k}"].any()
            continue
        assert np.array_equal(ours.view(np.uint8).ravel(), g[f"out_{k}"]), k


def test_config1_full_size_tiled_equals_plain_and_oracle_subset():
    """nchan 4096, 2^21 samples, 3643 DMs at 8 bits (30 GB of output): the
    tiled kernel equals the plain kernel on every output sample, and the
    oracle on a DM subset over all samples."""
    import torch
    cfg = sy.config1(nbits=8)
    d_in = sy.make_input_torch(cfg)
    params = (cfg.nchans, cfg.dt, cfg.f_top, cfg.df)
    p = dd.TDDPlan(*params)
    p.generate_dm_list(*cfg.dm_gen)
    ndm, md = p.get_dm_count(), p.get_max_delay()
    assert (ndm, md) == (3643, 35500)
    nout = cfg.nsamps - md
    out_t = torch.empty((ndm, nout), dtype=torch.float32, device="cuda")
    p.set_kernel(2)
    p.execute(cfg.nsamps, d_in, 8, out_t, 32, dd.DEDISP_DEVICE_POINTERS)
    # subset against the oracle: 6 DMs spread over the list, three windows
    # of 65536 output samples (start, middle, end of the series)
    pick = np.array([0, 1, 911, 1822, 2700, ndm - 1])
    dms = p.get_dm_list()
    delays = po.delay_table(cfg.nchans, np.float32(cfg.dt), np.float32(cfg.f_top),
                            np.float32(cfg.df))
    L = 65536
    for ta in (0, nout // 2, nout - L):
        win = d_in[ta:ta + L + md].cpu().numpy()
        ref = po.tdd(win, L + md, win.shape[1], 8, cfg.nchans, delays,
                     np.ones(cfg.nchans, np.int32), dms[pick], 32, L)
        got = out_t[torch.as_tensor(pick, device="cuda"), ta:ta + L].cpu().numpy()
        assert np.array_equal(got, ref), ta
    # whole output: tiled == plain, compared in chunks of DMs on the device
    q = dd.TDDPlan(*params)
    q.generate_dm_list(*cfg.dm_gen)
    q.set_kernel(1)
    step = 512
    for s0 in range(0, ndm, step):
        n = min(step, ndm - s0)
        part = torch.empty((n, nout), dtype=torch.float32, device="cuda")
        q.execute_guru(cfg.nsamps, d_in, 8, cfg.nchans, part, 32, nout * 4, s0, n,
                       dd.DEDISP_DEVICE_POINTERS)
        assert torch.equal(part.view(torch.int32), out_t[s0:s0 + n].view(torch.int32)), s0

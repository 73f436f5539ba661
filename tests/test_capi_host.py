"""C-ABI library: exported symbols and host-side behaviour (CPU only; no
compute is launched)."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

import dedisp_tests_b200 as dd
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dedisp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", dd.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r" T (\w+)", out))
    names = _declared("dedisp.h") + _declared("dedisp_b200.h")
    assert len(names) >= 30
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = dd.lib()
    for n in names:
        assert getattr(L, n) is not None


def test_reference_symbol_list_is_covered():
    # The reference version script libdedisp.version:3-29 minus the entries
    # its header comments out (adaptive dt, _guru DM list), plus
    # dedisp_select_implementation which the script forgot.
    live = ["dedisp_create_plan", "dedisp_destroy_plan", "dedisp_set_device",
            "dedisp_set_gulp_size", "dedisp_get_gulp_size", "dedisp_set_killmask",
            "dedisp_set_dm_list", "dedisp_generate_dm_list", "dedisp_get_max_delay",
            "dedisp_get_channel_count", "dedisp_get_dm_count", "dedisp_get_dm_delay",
            "dedisp_get_dm_list", "dedisp_get_killmask", "dedisp_get_dt", "dedisp_get_f0",
            "dedisp_get_df", "dedisp_get_error_string", "dedisp_execute", "dedisp_execute_adv",
            "dedisp_execute_guru", "dedisp_sync", "dedisp_select_implementation"]
    assert set(live) <= set(_declared("dedisp.h"))


def test_enum_values_match_reference():
    assert dd.ERROR_NAMES.index("DEDISP_UNKNOWN_ERROR") == 16
    assert dd.ERROR_NAMES.index("DEDISP_TOO_FEW_NSAMPS") == 8
    assert (dd.DEDISP_HOST_POINTERS, dd.DEDISP_DEVICE_POINTERS, dd.DEDISP_WAIT,
            dd.DEDISP_ASYNC) == (2, 4, 8, 16)
    L = dd.lib()
    assert L.dedisp_get_error_string(8) == b"No. samples < maximum delay"
    assert L.dedisp_get_error_string(99) == b"Invalid error code"


@pytest.mark.parametrize("cls", [dd.DedispPlan, dd.TDDPlan, dd.FDDGPUPlan])
def test_plan_setup_matches_oracle(cls):
    p = cls(4096, 64e-6, 1500.0, -0.078125)
    p.generate_dm_list(0, 2000, 40, 1.25)
    dms = po.generate_dm_list(4096, 64e-6, 1500.0, -0.078125, 0, 2000, 40, 1.25)
    assert p.get_dm_count() == 3643
    assert np.array_equal(p.get_dm_list().view(np.uint32), dms.view(np.uint32))
    assert p.get_max_delay() == 35500
    delays = po.delay_table(4096, np.float32(64e-6), 1500.0, -0.078125)
    for i in (0, 1, 1000, 3642):
        assert p.get_dm_delay(i) == po.max_delay(dms[: i + 1], delays)
    assert p.get_df() == np.float32(-0.078125)
    assert p.get_channel_count() == 4096
    assert np.all(p.get_killmask() == 1)
    km = np.ones(4096, np.int32)
    km[::3] = 0
    p.set_killmask(km)
    assert np.array_equal(p.get_killmask(), km)
    p.set_killmask(None)
    assert np.all(p.get_killmask() == 1)


def test_set_dm_list_and_getters():
    p = dd.TDDPlan(1024, 250e-6, 1581.8, -0.390625)
    assert p.get_max_delay() == 0 and p.get_dm_count() == 0
    dms = (500.0 * np.arange(512) / 511.0).astype(np.float32)
    p.set_dm_list(dms)
    assert p.get_max_delay() == 2622
    assert p.get_dm_delay(-1) == 0 and p.get_dm_delay(512) == 0
    assert p.get_gulp_size() > 0
    p.set_gulp_size(65536)
    assert p.get_gulp_size() == 65536


def test_fdd_rejects_gulp_size_and_adv():
    p = dd.FDDGPUPlan(64, 1e-3, 400.0, -1.0)
    with pytest.raises(dd.DedispError) as e:
        p.set_gulp_size(10)
    assert e.value.code == 4  # DEDISP_INVALID_PLAN
    assert p.get_gulp_size() == 0


def _err(fn):
    with pytest.raises(dd.DedispError) as e:
        fn()
    return dd.ERROR_NAMES[e.value.code], dd.ERROR_NAMES[e.value.detail]


def test_validation_order_matches_reference():
    """TDDPlan.cpp:167-195: pointer, stride, DM list, nsamps, nbits."""
    p = dd.TDDPlan(64, 1e-3, 400.0, -1.0)
    buf = np.zeros(1 << 16, np.uint8)
    # no DM list yet
    assert _err(lambda: p.execute(1000, buf, 8, buf, 32))[1] == "DEDISP_NO_DM_LIST_SET"
    p.set_dm_list(np.array([0.0, 30.0], np.float32))
    md = p.get_max_delay()
    assert md > 0
    # NULL pointer comes first
    assert _err(lambda: p.execute(1000, None, 8, buf, 32))[1] == "DEDISP_INVALID_POINTER"
    # stride before nsamps: execute_adv with a short output stride
    assert _err(lambda: p.execute_adv(1000, buf, 8, 64, buf, 32, 4))[1] == \
        "DEDISP_INVALID_STRIDE"
    # nsamps < max_delay through execute(): wraps to a matching stride, so the
    # nsamps check reports it
    assert _err(lambda: p.execute(md - 1, buf, 8, buf, 32))[1] == "DEDISP_TOO_FEW_NSAMPS"
    assert _err(lambda: p.execute(1000, buf, 3, buf, 32))[1] == "DEDISP_UNSUPPORTED_IN_NBITS"
    assert _err(lambda: p.execute(1000, buf, 8, buf, 12))[1] == "DEDISP_UNSUPPORTED_OUT_NBITS"
    # every plan-level failure is DEDISP_UNKNOWN_ERROR at the C boundary
    with pytest.raises(dd.DedispError) as e:
        p.execute(1000, None, 8, buf, 32)
    assert e.value.code == 16


def test_dedisp_plan_flag_combination():
    p = dd.DedispPlan(64, 1e-3, 400.0, -1.0)
    p.set_dm_list(np.array([0.0, 30.0], np.float32))
    buf = np.zeros(1 << 16, np.uint8)
    assert _err(lambda: p.execute(1000, buf, 8, buf, 32, dd.DEDISP_ASYNC | dd.DEDISP_WAIT))[1] \
        == "DEDISP_INVALID_FLAG_COMBINATION"


def test_nchans_limit():
    with pytest.raises(dd.DedispError) as e:
        dd.TDDPlan(8193, 1e-3, 400.0, -0.01)
    assert e.value.detail == 3  # DEDISP_NCHANS_EXCEEDS_LIMIT


def test_null_plan_handling():
    L = dd.lib()
    assert L.dedisp_set_dm_list(None, None, 0) == 4
    assert L.dedisp_get_dm_count(None) == 0
    assert L.dedisp_get_gulp_size(None) == 4  # reference returns the code as a size
    assert L.dedisp_execute(None, 0, None, 8, None, 32, 0) == 4
    L.dedisp_destroy_plan(None)


def test_fdd_output_row_length_follows_reference_geometry():
    p = dd.FDDGPUPlan(1024, 250e-6, 1581.8, -0.390625)
    p.set_dm_list((1000.0 * np.arange(2048) / 2047.0).astype(np.float32))
    assert p.get_max_delay() == 5243
    n = 1 << 20
    assert p.output_row_length(n) == 1064960            # spectrum: nfft floats
    p.set_options(segmented=1)
    assert p.output_row_length(n) == n - 5243           # segmented: time series
    p.set_options(segmented=0, timeseries=True)
    assert p.output_row_length(n) == n - 5243


def test_fdd_segment_length_rules():
    """Reference rule: doubling from 16384 while nfft * 0.2 < max delay
    (src/fdd/FDDGPUPlan.cpp:742,762-768). Automatic rule (tensor-core MAC):
    shorter segments while the MAC stays bound by phasor generation; on B200
    the config-3 beams below measured (MAC + transforms, ms) 488 / 296 / 182
    for 131072 / 65536 / 32768 points (beam 0) and 140 / 77 / 133 for 65536 /
    32768 / 16384 (beam 4), and the rule picks the fastest of each."""
    f = dd.fdd_segment_length
    assert f(1 << 20, 5243, 2048, 1024, 1, 0) == 32768
    assert f(850907, 14271, 3642, 1536, 1, 0) == 131072
    assert f(911111, 9918, 1481, 1536, 1, 0) == 65536
    assert f(850907, 14271, 3642, 1536, 1, "auto") == 32768
    assert f(911111, 9918, 1481, 1536, 1, "auto") == 32768
    assert f(414083, 29372, 3225, 1536, 1, "auto") <= 65536
    assert f(1000, 10, 16, 64, 1, 8192) == 8192
    assert f(1000, 9000, 16, 64, 1, 8192) == 0            # segment shorter than the max delay
    # FP32 MAC: the automatic rule is the reference rule
    assert f(850907, 14271, 3642, 1536, 0, "auto") == 131072
    # no power of two up to 2^20 exceeds the max delay: the reference rule
    assert f(5_000_000, 2_000_000, 512, 256, 1, "auto") == f(5_000_000, 2_000_000, 512, 256, 1, 0) > 2_000_000


def test_batch_api_argument_checks():
    """Host-side checks of the batch interface; no GPU work is launched."""
    L = dd._batch_lib()
    h = C.c_void_p()
    assert L.dedisp_b200_batch_create(None, 64, 1e-4, 1500.0, -1.0, 8, 32, 0) == 5  # invalid pointer
    assert L.dedisp_b200_batch_execute(None, None, 1) == 4                        # invalid plan
    assert L.dedisp_b200_batch_set_beams(None, None, 0) == 4
    assert L.dedisp_b200_batch_workspace_size(None) == 0
    L.dedisp_b200_batch_destroy(None)
    # unsupported widths are rejected before any device work
    assert L.dedisp_b200_batch_create(C.byref(h), 64, 1e-4, 1500.0, -1.0, 3, 32, 0) == 10
    assert L.dedisp_b200_batch_create(C.byref(h), 64, 1e-4, 1500.0, -1.0, 8, 12, 0) == 11
    assert not h.value


def test_fdd_extension_queries_reject_bad_handles():
    """The FDD queries and batch settings added with the phasor sources, MMA
    forms, segment lengths and MAC balance reject missing handles and
    pointers without touching a GPU."""
    L = dd.lib()
    B = dd._batch_lib()
    v = C.c_int(7)
    assert L.dedisp_b200_get_phasor_source(None, C.byref(v)) == 4      # invalid plan
    assert L.dedisp_b200_get_tc_form(None, C.byref(v)) == 4
    assert L.dedisp_b200_get_stage_times(None, None, 0) == 4
    assert B.dedisp_b200_fdd_batch_set_segment_nfft(None, 1) == 4
    assert B.dedisp_b200_fdd_batch_phasor_source(None, 0) == -1
    a, b = C.c_float(), C.c_float()
    assert B.dedisp_b200_fdd_batch_get_mac_balance(None, C.byref(a), C.byref(b)) == 4
    # a TDD plan has no FDD form; host-only plan objects need no GPU
    p = dd.TDDPlan(64, 250e-6, 1581.8, -1.5625)
    assert L.dedisp_b200_get_phasor_source(p._h, None) == 5            # invalid pointer
    assert L.dedisp_b200_get_tc_form(p._h, None) == 5
    assert L.dedisp_b200_get_phasor_source(p._h, C.byref(v)) == 0 and v.value == -1
    assert L.dedisp_b200_get_tc_form(p._h, C.byref(v)) == 0 and v.value == -1
    p.close()


def test_tile_variant_counts():
    """8-bit input: five shapes on channel-major packed rows and four on
    quad-strided rows; 1/2/4-bit: the packed-row kernel and the four
    quad-strided shapes; 16/32-bit one shape; the plans and the persistent
    batch kernel alike. Out-of-range variants are rejected."""
    assert dd.tdd_variant_count(8) == 9 and dd.batch_variant_count(8) == 9
    for nb in (1, 2, 4):
        assert dd.tdd_variant_count(nb) == 5 and dd.batch_variant_count(nb) == 5
    for nb in (16, 32):
        assert dd.tdd_variant_count(nb) == 1 and dd.batch_variant_count(nb) == 1
    p = dd.TDDPlan(64, 1e-4, 1500.0, -1.0)
    for bad in (-1, 9):
        with pytest.raises(dd.DedispError):
            p.set_tile_variant(bad)
    p.set_tile_variant(8)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="checks the no-GPU path")
def test_batch_create_without_gpu_fails_cleanly():
    L = dd._batch_lib()
    h = C.c_void_p()
    rc = L.dedisp_b200_batch_create(C.byref(h), 64, 1e-4, 1500.0, -1.0, 8, 32, 0)
    assert rc != 0 and not h.value
    with pytest.raises(dd.DedispError):
        dd.Batch(64, 1e-4, 1500.0, -1.0)


def test_server_api_host_checks():
    """Streaming-server argument checks that need no GPU work."""
    s = dd.StreamServer(256, 64e-6, 1500.0, -0.25, in_nbits=8, max_gulp=4096, tdd_workers=1)
    b = s.add_beam(np.linspace(0, 100, 20, dtype=np.float32), 0)
    assert b == 0 and s.max_delay(0) > 0
    with pytest.raises(dd.DedispError):
        s.add_beam(np.linspace(0, 100, 20, dtype=np.float32), 1)  # no FDD workers
    with pytest.raises(dd.DedispError):
        s.submit(0, np.zeros((10, 256), np.uint8), 10)            # before start()
    s.close()
    L = dd._server_lib()
    h = C.c_void_p()
    assert L.dedisp_b200_server_create(C.byref(h), 256, 64e-6, 1500.0, -0.25, 3, 0, 0, 4096, 1, 0, 1, 0, 0) == 10
    assert L.dedisp_b200_server_create(C.byref(h), 256, 64e-6, 1500.0, -0.25, 8, 0, 0, 4096, 0, 0, 1, 0, 0) != 0
    assert L.dedisp_b200_server_drain(None) == 4


def _prototypes():
    """name -> (returns void, parameter count) for every function declared in
    include/dedisp.h and include/dedisp_b200.h."""
    protos = {}
    for header in ("dedisp.h", "dedisp_b200.h"):
        text = open(os.path.join(ROOT, "include", header)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for ret, name, params in re.findall(r"([A-Za-z_][\w\s\*]*?)\b(dedisp_\w+)\s*\(([^;{}]*?)\)\s*;", text):
            params = " ".join(params.split())
            n = 0 if params in ("", "void") else params.count(",") + 1
            protos[name] = (ret.split()[-1] == "void" and "*" not in ret, n)
    return protos


def test_python_binding_matches_the_headers():
    """Every function the ctypes binding declares has the header's parameter
    count and void/non-void return."""
    protos = _prototypes()
    L = dd.lib()
    dd._batch_lib()
    dd._server_lib()
    dd._io_lib()
    checked = 0
    for name, (void, nparams) in protos.items():
        fn = getattr(L, name)
        if fn.argtypes is None:
            continue
        assert len(fn.argtypes) == nparams, name
        assert (fn.restype is None) == void, name
        checked += 1
    assert checked >= 50, checked


def test_wait_limit_setting_round_trip():
    """The bounded-wait limit is process-wide; 0 restores the 2 s default."""
    try:
        dd.set_wait_limit_ns(12345)
        assert dd.get_wait_limit_ns() == 12345
        dd.set_wait_expiry_test(True)
        dd.set_wait_expiry_test(False)
    finally:
        dd.set_wait_limit_ns(0)
    assert dd.get_wait_limit_ns() == 2_000_000_000

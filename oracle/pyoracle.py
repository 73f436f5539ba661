"""ctypes wrapper around the CPU oracle (oracle/liboracle.so) and the
reference pieces compiled into oracle/_ref/ by oracle/ref/Makefile.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the shipped package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# Root of the reference source tree (read only; present where the oracle is
# pinned, absent on machines that only run the prebuilt pieces). Override
# with DEDISP_REFERENCE_ROOT, as REF overrides it in oracle/ref/Makefile.
REFERENCE_ROOT = os.environ.get("DEDISP_REFERENCE_ROOT", "/root/reference")

_u8p = C.POINTER(C.c_uint8)
_f32p = C.POINTER(C.c_float)
_f64p = C.POINTER(C.c_double)
_i32p = C.POINTER(C.c_int32)
_u64p = C.POINTER(C.c_uint64)
_szp = C.POINTER(C.c_size_t)


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference tree is present, the
    reference pins in oracle/_ref)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref and os.path.isdir(REFERENCE_ROOT):
        subprocess.run(["make", "-s", "-j8", "-C", os.path.join(HERE, "ref"),
                        f"REF={REFERENCE_ROOT}", "all"], check=True)


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(ref=False)
        L = C.CDLL(path)
        L.orc_delay_table.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_float, _f32p]
        L.orc_generate_dm_list.argtypes = [C.c_float, C.c_float, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.c_size_t, C.c_double,
                                           _f32p, C.c_size_t]
        L.orc_generate_dm_list.restype = C.c_size_t
        L.orc_max_delay.argtypes = [C.c_float, C.c_float]
        L.orc_max_delay.restype = C.c_size_t
        L.orc_delay_rn.argtypes = [C.c_float, C.c_float]
        L.orc_delay_rn.restype = C.c_uint32
        L.orc_delay_trunc.argtypes = [C.c_float, C.c_float]
        L.orc_delay_trunc.restype = C.c_int32
        L.orc_scale_output.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_size_t, C.c_void_p]
        L.orc_tdd.argtypes = [_u8p, C.c_size_t, C.c_size_t, C.c_int, C.c_size_t, _f32p,
                              _i32p, _f32p, C.c_size_t, _u8p, C.c_int, C.c_size_t,
                              C.c_size_t, C.c_int]
        L.orc_tdd_sums.argtypes = [_u8p, C.c_size_t, C.c_size_t, C.c_int, C.c_size_t, _f32p,
                                   _i32p, _f32p, C.c_size_t, _u64p, C.c_size_t, C.c_int]
        L.orc_fdd_unpack.argtypes = [_u8p, C.c_size_t, C.c_size_t, C.c_int, C.c_size_t, _f32p]
        L.orc_fdd_timeseries.argtypes = [_f32p, C.c_size_t, C.c_size_t, _f32p, _i32p, _f32p,
                                         C.c_size_t, C.c_int, _f64p, C.c_size_t, C.c_int]
        L.orc_fdd_spectrum.argtypes = [_f32p, C.c_size_t, C.c_size_t, _f32p, _i32p, _f32p,
                                       C.c_size_t, C.c_int, C.c_size_t, _f64p, C.c_int]
        L.orc_fft.argtypes = [_f64p, _f64p, C.c_size_t, C.c_int]
        L.orc_fdd_nfft_spectrum.argtypes = [C.c_size_t, C.c_size_t]
        L.orc_fdd_nfft_spectrum.restype = C.c_size_t
        L.orc_fdd_segment_geometry.argtypes = [C.c_size_t, C.c_size_t, _szp, _szp, _szp]
        for name in ("orc_tdd", "orc_tdd_sums", "orc_fdd_unpack", "orc_fdd_timeseries",
                     "orc_fdd_spectrum", "orc_fft"):
            getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# Plan setup
# --------------------------------------------------------------------------

def delay_table(nchans: int, dt: float, f0: float, df: float) -> np.ndarray:
    out = np.zeros(nchans, np.float32)
    lib().orc_delay_table(nchans, dt, f0, df, _ptr(out, _f32p))
    return out


def generate_dm_list(nchans, dt, f0, df, dm_start, dm_end, ti, tol) -> np.ndarray:
    """Plan::generate_dm_list as called by the C API (all float arguments
    promoted to double, src/Plan.cpp:136-149)."""
    f32 = np.float32
    args = (f32(dm_start), f32(dm_end), float(f32(dt)), float(f32(ti)), float(f32(f0)),
            float(f32(df)), nchans, float(f32(tol)))
    n = lib().orc_generate_dm_list(*args, None, 0)
    if n == C.c_size_t(-1).value:
        raise ValueError("DM list recurrence does not advance")
    out = np.zeros(n, np.float32)
    lib().orc_generate_dm_list(*args, _ptr(out, _f32p), n)
    return out


def max_delay(dm_list: np.ndarray, delays: np.ndarray) -> int:
    return int(lib().orc_max_delay(float(dm_list[-1]), float(delays[-1])))


def delay_rn(dm: float, delay: float) -> int:
    return int(lib().orc_delay_rn(dm, delay))


def scale_output(s: int, in_nbits: int, out_nbits: int, nchans: int):
    buf = np.zeros(1, {8: np.uint8, 16: np.uint16, 32: np.float32}[out_nbits])
    lib().orc_scale_output(s, in_nbits, out_nbits, nchans, buf.ctypes.data)
    return buf[0]


# --------------------------------------------------------------------------
# TDD
# --------------------------------------------------------------------------

def tdd(inp: np.ndarray, nsamps: int, in_stride: int, in_nbits: int, nchans: int,
        delays: np.ndarray, killmask: np.ndarray, dms: np.ndarray, out_nbits: int,
        nsamps_out: int, nthreads: int = 0) -> np.ndarray:
    """Brute-force TDD; returns [ndm][nsamps_out] of the output type."""
    inp = np.ascontiguousarray(inp, dtype=np.uint8)
    delays = np.ascontiguousarray(delays, np.float32)
    killmask = np.ascontiguousarray(killmask, np.int32)
    dms = np.ascontiguousarray(dms, np.float32)
    dt = {8: np.uint8, 16: np.uint16, 32: np.float32}[out_nbits]
    out = np.zeros((len(dms), nsamps_out), dt)
    rc = lib().orc_tdd(_ptr(inp, _u8p), nsamps, in_stride, in_nbits, nchans,
                       _ptr(delays, _f32p), _ptr(killmask, _i32p), _ptr(dms, _f32p),
                       len(dms), out.ctypes.data_as(_u8p), out_nbits,
                       nsamps_out * out_nbits // 8, nsamps_out, nthreads)
    if rc != 0:
        raise RuntimeError(f"orc_tdd failed ({rc})")
    return out


def tdd_sums(inp, nsamps, in_stride, in_nbits, nchans, delays, killmask, dms,
             nsamps_out, nthreads: int = 0) -> np.ndarray:
    inp = np.ascontiguousarray(inp, dtype=np.uint8)
    sums = np.zeros((len(dms), nsamps_out), np.uint64)
    rc = lib().orc_tdd_sums(_ptr(inp, _u8p), nsamps, in_stride, in_nbits, nchans,
                            _ptr(np.ascontiguousarray(delays, np.float32), _f32p),
                            _ptr(np.ascontiguousarray(killmask, np.int32), _i32p),
                            _ptr(np.ascontiguousarray(dms, np.float32), _f32p),
                            len(dms), _ptr(sums, _u64p), nsamps_out, nthreads)
    if rc != 0:
        raise RuntimeError(f"orc_tdd_sums failed ({rc})")
    return sums


# --------------------------------------------------------------------------
# FDD
# --------------------------------------------------------------------------

def fdd_unpack(inp, nsamps, in_stride, in_nbits, nchans) -> np.ndarray:
    x = np.zeros((nchans, nsamps), np.float32)
    rc = lib().orc_fdd_unpack(_ptr(np.ascontiguousarray(inp, np.uint8), _u8p), nsamps,
                              in_stride, in_nbits, nchans, _ptr(x, _f32p))
    if rc != 0:
        raise RuntimeError("orc_fdd_unpack failed")
    return x


def fdd_timeseries(x, delays, killmask, dms, nsamps_out, round_delays=False,
                   nthreads: int = 0) -> np.ndarray:
    nchans, nsamps = x.shape
    y = np.zeros((len(dms), nsamps_out), np.float64)
    lib().orc_fdd_timeseries(_ptr(np.ascontiguousarray(x, np.float32), _f32p), nsamps,
                             nchans, _ptr(np.ascontiguousarray(delays, np.float32), _f32p),
                             _ptr(np.ascontiguousarray(killmask, np.int32), _i32p),
                             _ptr(np.ascontiguousarray(dms, np.float32), _f32p), len(dms),
                             int(round_delays), _ptr(y, _f64p), nsamps_out, nthreads)
    return y


def fdd_spectrum(x, delays, killmask, dms, nfft, round_delays=False,
                 nthreads: int = 0) -> np.ndarray:
    """Returns [ndm][nfft] float64: first nfft/2 bins interleaved re/im."""
    nchans, nsamps = x.shape
    spec = np.zeros((len(dms), nfft), np.float64)
    rc = lib().orc_fdd_spectrum(_ptr(np.ascontiguousarray(x, np.float32), _f32p), nsamps,
                                nchans, _ptr(np.ascontiguousarray(delays, np.float32), _f32p),
                                _ptr(np.ascontiguousarray(killmask, np.int32), _i32p),
                                _ptr(np.ascontiguousarray(dms, np.float32), _f32p),
                                len(dms), int(round_delays), nfft, _ptr(spec, _f64p),
                                nthreads)
    if rc != 0:
        raise RuntimeError(f"orc_fdd_spectrum failed ({rc})")
    return spec


def fft(z: np.ndarray, sign: int = -1) -> np.ndarray:
    re = np.ascontiguousarray(z.real, np.float64).copy()
    im = np.ascontiguousarray(z.imag, np.float64).copy()
    lib().orc_fft(_ptr(re, _f64p), _ptr(im, _f64p), len(re), sign)
    return re + 1j * im


def fdd_nfft_spectrum(nsamp: int, max_delay: int) -> int:
    return int(lib().orc_fdd_nfft_spectrum(nsamp, max_delay))


def fdd_segment_geometry(nsamp: int, max_delay: int):
    a, b, c = C.c_size_t(), C.c_size_t(), C.c_size_t()
    lib().orc_fdd_segment_geometry(nsamp, max_delay, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


# --------------------------------------------------------------------------
# Reference pins (oracle/_ref)
# --------------------------------------------------------------------------

def ref_available(name: str) -> bool:
    return os.path.exists(os.path.join(REF_DIR, name))


_ref_libs: dict = {}


def ref_lib(name: str) -> C.CDLL:
    if name not in _ref_libs:
        L = C.CDLL(os.path.join(REF_DIR, name))
        if name == "libref_plan.so":
            L.ref_plan_delay_table.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_float,
                                               _f32p]
            L.ref_plan_generate_dm_list.argtypes = [C.c_size_t, C.c_float, C.c_float,
                                                    C.c_float, C.c_float, C.c_float,
                                                    C.c_float, C.c_float, _f32p, C.c_size_t,
                                                    _szp]
            L.ref_plan_generate_dm_list.restype = C.c_long
            L.ref_plan_set_dm_list.argtypes = [C.c_size_t, C.c_float, C.c_float, C.c_float,
                                               _f32p, C.c_size_t]
            L.ref_plan_set_dm_list.restype = C.c_long
        elif name == "libref_epilogue.so":
            for fn in ("ref_scale_output_tdd", "ref_scale_output_legacy"):
                getattr(L, fn).argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_ulong,
                                           C.c_void_p]
                getattr(L, fn).restype = C.c_int
            L.ref_extract_subword.argtypes = [C.c_uint, C.c_int, C.c_int]
            L.ref_extract_subword.restype = C.c_uint
        else:
            L.ref_execute.argtypes = [C.c_int, C.c_size_t, C.c_float, C.c_float, C.c_float,
                                      _f32p, C.c_size_t, _i32p, C.c_size_t, _u8p,
                                      C.c_size_t, _u8p, C.c_size_t, C.c_size_t, C.c_int,
                                      _szp]
            L.ref_execute.restype = C.c_int
        _ref_libs[name] = L
    return _ref_libs[name]


def ref_delay_table(nchans, dt, f0, df) -> np.ndarray:
    out = np.zeros(nchans, np.float32)
    if ref_lib("libref_plan.so").ref_plan_delay_table(nchans, dt, f0, df, _ptr(out, _f32p)):
        raise RuntimeError("reference Plan construction failed")
    return out


def ref_generate_dm_list(nchans, dt, f0, df, dm_start, dm_end, ti, tol):
    L = ref_lib("libref_plan.so")
    cap = 1 << 20
    out = np.zeros(cap, np.float32)
    md = C.c_size_t()
    n = L.ref_plan_generate_dm_list(nchans, dt, f0, df, dm_start, dm_end, ti, tol,
                                    _ptr(out, _f32p), cap, C.byref(md))
    if n < 0:
        raise RuntimeError("reference generate_dm_list failed")
    return out[:n].copy(), md.value


def ref_set_dm_list_max_delay(nchans, dt, f0, df, dms) -> int:
    dms = np.ascontiguousarray(dms, np.float32)
    return int(ref_lib("libref_plan.so").ref_plan_set_dm_list(nchans, dt, f0, df,
                                                               _ptr(dms, _f32p), len(dms)))


def ref_scale_output(s: int, in_nbits: int, out_nbits: int, nchans: int, legacy=False):
    buf = np.zeros(1, {8: np.uint8, 16: np.uint16, 32: np.float32}[out_nbits])
    fn = "ref_scale_output_legacy" if legacy else "ref_scale_output_tdd"
    getattr(ref_lib("libref_epilogue.so"), fn)(s, in_nbits, out_nbits, nchans,
                                                buf.ctypes.data)
    return buf[0]


def ref_execute(plan: str, nchans, dt, f0, df, dms, killmask, nsamps, inp, in_nbits,
                out_nbits, out_elems, gulp_size=0, segmented=False, device=0):
    """Run the reference GPU plan ('tdd' | 'dedisp' | 'fdd'); needs a GPU."""
    L = ref_lib(f"libref_{plan}.so")
    dms = np.ascontiguousarray(dms, np.float32)
    km = None if killmask is None else np.ascontiguousarray(killmask, np.int32)
    inp = np.ascontiguousarray(inp, np.uint8)
    out = np.zeros(out_elems * out_nbits // 8, np.uint8)
    md = C.c_size_t()
    rc = L.ref_execute(device, nchans, dt, f0, df, _ptr(dms, _f32p), len(dms),
                       None if km is None else _ptr(km, _i32p), nsamps, _ptr(inp, _u8p),
                       in_nbits, _ptr(out, _u8p), out_nbits, gulp_size, int(segmented),
                       C.byref(md))
    if rc != 0:
        raise RuntimeError(f"reference {plan} plan failed")
    return out, md.value

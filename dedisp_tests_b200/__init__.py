"""B200-native dedispersion engine: Python mirror of the dedisp C interface.

The product is the C-ABI shared library ``lib/libdedisp.so`` (CUDA kernels for
sm_100a plus C++ plan classes; declarations in ``include/dedisp.h`` and
``include/dedisp_b200.h``). This module binds it with ctypes and mirrors the
reference's C++ plan classes (``DedispPlan``, ``TDDPlan``, ``FDDGPUPlan``;
reference src/Plan.hpp, src/tdd/TDDPlan.hpp, src/fdd/FDDGPUPlan.hpp) so that
tests and benchmarks read like the reference's own ``run<PlanType>()`` tests.

There is no CPU fallback: importing works without a GPU (plans can be built
and queried), but ``execute`` needs the library and a CUDA device and raises
otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

__all__ = [
    "DedispError", "lib", "build", "Plan", "DedispPlan", "TDDPlan", "FDDGPUPlan",
    "DEDISP_USE_DEFAULT", "DEDISP_HOST_POINTERS", "DEDISP_DEVICE_POINTERS",
    "DEDISP_WAIT", "DEDISP_ASYNC", "DEDISP_DEDISP", "DEDISP_TDD", "DEDISP_FDD", "Batch", "FddBatch",
    "ERROR_NAMES",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libdedisp.so")

DEDISP_USE_DEFAULT = 0
DEDISP_HOST_POINTERS = 1 << 1
DEDISP_DEVICE_POINTERS = 1 << 2
DEDISP_WAIT = 1 << 3
DEDISP_ASYNC = 1 << 4

DEDISP_DEDISP, DEDISP_TDD, DEDISP_FDD = 0, 1, 2

ERROR_NAMES = [
    "DEDISP_NO_ERROR", "DEDISP_MEM_ALLOC_FAILED", "DEDISP_MEM_COPY_FAILED",
    "DEDISP_NCHANS_EXCEEDS_LIMIT", "DEDISP_INVALID_PLAN", "DEDISP_INVALID_POINTER",
    "DEDISP_INVALID_STRIDE", "DEDISP_NO_DM_LIST_SET", "DEDISP_TOO_FEW_NSAMPS",
    "DEDISP_INVALID_FLAG_COMBINATION", "DEDISP_UNSUPPORTED_IN_NBITS",
    "DEDISP_UNSUPPORTED_OUT_NBITS", "DEDISP_INVALID_DEVICE_INDEX",
    "DEDISP_DEVICE_ALREADY_SET", "DEDISP_PRIOR_GPU_ERROR", "DEDISP_INTERNAL_GPU_ERROR",
    "DEDISP_UNKNOWN_ERROR",
]
DEDISP_UNKNOWN_ERROR = ERROR_NAMES.index("DEDISP_UNKNOWN_ERROR")


class DedispError(RuntimeError):
    """A dedisp_error code returned by the library. ``code`` is what the C
    call returned (DEDISP_UNKNOWN_ERROR for plan-level failures, as in the
    reference); ``detail`` is the specific code from dedisp_b200_last_error."""

    def __init__(self, code: int, detail: int = 0, message: str = ""):
        self.code = code
        self.detail = detail
        self.message = message
        super().__init__(f"{ERROR_NAMES[code] if 0 <= code < len(ERROR_NAMES) else code}"
                         f" ({ERROR_NAMES[detail] if 0 <= detail < len(ERROR_NAMES) else detail})"
                         f": {message}")


def build(jobs: int = 8) -> None:
    """Compile lib/libdedisp.so in-tree (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")], check=True)


_lib: Optional[C.CDLL] = None
_vp = C.c_void_p
_sz = C.c_ulong


def lib() -> C.CDLL:
    """Load libdedisp.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run dedisp_tests_b200.build() first")
    L = C.CDLL(LIB_PATH)
    err = C.c_int
    sig = {
        "dedisp_select_implementation": (err, [C.c_int]),
        "dedisp_create_plan": (err, [C.POINTER(_vp), _sz, C.c_float, C.c_float, C.c_float]),
        "dedisp_destroy_plan": (None, [_vp]),
        "dedisp_set_device": (err, [C.c_int]),
        "dedisp_set_gulp_size": (err, [_vp, _sz]),
        "dedisp_get_gulp_size": (_sz, [_vp]),
        "dedisp_set_killmask": (err, [_vp, _vp]),
        "dedisp_set_dm_list": (err, [_vp, _vp, _sz]),
        "dedisp_generate_dm_list": (err, [_vp, C.c_float, C.c_float, C.c_float, C.c_float]),
        "dedisp_get_max_delay": (_sz, [_vp]),
        "dedisp_get_dm_delay": (_sz, [_vp, C.c_int]),
        "dedisp_get_channel_count": (_sz, [_vp]),
        "dedisp_get_dm_count": (_sz, [_vp]),
        "dedisp_get_dm_list": (C.POINTER(C.c_float), [_vp]),
        "dedisp_get_killmask": (C.POINTER(C.c_int), [_vp]),
        "dedisp_get_dt": (C.c_float, [_vp]),
        "dedisp_get_f0": (C.c_float, [_vp]),
        "dedisp_get_df": (C.c_float, [_vp]),
        "dedisp_get_error_string": (C.c_char_p, [C.c_int]),
        "dedisp_execute": (err, [_vp, _sz, _vp, _sz, _vp, _sz, C.c_uint]),
        "dedisp_execute_adv": (err, [_vp, _sz, _vp, _sz, _sz, _vp, _sz, _sz, C.c_uint]),
        "dedisp_execute_guru": (err, [_vp, _sz, _vp, _sz, _sz, _vp, _sz, _sz, _sz, _sz,
                                      C.c_uint]),
        "dedisp_sync": (err, []),
        "dedisp_b200_set_tdd_kernel": (err, [_vp, C.c_int]),
        "dedisp_b200_set_tdd_variant": (err, [_vp, C.c_int]),
        "dedisp_b200_tdd_variant_count": (C.c_int, [_sz]),
        "dedisp_b200_set_stream": (err, [_vp, _vp]),
        "dedisp_b200_set_timing": (err, [_vp, C.c_int]),
        "dedisp_b200_get_timing": (err, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                         C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "dedisp_b200_last_error": (err, [C.c_char_p, _sz]),
        "dedisp_b200_set_fdd_options": (err, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _sz]),
        "dedisp_b200_output_row_length": (_sz, [_vp, _sz]),
        "dedisp_b200_get_stage_times": (err, [_vp, C.POINTER(C.c_float), C.c_int]),
        "dedisp_b200_get_phasor_source": (err, [_vp, C.POINTER(C.c_int)]),
        "dedisp_b200_get_tc_form": (err, [_vp, C.POINTER(C.c_int)]),
        "dedisp_b200_fdd_segment_length": (_sz, [_sz, _sz, _sz, _sz, C.c_int, _sz]),
        "dedisp_b200_set_wait_limit_ns": (err, [C.c_ulonglong]),
        "dedisp_b200_get_wait_limit_ns": (C.c_ulonglong, []),
        "dedisp_b200_set_wait_expiry_test": (err, [C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _check(code: int) -> None:
    if code != 0:
        buf = C.create_string_buffer(512)
        detail = lib().dedisp_b200_last_error(buf, 512)
        raise DedispError(code, detail, buf.value.decode(errors="replace"))


def _addr(x) -> int:
    """Address of a numpy array, a torch tensor (host or CUDA) or an int."""
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x)!r}")


class Plan:
    """Handle on a dedisp_plan (mirrors dedisp::Plan, src/Plan.hpp)."""

    IMPLEMENTATION = DEDISP_DEDISP

    def __init__(self, nchans: int, dt: float, f0: float, df: float, device_idx: int = 0):
        L = lib()
        _check(L.dedisp_set_device(device_idx))
        _check(L.dedisp_select_implementation(self.IMPLEMENTATION))
        h = _vp()
        _check(L.dedisp_create_plan(C.byref(h), nchans, dt, f0, df))
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().dedisp_destroy_plan(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # setup -------------------------------------------------------------
    def generate_dm_list(self, dm_start: float, dm_end: float, ti: float, tol: float) -> None:
        _check(lib().dedisp_generate_dm_list(self._h, dm_start, dm_end, ti, tol))

    def set_dm_list(self, dms) -> None:
        arr = np.ascontiguousarray(dms, np.float32)
        _check(lib().dedisp_set_dm_list(self._h, arr.ctypes.data, len(arr)))

    def set_killmask(self, killmask=None) -> None:
        if killmask is None:
            _check(lib().dedisp_set_killmask(self._h, None))
        else:
            km = np.ascontiguousarray(killmask, np.int32)
            _check(lib().dedisp_set_killmask(self._h, km.ctypes.data))

    def set_gulp_size(self, n: int) -> None:
        _check(lib().dedisp_set_gulp_size(self._h, n))

    def get_gulp_size(self) -> int:
        return int(lib().dedisp_get_gulp_size(self._h))

    # getters -----------------------------------------------------------
    def get_max_delay(self) -> int:
        return int(lib().dedisp_get_max_delay(self._h))

    def get_dm_delay(self, i: int) -> int:
        return int(lib().dedisp_get_dm_delay(self._h, i))

    def get_channel_count(self) -> int:
        return int(lib().dedisp_get_channel_count(self._h))

    def get_dm_count(self) -> int:
        return int(lib().dedisp_get_dm_count(self._h))

    def get_dm_list(self) -> np.ndarray:
        n = self.get_dm_count()
        p = lib().dedisp_get_dm_list(self._h)
        return np.ctypeslib.as_array(p, (n,)).copy() if n else np.zeros(0, np.float32)

    def get_killmask(self) -> np.ndarray:
        n = self.get_channel_count()
        p = lib().dedisp_get_killmask(self._h)
        return np.ctypeslib.as_array(p, (n,)).copy()

    def get_dt(self) -> float:
        return float(lib().dedisp_get_dt(self._h))

    def get_f0(self) -> float:
        return float(lib().dedisp_get_f0(self._h))

    def get_df(self) -> float:
        return float(lib().dedisp_get_df(self._h))

    def output_row_length(self, nsamps: int) -> int:
        return int(lib().dedisp_b200_output_row_length(self._h, nsamps))

    # execution ---------------------------------------------------------
    def execute(self, nsamps: int, inp, in_nbits: int, out, out_nbits: int,
                flags: int = 0) -> None:
        _check(lib().dedisp_execute(self._h, nsamps, _addr(inp), in_nbits, _addr(out),
                                    out_nbits, flags))

    def execute_adv(self, nsamps, inp, in_nbits, in_stride, out, out_nbits, out_stride,
                    flags: int = 0) -> None:
        _check(lib().dedisp_execute_adv(self._h, nsamps, _addr(inp), in_nbits, in_stride,
                                        _addr(out), out_nbits, out_stride, flags))

    def execute_guru(self, nsamps, inp, in_nbits, in_stride, out, out_nbits, out_stride,
                     first_dm_idx, dm_count, flags: int = 0) -> None:
        _check(lib().dedisp_execute_guru(self._h, nsamps, _addr(inp), in_nbits, in_stride,
                                         _addr(out), out_nbits, out_stride, first_dm_idx,
                                         dm_count, flags))

    def sync(self) -> None:
        _check(lib().dedisp_sync())

    # extensions ----------------------------------------------------------
    def set_stream(self, stream_ptr: int) -> None:
        _check(lib().dedisp_b200_set_stream(self._h, stream_ptr or None))

    def set_timing(self, enable: bool = True) -> None:
        _check(lib().dedisp_b200_set_timing(self._h, int(enable)))

    def get_timing(self) -> dict:
        k, p = C.c_float(), C.c_float()
        n, v = C.c_int(), C.c_int()
        _check(lib().dedisp_b200_get_timing(self._h, C.byref(k), C.byref(p), C.byref(n),
                                            C.byref(v)))
        return {"kernel_ms": k.value, "prep_ms": p.value, "launches": n.value,
                "variant": v.value}

    STAGES = ("unpack", "fft_fwd", "layout", "mac", "transpose", "fft_inv")

    def get_stage_times(self) -> dict:
        """FDD plans: device ms of each stage of the last timed execute."""
        v = (C.c_float * 6)()
        _check(lib().dedisp_b200_get_stage_times(self._h, v, 6))
        return dict(zip(self.STAGES, [float(x) for x in v]))

    PHASOR_SOURCES = {-1: None, 0: "table", 1: "quarter", 2: "hybrid", 3: "direct"}

    def get_phasor_source(self):
        """FDD plans: phasor source of the last tensor-core MAC ("table",
        "quarter", "hybrid", "direct"), None when none ran."""
        v = C.c_int()
        _check(lib().dedisp_b200_get_phasor_source(self._h, C.byref(v)))
        return self.PHASOR_SOURCES[v.value]

    TC_FORMS = {-1: None, 0: "three", 1: "fused", 2: "deep", 3: "pair", 4: "pair-deep", 5: "fused-wide"}

    def get_tc_form(self):
        """FDD plans: MMA form of the last tensor-core MAC launch."""
        v = C.c_int()
        _check(lib().dedisp_b200_get_tc_form(self._h, C.byref(v)))
        return self.TC_FORMS[v.value]


class DedispPlan(Plan):
    """Original dedisp interface (reference src/dedisp/DedispPlan.hpp)."""
    IMPLEMENTATION = DEDISP_DEDISP

    def set_kernel(self, kernel: int) -> None:
        """0 auto, 1 plain (one thread per sample pair), 2 tiled."""
        _check(lib().dedisp_b200_set_tdd_kernel(self._h, kernel))

    def set_tile_variant(self, variant: int) -> None:
        """Tile shape of the tiled kernel for 8-bit input (same sums)."""
        _check(lib().dedisp_b200_set_tdd_variant(self._h, variant))


class TDDPlan(DedispPlan):
    """Time-domain dedispersion (reference src/tdd/TDDPlan.hpp)."""
    IMPLEMENTATION = DEDISP_TDD


FDD_SEGMENT_AUTO = 1


def _segment_arg(segment_nfft) -> int:
    return FDD_SEGMENT_AUTO if segment_nfft == "auto" else int(segment_nfft)


def fdd_segment_length(nsamps: int, max_delay: int, dm_count: int, nchans: int, precision: int = 1,
                       segment_nfft=0) -> int:
    """Segment length (points) of segmented FDD for these sizes under the
    rule `segment_nfft` (0 reference, "auto", or a length); 0 if none fits."""
    return int(lib().dedisp_b200_fdd_segment_length(nsamps, max_delay, dm_count, nchans, precision,
                                                    _segment_arg(segment_nfft)))


class FDDGPUPlan(Plan):
    """Fourier-domain dedispersion (reference src/fdd/FDDGPUPlan.hpp)."""
    IMPLEMENTATION = DEDISP_FDD

    def set_options(self, segmented: int = -1, timeseries: bool = False, precision: int = 0,
                    round_delays: bool = False, segment_nfft=0) -> None:
        """segment_nfft: 0 the reference doubling rule, "auto" the power of two
        with the least modelled device time, else a power of two."""
        _check(lib().dedisp_b200_set_fdd_options(self._h, segmented, int(timeseries),
                                                 precision, int(round_delays),
                                                 _segment_arg(segment_nfft)))


def set_wait_limit_ns(ns: int) -> None:
    """Limit of the kernels' bounded waits on their own copies and MMAs
    (nanoseconds of GPU global time; 0 restores the default, 2 s)."""
    _check(lib().dedisp_b200_set_wait_limit_ns(int(ns)))


def get_wait_limit_ns() -> int:
    return int(lib().dedisp_b200_get_wait_limit_ns())


def set_wait_expiry_test(enable: bool) -> None:
    """Expiry test: each kernel with bounded waits also waits on a barrier
    that nothing arrives on, so its error path runs (for tests)."""
    _check(lib().dedisp_b200_set_wait_expiry_test(1 if enable else 0))


def tdd_variant_count(in_nbits: int = 8) -> int:
    """Number of tile-shape variants of the tiled TDD kernel for in_nbits."""
    return int(lib().dedisp_b200_tdd_variant_count(in_nbits))


def batch_variant_count(in_nbits: int = 8) -> int:
    """Number of tile-shape variants of the persistent multi-beam kernel
    (the same shapes as the plans' tiled kernel)."""
    return int(_batch_lib().dedisp_b200_batch_variant_count(in_nbits))


# ---------------------------------------------------------------------------
# Batched multi-beam TDD (dedisp_b200_batch_*; device buffers only)
# ---------------------------------------------------------------------------

class _Beam(C.Structure):
    _fields_ = [("in_", _vp), ("in_stride", _sz), ("nsamps", _sz), ("dm_list", _vp),
                ("dm_count", _sz), ("out", _vp), ("out_stride", _sz)]


_BATCH_SIGS = {
    "dedisp_b200_batch_create": (C.c_int, [C.POINTER(_vp), _sz, C.c_float, C.c_float, C.c_float,
                                           _sz, _sz, C.c_int]),
    "dedisp_b200_batch_destroy": (None, [_vp]),
    "dedisp_b200_batch_set_killmask": (C.c_int, [_vp, _vp]),
    "dedisp_b200_batch_set_beams": (C.c_int, [_vp, C.POINTER(_Beam), _sz]),
    "dedisp_b200_batch_workspace_size": (_sz, [_vp]),
    "dedisp_b200_batch_set_workspace": (C.c_int, [_vp, _vp, _sz]),
    "dedisp_b200_batch_set_shape": (C.c_int, [_vp, C.c_int, C.c_int]),
    "dedisp_b200_batch_variant_count": (C.c_int, [_sz]),
    "dedisp_b200_batch_autotune": (C.c_int, [_vp, _vp, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "dedisp_b200_batch_execute": (C.c_int, [_vp, _vp, C.c_int]),
    "dedisp_b200_batch_sync": (C.c_int, [_vp, _vp]),
    "dedisp_b200_batch_set_timing": (C.c_int, [_vp, C.c_int]),
    "dedisp_b200_batch_get_timing": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                               C.POINTER(C.c_int)]),
    "dedisp_b200_batch_max_delay": (_sz, [_vp, _sz]),
    "dedisp_b200_fdd_batch_create": (C.c_int, [C.POINTER(_vp), _sz, C.c_float, C.c_float, C.c_float,
                                               _sz, C.c_int]),
    "dedisp_b200_fdd_batch_destroy": (None, [_vp]),
    "dedisp_b200_fdd_batch_set_killmask": (C.c_int, [_vp, _vp]),
    "dedisp_b200_fdd_batch_set_beams": (C.c_int, [_vp, C.POINTER(_Beam), _sz]),
    "dedisp_b200_fdd_batch_workspace_size": (_sz, [_vp]),
    "dedisp_b200_fdd_batch_set_workspace": (C.c_int, [_vp, _vp, _sz]),
    "dedisp_b200_fdd_batch_execute": (C.c_int, [_vp, _vp, C.c_int]),
    "dedisp_b200_fdd_batch_sync": (C.c_int, [_vp, _vp]),
    "dedisp_b200_fdd_batch_set_timing": (C.c_int, [_vp, C.c_int]),
    "dedisp_b200_fdd_batch_get_timing": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                                   C.POINTER(C.c_float), C.POINTER(C.c_int)]),
    "dedisp_b200_fdd_batch_max_delay": (_sz, [_vp, _sz]),
    "dedisp_b200_fdd_batch_phasor_source": (C.c_int, [_vp, _sz]),
    "dedisp_b200_fdd_batch_get_mac_balance": (C.c_int, [_vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "dedisp_b200_fdd_batch_set_segment_nfft": (C.c_int, [_vp, _sz]),
}


def _batch_lib() -> C.CDLL:
    L = lib()
    if not getattr(L, "_batch_sigs", False):
        for name, (res, args) in _BATCH_SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L._batch_sigs = True
    return L


def _bcheck(code: int) -> None:
    if code != 0:
        buf = C.create_string_buffer(512)
        lib().dedisp_b200_last_error(buf, 512)
        raise DedispError(code, code, buf.value.decode(errors="replace"))


class Batch:
    """Many beams with one channel setup, dedispersed by one graph-captured
    persistent launch. Beams are (device input, nsamps, DM list, device
    output) with torch CUDA tensors or raw device addresses."""

    def __init__(self, nchans: int, dt: float, f0: float, df: float, in_nbits: int = 8,
                 out_nbits: int = 32, device: int = 0):
        self._h = _vp()
        _bcheck(_batch_lib().dedisp_b200_batch_create(C.byref(self._h), nchans, dt, f0, df,
                                                      in_nbits, out_nbits, device))
        self.nchans, self.in_nbits, self.out_nbits = nchans, in_nbits, out_nbits
        self._keep = []

    def close(self) -> None:
        if self._h:
            _batch_lib().dedisp_b200_batch_destroy(self._h)
            self._h = _vp()
        self._keep = []
        self._ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_killmask(self, killmask=None) -> None:
        if killmask is None:
            _bcheck(_batch_lib().dedisp_b200_batch_set_killmask(self._h, None))
            return
        km = np.ascontiguousarray(killmask, dtype=np.int32)
        _bcheck(_batch_lib().dedisp_b200_batch_set_killmask(self._h, km.ctypes.data))

    def set_beams(self, beams) -> None:
        """beams: sequence of (d_in, in_stride, nsamps, dm_list, d_out, out_stride)."""
        arr = (_Beam * max(len(beams), 1))()
        keep = []
        for i, (d_in, in_stride, nsamps, dms, d_out, out_stride) in enumerate(beams):
            dm = np.ascontiguousarray(dms, dtype=np.float32)
            keep.append(dm)
            arr[i] = _Beam(_addr(d_in), in_stride, nsamps, dm.ctypes.data, len(dm), _addr(d_out),
                           out_stride)
        _bcheck(_batch_lib().dedisp_b200_batch_set_beams(self._h, arr, len(beams)))
        self._keep = [b[0] for b in beams] + [b[4] for b in beams]

    def workspace_size(self) -> int:
        return int(_batch_lib().dedisp_b200_batch_workspace_size(self._h))

    def set_workspace(self, buf, nbytes: int) -> None:
        _bcheck(_batch_lib().dedisp_b200_batch_set_workspace(self._h, _addr(buf), nbytes))
        self._ws = buf

    def set_shape(self, variant: int, chan_per_stage: int = 0) -> None:
        _bcheck(_batch_lib().dedisp_b200_batch_set_shape(self._h, variant, chan_per_stage))

    def autotune(self, stream: int = 0):
        v, cs = C.c_int(), C.c_int()
        _bcheck(_batch_lib().dedisp_b200_batch_autotune(self._h, stream, C.byref(v), C.byref(cs)))
        return v.value, cs.value

    def execute(self, stream: int = 0, use_graph: bool = True) -> None:
        _bcheck(_batch_lib().dedisp_b200_batch_execute(self._h, stream, int(use_graph)))

    def sync(self, stream: int = 0) -> None:
        """Waits for the batch's work on `stream`; raises if a bounded wait
        of the last execute expired."""
        _bcheck(_batch_lib().dedisp_b200_batch_sync(self._h, stream))

    def set_timing(self, enable: bool = True) -> None:
        _bcheck(_batch_lib().dedisp_b200_batch_set_timing(self._h, int(enable)))

    def get_timing(self) -> dict:
        a, b, n = C.c_float(), C.c_float(), C.c_int()
        _bcheck(_batch_lib().dedisp_b200_batch_get_timing(self._h, C.byref(a), C.byref(b),
                                                          C.byref(n)))
        return {"transpose_ms": a.value, "dedisperse_ms": b.value, "launches": n.value}

    def max_delay(self, beam: int) -> int:
        return int(_batch_lib().dedisp_b200_batch_max_delay(self._h, beam))


# ---------------------------------------------------------------------------
# Streaming server (dedisp_b200_server_*)
# ---------------------------------------------------------------------------

class FddBatch:
    """Many beams with one channel setup, dedispersed in the Fourier domain
    (segmented time series, 3xBF16 tensor-core MAC) with one persistent MAC
    launch over all of them per MMA-form class (at most two), the whole
    sequence graph-captured. Beams are
    (device input, in_stride, nsamps, DM list, device output, out_stride);
    output rows hold nsamps - max_delay floats."""

    def __init__(self, nchans: int, dt: float, f0: float, df: float, in_nbits: int = 8,
                 device: int = 0):
        self._h = _vp()
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_create(C.byref(self._h), nchans, dt, f0, df,
                                                          in_nbits, device))
        self._keep = []
        self._ws = None

    def close(self) -> None:
        if self._h:
            _batch_lib().dedisp_b200_fdd_batch_destroy(self._h)
            self._h = _vp()
        self._keep = []
        self._ws = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_segment_nfft(self, segment_nfft) -> None:
        """0 the reference doubling rule (default), "auto" the least modelled
        time per beam, else a power of two; takes effect at set_beams."""
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_set_segment_nfft(self._h, _segment_arg(segment_nfft)))

    def set_killmask(self, killmask=None) -> None:
        if killmask is None:
            _bcheck(_batch_lib().dedisp_b200_fdd_batch_set_killmask(self._h, None))
            return
        km = np.ascontiguousarray(killmask, dtype=np.int32)
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_set_killmask(self._h, km.ctypes.data))

    def set_beams(self, beams) -> None:
        """beams: sequence of (d_in, in_stride, nsamps, dm_list, d_out, out_stride)."""
        arr = (_Beam * max(len(beams), 1))()
        for i, (d_in, in_stride, nsamps, dms, d_out, out_stride) in enumerate(beams):
            dm = np.ascontiguousarray(dms, dtype=np.float32)
            arr[i] = _Beam(_addr(d_in), in_stride, nsamps, dm.ctypes.data, len(dm), _addr(d_out),
                           out_stride)
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_set_beams(self._h, arr, len(beams)))
        self._keep = [b[0] for b in beams] + [b[4] for b in beams]

    def workspace_size(self) -> int:
        return int(_batch_lib().dedisp_b200_fdd_batch_workspace_size(self._h))

    def set_workspace(self, buf, nbytes: int) -> None:
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_set_workspace(self._h, _addr(buf), nbytes))
        self._ws = buf

    def execute(self, stream: int = 0, use_graph: bool = True) -> None:
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_execute(self._h, stream, int(use_graph)))

    def sync(self, stream: int = 0) -> None:
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_sync(self._h, stream))

    def set_timing(self, enable: bool = True) -> None:
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_set_timing(self._h, int(enable)))

    def get_timing(self) -> dict:
        p, m, q, n = C.c_float(), C.c_float(), C.c_float(), C.c_int()
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_get_timing(self._h, C.byref(p), C.byref(m),
                                                              C.byref(q), C.byref(n)))
        return {"prep_ms": p.value, "mac_ms": m.value, "post_ms": q.value, "launches": n.value}

    def get_mac_balance(self) -> dict:
        """After a direct execute with timing on: largest and mean per-CTA
        busy time of the MAC launch (ms)."""
        a, b = C.c_float(), C.c_float()
        _bcheck(_batch_lib().dedisp_b200_fdd_batch_get_mac_balance(self._h, C.byref(a), C.byref(b)))
        return {"cta_max_ms": a.value, "cta_mean_ms": b.value}

    def max_delay(self, beam: int) -> int:
        return int(_batch_lib().dedisp_b200_fdd_batch_max_delay(self._h, beam))

    def phasor_source(self, beam: int):
        """Phasor source planned for a beam's tensor-core MAC ("table",
        "quarter", "hybrid", "direct"), None without MAC work."""
        return Plan.PHASOR_SOURCES[int(_batch_lib().dedisp_b200_fdd_batch_phasor_source(self._h, beam))]


class _GulpRecord(C.Structure):
    _fields_ = [("beam", C.c_int), ("worker", C.c_int), ("nsamps", _sz), ("t_submit", C.c_double),
                ("t_start", C.c_double), ("t_done", C.c_double), ("device_ms", C.c_float)]


_SERVER_SIGS = {
    "dedisp_b200_server_create": (C.c_int, [C.POINTER(_vp), _sz, C.c_float, C.c_float, C.c_float,
                                            _sz, C.c_int, _sz, _sz, C.c_int, C.c_int, C.c_int, _sz,
                                            _sz]),
    "dedisp_b200_server_destroy": (None, [_vp]),
    "dedisp_b200_server_add_beam": (C.c_int, [_vp, _vp, _sz, C.c_int]),
    "dedisp_b200_server_max_delay": (_sz, [_vp, C.c_int]),
    "dedisp_b200_server_start": (C.c_int, [_vp, C.POINTER(_sz)]),
    "dedisp_b200_server_submit": (C.c_long, [_vp, C.c_int, _vp, _sz, _vp]),
    "dedisp_b200_server_done": (C.c_int, [_vp, C.c_long]),
    "dedisp_b200_server_wait": (C.c_int, [_vp, C.c_long]),
    "dedisp_b200_server_drain": (C.c_int, [_vp]),
    "dedisp_b200_server_record_count": (_sz, [_vp]),
    "dedisp_b200_server_records": (C.c_int, [_vp, C.POINTER(_GulpRecord), _sz]),
}


def _server_lib() -> C.CDLL:
    L = lib()
    if not getattr(L, "_server_sigs", False):
        for name, (res, args) in _SERVER_SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L._server_sigs = True
    return L


def _last_message() -> str:
    buf = C.create_string_buffer(512)
    lib().dedisp_b200_last_error(buf, 512)
    return buf.value.decode(errors="replace")


class StreamServer:
    """Streaming dedispersion of many beams' gulps with device-resident
    overlap tails (kind 0: TDD, 1: FDD). See include/dedisp_b200.h."""

    TDD, FDD = 0, 1

    def __init__(self, nchans: int, dt: float, f0: float, df: float, in_nbits: int = 8,
                 device: int = 0, hbm_budget: int = 0, max_gulp: int = 1 << 18,
                 tdd_workers: int = 2, fdd_workers: int = 0, fdd_precision: int = 1,
                 fdd_segment: int = 0, fdd_max_gulp: int = 0):
        self._h = _vp()
        _bcheck(_server_lib().dedisp_b200_server_create(
            C.byref(self._h), nchans, dt, f0, df, in_nbits, device, int(hbm_budget), max_gulp,
            tdd_workers, fdd_workers, fdd_precision, fdd_segment, fdd_max_gulp))
        self.nchans, self.in_nbits = nchans, in_nbits
        self._rows = {}

    def close(self) -> None:
        if self._h:
            _server_lib().dedisp_b200_server_destroy(self._h)
            self._h = _vp()
        self._rows = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_beam(self, dms, kind: int = 0) -> int:
        dm = np.ascontiguousarray(dms, dtype=np.float32)
        b = _server_lib().dedisp_b200_server_add_beam(self._h, dm.ctypes.data, len(dm), kind)
        if b < 0:
            raise DedispError(DEDISP_UNKNOWN_ERROR, DEDISP_UNKNOWN_ERROR, _last_message())
        return b

    def max_delay(self, beam: int) -> int:
        return int(_server_lib().dedisp_b200_server_max_delay(self._h, beam))

    def start(self) -> int:
        n = _sz()
        _bcheck(_server_lib().dedisp_b200_server_start(self._h, C.byref(n)))
        return int(n.value)

    def submit(self, beam: int, rows, nsamps: int, d_out=None) -> int:
        t = _server_lib().dedisp_b200_server_submit(self._h, beam, _addr(rows), nsamps, _addr(d_out))
        if t < 0:
            raise DedispError(DEDISP_UNKNOWN_ERROR, DEDISP_UNKNOWN_ERROR, _last_message())
        self._rows[t] = (rows, d_out)
        return t

    def done(self, ticket: int) -> bool:
        d = _server_lib().dedisp_b200_server_done(self._h, ticket)
        if d < 0:
            raise DedispError(DEDISP_UNKNOWN_ERROR, DEDISP_UNKNOWN_ERROR, _last_message())
        return bool(d)

    def wait(self, ticket: int) -> None:
        _bcheck(_server_lib().dedisp_b200_server_wait(self._h, ticket))
        self._rows.pop(ticket, None)

    def drain(self) -> None:
        _bcheck(_server_lib().dedisp_b200_server_drain(self._h))
        self._rows = {}

    def records(self) -> list:
        L = _server_lib()
        n = int(L.dedisp_b200_server_record_count(self._h))
        arr = (_GulpRecord * max(n, 1))()
        _bcheck(L.dedisp_b200_server_records(self._h, arr, n))
        return [{"beam": r.beam, "worker": r.worker, "nsamps": int(r.nsamps),
                 "t_submit": r.t_submit, "t_start": r.t_start, "t_done": r.t_done,
                 "device_ms": r.device_ms} for r in arr[:n]]


# ---------------------------------------------------------------------------
# SIGPROC filterbank I/O (dedisp_b200_fil_* / dedisp_b200_write_*)
# ---------------------------------------------------------------------------

class FilHeader(C.Structure):
    _fields_ = [("tsamp", C.c_double), ("tstart", C.c_double), ("fch1", C.c_double),
                ("foff", C.c_double), ("src_raj", C.c_double), ("src_dej", C.c_double),
                ("az_start", C.c_double), ("za_start", C.c_double), ("nchans", C.c_int),
                ("nifs", C.c_int), ("nbits", C.c_int), ("telescope_id", C.c_int),
                ("machine_id", C.c_int), ("nbeams", C.c_int), ("ibeam", C.c_int),
                ("nsamples", _sz), ("header_bytes", _sz), ("source_name", C.c_char * 80)]


_IO_SIGS = {
    "dedisp_b200_fil_read_header": (C.c_int, [C.c_char_p, C.POINTER(FilHeader)]),
    "dedisp_b200_fil_read_samples": (C.c_int, [C.c_char_p, C.POINTER(FilHeader), _sz, _sz, _vp]),
    "dedisp_b200_fil_decimate": (_sz, [_vp, _sz, _sz, _sz]),
    "dedisp_b200_write_dat": (C.c_int, [C.c_char_p, C.c_float, _vp, _sz]),
    "dedisp_b200_write_inf": (C.c_int, [C.c_char_p, C.c_float, C.POINTER(FilHeader), _sz]),
}


def _io_lib() -> C.CDLL:
    L = lib()
    if not getattr(L, "_io_sigs", False):
        for name, (res, args) in _IO_SIGS.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L._io_sigs = True
    return L


def fil_read_header(path: str) -> FilHeader:
    h = FilHeader()
    _bcheck(_io_lib().dedisp_b200_fil_read_header(path.encode(), C.byref(h)))
    return h


def fil_read(path: str, first: int = 0, count=None):
    """(header, time-major packed rows as a uint8 array [count][row bytes])."""
    h = fil_read_header(path)
    n = h.nsamples - first if count is None else count
    row = h.nchans * h.nifs * h.nbits // 8
    out = np.empty((n, row), np.uint8)
    _bcheck(_io_lib().dedisp_b200_fil_read_samples(path.encode(), C.byref(h), first, n, out.ctypes.data))
    return h, out


def fil_decimate(data: np.ndarray, nchans: int, factor: int) -> int:
    """8-bit rows averaged over `factor` samples in place; returns the new count."""
    return int(_io_lib().dedisp_b200_fil_decimate(data.ctypes.data, nchans, data.shape[0], factor))


def write_dat_inf(prefix: str, dm: float, series: np.ndarray, header: FilHeader) -> None:
    s = np.ascontiguousarray(series, dtype=np.float32)
    _bcheck(_io_lib().dedisp_b200_write_dat(prefix.encode(), dm, s.ctypes.data, s.size))
    _bcheck(_io_lib().dedisp_b200_write_inf(prefix.encode(), dm, C.byref(header), s.size))


def fil_tool_path() -> str:
    """The dedisp_fil command-line program built beside the library."""
    return os.path.join(HERE, "bin", "dedisp_fil")

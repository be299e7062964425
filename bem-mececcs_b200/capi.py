"""ctypes bindings of libbem_b200.so (include/bem_capi.h).

The library is the product: every call here goes to the sm_100a kernels.
There is no CPU fallback; a missing or unloadable library raises.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbem_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "bem_capi.h")

BEM_OK = 0
BEM_ERR_DEGENERATE = 1
BEM_ERR_SINGULAR = 2
BEM_ERR_ARG = 3
BEM_ERR_CUDA = 4
BEM_ERR_NOMEM = 5
BEM_ERR_STATE = 6
BEM_ERR_TIMEOUT = 7
BEM_FAST_SINGULAR = 1
BEM_KEEP_PRESWAP = 2
BEM_FORM_PLAIN = 0
BEM_FORM_MIXED = 1
PROF_CLASSES = ["assembly", "panel", "laswp_trsm", "gemm", "solves", "residual"]

_lib = None


class BemError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def header_functions() -> list:
    """Names of every function the C-ABI header declares."""
    with open(HEADER) as fh:
        text = fh.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", text)) - {"if", "defined"})


def lib():
    """Loads the library; raises when it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    P = ctypes.POINTER
    L.bem_ctx_create.argtypes = [ip, P(vp)]
    L.bem_ctx_destroy.argtypes = [vp]
    L.bem_ctx_set_stream.argtypes = [vp, vp]
    L.bem_status_string.argtypes = [ip]
    L.bem_status_string.restype = ctypes.c_char_p
    L.bem_last_error.argtypes = [vp]
    L.bem_last_error.restype = ctypes.c_char_p
    L.bem_ctx_set_option.argtypes = [vp, ctypes.c_char_p, ip]
    L.bem_ctx_get_option.argtypes = [vp, ctypes.c_char_p, P(ip)]
    L.bem_ctx_launch_count.argtypes = [vp]
    L.bem_ctx_launch_count.restype = ctypes.c_longlong
    L.bem_mesh_upload.argtypes = [vp, ip, ip, ip, ip] + [vp] * 10
    L.bem_ghmatece.argtypes = [vp, vp, ip, vp, vp]
    L.bem_set_gestdiag.argtypes = [vp, vp]
    L.bem_set_hestdiag.argtypes = [vp, vp]
    L.bem_static_h.argtypes = [vp, vp, vp]
    L.bem_dyn_upload.argtypes = [vp, vp, vp]
    L.bem_ghmatecd.argtypes = [vp, vp, vp, vp, vp, dp, ip]
    L.bem_get_system.argtypes = [vp, vp, vp]
    L.bem_get_preswap.argtypes = [vp, vp, vp]
    L.bem_ghmatecd_noalloc.argtypes = [vp, vp, vp, vp, vp, dp, ip, vp, ctypes.c_size_t]
    L.bem_linsolve.argtypes = [vp, vp]
    L.bem_solve_dense.argtypes = [vp, ip, vp, vp, vp]
    L.bem_unswap.argtypes = [vp, vp, vp]
    L.bem_sync.argtypes = [vp]
    L.bem_linsolve_async.argtypes = [vp]
    L.bem_prof_enable.argtypes = [vp, ip]
    L.bem_prof_reset.argtypes = [vp]
    L.bem_prof_read.argtypes = [vp, vp, vp, vp]
    L.bem_prof_bytes.argtypes = [vp, vp]
    L.bem_measure_fp64_peak.argtypes = [vp, vp]
    L.bem_measure_peaks.argtypes = [vp, vp]
    L.bem_wait_selftest.argtypes = [vp, ip]
    L.bem_static_solve.argtypes = [vp, vp, dp, vp, vp, vp, vp]
    L.bem_batch_solve.argtypes = [vp, ip, vp, vp, vp, vp, vp, vp, ip, ip, vp, vp]
    L.bem_interior.argtypes = [vp, vp, vp, vp, dp, dp, ip, vp, vp, vp, vp, vp, vp, vp]
    L.bem_sweep.argtypes = [vp, vp, vp, vp, vp, vp, ip, ip, ip, ip, vp, vp]
    L.bem_sweep_async.argtypes = [vp, vp, vp, vp, vp, vp, ip, ip, ip, ip, vp]
    L.bem_sweep_batch_limit.argtypes = [vp, ip, P(ip)]
    _lib = L
    return L


def ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class Context:
    """One bem_ctx (one mesh resident on one GPU)."""

    def __init__(self, device: int = 0):
        self.L = lib()
        self.h = ctypes.c_void_p()
        rc = self.L.bem_ctx_create(device, ctypes.byref(self.h))
        if rc != BEM_OK:
            raise BemError(rc, f"bem_ctx_create(device={device}) failed")

    def check(self, rc: int, what: str, allow=()):
        if rc != BEM_OK and rc not in allow:
            raise BemError(rc, f"{what}: {self.L.bem_last_error(self.h).decode()}")
        return rc

    def close(self):
        if self.h:
            self.L.bem_ctx_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    INT_OPTIONS = ("gemm_ctas", "trsv_ctas", "wait_limit_ms")

    def set_option(self, name: str, value) -> None:
        """bem_ctx_set_option: switches tcgen05, trsv_coop, lu_pairs, lu_quads,
        f64_pairs, tc_pair, panel_calu, panel_push, panel_async, laswp_tc, trsv_inv, graphs; CTA
        budgets gemm_ctas, trsv_ctas (0 = device); wait_limit_ms, the bound of
        every device-side wait (1..60000, default 2000)."""
        v = int(value) if name in self.INT_OPTIONS else int(bool(value))
        self.check(self.L.bem_ctx_set_option(self.h, name.encode(), v), "bem_ctx_set_option")

    def get_option(self, name: str):
        out = ctypes.c_int(0)
        self.check(self.L.bem_ctx_get_option(self.h, name.encode(), ctypes.byref(out)), "bem_ctx_get_option")
        return out.value if name in self.INT_OPTIONS else bool(out.value)

    @property
    def launches(self) -> int:
        return int(self.L.bem_ctx_launch_count(self.h))

    def prof(self, on: bool):
        self.check(self.L.bem_prof_enable(self.h, int(on)), "bem_prof_enable")

    def prof_reset(self):
        self.check(self.L.bem_prof_reset(self.h), "bem_prof_reset")

    def prof_read(self) -> dict:
        nc = len(PROF_CLASSES)
        ms = np.zeros(nc)
        n = np.zeros(nc, dtype=np.int64)
        work = np.zeros(nc)
        self.check(self.L.bem_prof_read(self.h, ptr(ms), ptr(n), ptr(work)), "bem_prof_read")
        nbytes = np.zeros(nc)
        self.check(self.L.bem_prof_bytes(self.h, ptr(nbytes)), "bem_prof_bytes")
        return {k: {"ms": float(ms[i]), "launches": int(n[i]), "work": float(work[i]),
                    "bytes": float(nbytes[i])}
                for i, k in enumerate(PROF_CLASSES)}

    def wait_selftest(self, which: int) -> int:
        """bem_wait_selftest: the status of one bounded wait on an event that
        never happens (0: bulk-copy mbarrier, 1: grid barrier); BEM_ERR_TIMEOUT
        when the wait gave up as it should."""
        return int(self.L.bem_wait_selftest(self.h, int(which)))

    def fp64_peak_tflops(self) -> float:
        out = np.zeros(1)
        self.check(self.L.bem_measure_fp64_peak(self.h, ptr(out)), "bem_measure_fp64_peak")
        return float(out[0])

    def peaks(self) -> dict:
        """bem_measure_peaks: measured arithmetic peaks, TFLOP/s."""
        out = np.zeros(5)
        self.check(self.L.bem_measure_peaks(self.h, ptr(out)), "bem_measure_peaks")
        keys = ["fp64_fma", "fp32_fma", "fp64_dmma", "tf32_umma_n128", "tf32_umma_n256"]
        return {k: round(float(v), 2) for k, v in zip(keys, out)}

    def sync(self):
        return self.check(self.L.bem_sync(self.h), "bem_sync")

    def set_stream(self, stream_handle: int | None):
        self.check(self.L.bem_ctx_set_stream(self.h, ctypes.c_void_p(stream_handle or 0)),
                   "bem_ctx_set_stream")

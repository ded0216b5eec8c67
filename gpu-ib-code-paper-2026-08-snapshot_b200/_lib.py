"""ctypes binding of ``include/pyib_b200.h`` (the C ABI of ``libpyib_b200.so``).

The library is built in-tree (``build.py``) and loaded from the package
directory.  There is no fallback: if the shared library is missing or a call
fails, a ``B200Error`` is raised with the library's own message.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpyib_b200.so"
MAX_LEVELS = 8

# status codes
OK, E_ARG, E_CUDA, E_STATE, E_NOCONV, E_NONFINITE, E_DEVICE = range(7)

# tables (enum pyib_table)
TABLES = [
    "PREC", "INLET_IDX", "INLET_VAL", "CURL_PTR", "CURL_COL", "CURL_VAL", "ROT_PTR", "ROT_COL",
    "ROT_VAL", "P_PTR", "P_COL", "P_VAL3", "I_PTR", "I_COL", "I_VAL3", "CF_PTR", "CF_FACE",
    "F_LO", "F_HI", "F_AOL", "VOLCI", "BF_FACE", "BF_CELL", "BF_INFO", "BF_AF",
    "PA_BITS", "PA_ROW", "PA_PTR", "PA_COL", "PA_VAL",
    "PV_BITS", "PV_ROW", "PV_PTR", "PV_COL", "PV_VAL",
    "PR_BITS", "PR_ROW", "PR_PTR", "PR_COL", "PR_VAL",
    "LC_CAND", "LC_FIDX", "LC_CPOS", "PREC_BITS", "PREC_REG", "PA_IDS", "PV_IDS", "PR_IDS",
]
T = {name: i for i, name in enumerate(TABLES)}

FIELDS = [
    "S", "S_OLD", "U", "VC", "VC_GHOST", "RES_C", "RES_E", "FE", "FL", "MARKERS", "MVEL", "DS",
    "WORK_E", "WORK_E2", "WORK_C3", "WORK_F", "IB_CELL", "IB_W", "IB_BASE", "LAG_TMP", "DINV",
]
F = {name: i for i, name in enumerate(FIELDS)}

EXPORTS = [
    "pyib_version", "pyib_last_error", "pyib_create", "pyib_destroy", "pyib_upload", "pyib_finalize",
    "pyib_set_params", "pyib_set_ib_geometry", "pyib_set_field", "pyib_get_field", "pyib_matvec",
    "pyib_operator", "pyib_calc_vel", "pyib_conv_diff", "pyib_helm_solve", "pyib_step",
    "pyib_ib_stencil", "pyib_ib_interp", "pyib_ib_spread", "pyib_loads", "pyib_diagnostics",
    "pyib_cg_timing", "pyib_matvec_plan", "pyib_event", "pyib_bench_matvec", "pyib_bench_matvec_fused", "pyib_spread_noalloc", "pyib_ib_interp_dx", "pyib_graph_pcg",
    "pyib_recover_pressure", "pyib_batch_create", "pyib_batch_destroy", "pyib_batch_last_error",
    "pyib_batch_step", "pyib_batch_timing",
]


class Layout(C.Structure):
    _fields_ = [
        ("nlevels", C.c_int32),
        ("n", (C.c_int32 * 3) * MAX_LEVELS),
        ("hole_lo", (C.c_int32 * 3) * MAX_LEVELS),
        ("hole_n", (C.c_int32 * 3) * MAX_LEVELS),
        ("h", C.c_double * MAX_LEVELS),
        ("lo", (C.c_double * 3) * MAX_LEVELS),
        ("ncell", C.c_int64), ("nface", C.c_int64), ("nedge", C.c_int64),
        ("nbface", C.c_int32), ("device", C.c_int32),
    ]


class Params(C.Structure):
    _fields_ = [
        ("rou", C.c_double), ("visc", C.c_double), ("ac", C.c_double), ("ad", C.c_double),
        ("tol1", C.c_double), ("tol2", C.c_double),
        ("cavity", C.c_int32), ("check", C.c_int32), ("cg_max", C.c_int32), ("strict", C.c_int32),
        ("precision", C.c_int32), ("nmarkers", C.c_int32),
        ("hh", C.c_double), ("hh3", C.c_double),
        ("mixed_tol", C.c_double), ("mixed_max_sweeps", C.c_int32), ("ib_mode", C.c_int32),
        ("ib_alpha", C.c_double),
    ]


class SolveStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("converged", C.c_int32),
        ("rel_residual", C.c_double), ("tol_ratio", C.c_double),
        ("eta0", C.c_double), ("threshold", C.c_double),
        ("refinements", C.c_int32), ("pad", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int32), ("total_iterations", C.c_int32),
        ("all_converged", C.c_int32), ("ib_updates", C.c_int32),
        ("max_rel_residual", C.c_double), ("max_tol_ratio", C.c_double),
    ]


class B200Error(RuntimeError):
    """A call into libpyib_b200 failed; ``code`` is the PYIB_E_* status."""

    def __init__(self, code, message):
        super().__init__(message)
        self.code = code


_lib = None


def load():
    """Load the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise B200Error(E_STATE, f"{LIB_PATH.name} is not built; run build.build_library() "
                                 "(the B200 path has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "pyib_version": [C.c_char_p, C.c_size_t],
        "pyib_last_error": [vp, C.c_char_p, C.c_size_t],
        "pyib_create": [C.POINTER(Layout), C.POINTER(vp)],
        "pyib_destroy": [vp],
        "pyib_upload": [vp, C.c_int32, vp, C.c_size_t],
        "pyib_finalize": [vp, C.POINTER(C.c_int64), C.c_int32],
        "pyib_set_params": [vp, C.POINTER(Params)],
        "pyib_set_ib_geometry": [vp, C.POINTER(C.c_double), C.c_double],
        "pyib_set_field": [vp, C.c_int32, vp, C.c_size_t],
        "pyib_get_field": [vp, C.c_int32, vp, C.c_size_t],
        "pyib_matvec": [vp, C.c_int32, C.c_int32, C.c_double, C.c_int32],
        "pyib_operator": [vp, C.c_int32],
        "pyib_calc_vel": [vp],
        "pyib_conv_diff": [vp],
        "pyib_helm_solve": [vp, C.c_double, C.POINTER(SolveStats)],
        "pyib_step": [vp, C.c_double, C.c_double, C.c_int32, vp, vp, C.POINTER(StepStats)],
        "pyib_ib_stencil": [vp],
        "pyib_ib_interp": [vp],
        "pyib_ib_spread": [vp],
        "pyib_loads": [vp, C.POINTER(C.c_double), C.c_double, C.c_double, C.c_double, C.c_int32,
                       C.POINTER(C.c_double), C.POINTER(C.c_double)],
        "pyib_diagnostics": [vp, C.POINTER(C.c_double)],
        "pyib_cg_timing": [vp, C.POINTER(C.c_double), C.c_int32],
        "pyib_matvec_plan": [vp, C.POINTER(C.c_int32)],
        "pyib_event": [vp, C.c_int32, C.POINTER(C.c_double)],
        "pyib_bench_matvec": [vp, C.c_int32, C.c_double, C.POINTER(C.c_double)],
        "pyib_bench_matvec_fused": [vp, C.c_int32, C.c_double, C.POINTER(C.c_double)],
        "pyib_spread_noalloc": [vp, vp, vp, vp, C.c_int32, C.c_int64, vp, vp],
        "pyib_ib_interp_dx": [vp, C.POINTER(C.c_double)],
        "pyib_graph_pcg": [vp, C.c_int64, vp, vp, vp, vp, vp, C.c_double, C.c_int32, C.POINTER(C.c_int32),
                           C.POINTER(C.c_double)],
        "pyib_recover_pressure": [vp, C.c_int64, vp, C.c_int64, vp, vp, vp, C.c_double, C.c_int32, vp, vp],
        "pyib_batch_create": [C.POINTER(vp), C.c_int32, C.POINTER(vp)],
        "pyib_batch_destroy": [vp],
        "pyib_batch_last_error": [vp, C.c_char_p, C.c_size_t],
        "pyib_batch_step": [vp, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int32, C.POINTER(vp),
                            C.POINTER(vp), C.POINTER(StepStats)],
        "pyib_batch_timing": [vp, C.POINTER(C.c_double), C.c_int32],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    _lib = lib
    return lib


def version():
    """The library's version string (pyib_version)."""
    buf = C.create_string_buffer(128)
    load().pyib_version(buf, len(buf))
    return buf.value.decode()


def exported_symbols():
    """Names the header declares that the loaded library resolves."""
    lib = load()
    return [n for n in EXPORTS if hasattr(lib, n)]


class Handle:
    """Owner of one ``pyib_ctx``; every call is checked."""

    def __init__(self, layout: Layout):
        self.lib = load()
        self.ptr = C.c_void_p()
        rc = self.lib.pyib_create(C.byref(layout), C.byref(self.ptr))
        if rc != OK:
            msg = self.error() if self.ptr else "pyib_create rejected the layout"
            if self.ptr:
                self.lib.pyib_destroy(self.ptr)
                self.ptr = C.c_void_p()
            raise B200Error(rc, msg)

    def error(self):
        buf = C.create_string_buffer(1024)
        self.lib.pyib_last_error(self.ptr, buf, 1024)
        return buf.value.decode(errors="replace")

    def call(self, name, *args):
        rc = getattr(self.lib, name)(self.ptr, *args)
        if rc != OK:
            raise B200Error(rc, f"{name}: {self.error()}")
        return rc

    def close(self):
        if self.ptr:
            self.lib.pyib_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- convenience -------------------------------------------------------
    def upload(self, name, arr):
        arr = np.ascontiguousarray(arr)
        self.call("pyib_upload", T[name], arr.ctypes.data_as(C.c_void_p), arr.nbytes)

    def set_field(self, name, arr, dtype=np.float64):
        arr = np.ascontiguousarray(arr, dtype=dtype).reshape(-1)
        self.call("pyib_set_field", F[name], arr.ctypes.data_as(C.c_void_p), arr.size)

    def get_field(self, name, count, dtype=np.float64):
        out = np.empty(int(count), dtype=dtype)
        self.call("pyib_get_field", F[name], out.ctypes.data_as(C.c_void_p), out.size)
        return out


class Batch:
    """Owner of one ``pyib_batch`` over the contexts of ``handles`` (which it does not own)."""

    def __init__(self, handles):
        self.lib = load()
        self.handles = list(handles)
        arr = (C.c_void_p * len(self.handles))(*[h.ptr.value for h in self.handles])
        self.ptr = C.c_void_p()
        rc = self.lib.pyib_batch_create(arr, len(self.handles), C.byref(self.ptr))
        if rc != OK:
            raise B200Error(rc, "pyib_batch_create: " + self.handles[0].error())

    def error(self):
        buf = C.create_string_buffer(1024)
        self.lib.pyib_batch_last_error(self.ptr, buf, 1024)
        return buf.value.decode(errors="replace")

    def call(self, name, *args):
        rc = getattr(self.lib, name)(self.ptr, *args)
        if rc != OK:
            raise B200Error(rc, f"{name}: {self.error()}")
        return rc

    def close(self):
        if self.ptr:
            self.lib.pyib_batch_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

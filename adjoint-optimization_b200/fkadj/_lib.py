"""ctypes binding of libfkadj.so (the C ABI declared in include/fkadj.h).

The library is built in-tree by ``make -C adjoint-optimization_b200`` (or
``__graft_entry__.build()``).  There is no fallback: when the shared library
is missing or cannot be loaded every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .params import CFkParams

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# FKADJ_LIB selects another build of the library (a variant compiled with
# different switches); the default is the in-tree build.
LIB_PATH = os.environ.get("FKADJ_LIB") or os.path.join(PKG_DIR, "libfkadj.so")

OK, ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_NUMERIC, ERR_NODEVICE, ERR_BUSY, ERR_TIMEOUT = range(8)
GRAD_REF, GRAD_EXACT = 0, 1
CKPT_AUTO, CKPT_FULL, CKPT_SQRT, CKPT_BINOMIAL = 0, 1, 2, 3

# Every symbol include/fkadj.h declares (checked by the CPU tests).
EXPORTS = (
    "fkadj_default_options", "fkadj_default_params", "fkadj_forward", "fkadj_grad",
    "fkadj_param_string", "fkadj_last_error", "fkadj_release_cached_memory", "fkadj_problem_create",
    "fkadj_problem_destroy",
    "fkadj_problem_device_bytes", "fkadj_problem_objective", "fkadj_problem_grad",
    "fkadj_problem_last_timing", "fkadj_problem_last_launches", "fkadj_problem_set_profiling",
    "fkadj_problem_kernel_time", "fkadj_problem_tiles", "fkadj_problem_last_plan",
    "fkadj_problem_adjoint_kernel",
)


class FkadjError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"libfkadj status {status}: {msg}")
        self.status = status


class COptions(C.Structure):
    _fields_ = [("grad_mode", C.c_int), ("ckpt_policy", C.c_int), ("ckpt_budget_bytes", C.c_int64),
                ("device", C.c_int), ("stream", C.c_void_p), ("tile", C.c_int), ("verbose", C.c_int)]


_lib = None


def load():
    """Loads libfkadj.so; raises when it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C {PKG_DIR}` "
                          "(nvcc, sm_100a).  There is no CPU fallback.")
    L = C.CDLL(LIB_PATH)
    dp, ip, i64p = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int64)
    P, O = C.POINTER(CFkParams), C.POINTER(COptions)
    L.fkadj_default_options.argtypes = [O]
    L.fkadj_default_params.argtypes = [P, C.c_double]
    L.fkadj_forward.argtypes = [P, C.c_double, dp, C.c_int, dp, ip, C.c_int, C.c_int, C.c_int, dp,
                                C.c_int, C.c_int, dp, dp, O]
    L.fkadj_grad.argtypes = [P, C.c_double, dp, C.c_int, dp, ip, C.c_int, C.c_int, C.c_int, dp, dp,
                             C.c_int64, i64p, i64p, dp, C.c_double, dp, dp, dp, dp, dp, O]
    L.fkadj_param_string.argtypes = [P]
    L.fkadj_param_string.restype = C.c_char_p
    L.fkadj_last_error.restype = C.c_char_p
    L.fkadj_release_cached_memory.restype = C.c_int
    L.fkadj_release_cached_memory.argtypes = []
    L.fkadj_problem_create.argtypes = [C.POINTER(C.c_void_p), P, C.c_double, C.c_int, ip, C.c_int,
                                       C.c_int, C.c_int, dp, dp, C.c_int64, i64p, i64p, dp, C.c_double, O]
    L.fkadj_problem_destroy.argtypes = [C.c_void_p]
    L.fkadj_problem_device_bytes.argtypes = [C.c_void_p]
    L.fkadj_problem_device_bytes.restype = C.c_int64
    L.fkadj_problem_objective.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp]
    L.fkadj_problem_grad.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp, dp]
    L.fkadj_problem_last_timing.argtypes = [C.c_void_p, dp]
    L.fkadj_problem_last_launches.argtypes = [C.c_void_p]
    L.fkadj_problem_last_launches.restype = C.c_int64
    L.fkadj_problem_set_profiling.argtypes = [C.c_void_p, C.c_int]
    L.fkadj_problem_kernel_time.argtypes = [C.c_void_p, C.c_int, dp, i64p]
    L.fkadj_problem_tiles.argtypes = [C.c_void_p, ip, ip]
    L.fkadj_problem_last_plan.argtypes = [C.c_void_p, i64p]
    L.fkadj_problem_adjoint_kernel.argtypes = [C.c_void_p, ip]
    for name in ("fkadj_forward", "fkadj_grad", "fkadj_problem_create", "fkadj_problem_objective",
                 "fkadj_problem_grad"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(status: int) -> None:
    if status != OK:
        raise FkadjError(status, load().fkadj_last_error().decode())


def options(grad_mode=GRAD_REF, ckpt_policy=CKPT_AUTO, ckpt_budget_bytes=0, device=-1,
            stream=None, tile=0, verbose=0) -> COptions:
    o = COptions()
    load().fkadj_default_options(C.byref(o))
    o.grad_mode, o.ckpt_policy, o.ckpt_budget_bytes = int(grad_mode), int(ckpt_policy), int(ckpt_budget_bytes)
    o.device, o.stream, o.tile, o.verbose = int(device), stream, int(tile), int(verbose)
    return o

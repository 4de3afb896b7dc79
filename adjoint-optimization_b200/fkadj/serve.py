"""Continuous-batching request server (C ABI fkadj_server_*).

A worker thread inside the library owns the GPU; requests submitted from any
thread are admitted between ticks by device-memory footprint and share the
batched launches with the requests already running.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from ._lib import ERR_TIMEOUT, FkadjError, check, load, options
from .params import CFkParams, FkParams

_bound = False


def _bind():
    global _bound
    L = load()
    if _bound:
        return L
    dp, ip, i64p, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int64), C.c_void_p
    L.fkadj_server_create.argtypes = [C.POINTER(vp), vp, C.c_int64]
    L.fkadj_server_destroy.argtypes = [vp]
    L.fkadj_server_submit.argtypes = [vp, C.POINTER(CFkParams), C.c_double, C.c_int, ip, C.c_int, C.c_int, C.c_int,
                                      dp, dp, C.c_int64, i64p, i64p, dp, C.c_double, dp, dp, C.c_int, i64p]
    L.fkadj_server_poll.argtypes = [vp, C.c_int64]
    L.fkadj_server_wait.argtypes = [vp, C.c_int64, C.c_double]
    L.fkadj_server_result.argtypes = [vp, C.c_int64, dp, dp, dp, dp, C.c_int64, dp]
    L.fkadj_server_stats.argtypes = [vp, i64p]
    for n in ("fkadj_server_create", "fkadj_server_submit", "fkadj_server_wait", "fkadj_server_result"):
        getattr(L, n).restype = C.c_int
    L.fkadj_server_poll.restype = C.c_int
    _bound = True
    return L


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Server:
    def __init__(self, opts=None, hbm_budget_bytes: int = 0):
        self._L = _bind()
        self._h = C.c_void_p()
        o = opts if opts is not None else options()
        check(self._L.fkadj_server_create(C.byref(self._h), C.byref(o), int(hbm_budget_bytes)))
        self._nt = {}

    def close(self):
        if getattr(self, "_h", None):
            self._L.fkadj_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, inst, Et=None, y0=None, want_grad=True) -> int:
        ai = np.ascontiguousarray(inst.active_index, dtype=np.int32)
        S = sp.csc_matrix(inst.S)
        S.sort_indices()
        Jc = np.ascontiguousarray(S.indptr, dtype=np.int64)
        Ir = np.ascontiguousarray(S.indices, dtype=np.int64)
        Sv, gh, g = _f64(S.data), _f64(inst.ghost), _f64(inst.gamma)
        Et = _f64(inst.Et if Et is None else Et)
        y = _f64(inst.y0 if y0 is None else y0)
        cp = CFkParams.of(inst.params or FkParams())
        i64 = C.POINTER(C.c_int64)
        rid = C.c_int64()
        check(self._L.fkadj_server_submit(self._h, C.byref(cp), float(inst.dt), int(inst.nt),
                                          ai.ctypes.data_as(C.POINTER(C.c_int)), inst.nrows, inst.ncols,
                                          int((ai > 0).sum()), _dp(gh), _dp(g), S.shape[1],
                                          Jc.ctypes.data_as(i64), Ir.ctypes.data_as(i64), _dp(Sv),
                                          float(inst.alpha), _dp(Et), _dp(y), 1 if want_grad else 0,
                                          C.byref(rid)))
        self._nt[rid.value] = (int(inst.nt), want_grad)
        return rid.value

    def poll(self, rid: int) -> int:
        return int(self._L.fkadj_server_poll(self._h, int(rid)))

    def wait(self, rid: int, timeout_s: float = 600.0) -> bool:
        st = self._L.fkadj_server_wait(self._h, int(rid), float(timeout_s))
        if st == ERR_TIMEOUT:
            return False
        check(st)
        return True

    def result(self, rid: int):
        nt, want_grad = self._nt.pop(rid)
        g = np.empty(nt + 1) if want_grad else None
        L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
        lat = (C.c_double * 2)()
        check(self._L.fkadj_server_result(self._h, int(rid), C.byref(L0), C.byref(LE), C.byref(Lc),
                                          _dp(g) if g is not None else None, nt + 1 if want_grad else 0, lat))
        r = dict(Lcost=Lc.value, L0=L0.value, LE=LE.value, latency_s=lat[0], queue_s=lat[1])
        if want_grad:
            r["gradE"] = g
        return r

    @property
    def stats(self):
        out = (C.c_int64 * 6)()
        self._L.fkadj_server_stats(self._h, out)
        return dict(completed=out[0], failed=out[1], queued=out[2], running=out[3], peak_running=out[4],
                    reserved_bytes=out[5])

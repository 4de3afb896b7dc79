"""Batched execution of many independent FK problems (C ABI fkadj_batch_*).

Every tick advances every running job by one step; the steps of all jobs run
as at most three launches of the persistent batched kernels, so instances of
different grid sizes and horizons fill the GPU together.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from ._lib import CKPT_AUTO, GRAD_REF, check, load, options
from .params import CFkParams, FkParams

_bound = False


def _bind():
    global _bound
    L = load()
    if _bound:
        return L
    dp, ip, i64p, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int64), C.c_void_p
    L.fkadj_batch_create.argtypes = [C.POINTER(vp), vp]
    L.fkadj_batch_destroy.argtypes = [vp]
    L.fkadj_batch_add_problem.argtypes = [vp, C.POINTER(CFkParams), C.c_double, C.c_int, ip, C.c_int, C.c_int,
                                          C.c_int, dp, dp, C.c_int64, i64p, i64p, dp, C.c_double, C.c_int,
                                          C.c_int, C.c_int64, ip]
    L.fkadj_batch_remove_problem.argtypes = [vp, C.c_int]
    L.fkadj_batch_submit.argtypes = [vp, C.c_int, dp, dp, C.c_int, ip]
    L.fkadj_batch_tick.argtypes = [vp, ip]
    L.fkadj_batch_run.argtypes = [vp]
    L.fkadj_batch_job_done.argtypes = [vp, C.c_int]
    L.fkadj_batch_result.argtypes = [vp, C.c_int, dp, dp, dp, dp, C.c_int64]
    L.fkadj_batch_release.argtypes = [vp, C.c_int]
    L.fkadj_batch_stats.argtypes = [vp, i64p]
    for n in ("fkadj_batch_create", "fkadj_batch_add_problem", "fkadj_batch_remove_problem", "fkadj_batch_submit",
              "fkadj_batch_tick", "fkadj_batch_run", "fkadj_batch_result", "fkadj_batch_release"):
        getattr(L, n).restype = C.c_int
    L.fkadj_batch_job_done.restype = C.c_int
    _bound = True
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


class Batch:
    def __init__(self, opts=None, tile: int = 0, stream=None):
        self._L = _bind()
        self._h = C.c_void_p()
        o = opts if opts is not None else options(tile=tile, stream=stream)
        check(self._L.fkadj_batch_create(C.byref(self._h), C.byref(o)))
        self._nt = {}
        self._keep = {}

    def close(self):
        if getattr(self, "_h", None):
            self._L.fkadj_batch_destroy(self._h)
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

    def add_problem(self, inst, grad_mode=GRAD_REF, ckpt_policy=CKPT_AUTO, ckpt_budget_bytes=0) -> int:
        ai = np.ascontiguousarray(inst.active_index, dtype=np.int32)
        gh = _f64(inst.ghost)
        S = sp.csc_matrix(inst.S)
        S.sort_indices()
        Jc = np.ascontiguousarray(S.indptr, dtype=np.int64)
        Ir = np.ascontiguousarray(S.indices, dtype=np.int64)
        Sv = _f64(S.data)
        g = _f64(inst.gamma)
        cp = CFkParams.of(inst.params or FkParams())
        i64 = C.POINTER(C.c_int64)
        pid = C.c_int()
        check(self._L.fkadj_batch_add_problem(self._h, C.byref(cp), float(inst.dt), int(inst.nt),
                                              ai.ctypes.data_as(C.POINTER(C.c_int)), inst.nrows, inst.ncols,
                                              int((ai > 0).sum()), _dp(gh), _dp(g), S.shape[1],
                                              Jc.ctypes.data_as(i64), Ir.ctypes.data_as(i64), _dp(Sv),
                                              float(inst.alpha), int(grad_mode), int(ckpt_policy),
                                              int(ckpt_budget_bytes), C.byref(pid)))
        self._nt[pid.value] = int(inst.nt)
        return pid.value

    def remove_problem(self, pid: int):
        check(self._L.fkadj_batch_remove_problem(self._h, int(pid)))

    def submit(self, pid: int, Et, y0=None, want_grad=True) -> int:
        Et = _f64(Et)
        y = None if y0 is None else _f64(y0)
        jid = C.c_int()
        check(self._L.fkadj_batch_submit(self._h, int(pid), _dp(Et), None if y is None else _dp(y),
                                         1 if want_grad else 0, C.byref(jid)))
        self._keep[jid.value] = (pid, want_grad)
        return jid.value

    def tick(self) -> int:
        a = C.c_int()
        check(self._L.fkadj_batch_tick(self._h, C.byref(a)))
        return a.value

    def run(self):
        check(self._L.fkadj_batch_run(self._h))

    def done(self, jid: int) -> bool:
        return bool(self._L.fkadj_batch_job_done(self._h, int(jid)))

    def result(self, jid: int, release=True):
        pid, want_grad = self._keep[jid]
        nt = self._nt[pid]
        g = np.empty(nt + 1) if want_grad else None
        L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
        check(self._L.fkadj_batch_result(self._h, int(jid), C.byref(L0), C.byref(LE), C.byref(Lc),
                                         _dp(g) if g is not None else None, nt + 1))
        if release:
            check(self._L.fkadj_batch_release(self._h, int(jid)))
            self._keep.pop(jid, None)
        r = dict(Lcost=Lc.value, L0=L0.value, LE=LE.value)
        if want_grad:
            r["gradE"] = g
        return r

    @property
    def stats(self):
        out = (C.c_int64 * 3)()
        self._L.fkadj_batch_stats(self._h, out)
        return dict(launches=out[0], ticks=out[1], device_bytes=out[2])

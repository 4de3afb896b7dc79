"""Python mirror of the reference's two MEX entry points, backed by libfkadj.

Reference gateways (agarzon27/adjoint-optimization):
  [ys, yf, param_str] = fk_forward_Et_mex(Et, dt, nt, y0, active_index, ncols, nrows,
                                          ghost_lr, nstep)
      src/cuda/fk_forward_Et_param_mex.cpp:33-121
  [gradE, Lcost, L0, LE, param_str] = fk_grad_Et_mex(Et, dt, nt, y0, active_index, ncols,
                                                     nrows, ghost_lr, gamma, S, alpha)
      src/cuda/fk_grad_Et_param_mex.cpp:11-92
Same argument order, meaning and outputs (slot 6 is ``ncols`` and slot 7 is
``nrows``, as in the gateways); the FK parameter set and engine options are
extra keyword arguments.  Errors raise ``FkadjError`` (the gateways raise
mexErrMsgIdAndTxt for argument-count errors and exit() on the rest).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import FkadjError, check, load, options
from .params import CFkParams, FkParams

__all__ = ["fk_forward_Et", "fk_grad_Et", "Problem", "compute_ns", "FkadjError", "options"]


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def compute_ns(nt: int, nstep: int) -> int:
    """Number of forward snapshots (fk_forward_Et_param_mex.cpp:7-25): the final
    step is not stored when nt/nstep is an integer.  nstep <= 0 asks for no
    snapshots (the reference's rule divides by nstep)."""
    if nstep <= 0:
        return 0
    r = nt / nstep
    rn = round(r)
    if abs(r - rn) < 5e-16 * r:
        return int(rn) - 1
    return int(math.floor(r))


def _csc(S, n_num):
    S = sp.csc_matrix(S)
    S.sort_indices()
    if S.shape[1] != n_num:
        raise FkadjError(_lib.ERR_ARG, "Numbers of not-NaN do not agree")
    return (np.ascontiguousarray(S.indptr, dtype=np.int64),
            np.ascontiguousarray(S.indices, dtype=np.int64), _f64(S.data))


def _grid_args(y0, active_index, ncols, nrows, ghost_lr):
    y0 = _f64(y0)
    ai = np.ascontiguousarray(np.asarray(active_index).ravel(), dtype=np.int32)
    n_num = y0.size // 3
    gh = _f64(ghost_lr)
    nrows, ncols = int(nrows), int(ncols)
    if ai.size != nrows * ncols:
        raise FkadjError(_lib.ERR_ARG, "active_index must have nrows*ncols entries")
    return y0, ai, n_num, gh, nrows, ncols


def fk_forward_Et(Et, dt, nt, y0, active_index, ncols, nrows, ghost_lr, nstep, *,
                  params: FkParams | None = None, opts=None):
    """Returns (ys[3n, ns] column-major like the gateway, yf[3n], param_str)."""
    L = load()
    P = params or FkParams()
    Et = _f64(Et)
    nt = int(nt)
    y0, ai, n_num, gh, nrows, ncols = _grid_args(y0, active_index, ncols, nrows, ghost_lr)
    ns = compute_ns(nt, int(nstep))
    n3 = 3 * nrows * ncols
    ys = np.empty((max(ns, 0), n3))
    yf = np.empty(n3)
    cp = CFkParams.of(P)
    o = opts if opts is not None else options()
    check(L.fkadj_forward(C.byref(cp), float(dt), _dp(Et), nt, _dp(y0),
                          ai.ctypes.data_as(C.POINTER(C.c_int)), nrows, ncols, n_num, _dp(gh),
                          int(nstep), ns, _dp(ys) if ns > 0 else None, _dp(yf), C.byref(o)))
    return ys.T, yf, L.fkadj_param_string(C.byref(cp)).decode()


def release_cached_memory():
    """Hands back the device memory and pinned host staging that fk_forward_Et /
    fk_grad_Et keep between calls (fkadj_release_cached_memory)."""
    check(load().fkadj_release_cached_memory())


def fk_grad_Et(Et, dt, nt, y0, active_index, ncols, nrows, ghost_lr, gamma, S, alpha, *,
               params: FkParams | None = None, opts=None, return_yf=False):
    """Returns (gradE[nt+1], Lcost, L0, LE, param_str) (+ yf when return_yf)."""
    L = load()
    P = params or FkParams()
    Et = _f64(Et)
    nt = int(nt)
    y0, ai, n_num, gh, nrows, ncols = _grid_args(y0, active_index, ncols, nrows, ghost_lr)
    Jc, Ir, Sv = _csc(S, n_num)
    gamma = _f64(gamma)
    gradE = np.empty(nt + 1)
    yf = np.empty(3 * nrows * ncols) if return_yf else None
    L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
    cp = CFkParams.of(P)
    o = opts if opts is not None else options()
    i64 = C.POINTER(C.c_int64)
    check(L.fkadj_grad(C.byref(cp), float(dt), _dp(Et), nt, _dp(y0),
                       ai.ctypes.data_as(C.POINTER(C.c_int)), nrows, ncols, n_num, _dp(gh), _dp(gamma),
                       n_num, Jc.ctypes.data_as(i64), Ir.ctypes.data_as(i64), _dp(Sv), float(alpha),
                       C.byref(L0), C.byref(LE), C.byref(Lc), _dp(gradE),
                       _dp(yf) if yf is not None else None, C.byref(o)))
    out = (gradE, Lc.value, L0.value, LE.value, L.fkadj_param_string(C.byref(cp)).decode())
    return out + (yf,) if return_yf else out


class Problem:
    """A resident problem (geometry, objective and buffers stay on the GPU)."""

    def __init__(self, inst=None, *, params=None, dt=None, nt=None, active_index=None, nrows=None,
                 ncols=None, ghost_lr=None, gamma=None, S=None, alpha=0.0, opts=None):
        if inst is not None:
            params, dt, nt = inst.params, inst.dt, inst.nt
            active_index, nrows, ncols = inst.active_index, inst.nrows, inst.ncols
            ghost_lr, gamma, S, alpha = inst.ghost, inst.gamma, inst.S, inst.alpha
        L = load()
        self._L = L
        self.nt, self.nrows, self.ncols = int(nt), int(nrows), int(ncols)
        ai = np.ascontiguousarray(np.asarray(active_index).ravel(), dtype=np.int32)
        self.n_num = int((ai > 0).sum())
        gh = _f64(ghost_lr)
        self._keep = []
        h = C.c_void_p()
        cp = CFkParams.of(params or FkParams())
        o = opts if opts is not None else options()
        i64 = C.POINTER(C.c_int64)
        if S is not None:
            Jc, Ir, Sv = _csc(S, self.n_num)
            g = _f64(gamma)
            self._keep += [Jc, Ir, Sv, g]
            args = (_dp(g), self.n_num, Jc.ctypes.data_as(i64), Ir.ctypes.data_as(i64), _dp(Sv))
        else:
            args = (None, 0, None, None, None)
        check(L.fkadj_problem_create(C.byref(h), C.byref(cp), float(dt), self.nt,
                                     ai.ctypes.data_as(C.POINTER(C.c_int)), self.nrows, self.ncols,
                                     self.n_num, _dp(gh), *args, float(alpha), C.byref(o)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            self._L.fkadj_problem_destroy(self._h)
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

    @property
    def device_bytes(self) -> int:
        return int(self._L.fkadj_problem_device_bytes(self._h))

    @property
    def last_timing(self):
        out = (C.c_double * 3)()
        self._L.fkadj_problem_last_timing(self._h, out)
        return dict(fwd_ms=out[0], bwd_ms=out[1], total_ms=out[2])

    @property
    def last_launches(self) -> int:
        return int(self._L.fkadj_problem_last_launches(self._h))

    @property
    def last_plan(self):
        """Trajectory store of the last gradient: policy (FULL/SQRT/BINOMIAL
        name), stored slots, segment/scratch slots, recomputed forward steps."""
        out = (C.c_int64 * 4)()
        self._L.fkadj_problem_last_plan(self._h, out)
        names = {0: None, _lib.CKPT_FULL: "full", _lib.CKPT_SQRT: "sqrt", _lib.CKPT_BINOMIAL: "binomial"}
        return {"policy": names.get(int(out[0]), int(out[0])), "slots": int(out[1]), "segment_slots": int(out[2]),
                "recompute_steps": int(out[3])}

    @property
    def adjoint_kernel(self):
        """The reference-mode backward step: path ("split", "fused" with the
        J cache, "fused-recompute") and the fused kernel's (TX, TY, threads)."""
        out = (C.c_int * 4)()
        self._L.fkadj_problem_adjoint_kernel(self._h, out)
        return {"path": ("split", "fused", "fused-recompute")[out[0]], "tile": (out[1], out[2], out[3])}

    def set_profiling(self, on: bool = True) -> None:
        self._L.fkadj_problem_set_profiling(self._h, 1 if on else 0)

    @property
    def tiles(self):
        """Tile shapes (tx, ty, threads) in use per kernel kind."""
        out, shp = (C.c_int * 4)(), (C.c_int * 12)()
        self._L.fkadj_problem_tiles(self._h, out, shp)
        names = ("fwd_step", "adj_mid", "adj_step", "adj_exact")
        return {n: (shp[3 * k], shp[3 * k + 1], shp[3 * k + 2]) for k, n in enumerate(names)}

    def kernel_time(self, kernel: int):
        """(average ms per launch, samples) of kernel 0 forward step,
        1 adjoint midpoint, 2 adjoint step, over the last call."""
        ms, n = C.c_double(), C.c_int64()
        self._L.fkadj_problem_kernel_time(self._h, int(kernel), C.byref(ms), C.byref(n))
        return ms.value, n.value

    def objective(self, Et, y0=None, return_yf=False):
        """y0 None re-uses the resident initial state of the previous call."""
        Et = _f64(Et)
        y0 = None if y0 is None else _f64(y0)
        L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
        yf = np.empty(3 * self.nrows * self.ncols) if return_yf else None
        check(self._L.fkadj_problem_objective(self._h, _dp(Et), None if y0 is None else _dp(y0),
                                              C.byref(L0), C.byref(LE),
                                              C.byref(Lc), _dp(yf) if yf is not None else None))
        r = dict(Lcost=Lc.value, L0=L0.value, LE=LE.value)
        if return_yf:
            r["yf"] = yf
        return r

    def grad(self, Et, y0=None, return_yf=False):
        """y0 None re-uses the resident initial state of the previous call."""
        Et = _f64(Et)
        y0 = None if y0 is None else _f64(y0)
        L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
        gradE = np.empty(self.nt + 1)
        yf = np.empty(3 * self.nrows * self.ncols) if return_yf else None
        check(self._L.fkadj_problem_grad(self._h, _dp(Et), None if y0 is None else _dp(y0),
                                         C.byref(L0), C.byref(LE),
                                         C.byref(Lc), _dp(gradE), _dp(yf) if yf is not None else None))
        r = dict(gradE=gradE, Lcost=Lc.value, L0=L0.value, LE=LE.value)
        if return_yf:
            r["yf"] = yf
        return r

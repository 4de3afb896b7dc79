"""ctypes front of the reference's own CUDA routines compiled from source by
oracle/ref_build.sh into oracle/_ref/ (test infrastructure; GPU only).

Same argument layouts as the reference's comp routines: compact y_ini
[u;v;w], 1-based active_index, gh_num = ghost_lr (the routine scales it by
Du*2/h), S in CSC; grid sides must be multiples of 16 (cu-G:1666-1673).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")


def available(dx_tag: str = "dx0p025") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libfkref_grad_{dx_tag}.so"))


def _load(kind, dx_tag):
    L = C.CDLL(os.path.join(REF_DIR, f"libfkref_{kind}_{dx_tag}.so"))
    dp, ip, i64 = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int64)
    if kind == "fwd":
        L.fkref_forward.argtypes = [C.c_double, dp, C.c_int, dp, ip, C.c_int, C.c_int, C.c_int, dp, C.c_int,
                                    C.c_int, dp, dp]
        L.fkref_forward.restype = C.c_int
    else:
        L.fkref_grad.argtypes = [C.c_double, dp, C.c_int, dp, ip, C.c_int, C.c_int, C.c_int, dp, dp, C.c_int64,
                                 i64, i64, dp, C.c_double, dp, dp, dp, dp]
        L.fkref_grad.restype = C.c_int
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())


def forward(dt, Et, nt, y0, active_index, nrows, ncols, ghost, nstep, ns, dx_tag="dx0p025"):
    L = _load("fwd", dx_tag)
    Et, y0, gh = _f(Et), _f(y0), _f(ghost)
    ai = np.ascontiguousarray(active_index, dtype=np.int32)
    n3 = 3 * nrows * ncols
    ys = np.zeros((max(ns, 1), n3))
    yf = np.zeros(n3)
    rc = L.fkref_forward(float(dt), _dp(Et), int(nt), _dp(y0), ai.ctypes.data_as(C.POINTER(C.c_int)), nrows,
                         ncols, y0.size // 3, _dp(gh), int(nstep), int(ns), _dp(ys), _dp(yf))
    assert rc == 0
    return ys[:ns], yf


def grad(dt, Et, nt, y0, active_index, nrows, ncols, ghost, gamma, S, alpha, dx_tag="dx0p025"):
    import scipy.sparse as sp
    L = _load("grad", dx_tag)
    Et, y0, gh, gm = _f(Et), _f(y0), _f(ghost), _f(gamma)
    ai = np.ascontiguousarray(active_index, dtype=np.int32)
    S = sp.csc_matrix(S)
    S.sort_indices()
    Jc = np.ascontiguousarray(S.indptr, dtype=np.int64)
    Ir = np.ascontiguousarray(S.indices, dtype=np.int64)
    Sv = _f(S.data)
    gradE = np.zeros(int(nt) + 1)
    L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
    i64 = C.POINTER(C.c_int64)
    rc = L.fkref_grad(float(dt), _dp(Et), int(nt), _dp(y0), ai.ctypes.data_as(C.POINTER(C.c_int)), nrows, ncols,
                      y0.size // 3, _dp(gh), _dp(gm), S.shape[1], Jc.ctypes.data_as(i64), Ir.ctypes.data_as(i64),
                      _dp(Sv), float(alpha), C.byref(L0), C.byref(LE), C.byref(Lc), _dp(gradE))
    assert rc == 0
    return dict(gradE=gradE, L0=L0.value, LE=LE.value, Lcost=Lc.value)

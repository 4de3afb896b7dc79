"""ctypes front of the CPU oracle (oracle/fk_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker that tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg compare the CUDA library against.  The
product path never imports this module.

Arrays follow the reference layout: a state is three dense grids (u, v, w)
stacked into one float64 vector of length 3*nrows*ncols, row-major, NaN at
holes; ``gh`` is the dense virtual-electrode vector ``(Du*2/h)*ghost_lr`` with
NaN at holes (src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1581-1595).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libfkoracle.so")

PARAM_FIELDS = ("u_c", "u_v", "tau_d", "tau_v1_minus", "tau_v2_minus", "tau_v_plus",
                "tau_0", "tau_r", "tau_si", "u_csi", "k_fk", "tau_w_minus", "tau_w_plus",
                "Du", "Dv", "Dw", "ksm", "h")


class _Params(C.Structure):
    _fields_ = [(f, C.c_double) for f in PARAM_FIELDS]


class _Objective(C.Structure):
    _fields_ = [("n_num", C.c_int), ("Jc", C.POINTER(C.c_int64)), ("Ir", C.POINTER(C.c_int64)),
                ("Sv", C.POINTER(C.c_double)), ("gamma", C.c_double * 3)]


_lib = None


def build() -> str:
    """Compile the oracle (gcc, OpenMP) if the shared library is missing or stale."""
    src = os.path.join(HERE, "fk_oracle.c")
    if (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        P = C.POINTER(_Params)
        O = C.POINTER(_Objective)
        L.ora_rhs.argtypes = [P, C.c_int, C.c_int, dp, dp, C.c_double, dp]
        L.ora_adj_rhs.argtypes = [P, C.c_int, C.c_int, dp, dp, dp]
        L.ora_spline_ypp.argtypes = [C.c_int, C.c_double, dp, dp]
        L.ora_spline_ypp.restype = C.c_int
        L.ora_spline_val.argtypes = [C.c_int, C.c_double, dp, dp, C.c_double]
        L.ora_spline_val.restype = C.c_double
        L.ora_forward.argtypes = [P, C.c_double, dp, C.c_int, C.c_int, C.c_int, dp, dp,
                                  C.c_int, C.c_int, dp, dp]
        L.ora_forward.restype = C.c_int
        L.ora_objective_eval.argtypes = [O, ip, C.c_int, dp, dp, dp]
        L.ora_objective_eval.restype = C.c_int
        for fn in (L.ora_grad_ref, L.ora_grad_exact):
            fn.argtypes = [P, C.c_double, dp, C.c_int, C.c_int, C.c_int, dp, dp, ip, O, C.c_double,
                           dp, dp, dp, dp, dp]
            fn.restype = C.c_int
        L.ora_set_threads.argtypes = [C.c_int]
        L.ora_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _params(p) -> _Params:
    get = (lambda k: p[k]) if isinstance(p, dict) else (lambda k: getattr(p, k))
    return _Params(*[float(get(f)) for f in PARAM_FIELDS])


class Objective:
    """L0 = sum_v gamma_v y_v^T S y_v with S given as scipy CSC (n_num x n_num)."""

    def __init__(self, S, gamma):
        S = S.tocsc()
        S.sort_indices()
        self.n_num = S.shape[1]
        self.Jc = np.ascontiguousarray(S.indptr, dtype=np.int64)
        self.Ir = np.ascontiguousarray(S.indices, dtype=np.int64)
        self.Sv = _f64(S.data)
        self.gamma = [float(g) for g in gamma]

    def c(self) -> _Objective:
        return _Objective(self.n_num, self.Jc.ctypes.data_as(C.POINTER(C.c_int64)),
                          self.Ir.ctypes.data_as(C.POINTER(C.c_int64)), _dp(self.Sv),
                          (C.c_double * 3)(*self.gamma))


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def threads() -> int:
    return int(lib().ora_get_threads())


def rhs(p, nrows, ncols, y, gh, E):
    y, gh = _f64(y), _f64(gh)
    f = np.empty_like(y)
    lib().ora_rhs(C.byref(_params(p)), nrows, ncols, _dp(y), _dp(gh), float(E), _dp(f))
    return f


def adj_rhs(p, nrows, ncols, z, y):
    z, y = _f64(z), _f64(y)
    fz = np.empty_like(z)
    lib().ora_adj_rhs(C.byref(_params(p)), nrows, ncols, _dp(z), _dp(y), _dp(fz))
    return fz


def spline_ypp(Et, dt):
    Et = _f64(Et)
    ypp = np.empty_like(Et)
    if lib().ora_spline_ypp(len(Et), float(dt), _dp(Et), _dp(ypp)):
        raise ValueError("spline needs at least 4 samples")
    return ypp


def spline_val(Et, ypp, dt, t):
    Et, ypp = _f64(Et), _f64(ypp)
    return float(lib().ora_spline_val(len(Et), float(dt), _dp(Et), _dp(ypp), float(t)))


def forward(p, dt, Et, nt, nrows, ncols, y0, gh, nstep=0, ns=0):
    """Returns (ys[ns, 3n], yf[3n]) on the NaN grid (cu-F:646-849)."""
    Et, y0, gh = _f64(Et), _f64(y0), _f64(gh)
    n3 = 3 * nrows * ncols
    ys = np.empty((max(ns, 0), n3))
    yf = np.empty(n3)
    rc = lib().ora_forward(C.byref(_params(p)), float(dt), _dp(Et), int(nt), nrows, ncols,
                           _dp(y0), _dp(gh), int(nstep), int(ns), _dp(ys), _dp(yf))
    if rc:
        raise RuntimeError(f"ora_forward failed: {rc}")
    return ys, yf


def objective_eval(obj: Objective, active_index, yT):
    ai = np.ascontiguousarray(active_index, dtype=np.int32)
    yT = _f64(yT)
    zT = np.empty_like(yT)
    L0 = C.c_double()
    o = obj.c()
    rc = lib().ora_objective_eval(C.byref(o), ai.ctypes.data_as(C.POINTER(C.c_int)), len(ai),
                                  _dp(yT), C.byref(L0), _dp(zT))
    if rc:
        raise RuntimeError(f"ora_objective_eval failed: {rc}")
    return L0.value, zT


def grad(p, dt, Et, nt, nrows, ncols, y0, gh, active_index, obj: Objective, alpha, mode="ref"):
    """Returns dict(gradE, L0, LE, Lcost, yf).  mode 'ref' follows the reference
    continuous adjoint (cu-G:1569-1938); 'exact' is the discrete adjoint with
    gradE = (1/dt) dLcost/dEt."""
    Et, y0, gh = _f64(Et), _f64(y0), _f64(gh)
    ai = np.ascontiguousarray(active_index, dtype=np.int32)
    n3 = 3 * nrows * ncols
    gradE = np.empty(nt + 1)
    yf = np.empty(n3)
    L0, LE, Lc = C.c_double(), C.c_double(), C.c_double()
    o = obj.c()
    fn = lib().ora_grad_ref if mode == "ref" else lib().ora_grad_exact
    rc = fn(C.byref(_params(p)), float(dt), _dp(Et), int(nt), nrows, ncols, _dp(y0), _dp(gh),
            ai.ctypes.data_as(C.POINTER(C.c_int)), C.byref(o), float(alpha), _dp(gradE),
            C.byref(L0), C.byref(LE), C.byref(Lc), _dp(yf))
    if rc:
        raise RuntimeError(f"oracle grad ({mode}) failed: {rc}")
    return dict(gradE=gradE, L0=L0.value, LE=LE.value, Lcost=Lc.value, yf=yf)

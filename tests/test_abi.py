"""CPU checks of the C-ABI boundary: the library loads and exports every
function include/*.h declares; host-side argument checks reject bad input
before any device work."""
import ctypes as C
import glob
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(fkadj_\w+)\s*\(", txt))
    return names


def test_library_exports_every_declared_function():
    from fkadj import _lib
    L = _lib.load()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (fkadj_\w+)", out))
    declared = _declared()
    assert declared, "no declarations found"
    missing = declared - exported
    assert not missing, missing
    for name in declared:
        assert hasattr(L, name)
    assert set(_lib.EXPORTS) <= declared


def test_default_params_and_param_string():
    from fkadj import _lib
    from fkadj.params import CFkParams, FkParams
    L = _lib.load()
    p = CFkParams()
    L.fkadj_default_params(C.byref(p), 0.025)
    ref = FkParams().with_h(0.025)
    for f in ref.__dataclass_fields__:
        assert getattr(p, f) == getattr(ref, f)
    s = L.fkadj_param_string(C.byref(p)).decode()
    assert "tau_w_plus = 399.99999999999994" in s and "h = 0.025" in s


def test_argument_errors_return_status_without_device_work():
    from fkadj import _lib
    from fkadj.params import CFkParams, FkParams
    L = _lib.load()
    p = CFkParams.of(FkParams())
    Et = np.zeros(11)
    ai = np.arange(1, 17, dtype=np.int32)
    y0 = np.zeros(48)
    gh = np.zeros(16)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    o = _lib.options()
    # nt < 3
    st = L.fkadj_forward(C.byref(p), 0.1, dp(Et), 2, dp(y0), ai.ctypes.data_as(C.POINTER(C.c_int)), 4, 4,
                         16, dp(gh), 0, 0, None, dp(np.empty(48)), C.byref(o))
    assert st == _lib.ERR_ARG
    assert b"nt" in L.fkadj_last_error()
    # n_num mismatch
    st = L.fkadj_forward(C.byref(p), 0.1, dp(Et), 10, dp(y0), ai.ctypes.data_as(C.POINTER(C.c_int)), 4, 4,
                         15, dp(gh), 0, 0, None, dp(np.empty(48)), C.byref(o))
    assert st == _lib.ERR_ARG
    # dt <= 0
    st = L.fkadj_forward(C.byref(p), 0.0, dp(Et), 10, dp(y0), ai.ctypes.data_as(C.POINTER(C.c_int)), 4, 4,
                         16, dp(gh), 0, 0, None, dp(np.empty(48)), C.byref(o))
    assert st == _lib.ERR_ARG


def test_compute_ns_matches_gateway_rule():
    from fkadj.api import compute_ns
    assert compute_ns(2000, 100) == 19
    assert compute_ns(2000, 300) == 6
    assert compute_ns(10, 10) == 0


def test_mex_compat_shim_compiles_and_links(tmp_path):
    """The drop-in shim (reference names and signatures) compiles against a
    MEX-API stand-in and links against libfkadj; the call with a bad grid
    returns the status instead of exiting (no device work)."""
    from fkadj import _lib
    src = tmp_path / "gw.cpp"
    src.write_text(r'''
#include "matrix.h"
#include "fkadj_mex_compat.h"
#include <cstdio>
int main() {
    double Et[4] = {0, 0, 0, 0}, y0[3] = {0, 0, 0}, gh[1] = {0}, ys[3], yf[3];
    int ai[1] = {1};
    char *ps = nullptr;
    int rc = fk_forward_Et_comp(0.1, Et, 3, y0, ai, 1, 1, 1, gh, 1, 0, ys, yf, &ps);
    std::printf("rc=%d str=%d\n", rc, ps != nullptr && std::strstr(ps, "h = 0.035") != nullptr);
    return rc == 1 ? 0 : 1;
}
''')
    exe = tmp_path / "gw"
    inc = [f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(ROOT, 'oracle', 'ref_shim')}"]
    subprocess.run(["g++", "-std=c++17", *inc, str(src), "-o", str(exe), _lib.LIB_PATH,
                    f"-Wl,-rpath,{os.path.dirname(_lib.LIB_PATH)}"], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "rc=1 str=1" in out.stdout

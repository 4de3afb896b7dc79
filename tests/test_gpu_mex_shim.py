"""The reference-name shim (include/fkadj_mex_compat.h) on real data: a
gateway-shaped caller (tests/mex_gateway_caller.cpp) built against the
MEX-API stand-in passes the reference's shipped 256^2 x 3000-step problem
(h = 0.035, the shim's default spacing) to fk_grad_Et_comp with the objective
matrix as a CSC mxArray of mwIndex indices, the way the unmodified gateway
does (src/cuda/fk_grad_Et_param_mex.cpp:26-38, 69-79).  The gradient must
match the reference's own golden gradient to 1e-9 relative, as the direct
C-ABI call does (test_gpu_parity.py::test_golden_reference_gradient)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from fkadj import _lib, geometry as G

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _build(out):
    L = _lib.LIB_PATH
    inc = [f"-I{os.path.join(ROOT, 'include')}", f"-I{os.path.join(ROOT, 'oracle', 'ref_shim')}"]
    gxx = shutil.which("g++") or pytest.skip("g++ not found")
    subprocess.run([gxx, "-std=c++17", "-O2", *inc, os.path.join(HERE, "mex_gateway_caller.cpp"), "-o", out, L,
                    f"-Wl,-rpath,{os.path.dirname(L)}"], check=True, capture_output=True, timeout=300)
    return out


@pytest.mark.parametrize("k", [0, 3])
def test_shim_gradient_matches_the_reference_golden_file(golden, tmp_path, k):
    exe = _build(str(tmp_path / "gw"))
    ai = golden["active_index"].astype(np.int32)
    n = int(golden["nrows"])
    mask = (ai > 0).reshape(n, n)
    S = G.objective_matrix(mask).tocsc()
    S.sort_indices()
    n_num = int(mask.sum())
    nt = int(golden["nt"])
    files = {
        "scalars.f64": np.array([golden["dt"], nt, n, n, n_num, golden["alpha"], S.nnz], np.float64),
        "Et.f64": np.ascontiguousarray(golden["Et"][k], np.float64),
        "y0.f64": np.ascontiguousarray(golden["y0"], np.float64),
        "active_index.i32": ai,
        "ghost.f64": golden["ghost_lr"].astype(np.float64),
        "gamma.f64": np.ascontiguousarray(golden["gamma"], np.float64),
        "S_jc.u64": S.indptr.astype(np.uint64),
        "S_ir.u64": S.indices.astype(np.uint64),
        "S_pr.f64": S.data.astype(np.float64),
    }
    for name, arr in files.items():
        arr.tofile(str(tmp_path / name))
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (r.returncode, r.stdout, r.stderr)
    out = np.fromfile(str(tmp_path / "out.f64"), np.float64)
    status, Lcost, L0, LE, gradE = out[0], out[1], out[2], out[3], out[4:]
    assert status == 0 and gradE.size == nt + 1
    ge = golden["gradE"][k]
    assert abs(Lcost - golden["Lcost"][k]) <= 1e-10 * abs(golden["Lcost"][k])
    assert np.linalg.norm(gradE - ge) <= 1e-9 * np.linalg.norm(ge)
    assert "h = 0.035" in (tmp_path / "param.txt").read_text()

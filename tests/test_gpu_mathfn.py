"""The kernels' own math functions on the GPU.

Reciprocal (fk_device.cuh `own_rcp`: the hardware estimate refined without a
division, by either refinement FKADJ_RCP_CUBIC selects) against the correctly rounded quotient: within one ulp over the
denominators the model produces (1 + e^{...} from 1 to 1e300, the tau_v-
range), exact at powers of two, 0 at +inf and beyond 2^1022.

Exponential (`fk_exp`, each form FKADJ_OWN_EXP selects) against CUDA's exp:
within 3 ulp (each within about one ulp of e^x) over the arguments the smoothed steps see and far beyond them,
NaN for NaN, and saturated (never inf, never 0) at the ends of the range.

The probe source is compiled here for sm_100a; the build check runs without a
GPU."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE = os.path.join(HERE, "mathfn_probe.cu")


def _nvcc():
    for p in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if p and os.path.exists(p):
            return p
    pytest.skip("nvcc not found")


def _build(out, defs=()):
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
           *defs, "-shared", "-o", out, PROBE]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    return out


def test_probe_builds_for_sm100a(tmp_path):
    assert os.path.getsize(_build(str(tmp_path / "probe.so"))) > 0


def _inputs():
    rng = np.random.default_rng(11)
    logistic = 1.0 + np.exp(rng.uniform(-60.0, 690.0, 400_000))   # 1 + e^{-2x}, e up to ~1e300
    near_one = 1.0 + np.exp(rng.uniform(-40.0, 2.0, 200_000))
    tau = rng.uniform(10.0, 2000.0, 200_000)                       # tau_v- = q tau_v1- + (1-q) tau_v2-
    pow2 = np.ldexp(1.0, np.arange(0, 1022))
    return np.concatenate([logistic, near_one, tau, pow2, pow2 * (1 + 2.0 ** -52), [1.0, 3.0, 7.0]])


@pytest.mark.gpu
@pytest.mark.parametrize("cubic", [0, 1])
def test_own_reciprocal_within_one_ulp(tmp_path, cubic):
    lib = ctypes.CDLL(_build(str(tmp_path / f"probe_rcp{cubic}.so"), (f"-DFKADJ_RCP_CUBIC={cubic}",)))
    lib.probe_rcp.restype = ctypes.c_int
    lib.probe_rcp.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_longlong]

    def run(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        own, ieee = np.empty_like(x), np.empty_like(x)
        assert lib.probe_rcp(x.ctypes.data, own.ctypes.data, ieee.ctypes.data, x.size) == 0
        return own, ieee

    x = _inputs()
    own, ieee = run(x)
    np.testing.assert_array_equal(ieee, 1.0 / x)          # the device quotient is the IEEE one
    ulps = np.abs(own.view(np.int64) - ieee.view(np.int64))
    assert ulps.max() <= 1, f"max {ulps.max()} ulp at x={x[ulps.argmax()]!r}"
    p2 = np.ldexp(1.0, np.arange(0, 1022))
    own_p2, _ = run(p2)
    np.testing.assert_array_equal(own_p2, 1.0 / p2)       # exact at powers of two
    big, _ = run(np.array([np.ldexp(1.5, 1022), 1.7e308, np.inf]))  # quotients below 2^-1022 flush to 0
    assert np.all(big == 0.0)                             # the logistic then takes s = 0, 1 - s = 1
    nan, _ = run(np.array([np.nan]))
    assert np.isnan(nan[0])


@pytest.mark.gpu
@pytest.mark.parametrize("form", [1, 2])
def test_own_exponential_within_three_ulp_of_cuda_exp(tmp_path, form):
    lib = ctypes.CDLL(_build(str(tmp_path / f"probe_exp{form}.so"), (f"-DFKADJ_OWN_EXP={form}",)))
    lib.probe_exp.restype = ctypes.c_int
    lib.probe_exp.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_longlong]

    def run(x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        own, ref = np.empty_like(x), np.empty_like(x)
        assert lib.probe_exp(x.ctypes.data, own.ctypes.data, ref.ctypes.data, x.size) == 0
        return own, ref

    rng = np.random.default_rng(12)
    # -2 ksm (u - u_c) and -2 k_fk (u - u_csi) for u in [-1, 2], then the whole normal range
    x = np.concatenate([rng.uniform(-400.0, 250.0, 600_000), rng.uniform(-40.0, 40.0, 200_000),
                        rng.uniform(-707.0, 692.0, 200_000), rng.uniform(-1e-3, 1e-3, 50_000),
                        np.arange(-2040, 1996) * (np.log(2.0) / 4.0),  # about the reduction's breakpoints
                        [0.0, -0.0, 1.0, -1.0, 1e-300]])
    own, ref = run(x)
    ulps = np.abs(own.view(np.int64) - ref.view(np.int64))
    assert ulps.max() <= 3, f"max {ulps.max()} ulp at x={x[ulps.argmax()]!r}"
    edge, _ = run(np.array([693.0, 710.0, 1e4, 1e12, -710.0, -1e4, -1e12]))
    assert np.all(np.isfinite(edge)) and np.all(edge > 0) and np.all(edge < 2.0 ** 1000)
    nan, _ = run(np.array([np.nan]))
    assert np.isnan(nan[0])

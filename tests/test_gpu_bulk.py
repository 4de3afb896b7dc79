"""The bulk-copy helpers the step kernels load their tile windows with
(fk_bulk.cuh): a window of three planes arrives in shared memory exactly as
the vector loads would place it, for full and cut tiles at even column
offsets; and the bounded wait expires on time when more bytes are posted than
any copy delivers (the failure it guards against), reports it, and leaves the
context usable for the next call.  The probe source is compiled here for
sm_100a; the build check runs without a GPU."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
PROBE = os.path.join(HERE, "bulk_probe.cu")
WIDTH = 72


def _nvcc():
    for p in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if p and os.path.exists(p):
            return p
    pytest.skip("nvcc not found")


def _build(out):
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
           "-shared", "-o", out, PROBE]
    subprocess.run(cmd, check=True, capture_output=True, timeout=600)
    return out


def test_bulk_probe_builds_for_sm100a(tmp_path):
    assert os.path.getsize(_build(str(tmp_path / "bulk.so"))) > 0


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    lib = ctypes.CDLL(_build(str(tmp_path_factory.mktemp("bulk") / "bulk.so")))
    lib.probe_bulk.restype = ctypes.c_int
    lib.probe_bulk.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.c_uint, ctypes.c_ulonglong, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                               ctypes.POINTER(ctypes.c_float), ctypes.c_int, ctypes.POINTER(ctypes.c_uint)]

    def run(src, rows_alloc, ld, rows, col0, extra=0, limit_ns=1_000_000_000, cta_mode=False, with_fault=False):
        out = np.full(3 * rows * WIDTH, np.nan)
        status, ms, fault = ctypes.c_int(-1), ctypes.c_float(0), ctypes.c_uint(7)
        rc = lib.probe_bulk(src.ctypes.data, rows_alloc, ld, rows, col0, extra, limit_ns, out.ctypes.data,
                            ctypes.byref(status), ctypes.byref(ms), 1 if cta_mode else 0, ctypes.byref(fault))
        assert rc == 0, f"CUDA error {rc}"
        r = (out.reshape(3, rows, WIDTH), status.value, ms.value)
        return r + (fault.value,) if with_fault else r

    return run


def _planes(rows_alloc, ld, seed):
    return np.random.default_rng(seed).standard_normal(3 * rows_alloc * ld)


@pytest.mark.gpu
@pytest.mark.parametrize("rows,col0", [(40, 0), (17, 6), (1, 8)])
def test_bulk_window_matches_source(probe, rows, col0):
    rows_alloc, ld = 40, 80
    src = _planes(rows_alloc, ld, rows)
    out, status, _ = probe(src, rows_alloc, ld, rows, col0)
    assert status == 1
    want = src.reshape(3, rows_alloc, ld)[:, :rows, col0:col0 + WIDTH]
    np.testing.assert_array_equal(out, want)


@pytest.mark.gpu
def test_bounded_wait_expires_reports_and_leaves_the_context_usable(probe):
    rows_alloc, ld = 40, 80
    src = _planes(rows_alloc, ld, 5)
    limit_ns = 50_000_000
    _, status, ms = probe(src, rows_alloc, ld, 24, 0, extra=16, limit_ns=limit_ns)
    assert status == 0                          # the 16 posted bytes never arrive: the wait gave up
    assert 40.0 <= ms < 5000.0, ms              # after its limit, not forever
    out, status, _ = probe(src, rows_alloc, ld, 24, 0)  # the next call on the same context works
    assert status == 1
    np.testing.assert_array_equal(out, src.reshape(3, rows_alloc, ld)[:, :24, :WIDTH])


@pytest.mark.gpu
def test_expired_wait_in_a_step_kernel_skips_the_tile_and_sets_the_fault_word(probe):
    """The step kernels wait with bulk_wait_cta: when the wait expires the CTA
    sets its problem's fault word, waits once more (bounded) and returns
    before computing or storing anything; the next call is correct."""
    rows_alloc, ld = 40, 80
    src = _planes(rows_alloc, ld, 6)
    limit_ns = 50_000_000
    out, status, ms, fault = probe(src, rows_alloc, ld, 24, 0, extra=16, limit_ns=limit_ns, cta_mode=True,
                                   with_fault=True)
    assert fault == 1                           # the fault word passed to the kernel is set
    assert status == -1                         # the CTA returned before it wrote its outcome ...
    assert np.isnan(out).all()                  # ... or any of the window
    assert 80.0 <= ms < 10000.0, ms             # two bounded waits, then out
    out, status, ms, fault = probe(src, rows_alloc, ld, 24, 0, cta_mode=True, with_fault=True)
    assert fault == 0 and status == 1
    np.testing.assert_array_equal(out, src.reshape(3, rows_alloc, ld)[:, :24, :WIDTH])

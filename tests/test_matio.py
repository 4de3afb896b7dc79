"""MAT-file reader/writer of libfkadj (include/fkadj_matio.h) and the
configuration/input handling of the native drivers, on the CPU.

The reader is checked against scipy.io on files scipy writes (every numeric
class, compressed and not, logical, char, sparse) and on the reference's own
data files when the reference tree is present; the writer is checked by
reading its files back with scipy.  The drivers are checked up to the point
where they need a GPU: configuration errors and input-class errors come out
as the reference's messages with exit status 1."""
import os
import subprocess

import numpy as np
import pytest
import scipy.io as sio
import scipy.sparse as sp

from fkadj import matio
from fkadj._lib import FkadjError

from conftest import reference_dir

REF_DATA = os.path.join(reference_dir() or "", "src", "cuda", "data")
BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "adjoint-optimization_b200",
                   "bin")


def _same(a, b):
    if sp.issparse(a):
        return sp.issparse(b) and a.shape == b.shape and (a != b).nnz == 0
    if isinstance(a, str):
        return a == (str(b[0]) if np.size(b) else "")
    b = np.asarray(b)
    return a.shape == b.shape and np.array_equal(a.astype(np.float64), b.astype(np.float64), equal_nan=True)


@pytest.mark.parametrize("compress", [True, False])
def test_reader_matches_scipy_on_every_class(tmp_path, compress):
    rng = np.random.default_rng(3)
    v = {
        "d": rng.standard_normal((9, 4)),
        "nanvec": np.array([[1.0, np.nan, -np.inf, 2.5]]),
        "i8": np.array([[-5, 7]], dtype=np.int8), "u8": np.array([[250, 3]], dtype=np.uint8),
        "i16": np.arange(-6, 6, dtype=np.int16).reshape(3, 4), "u16": np.array([[65000]], dtype=np.uint16),
        "i32": np.array([[-(2 ** 31), 2 ** 31 - 1]], dtype=np.int32), "u32": np.array([[7]], dtype=np.uint32),
        "i64": np.array([[-3, 2 ** 40]], dtype=np.int64), "f32": np.array([[1.5, -2.25]], dtype=np.float32),
        "b": np.array([[True, False, True]]), "txt": "spirals.mat",
        "S": sp.random(30, 20, density=0.2, random_state=4, format="csc"),
        "E": np.zeros((0, 0)), "scal": 2.0,
        "intlike": np.array([[1.0, -1.0, 0.0, 2.0]]),   # scipy may store these as small ints
    }
    p = str(tmp_path / "x.mat")
    sio.savemat(p, v, do_compression=compress)
    ref = sio.loadmat(p)
    got = matio.loadmat(p, integer_as_int32=False)
    for k in v:
        assert k in got, k
        assert _same(got[k], ref[k]), k
    got32 = matio.loadmat(p)
    assert got32["i32"].dtype == np.int32 and np.array_equal(got32["i32"], v["i32"])


def test_int32_read_rejects_out_of_range_values(tmp_path):
    p = str(tmp_path / "x.mat")
    sio.savemat(p, {"big": np.array([[2.0 ** 40]]), "frac": np.array([[0.5]])})
    L = matio._lib()
    import ctypes as C
    h = C.c_void_p()
    assert L.fkadj_mat_open(p.encode(), C.byref(h)) == 0
    out = np.zeros(1, np.int32)
    for name in (b"big", b"frac"):
        assert L.fkadj_mat_read_int32(h, name, out.ctypes.data_as(C.POINTER(C.c_int32)), 1) != 0
    assert L.fkadj_mat_read_int32(h, b"missing", out.ctypes.data_as(C.POINTER(C.c_int32)), 1) != 0
    L.fkadj_mat_close(h)


@pytest.mark.parametrize("compress", [True, False])
def test_writer_round_trips_through_scipy(tmp_path, compress):
    rng = np.random.default_rng(5)
    S = sp.random(40, 25, density=0.15, random_state=6, format="csc")
    v = {"Et": rng.standard_normal(301), "gamma": np.array([[1.0, 0.2, 0.2]]),
         "active_index": np.arange(-2, 10, dtype=np.int32), "ghost_lr": np.array([0, 1, -1, 2], dtype=np.int16),
         "m": np.array([[0, 255]], dtype=np.uint8), "param_str": "u_c = 0.13\nksm = 100", "empty": "",
         "S": S, "S0": sp.csc_matrix((3, 4)), "x": 0.1, "ys": rng.standard_normal((12, 3))}
    p = str(tmp_path / "w.mat")
    matio.savemat(p, v, compress=compress)
    ref = sio.loadmat(p)
    for k, x in v.items():
        if isinstance(x, np.ndarray) and x.ndim == 1:
            x = x.reshape(-1, 1)
        elif isinstance(x, float):
            x = np.array([[x]])
        if isinstance(x, np.ndarray):
            assert ref[k].dtype == x.dtype and np.array_equal(ref[k], x), k
        else:
            assert _same(x, ref[k]), k
    back = matio.loadmat(p)
    assert sorted(back) == sorted(v)
    assert back["param_str"] == v["param_str"]


def test_reader_errors_are_statuses_not_crashes(tmp_path):
    with pytest.raises(FkadjError):
        matio.loadmat(str(tmp_path / "missing.mat"))
    bad = tmp_path / "bad.mat"
    bad.write_bytes(b"not a mat file" * 20)
    with pytest.raises(FkadjError):
        matio.loadmat(str(bad))
    good = tmp_path / "good.mat"
    sio.savemat(str(good), {"a": np.arange(1000.0)}, do_compression=True)
    raw = good.read_bytes()
    trunc = tmp_path / "trunc.mat"
    trunc.write_bytes(raw[: len(raw) - 40])
    with pytest.raises(FkadjError):
        matio.loadmat(str(trunc))


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data not present")
def test_reader_matches_scipy_on_the_reference_data_files():
    names = sorted(f for f in os.listdir(REF_DATA) if f.endswith(".mat"))
    assert len(names) >= 8
    for f in names:
        p = os.path.join(REF_DATA, f)
        ref = sio.loadmat(p)
        got = matio.loadmat(p, integer_as_int32=False)
        skipped = set(ref) - set(got) - {"__header__", "__version__", "__globals__"}
        assert skipped <= {"mex_function"}, (f, skipped)   # a MATLAB function handle
        for k, x in got.items():
            assert _same(x, ref[k]), (f, k)


def _run(binary, cwd, arg=None):
    cmd = [os.path.join(BIN, binary)] + ([arg] if arg else [])
    return subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=120)


def test_drivers_report_missing_configuration_variables(tmp_path):
    (tmp_path / "infile_grad").write_text("% -*-octave-*-\nalpha=0.5; % weight\nds=1e-3;\nbogus line\n")
    r = _run("fkadj_simple_grad_desc", tmp_path)
    assert r.returncode == 1
    assert "The following variables were not found: ns final_time gamma nmod" in r.stderr
    assert "Expression 'bogus line' not evaluated" in r.stdout
    (tmp_path / "fwd.cfg").write_text("Et_file = '';\n")
    r = _run("fkadj_save_fk_forward_Et", tmp_path, "fwd.cfg")
    assert r.returncode == 1 and "final_time nstep icondfile" in r.stderr


def test_forward_driver_requires_int32_active_index(tmp_path):
    n = 8
    ai = np.arange(1, n * n + 1, dtype=np.float64)          # double, not int32
    sio.savemat(str(tmp_path / "grid.mat"), {"active_index": ai.reshape(-1, 1), "ghost_lr": np.zeros((n * n, 1))})
    sio.savemat(str(tmp_path / "ic.mat"), {"yf": np.zeros((3 * n * n, 1))})
    (tmp_path / "infile_forward").write_text(
        "Et_file = '';\nfinal_time = 1;\nnstep = 5;\nicondfile = 'ic.mat';\noutfile = 'o.mat';\n"
        "outfile_prefix = 'ys_';\nmex_function = @fk_forward_Et_mex;\ngrid_file = 'grid.mat';\n"
        "in_path = './';\nout_path = './';\n")
    r = _run("fkadj_save_fk_forward_Et", tmp_path)
    assert r.returncode == 1
    assert 'Variable "active_index" must be of type int32' in r.stderr
    assert "Et_file string is empty, will set Et to zero" in r.stdout


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference data not present")
def test_gradient_driver_loads_the_reference_inputs(tmp_path):
    """With the reference's own infile_grad (paths pointed at its data) the
    driver reads every input through the native reader; without a GPU it
    stops at device setup, after echoing the reference's parameter lines."""
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present: this test covers the host-side path only")
    text = open(os.path.join(os.path.dirname(REF_DATA), "infile_grad")).read()
    text = text.replace("in_path = './data/';", f"in_path = '{REF_DATA}/';")
    text = text.replace("out_path = './data/';", "out_path = './';")
    (tmp_path / "infile_grad").write_text(text)
    r = _run("fkadj_simple_grad_desc", tmp_path)
    assert "gamma=[1.00, 0.20, 0.20]" in r.stdout
    assert "Et_seed_file=Et_pulse_N_1_E0_5.00_t0_20.0_300ms.mat" in r.stdout
    assert r.returncode == 1 and "error: problem:" in r.stderr

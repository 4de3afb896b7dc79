"""Native drivers end to end on the GPU, through MAT files only.

fkadj_simple_grad_desc: the reference's 256^2 x 3000-step gradient-descent
run restarted at iteration 51 from files the native writer makes (grid,
objective matrix, initial state, seed pulse) and run for nmod = 50
iterations writes the iteration-100 snapshot; its Et, gradE, Lcost and the
Lcost/L0/LE vectors are compared with the reference's own iteration-100 file
(read with scipy).

fkadj_save_fk_forward_Et: a 64^2 forward run with snapshots; ys and yf are
compared with the library's Python binding (same engine, bit for bit) and yf
with the oracle."""
import os
import subprocess

import numpy as np
import pytest
import scipy.io as sio

from fkadj import api, geometry as G, matio, workloads as W

pytestmark = pytest.mark.gpu

BIN = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "adjoint-optimization_b200",
                   "bin")


def _run(binary, cwd, timeout=600):
    r = subprocess.run([os.path.join(BIN, binary)], cwd=cwd, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, (r.stdout[-2000:], r.stderr[-2000:])
    return r


def _nan_grid(y_compact, active_index):
    n = active_index.size
    y = np.full(3 * n, np.nan)
    act = np.flatnonzero(active_index > 0)
    k = active_index[act] - 1
    for f in range(3):
        y[f * n + act] = y_compact[f * len(act) + k]
    return y


def test_gradient_descent_driver_reproduces_the_reference_iteration_100_file(golden, tmp_path):
    ai = golden["active_index"].astype(np.int32)
    n = int(golden["nrows"])
    mask = (ai > 0).reshape(n, n)
    ds = 1e-3
    k50 = list(golden["iters"]).index(50)
    Et51 = golden["Et"][k50] - ds * golden["gradE"][k50]   # the reference's update at iteration 50
    matio.savemat(str(tmp_path / "grid.mat"), {"active_index": ai, "ghost_lr": golden["ghost_lr"].astype(np.int16)})
    matio.savemat(str(tmp_path / "S.mat"), {"S": G.objective_matrix(mask)})
    matio.savemat(str(tmp_path / "ic.mat"), {"yf": _nan_grid(golden["y0"], ai)})
    matio.savemat(str(tmp_path / "seed.mat"), {"Et": Et51.reshape(1, -1), "dt": 0.1, "final_time": 300.0})
    (tmp_path / "infile_grad").write_text(
        "% -*-octave-*-\nalpha=0.5; % weight of electric field integral\nds=1e-3;\nns=50;\nfinal_time=300;\n"
        "gamma = [1, 0.2, 0.2];\nnmod = 50;\nEt_seed_file = 'seed.mat';\nicondfile = 'ic.mat';\n"
        "grid_file = 'grid.mat';\nS_file = 'S.mat';\nmex_function = @fk_grad_Et_mex;\nin_path = './';\n"
        "out_path = './out/';\njobid = '000001';\n")
    os.makedirs(tmp_path / "out")
    r = _run("fkadj_simple_grad_desc", tmp_path)
    assert "i_grad = 50 of 50" in r.stdout
    outs = [f for f in os.listdir(tmp_path / "out") if f.startswith("simple_grad_desc_step_")]
    assert len(outs) == 1 and outs[0].endswith("_000001_50.mat"), outs
    got = sio.loadmat(str(tmp_path / "out" / outs[0]))
    k = list(golden["iters"]).index(100)
    rel = lambda a, b: np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b))
    assert rel(got["Et"], golden["Et"][k]) <= 1e-12
    assert rel(got["gradE"], golden["gradE"][k]) <= 1e-8
    assert abs(got["Lcost"][0, 0] - golden["Lcost"][k]) <= 1e-9 * golden["Lcost"][k]
    for key in ("Lcost_vec", "L0_vec", "LE_vec"):
        assert np.max(np.abs(got[key].ravel() - golden[key][k]) / np.abs(golden[key][k])) <= 1e-9, key
    for key in ("alpha", "dt", "final_time", "ds", "nmod"):
        assert got[key].shape == (1, 1)
    assert str(got["icondfile"][0]) == "ic.mat" and str(got["mex_function"][0]) == "fk_grad_Et_mex"
    assert got["gamma"].shape == (1, 3)


def test_forward_driver_writes_the_snapshots_the_library_computes(tmp_path):
    import oracle as O  # the checker
    inst = W.plain_instance(64, 200, seed=17, n_obstacles=5, intervals=10)
    ai = inst.active_index.astype(np.int32)
    matio.savemat(str(tmp_path / "grid.mat"), {"active_index": ai, "ghost_lr": inst.ghost.astype(np.float64)})
    matio.savemat(str(tmp_path / "ic.mat"), {"yf": _nan_grid(inst.y0, ai)})
    matio.savemat(str(tmp_path / "pulse.mat"), {"Et": inst.Et.reshape(1, -1), "dt": inst.dt,
                                                "final_time": inst.dt * inst.nt, "alpha": 0.25})
    (tmp_path / "infile_forward").write_text(
        "% -*-octave-*-\nEt_file = 'pulse.mat';\nfinal_time = 1; % ignored\nnstep = 50;\nicondfile = 'ic.mat';\n"
        "outfile = '';\noutfile_prefix = 'ys_mex_';\nmex_function = @fk_forward_Et_mex;\n"
        f"grid_file = 'grid.mat';\nin_path = './';\nout_path = './';\ndx = {inst.dx!r};\n")
    r = _run("fkadj_save_fk_forward_Et", tmp_path)
    assert "alpha=0.25" in r.stdout and "ns=nt/nstep-1=3" in r.stdout
    got = sio.loadmat(str(tmp_path / "ys_mex_pulse.mat"))
    ys, yf, pstr = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, ai, inst.ncols, inst.nrows,
                                     inst.ghost.astype(np.float64), 50, params=inst.params)
    assert got["ys"].shape == ys.shape == (3 * inst.n, 3)
    assert np.array_equal(got["ys"], ys, equal_nan=True)
    assert np.array_equal(got["yf"].ravel(), yf, equal_nan=True)
    assert str(got["param_str"][0]) == pstr
    assert int(got["nrows"][0, 0]) == 64 and int(got["nstep"][0, 0]) == 50
    _, ora = O.forward(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid)
    act = np.isfinite(yf)
    assert np.max(np.abs(yf[act] - ora[act])) <= 1e-10 * np.max(np.abs(ora[act]))


def test_gradient_descent_driver_armijo_mode_decreases_the_cost(tmp_path):
    """line_search = 'armijo' with the exact gradient: trial steps as one batch
    of objective-only jobs; every accepted step lowers Lcost, so the recorded
    Lcost_vec never increases."""
    inst = W.make_instance(64, 300, seed=71, n_obstacles=5, intervals=12, objective="gradient", alpha=0.02)
    ai = inst.active_index.astype(np.int32)
    matio.savemat(str(tmp_path / "grid.mat"), {"active_index": ai, "ghost_lr": inst.ghost.astype(np.float64)})
    matio.savemat(str(tmp_path / "S.mat"), {"S": inst.S})
    matio.savemat(str(tmp_path / "ic.mat"), {"yf": _nan_grid(inst.y0, ai)})
    matio.savemat(str(tmp_path / "seed.mat"), {"Et": inst.Et.reshape(1, -1)})
    (tmp_path / "infile_grad").write_text(
        f"alpha = 0.02;\nds = 1e-2;\nns = 4;\nfinal_time = {inst.dt * inst.nt!r};\ndt = {inst.dt!r};\n"
        "gamma = [1, 0.2, 0.2];\nnmod = 4;\nEt_seed_file = 'seed.mat';\nicondfile = 'ic.mat';\n"
        "grid_file = 'grid.mat';\nS_file = 'S.mat';\nmex_function = @fk_grad_Et_mex;\nin_path = './';\n"
        f"out_path = './';\njobid = 'armijo';\ndx = {inst.dx!r};\ngrad_mode = 'exact';\n"
        "line_search = 'armijo';\nprobes = 5;\n")
    r = _run("fkadj_simple_grad_desc", tmp_path)
    assert r.stdout.count("armijo:") == 4
    outs = [f for f in os.listdir(tmp_path) if f.startswith("simple_grad_desc_step_") and f.endswith("_armijo_4.mat")]
    assert len(outs) == 1, os.listdir(tmp_path)
    L = sio.loadmat(str(tmp_path / outs[0]))["Lcost_vec"].ravel()
    assert np.all(np.diff(L) <= 0), L
    assert "accepted" in r.stdout

"""The reference's own CUDA routines (compiled from its sources into
oracle/_ref by oracle/ref_build.sh) vs libfkadj and the CPU oracle on the
same seeded inputs.  Skipped where the reference build is absent."""
import numpy as np
import pytest

import oracle as O
import refbin
from fkadj import api, geometry as G, workloads as W
from fkadj.params import FkParams

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refbin.available(), reason="oracle/_ref not built")]


def _rel(a, b):
    m = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), m)
    return np.abs(a[m] - b[m]).max() / np.abs(b[m]).max()


def test_reference_forward_binary_vs_fkadj():
    inst = W.make_instance(64, 200, seed=51, n_obstacles=6, ncols=80)
    ns = api.compute_ns(inst.nt, 50)
    ys_r, yf_r = refbin.forward(inst.dt, inst.Et, inst.nt, inst.y0, inst.active_index, inst.nrows, inst.ncols,
                                inst.ghost, 50, ns)
    ys, yf, _ = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                  inst.nrows, inst.ghost, 50, params=inst.params)
    assert _rel(yf, yf_r) <= 1e-10
    for k in range(ns):
        assert _rel(ys[:, k], ys_r[k]) <= 1e-10


@pytest.mark.parametrize("objective", ["mean_u2", "gradient"])
def test_reference_gradient_binary_vs_fkadj_and_oracle(objective):
    inst = W.make_instance(64, 200, seed=52, n_obstacles=6, objective=objective)
    alpha = 0.25
    r = refbin.grad(inst.dt, inst.Et, inst.nt, inst.y0, inst.active_index, inst.nrows, inst.ncols,
                    inst.ghost, inst.gamma, inst.S, alpha)
    g, Lc, L0, LE, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                      inst.nrows, inst.ghost, inst.gamma, inst.S, alpha, params=inst.params)
    o = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, O.Objective(inst.S, inst.gamma), alpha, mode="ref")
    assert abs(Lc - r["Lcost"]) <= 1e-10 * abs(r["Lcost"])
    assert np.linalg.norm(g - r["gradE"]) <= 1e-8 * np.linalg.norm(r["gradE"])
    assert np.linalg.norm(o["gradE"] - r["gradE"]) <= 1e-8 * np.linalg.norm(r["gradE"])


def test_reference_binary_reproduces_its_golden_file(golden):
    """The reference built here reproduces its own shipped gradient (GD
    iteration 200, 256^2 x 3000 steps, h = 0.035)."""
    k = 3
    ai = golden["active_index"]
    n = int(golden["nrows"])
    S = G.objective_matrix((ai > 0).reshape(n, n))
    r = refbin.grad(float(golden["dt"]), golden["Et"][k], int(golden["nt"]), golden["y0"], ai, n, n,
                    golden["ghost_lr"].astype(float), golden["gamma"], S, float(golden["alpha"]),
                    dx_tag="dx0p035")
    ge = golden["gradE"][k]
    assert abs(r["Lcost"] - golden["Lcost"][k]) <= 1e-10 * golden["Lcost"][k]
    assert np.linalg.norm(r["gradE"] - ge) <= 1e-9 * np.linalg.norm(ge)

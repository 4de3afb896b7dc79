"""Optimisation drivers: the reference's fixed-step loop reproduces its own
gradient-descent history (golden files), and the Armijo descent with batched
probes decreases the cost with every accepted step satisfying the Armijo
condition."""
import numpy as np
import pytest

from fkadj import geometry as G, optimize, workloads as W
from fkadj.params import FkParams

pytestmark = pytest.mark.gpu


def test_simple_grad_desc_follows_the_reference_history(golden):
    """Start at the pulse of gradient-descent iteration 50 (ds = 1e-3) and take
    two iterations: iteration 50's Lcost and the LE / Lcost of iteration 51
    (the first entries of the iteration-100 file's vectors) come out."""
    ai = golden["active_index"]
    n = int(golden["nrows"])
    mask = (ai > 0).reshape(n, n)
    P = FkParams().with_h(float(golden["h"]))
    inst = W.Instance(n, n, P.h, float(golden["dt"]), int(golden["nt"]), P, mask, ai,
                      golden["ghost_lr"].astype(float), golden["y0"], golden["Et"][0], np.zeros(1),
                      np.zeros(int(golden["nt"]) + 1, dtype=int), G.objective_matrix(mask), golden["gamma"],
                      float(golden["alpha"]), 0)
    out = optimize.simple_grad_desc(inst, 2, 1e-3)
    assert abs(out["Lcost_vec"][0] - golden["Lcost"][0]) <= 1e-10 * golden["Lcost"][0]
    assert abs(out["LE_vec"][1] - golden["LE_vec"][1][0]) <= 1e-9 * golden["LE_vec"][1][0]
    assert abs(out["L0_vec"][1] - golden["L0_vec"][1][0]) <= 1e-9 * golden["L0_vec"][1][0]
    assert abs(out["Lcost_vec"][1] - golden["Lcost_vec"][1][0]) <= 1e-9 * golden["Lcost_vec"][1][0]


def test_armijo_descent_with_batched_probes_decreases_the_cost():
    inst = W.make_instance(64, 300, seed=61, n_obstacles=6, intervals=12, alpha=0.02)
    out = optimize.armijo_descent(inst, iters=4, probes=5)
    J = out["J"]
    assert all(out["armijo_ok"])
    assert np.all(np.diff(J) < 0), J
    for (steps_js, j0, s) in zip(out["probes"], J, out["step"]):
        assert any(abs(st - s) == 0 for st, _ in steps_js)

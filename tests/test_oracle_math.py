"""Self-checks of the oracle: spline vs scipy, exact-mode adjoint vs central
finite differences, reference mode vs exact mode on a smooth problem."""
import numpy as np
import pytest
import scipy.interpolate as si

import oracle as O
from fkadj import geometry as G
from fkadj import workloads as W
from fkadj.params import FkParams


def test_spline_not_a_knot_matches_scipy():
    rng = np.random.default_rng(3)
    for n in (4, 5, 9, 101):
        dt = 0.1
        E = rng.standard_normal(n)
        ypp = O.spline_ypp(E, dt)
        cs = si.CubicSpline(np.arange(n) * dt, E, bc_type="not-a-knot")
        assert np.allclose(ypp, cs(np.arange(n) * dt, 2), rtol=1e-10, atol=1e-10)
        for t in (0.05, (n - 1.5) * dt, (n - 1) * dt * 0.37):
            assert abs(O.spline_val(E, ypp, dt, t) - cs(t)) <= 1e-12 * (1 + abs(cs(t)))


def _small_problem(n=32, nt=40, seed=5):
    inst = W.plain_instance(n=n, nt=nt, seed=seed, n_obstacles=3, intervals=8)
    return inst


@pytest.mark.parametrize("seed", [1, 2])
def test_exact_gradient_matches_central_fd(seed):
    inst = _small_problem(seed=seed)
    P = inst.params
    obj = O.Objective(inst.S, inst.gamma)
    args = (P, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
            inst.active_index, obj, 0.3)
    r = O.grad(*args, mode="exact")
    rng = np.random.default_rng(seed)
    h = 1e-6
    for i in rng.choice(inst.nt + 1, size=5, replace=False):
        Ep, Em = inst.Et.copy(), inst.Et.copy()
        Ep[i] += h
        Em[i] -= h
        a = list(args)
        a[2] = Ep
        lp = O.grad(*a, mode="exact")["Lcost"]
        a[2] = Em
        lm = O.grad(*a, mode="exact")["Lcost"]
        fd = (lp - lm) / (2 * h)
        an = r["gradE"][i] * inst.dt
        assert abs(fd - an) <= 2e-6 * max(abs(fd), 1e-4), (i, fd, an)


def test_ref_and_exact_modes_agree_to_discretisation_error():
    """The reference's continuous-adjoint density and the discrete gradient
    (scaled by 1/dt) agree on interval sums to O(dt): halving dt halves the
    gap (measured 0.021 -> 0.0097 at dt 0.02 -> 0.01)."""
    gaps = []
    for nt, dt in ((60, 0.02), (120, 0.01)):
        inst = W.plain_instance(n=32, nt=nt, seed=4, n_obstacles=3, intervals=8, dt=dt)
        obj = O.Objective(inst.S, inst.gamma)
        args = (inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid,
                inst.gh_grid, inst.active_index, obj, 0.0)
        gr = O.grad(*args, mode="ref")["gradE"]
        ge = O.grad(*args, mode="exact")["gradE"]
        starts = np.arange(0, nt, nt // 8)
        sr, se = np.add.reduceat(gr[:-1], starts), np.add.reduceat(ge[:-1], starts)
        gaps.append(np.linalg.norm(sr - se) / np.linalg.norm(sr))
    assert gaps[0] < 0.03 and gaps[1] < 0.6 * gaps[0], gaps

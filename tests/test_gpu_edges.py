"""Edge cases of the CUDA path against the oracle (through the C ABI): a grid
without holes, cells whose two opposite neighbours are both holes (the
reference's mirroring leaves such a cell NaN; its neighbours treat it as a
hole), the shortest horizon the not-a-knot spline allows (3 steps), a tiny
ragged grid, and a zero pulse.  Tolerances as in the parity tests: states 1e-10
relative, gradients 1e-8 relative."""
import numpy as np
import pytest

import oracle as O
from fkadj import _lib, api, geometry as G, workloads as W
from fkadj._lib import FkadjError
from fkadj.params import FkParams

pytestmark = pytest.mark.gpu


def _custom(mask, nt, seed=3, dx=0.025, dt=0.02, objective="gradient", alpha=0.1, Et=None):
    mask = np.asarray(mask, dtype=bool)
    nr, nc = mask.shape
    rng = np.random.default_rng(seed)
    u, v, w = W.broken_wavefront_ic(mask, rng)
    y0 = np.concatenate([f[mask] for f in (u, v, w)])
    amps = rng.uniform(0.0, 1.0, 4)
    E, iv = W.piecewise_constant(nt, amps)
    if Et is not None:
        E = np.asarray(Et, dtype=np.float64)
    n_num = int(mask.sum())
    if objective == "gradient":
        S, gamma = G.objective_matrix(mask), np.array([1.0, 0.2, 0.2])
    else:
        S, gamma = G.mean_square_matrix(n_num), np.array([1.0, 0.0, 0.0])
    return W.Instance(nr, nc, dx, dt, nt, FkParams().with_h(dx), mask, G.active_index(mask), G.ghost_lr(mask),
                      y0, E, amps, iv, S, gamma, float(alpha), seed, "edge")


def _rel_states(a, b):
    m = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), m), "NaN pattern differs"
    return np.abs(a[m] - b[m]).max() / np.abs(b[m]).max()


def _forward_matches(inst):
    _, yf, _ = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                 inst.ghost, 0, params=inst.params)
    _, yo = O.forward(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid)
    assert _rel_states(yf, yo) <= 1e-10
    return yf


def _grad_matches(inst, mode):
    g, Lc, _, _, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                    inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params,
                                    opts=api.options(grad_mode=mode))
    o = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, O.Objective(inst.S, inst.gamma), inst.alpha,
               mode="ref" if mode == _lib.GRAD_REF else "exact")
    assert abs(Lc - o["Lcost"]) <= 1e-10 * abs(o["Lcost"])
    assert np.linalg.norm(g - o["gradE"]) <= 1e-8 * np.linalg.norm(o["gradE"])


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_grid_without_holes(mode):
    inst = _custom(np.ones((40, 56), bool), 150)
    _forward_matches(inst)
    _grad_matches(inst, mode)


def test_cells_between_two_holes_stay_nan_and_do_not_spread():
    mask = np.ones((32, 48), bool)
    mask[10, 10] = mask[12, 10] = False      # (11, 10): north and south are holes
    mask[20, 30] = mask[20, 32] = False      # (20, 31): west and east are holes
    inst = _custom(mask, 120, objective="gradient")
    yf = _forward_matches(inst)
    n = 32 * 48
    u = yf[:n].reshape(32, 48)
    assert np.isnan(u[11, 10]) and np.isnan(u[20, 31])
    assert np.isfinite(u[mask]).sum() == mask.sum() - 2
    # the objective sees the NaN cells, as the reference's does: a numeric error
    with pytest.raises(FkadjError) as e:
        api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost,
                       inst.gamma, inst.S, inst.alpha, params=inst.params)
    assert e.value.status == _lib.ERR_NUMERIC


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_shortest_horizon(mode):
    mask = np.ones((48, 64), bool)
    mask[20:24, 30:33] = False
    inst = _custom(mask, 3)
    _forward_matches(inst)
    _grad_matches(inst, mode)


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_tiny_ragged_grid(mode):
    mask = np.ones((5, 7), bool)
    inst = _custom(mask, 60, objective="mean_u2", alpha=0.0)
    _forward_matches(inst)
    _grad_matches(inst, mode)


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_zero_pulse(mode):
    mask = np.ones((48, 48), bool)
    mask[10:14, 10:14] = False
    inst = _custom(mask, 100, Et=np.zeros(101))
    _forward_matches(inst)
    _grad_matches(inst, mode)


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_nonfinite_gradient_with_finite_objective_is_a_numeric_error(mode):
    """The adjoint's z.gh sums overflow while y(T) and the objective stay
    finite: the pulse is zero, so gh never enters the forward sweep, and one
    active cell gets a ghost_lr near the largest double while gamma_u scales
    z(T) = -gamma_u S u(T) past 1 there.  The objective-only call succeeds with
    a finite J; the gradient call reports a numeric error instead of returning
    an infinite gradient with FKADJ_OK.  The failure is made on the host (the
    inputs); nothing on the GPU faults."""
    mask = np.ones((48, 48), bool)
    mask[20:24, 20:24] = False
    inst = _custom(mask, 60, Et=np.zeros(61), objective="mean_u2", alpha=0.0)
    _, yf, _ = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                 inst.ghost, 0, params=inst.params)
    uT = G.compact(yf, inst.active_index)[:inst.n_num]
    k = int(np.argmax(np.abs(uT)))
    assert abs(uT[k]) > 0.05
    ghost = inst.ghost.astype(np.float64).copy()
    ghost[k] = 1.7e308
    gamma = np.array([1.0e5 * inst.n_num, 0.0, 0.0])
    with api.Problem(params=inst.params, dt=inst.dt, nt=inst.nt, active_index=inst.active_index,
                     nrows=inst.nrows, ncols=inst.ncols, ghost_lr=ghost, gamma=gamma, S=inst.S, alpha=0.0,
                     opts=api.options(grad_mode=mode)) as pb:
        r = pb.objective(inst.Et, inst.y0)
        assert np.isfinite(r["Lcost"]) and r["Lcost"] > 0
        with pytest.raises(FkadjError) as e:
            pb.grad(inst.Et, inst.y0)
        assert e.value.status == _lib.ERR_NUMERIC
        assert "gradient is not finite" in str(e.value)
    with pytest.raises(FkadjError) as e:
        api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, ghost, gamma,
                       inst.S, 0.0, params=inst.params, opts=api.options(grad_mode=mode))
    assert e.value.status == _lib.ERR_NUMERIC

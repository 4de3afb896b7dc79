"""CUDA path vs the CPU oracle on the same seeded inputs (through the C ABI).

Tolerances: states 1e-10 relative (max-norm, at horizons short enough that
round-off growth stays below it), J and gradE 1e-8 relative (2-norm); the
golden 256^2 x 3000-step gradient of the reference to 1e-9 relative.
"""
import numpy as np
import pytest

import oracle as O
from fkadj import api, geometry as G, workloads as W
from fkadj import _lib

pytestmark = pytest.mark.gpu


def _rel(a, b):
    m = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), m), "NaN pattern differs"
    return np.abs(a[m] - b[m]).max() / max(np.abs(b[m]).max(), 1e-300)


def _inst(n=64, nt=200, seed=11, ncols=None, **kw):
    return W.make_instance(n, nt, seed=seed, ncols=ncols, n_obstacles=kw.pop("n_obstacles", 6), **kw)


@pytest.mark.parametrize("shape", [(64, 64), (48, 80), (50, 70), (33, 129)])
def test_forward_matches_oracle(shape):
    nr, nc = shape
    inst = _inst(nr, 150, seed=nr * 7 + nc, ncols=nc)
    ys, yf, pstr = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                     inst.nrows, inst.ghost, 50, params=inst.params)
    ns = api.compute_ns(inst.nt, 50)
    ys_o, yf_o = O.forward(inst.params, inst.dt, inst.Et, inst.nt, nr, nc, inst.y0_grid, inst.gh_grid,
                           50, ns)
    assert _rel(yf, yf_o) <= 1e-10
    assert ys.shape == (3 * nr * nc, ns)
    for k in range(ns):
        assert _rel(ys[:, k], ys_o[k]) <= 1e-10
    assert "h = 0.025" in pstr


@pytest.mark.parametrize("tile", [1, 2, 3, 4, 5, 6, 7, 8, 9])
def test_forward_state_is_independent_of_tile_shape(tile):
    """options.tile k >= 1 fixes preset k-1 for every kernel; 0 autotunes."""
    inst = _inst(96, 40, seed=3, ncols=72)
    ref = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                            inst.ghost, 40, params=inst.params, opts=api.options(tile=1))[1]
    yf = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                           inst.ghost, 40, params=inst.params, opts=api.options(tile=tile))[1]
    assert np.array_equal(np.isnan(ref), np.isnan(yf))
    assert np.array_equal(ref[~np.isnan(ref)], yf[~np.isnan(yf)])


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_gradient_bits_are_independent_of_tile_and_autotune(mode):
    """Fixed-order 16x16 sub-block reductions: every tile preset and the
    autotuned choice give bit-identical gradients."""
    inst = _inst(80, 60, seed=13, ncols=112, objective="gradient")
    outs = []
    for tile in (0, 1, 2, 3, 4, 5, 6, 7, 8, 9):
        outs.append(api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                   inst.nrows, inst.ghost, inst.gamma, inst.S, 0.1, params=inst.params,
                                   opts=api.options(tile=tile, grad_mode=mode)))
    for o in outs[1:]:
        assert np.array_equal(o[0], outs[0][0])
        assert o[1] == outs[0][1]


@pytest.mark.parametrize("objective", ["mean_u2", "gradient"])
def test_ref_gradient_matches_oracle(objective):
    inst = _inst(64, 120, seed=21, objective=objective, ncols=80)
    alpha = 0.3
    g, Lc, L0, LE, _, yf = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                          inst.nrows, inst.ghost, inst.gamma, inst.S, alpha,
                                          params=inst.params, return_yf=True)
    obj = O.Objective(inst.S, inst.gamma)
    r = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, obj, alpha, mode="ref")
    assert _rel(yf, r["yf"]) <= 1e-10
    assert abs(L0 - r["L0"]) <= 1e-10 * abs(r["L0"])
    assert abs(LE - r["LE"]) <= 1e-13 * abs(r["LE"])
    assert abs(Lc - r["Lcost"]) <= 1e-10 * abs(r["Lcost"])
    assert np.linalg.norm(g - r["gradE"]) <= 1e-8 * np.linalg.norm(r["gradE"])


def test_sqrt_checkpointing_equals_full_storage():
    inst = _inst(64, 150, seed=5)
    args = (inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost,
            inst.gamma, inst.S, 0.0)
    full = api.fk_grad_Et(*args, params=inst.params, opts=api.options(ckpt_policy=_lib.CKPT_FULL))
    sq = api.fk_grad_Et(*args, params=inst.params, opts=api.options(ckpt_policy=_lib.CKPT_SQRT))
    assert np.array_equal(full[0], sq[0])
    assert full[1] == sq[1]


def test_golden_reference_gradient(golden):
    """The reference's shipped 256^2 x 3000-step gradient (GD iteration 50)."""
    k = 0
    ai = golden["active_index"]
    n = int(golden["nrows"])
    mask = (ai > 0).reshape(n, n)
    S = G.objective_matrix(mask)
    from fkadj.params import FkParams
    P = FkParams().with_h(float(golden["h"]))
    g, Lc, L0, LE, _ = api.fk_grad_Et(golden["Et"][k], float(golden["dt"]), int(golden["nt"]), golden["y0"],
                                      ai, n, n, golden["ghost_lr"].astype(float), golden["gamma"], S,
                                      float(golden["alpha"]), params=P)
    ge = golden["gradE"][k]
    assert abs(Lc - golden["Lcost"][k]) <= 1e-10 * abs(golden["Lcost"][k])
    assert np.linalg.norm(g - ge) <= 1e-9 * np.linalg.norm(ge)


def test_problem_handle_repeated_calls_are_deterministic():
    inst = _inst(64, 100, seed=8)
    with api.Problem(inst) as pb:
        a = pb.grad(inst.Et, inst.y0)
        b = pb.grad(inst.Et, inst.y0)
        o = pb.objective(inst.Et, inst.y0)
        assert pb.last_launches > 0
        assert pb.device_bytes > 0
    assert np.array_equal(a["gradE"], b["gradE"])
    assert a["Lcost"] == b["Lcost"] == o["Lcost"]


def _exact(inst, alpha=0.2, ckpt=_lib.CKPT_AUTO, Et=None):
    Et = inst.Et if Et is None else Et
    return api.fk_grad_Et(Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                          inst.ghost, inst.gamma, inst.S, alpha, params=inst.params,
                          opts=api.options(grad_mode=_lib.GRAD_EXACT, ckpt_policy=ckpt))


@pytest.mark.parametrize("objective", ["mean_u2", "gradient"])
def test_exact_gradient_matches_oracle(objective):
    inst = _inst(48, 90, seed=31, objective=objective, ncols=64)
    g, Lc, L0, LE, _ = _exact(inst)
    r = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, O.Objective(inst.S, inst.gamma), 0.2, mode="exact")
    assert abs(Lc - r["Lcost"]) <= 1e-10 * abs(r["Lcost"])
    assert np.linalg.norm(g - r["gradE"]) <= 1e-8 * np.linalg.norm(r["gradE"])


def test_exact_sqrt_equals_full():
    inst = _inst(64, 130, seed=9)
    a = _exact(inst, ckpt=_lib.CKPT_FULL)
    b = _exact(inst, ckpt=_lib.CKPT_SQRT)
    assert np.array_equal(a[0], b[0])


def test_exact_gradient_central_fd_on_intervals():
    """dJ/dA_k for piecewise-constant amplitudes (central FD, h = 1e-6) on
    10 seeded intervals vs the discrete adjoint: dJ/dA_k = dt * sum_{i in k} gradE[i]."""
    inst = W.make_instance(64, 400, seed=41, n_obstacles=8, intervals=40, wavefronts=4)
    alpha = 0.0
    g = _exact(inst, alpha)[0]
    K = len(inst.amplitudes)
    dJdA = np.array([inst.dt * g[inst.interval_of_sample == k].sum() for k in range(K)])
    rng = np.random.default_rng(2024)
    h = 1e-6
    with api.Problem(inst, opts=api.options(grad_mode=_lib.GRAD_EXACT)) as pb:
        for k in rng.choice(K, size=10, replace=False):
            Ap, Am = inst.amplitudes.copy(), inst.amplitudes.copy()
            Ap[k] += h
            Am[k] -= h
            Jp = pb.objective(W.piecewise_constant(inst.nt, Ap)[0], inst.y0)["Lcost"]
            Jm = pb.objective(W.piecewise_constant(inst.nt, Am)[0], inst.y0)["Lcost"]
            fd = (Jp - Jm) / (2 * h)
            assert abs(fd - dJdA[k]) <= 1e-6 * np.abs(dJdA).max() + 1e-5 * abs(fd), (k, fd, dJdA[k])


def _state_bytes(nrows, ncols):
    rows = (nrows + 63) // 64 * 64 + 8
    ld = ((ncols + 63) // 64 * 64 + 8 + 7) // 8 * 8
    return 3 * rows * ld * 8


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
@pytest.mark.parametrize("slots", [2, 4, 9, 60])
def test_binomial_checkpointing_equals_full_storage(mode, slots):
    """Binomial reversal with a budget of `slots` states (2 = no free snapshot,
    every state replayed from y_0; 60 = a long chain of checkpoints stored by
    the forward sweep itself) gives the same bits as full storage."""
    inst = _inst(48, 70 if slots == 2 else 130, seed=23, ncols=64, objective="gradient")
    args = (inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost,
            inst.gamma, inst.S, 0.2)
    full = api.fk_grad_Et(*args, params=inst.params,
                          opts=api.options(grad_mode=mode, ckpt_policy=_lib.CKPT_FULL))
    budget = (slots + 1) * _state_bytes(inst.nrows, inst.ncols)
    bino = api.fk_grad_Et(*args, params=inst.params,
                          opts=api.options(grad_mode=mode, ckpt_policy=_lib.CKPT_BINOMIAL,
                                           ckpt_budget_bytes=budget))
    assert np.array_equal(full[0], bino[0])
    assert full[1] == bino[1]


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_windowed_zgh_reduction_matches_oracle_and_batch(mode):
    """1300 steps: the standalone sweep reduces its z.gh partials in blocks of
    rows as it goes (three blocks here); the batch engine keeps every row and
    reduces once.  The two agree to 1e-12 (the batch tests' bound), and the
    oracle within 1e-8."""
    from fkadj.batch import Batch
    inst = _inst(48, 1300, seed=33, ncols=64, objective="gradient", alpha=0.1)
    g, Lc, _, _, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                    inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params,
                                    opts=api.options(grad_mode=mode))
    with Batch() as b:
        p = b.add_problem(inst, grad_mode=mode)
        r = b.result((b.submit(p, inst.Et, inst.y0), b.run())[0])
    assert np.linalg.norm(r["gradE"] - g) <= 1e-12 * np.linalg.norm(g)
    assert abs(r["Lcost"] - Lc) <= 1e-12 * abs(Lc)
    o = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, O.Objective(inst.S, inst.gamma), inst.alpha,
               mode="ref" if mode == _lib.GRAD_REF else "exact")
    assert np.linalg.norm(g - o["gradE"]) <= 1e-8 * np.linalg.norm(o["gradE"])


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_auto_store_takes_the_schedule_that_recomputes_less(mode):
    """AUTO with a budget below the full trajectory (131 states): 100 states
    let the binomial schedule recompute 32 steps against sqrt's 119, 30 states
    102.  The exact mode takes binomial both times; the reference mode, whose
    binomial reversal also loses the kept k1 and copies a state per step (0.9
    of a forward step per backward step, as measured), keeps sqrt.  Every
    choice gives the bits of full storage."""
    inst = _inst(48, 130, seed=23, ncols=64, objective="gradient", alpha=0.2)
    args = (inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost,
            inst.gamma, inst.S, inst.alpha)
    full = api.fk_grad_Et(*args, params=inst.params,
                          opts=api.options(grad_mode=mode, ckpt_policy=_lib.CKPT_FULL))
    sb = _state_bytes(inst.nrows, inst.ncols)
    want = "binomial" if mode == _lib.GRAD_EXACT else "sqrt"
    for states in (100, 30):
        opts = api.options(grad_mode=mode, ckpt_policy=_lib.CKPT_AUTO, ckpt_budget_bytes=states * sb)
        with api.Problem(inst, opts=opts) as pb:
            r = pb.grad(inst.Et, inst.y0)
            plan = pb.last_plan
        assert plan["policy"] == want, (states, plan)
        assert plan["recompute_steps"] == {"sqrt": 119, "binomial": 32 if states == 100 else 102}[want]
        assert np.array_equal(r["gradE"], full[0])
        assert r["Lcost"] == full[1]


@pytest.mark.parametrize("ckpt", [_lib.CKPT_SQRT, _lib.CKPT_FULL])
def test_zgh_row_segment_lattice_agrees_with_16x16_lattice(monkeypatch, ckpt):
    """The reference-mode step's z.gh partials on 16-cell row segments (tiles of
    any height, the default where 64x32 tiles fit one wave) and on 16x16
    sub-blocks (FKADJ_ZGH_SEGMENTS=0) sum the same terms in two fixed orders:
    gradients within 1e-13, objectives equal; on a ragged grid (rows and
    columns not multiples of 16) and a horizon whose rows span several windows."""
    inst = _inst(90, 700, seed=41, ncols=75, objective="gradient", alpha=0.1)
    args = (inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost, inst.gamma,
            inst.S, inst.alpha)
    seg = api.fk_grad_Et(*args, params=inst.params, opts=api.options(ckpt_policy=ckpt))
    monkeypatch.setenv("FKADJ_ZGH_SEGMENTS", "0")
    blk = api.fk_grad_Et(*args, params=inst.params, opts=api.options(ckpt_policy=ckpt))
    assert np.linalg.norm(seg[0] - blk[0]) <= 1e-13 * np.linalg.norm(blk[0])
    assert seg[1] == blk[1]

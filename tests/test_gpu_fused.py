"""The fused reference-adjoint step (k_adj_fused: the midpoint reconstruction
and the four backward stages in one launch) against the split kernels
(k_adj_mid + k_adj_step) and the CPU oracle, through the C ABI.

Both paths do the same arithmetic on the same values, so the gradients must
agree to round-off of the order of the last bit (1e-13 relative) under every
trajectory store (full with kept f, sqrt with the recompute's kept f, binomial
with the f carry), for every fused tile preset and with the J_F(y)^T cache or
without it; and the oracle within the parity tolerance (1e-8)."""
import numpy as np
import pytest

import oracle as O
from fkadj import _lib, api, workloads as W

pytestmark = pytest.mark.gpu


def _inst(nr=80, nc=112, nt=90, seed=61):
    return W.make_instance(nr, nt, seed=seed, ncols=nc, n_obstacles=7, objective="gradient", alpha=0.2,
                           wavefronts=2)


def _state_bytes(nrows, ncols):
    rows = (nrows + 63) // 64 * 64 + 8
    ld = ((ncols + 63) // 64 * 64 + 8 + 7) // 8 * 8
    return 3 * rows * ld * 8


def _grad(inst, monkeypatch, path, tile=None, ckpt=_lib.CKPT_SQRT, budget=0):
    monkeypatch.setenv("FKADJ_ADJ_PATH", path)
    if tile is None:
        monkeypatch.delenv("FKADJ_FUSED_TILE", raising=False)
    else:
        monkeypatch.setenv("FKADJ_FUSED_TILE", str(tile))
    with api.Problem(inst, opts=api.options(ckpt_policy=ckpt, ckpt_budget_bytes=budget)) as pb:
        r = pb.grad(inst.Et, inst.y0)
        r2 = pb.grad(inst.Et)   # a second call replays the captured graph
        kern = pb.adjoint_kernel
    assert np.array_equal(r["gradE"], r2["gradE"])
    return r, kern


def _close(a, b, tol=1e-13):
    return np.linalg.norm(a - b) <= tol * np.linalg.norm(b)


@pytest.mark.parametrize("tile", [0, 1, 2, 3])
@pytest.mark.parametrize("path", ["fused", "fused-recompute"])
def test_fused_step_gives_the_split_gradient(monkeypatch, tile, path):
    inst = _inst()
    split, k0 = _grad(inst, monkeypatch, "split")
    fused, k1 = _grad(inst, monkeypatch, path, tile)
    assert k0["path"] == "split" and k1["path"] == path
    assert _close(fused["gradE"], split["gradE"])
    assert abs(fused["Lcost"] - split["Lcost"]) <= 1e-15 * abs(split["Lcost"])


@pytest.mark.parametrize("store", ["full", "binomial"])
def test_fused_step_under_other_stores(monkeypatch, store):
    """Full storage keeps k1 = f(y) for every state (the fused kernel reads f of
    both ends); the binomial schedule keeps none (it evaluates f(y_{i-1}) and
    carries it to the next step as f(y_i))."""
    inst = _inst(64, 80, 70, seed=62)
    if store == "full":
        kw = dict(ckpt=_lib.CKPT_FULL)
    else:
        kw = dict(ckpt=_lib.CKPT_BINOMIAL, budget=12 * _state_bytes(64, 80))
    split, _ = _grad(inst, monkeypatch, "split", **kw)
    for path in ("fused", "fused-recompute"):
        fused, _ = _grad(inst, monkeypatch, path, 0, **kw)
        assert _close(fused["gradE"], split["gradE"]), path


def test_fused_step_matches_the_oracle(monkeypatch):
    inst = _inst(72, 96, 150, seed=63)
    fused, _ = _grad(inst, monkeypatch, "fused", 1)
    o = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, O.Objective(inst.S, inst.gamma), inst.alpha, mode="ref")
    assert abs(fused["Lcost"] - o["Lcost"]) <= 1e-10 * abs(o["Lcost"])
    assert np.linalg.norm(fused["gradE"] - o["gradE"]) <= 1e-8 * np.linalg.norm(o["gradE"])


def test_autotuner_reports_the_path_it_chose(monkeypatch):
    """Unforced, the autotuner times the fused presets (with and without the J
    cache) against the split pair and keeps the fastest; the gradient is the
    same whichever it picks."""
    inst = _inst(96, 96, 60, seed=64)
    monkeypatch.delenv("FKADJ_ADJ_PATH", raising=False)
    monkeypatch.delenv("FKADJ_FUSED_TILE", raising=False)
    with api.Problem(inst) as pb:
        r = pb.grad(inst.Et, inst.y0)
        k = pb.adjoint_kernel
    assert k["path"] in ("split", "fused", "fused-recompute")
    assert (k["tile"] == (0, 0, 0)) == (k["path"] == "split")
    split, _ = _grad(inst, monkeypatch, "split")
    assert _close(r["gradE"], split["gradE"])

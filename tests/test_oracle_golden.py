"""Pins the CPU oracle against the reference's own golden vectors
(src/cuda/data/*.mat, converted by tests/golden/make_golden.py)."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
from fkadj import geometry as G
from fkadj.params import FkParams


def _setup(golden):
    ai = golden["active_index"]
    n = int(golden["nrows"])
    mask = (ai > 0).reshape(n, n)
    P = FkParams().with_h(float(golden["h"]))
    y0 = G.nan_grid(golden["y0"], ai)
    gh = G.gh_grid(golden["ghost_lr"], ai, P.Du, P.h)
    return ai, n, mask, P, y0, gh


def test_generators_reproduce_shipped_grid_files(golden):
    ai, n, mask, P, y0, gh = _setup(golden)
    assert np.array_equal(G.active_index(mask), ai)
    assert np.array_equal(G.ghost_lr(mask), golden["ghost_lr"].astype(float))
    S = G.objective_matrix(mask)
    Sref = sp.csc_matrix((golden["S_data4"] / 4.0, golden["S_indices"], golden["S_indptr"]),
                         shape=S.shape)
    assert abs(S - Sref).max() == 0.0
    L = G.laplacian(mask)
    Lref = sp.csc_matrix((golden["lap_data"].astype(float), golden["lap_indices"],
                          golden["lap_indptr"]), shape=S.shape)
    assert abs(L - Lref).max() == 0.0
    assert np.array_equal(G.clean_mask(mask), mask)


def test_oracle_rhs_equals_shipped_laplacian(golden):
    """The stencil with NaN mirroring equals the shipped sparse lap matrix."""
    ai, n, mask, P, y0, gh = _setup(golden)
    Lref = sp.csc_matrix((golden["lap_data"].astype(float), golden["lap_indices"],
                          golden["lap_indptr"]), shape=(int(mask.sum()),) * 2)
    y0c = golden["y0"]
    nn = int(mask.sum())
    # zero ionic part: subtract rhs at the same state with D = 0
    P0 = FkParams(**{**P.as_dict(), "Du": 0.0, "Dv": 0.0, "Dw": 0.0})
    f = G.compact(O.rhs(P, n, n, y0, np.where(np.isnan(gh), np.nan, 0.0), 0.0), ai)
    f0 = G.compact(O.rhs(P0, n, n, y0, np.where(np.isnan(gh), np.nan, 0.0), 0.0), ai)
    for c, D in enumerate((P.Du, P.Dv, P.Dw)):
        lap = (f - f0)[c * nn:(c + 1) * nn]
        want = D / P.h ** 2 * (Lref @ y0c[c * nn:(c + 1) * nn])
        assert np.abs(lap - want).max() <= 1e-12 * np.abs(want).max()


def test_oracle_objective_matches_golden_LE(golden):
    dt = float(golden["dt"])
    for k in range(len(golden["iters"])):
        Et = golden["Et"][k]
        LE = dt * float(np.dot(Et, Et))
        assert abs(LE - golden["LE_vec"][k][-1]) <= 1e-13 * LE
        Lc = golden["Lcost"][k]
        assert abs(0.5 * golden["L0_vec"][k][-1] + 0.5 * float(golden["alpha"]) * LE - Lc) <= 1e-12 * Lc


@pytest.mark.slow
@pytest.mark.parametrize("k", [0, 3])
def test_oracle_ref_gradient_matches_golden(golden, k):
    """Full 256^2 x 3000-step gradient at gradient-descent iterations 50 and
    200.  Measured: Lcost rel 5e-16, gradE rel (2-norm) 2.4e-12."""
    ai, n, mask, P, y0, gh = _setup(golden)
    obj = O.Objective(G.objective_matrix(mask), golden["gamma"])
    r = O.grad(P, float(golden["dt"]), golden["Et"][k], int(golden["nt"]), n, n, y0, gh, ai, obj,
               float(golden["alpha"]), mode="ref")
    ge = golden["gradE"][k]
    assert abs(r["Lcost"] - golden["Lcost"][k]) <= 1e-12 * abs(golden["Lcost"][k])
    assert abs(r["L0"] - golden["L0_vec"][k][-1]) <= 1e-12 * abs(golden["L0_vec"][k][-1])
    assert np.linalg.norm(r["gradE"] - ge) <= 1e-9 * np.linalg.norm(ge)

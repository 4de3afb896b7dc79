"""CUDA-graph replay of the gradient: the launch sequence captured once per
configuration and replayed with new pulses (written into the device E tables)
gives the same bits as plain launches, for every trajectory store and both
gradient modes, across calls with different pulses and initial states."""
import os

import numpy as np
import pytest

from fkadj import _lib, api, workloads as W

pytestmark = pytest.mark.gpu


def _problem(inst, graphs, **kw):
    old = os.environ.pop("FKADJ_NO_GRAPHS", None)
    if not graphs:
        os.environ["FKADJ_NO_GRAPHS"] = "1"
    try:
        return api.Problem(inst, opts=api.options(**kw))
    finally:
        os.environ.pop("FKADJ_NO_GRAPHS", None)
        if old is not None:
            os.environ["FKADJ_NO_GRAPHS"] = old


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
@pytest.mark.parametrize("ckpt,budget", [(_lib.CKPT_FULL, 0), (_lib.CKPT_SQRT, 0), (_lib.CKPT_BINOMIAL, 6)])
def test_graph_replay_is_bit_identical_to_plain_launches(mode, ckpt, budget):
    inst = W.make_instance(64, 120, seed=81, n_obstacles=5, intervals=12, ncols=80,
                           objective="gradient", alpha=0.1)
    kw = dict(grad_mode=mode, ckpt_policy=ckpt)
    if budget:
        # room for `budget` padded states (72 rows x 136 columns x 3 fields): a
        # binomial schedule with few snapshots
        kw["ckpt_budget_bytes"] = budget * 3 * 8 * 72 * 136
    rng = np.random.default_rng(5)
    pulses = [inst.Et, inst.Et * 0.5 + 0.1, inst.Et + rng.uniform(0, 0.2, inst.Et.size)]
    with _problem(inst, True, **kw) as pg, _problem(inst, False, **kw) as pp:
        for k, E in enumerate(pulses):
            y0 = inst.y0 if k != 1 else None      # the second call re-uses the resident state
            a = pg.grad(E, y0)
            b = pp.grad(E, y0)
            assert np.array_equal(a["gradE"], b["gradE"]), k
            assert a["Lcost"] == b["Lcost"] and a["L0"] == b["L0"]
            if k > 0:  # the first call of the first problem also runs the autotuner's trials
                assert pg.last_launches == pp.last_launches


def test_profiling_and_graph_runs_agree():
    inst = W.make_instance(64, 80, seed=82, n_obstacles=4, intervals=8)
    with api.Problem(inst) as pb:
        a = pb.grad(inst.Et, inst.y0)
        pb.set_profiling(True)                    # sampled events: plain launches
        b = pb.grad(inst.Et)
        pb.set_profiling(False)
        c = pb.grad(inst.Et)                      # replay again
    assert np.array_equal(a["gradE"], b["gradE"]) and np.array_equal(a["gradE"], c["gradE"])


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
@pytest.mark.parametrize("nt", [120, 97])
def test_one_shot_segment_graphs_are_bit_identical(monkeypatch, mode, nt):
    """A gradient that runs as plain launches (here the drop-in call) launches
    each segment of its sqrt store from a graph captured while the GPU runs the
    previous one; the result equals plain launches (FKADJ_SEGMENT_GRAPHS=0)
    bit for bit, with a short last segment too (nt = 97)."""
    inst = W.make_instance(64, nt, seed=82, n_obstacles=5, intervals=12, ncols=80,
                           objective="gradient", alpha=0.1)
    out = {}
    for v in ("0", "1"):
        monkeypatch.setenv("FKADJ_SEGMENT_GRAPHS", v)
        out[v] = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params,
                                opts=api.options(grad_mode=mode, ckpt_policy=_lib.CKPT_SQRT), return_yf=True)
    a, b = out["0"], out["1"]
    assert np.array_equal(a[0], b[0])
    assert a[1] == b[1] and a[2] == b[2]
    assert np.array_equal(a[5][~np.isnan(a[5])], b[5][~np.isnan(b[5])])

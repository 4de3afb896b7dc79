"""Batched execution (fkadj_batch_*): uneven instances in one tick loop give
the same results as the one-shot entry point, and a job's result is the same
alone and in the mix (bit for bit)."""
import numpy as np
import pytest

from fkadj import _lib, api, workloads as W
from fkadj.batch import Batch

pytestmark = pytest.mark.gpu


def _mixed(seed=0):
    specs = [(48, 64, 90), (64, 64, 150), (96, 80, 60), (32, 128, 200), (80, 48, 120)]
    insts = []
    for k, (nr, nc, nt) in enumerate(specs):
        insts.append(W.make_instance(nr, nt, seed=seed * 10 + k, ncols=nc, n_obstacles=4, intervals=10,
                                     objective="gradient" if k % 2 else "mean_u2", alpha=0.05 * k))
    return insts


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
@pytest.mark.parametrize("ckpt", [_lib.CKPT_FULL, _lib.CKPT_SQRT])
def test_batch_matches_one_shot_gradients(mode, ckpt):
    insts = _mixed(1)
    with Batch() as b:
        pids = [b.add_problem(i, grad_mode=mode, ckpt_policy=ckpt) for i in insts]
        jobs = [b.submit(p, i.Et, i.y0) for p, i in zip(pids, insts)]
        b.run()
        res = [b.result(j) for j in jobs]
        assert b.stats["ticks"] > 0
    for inst, r in zip(insts, res):
        g, Lc, L0, LE, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                          inst.nrows, inst.ghost, inst.gamma, inst.S, inst.alpha,
                                          params=inst.params, opts=api.options(grad_mode=mode, ckpt_policy=ckpt))
        assert abs(r["Lcost"] - Lc) <= 1e-12 * abs(Lc)
        assert np.linalg.norm(r["gradE"] - g) <= 1e-12 * np.linalg.norm(g)


def test_result_is_the_same_alone_and_in_the_mix():
    insts = _mixed(2)
    target = insts[1]
    with Batch() as b:
        p = b.add_problem(target)
        alone = b.result((b.submit(p, target.Et, target.y0), b.run())[0])
    with Batch() as b:
        pids = [b.add_problem(i) for i in insts]
        # the others start at different ticks
        jobs = {}
        jobs[1] = b.submit(pids[1], target.Et, target.y0)
        for _ in range(7):
            b.tick()
        jobs[0] = b.submit(pids[0], insts[0].Et, insts[0].y0)
        for _ in range(13):
            b.tick()
        for k in (2, 3, 4):
            jobs[k] = b.submit(pids[k], insts[k].Et, insts[k].y0)
        b.run()
        mixed = b.result(jobs[1])
    assert np.array_equal(alone["gradE"], mixed["gradE"])
    assert alone["Lcost"] == mixed["Lcost"]


def test_objective_only_jobs_and_resident_initial_state():
    inst = _mixed(3)[2]
    with Batch() as b:
        p = b.add_problem(inst)
        j1 = b.submit(p, inst.Et, inst.y0, want_grad=False)
        b.run()
        r1 = b.result(j1)
        j2 = b.submit(p, inst.Et, None, want_grad=False)
        b.run()
        r2 = b.result(j2)
    ref = api.Problem(inst).objective(inst.Et, inst.y0)
    assert r1["Lcost"] == r2["Lcost"]
    assert abs(r1["Lcost"] - ref["Lcost"]) <= 1e-12 * abs(ref["Lcost"])


@pytest.mark.parametrize("mode", [_lib.GRAD_REF, _lib.GRAD_EXACT])
def test_tick_blocks_replayed_as_graphs_give_the_bits_of_single_ticks(monkeypatch, mode):
    """Runs of ticks without host work are planned together and replayed from
    a CUDA graph whose launches read their queues from device headers; the
    results are the bits of one tick at a time (FKADJ_BATCH_GRAPHS=0)."""
    insts = _mixed(4)
    out = {}
    for graphs in ("0", "1"):
        monkeypatch.setenv("FKADJ_BATCH_GRAPHS", graphs)
        with Batch() as b:
            pids = [b.add_problem(i, grad_mode=mode, ckpt_policy=_lib.CKPT_SQRT) for i in insts]
            jobs = [b.submit(p, i.Et, i.y0) for p, i in zip(pids, insts)]
            b.run()
            out[graphs] = ([b.result(j) for j in jobs], b.stats)
    assert out["1"][1]["ticks"] > 0 and out["0"][1]["ticks"] > 0
    for a, c in zip(out["0"][0], out["1"][0]):
        assert np.array_equal(a["gradE"], c["gradE"]) and a["Lcost"] == c["Lcost"]


@pytest.mark.parametrize("path", ["fused", "fused-recompute"])
def test_batched_fused_adjoint_step_matches_the_split_kernels(monkeypatch, path):
    insts = _mixed(5)
    out = {}
    for p in ("split", path):
        monkeypatch.setenv("FKADJ_ADJ_PATH", p)
        with Batch() as b:
            pids = [b.add_problem(i, ckpt_policy=_lib.CKPT_SQRT) for i in insts]
            jobs = [b.submit(q, i.Et, i.y0) for q, i in zip(pids, insts)]
            b.run()
            out[p] = [b.result(j) for j in jobs]
    for a, c in zip(out["split"], out[path]):
        assert np.linalg.norm(c["gradE"] - a["gradE"]) <= 1e-13 * np.linalg.norm(a["gradE"])


def test_presets_set_after_objective_only_ticks(monkeypatch):
    """An objective-only job runs blocks of ticks (replayed from graphs) with
    the engine's first presets (32x32 tiles) before a gradient job arrives and
    the presets are set for it (here by FKADJ_TILES, to 16x16 tiles, as the
    autotuner may do): blocks from then on launch the new presets' kernels,
    whose tiles the queues are cut into.  Both results equal the one-shot ones."""
    monkeypatch.setenv("FKADJ_TILES", "4,4,4,4")
    insts = _mixed(6)
    obj, grad = insts[2], insts[1]
    with Batch() as b:
        po, pg = b.add_problem(obj), b.add_problem(grad)
        jo = b.submit(po, obj.Et, obj.y0, want_grad=False)
        b.tick()
        b.tick()
        jg = b.submit(pg, grad.Et, grad.y0)
        b.run()
        ro, rg = b.result(jo), b.result(jg)
    g, Lc, L0, LE, _ = api.fk_grad_Et(grad.Et, grad.dt, grad.nt, grad.y0, grad.active_index, grad.ncols,
                                      grad.nrows, grad.ghost, grad.gamma, grad.S, grad.alpha, params=grad.params)
    assert abs(rg["Lcost"] - Lc) <= 1e-12 * abs(Lc)
    assert np.linalg.norm(rg["gradE"] - g) <= 1e-12 * np.linalg.norm(g)
    ref = api.Problem(obj).objective(obj.Et, obj.y0)
    assert abs(ro["Lcost"] - ref["Lcost"]) <= 1e-12 * abs(ref["Lcost"])

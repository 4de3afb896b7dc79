"""Serving (fkadj_server_*): requests of different sizes arriving while others
run are admitted and computed together (concurrent single-instance solves on
a pool of streams, or the tick engine's batched launches); each result equals
the one-shot result and is the same alone and in the mix; waits are bounded."""
import threading
import time

import numpy as np
import pytest

from fkadj import _lib, api, workloads as W
from fkadj.serve import Server

pytestmark = pytest.mark.gpu


def _requests(seed):
    specs = [(64, 80, 200, True), (48, 48, 120, False), (96, 64, 90, True), (32, 128, 300, True),
             (80, 80, 60, False), (64, 64, 150, True)]
    return [(W.make_instance(nr, nt, seed=seed + k, ncols=nc, n_obstacles=5, intervals=10,
                             objective="gradient" if k % 2 else "mean_u2", alpha=0.1), g)
            for k, (nr, nc, nt, g) in enumerate(specs)]


@pytest.mark.parametrize("mode", ["streams", "ticks"])
def test_served_results_match_one_shot_and_are_mix_invariant(monkeypatch, mode):
    """Both ways of running admitted requests: concurrent single-instance
    solves on a pool of streams (the default) and the tick engine's batched
    launches (FKADJ_SERVE_MODE=ticks)."""
    monkeypatch.setenv("FKADJ_SERVE_MODE", mode)
    reqs = _requests(300)
    target, _ = reqs[0]
    with Server() as srv:
        rid = srv.submit(target)
        assert srv.wait(rid, 120)
        alone = srv.result(rid)
    with Server() as srv:
        ids = []
        # staggered arrivals from another thread while earlier requests run
        def client():
            for inst, g in reqs[1:]:
                ids.append((srv.submit(inst, want_grad=g), inst, g))
                time.sleep(0.002)
        th = threading.Thread(target=client)
        th.start()
        time.sleep(0.001)
        rid = srv.submit(target)
        th.join()
        assert srv.wait(rid, 120)
        mixed = srv.result(rid)
        results = []
        for r, inst, g in ids:
            assert srv.wait(r, 120)
            results.append((srv.result(r), inst, g))
        st = srv.stats
        assert st["failed"] == 0 and st["completed"] == len(reqs)
    assert np.array_equal(alone["gradE"], mixed["gradE"]) and alone["Lcost"] == mixed["Lcost"]
    for res, inst, g in results:
        if g:
            ref = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                 inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params)
            assert np.linalg.norm(res["gradE"] - ref[0]) <= 1e-12 * np.linalg.norm(ref[0])
            assert abs(res["Lcost"] - ref[1]) <= 1e-12 * abs(ref[1])
        else:
            ref = api.Problem(inst).objective(inst.Et, inst.y0)
            assert abs(res["Lcost"] - ref["Lcost"]) <= 1e-12 * abs(ref["Lcost"])
        assert res["latency_s"] >= res["queue_s"] >= 0


@pytest.mark.parametrize("mode", ["streams", "ticks"])
def test_admission_respects_the_hbm_budget(monkeypatch, mode):
    monkeypatch.setenv("FKADJ_SERVE_MODE", mode)
    reqs = _requests(400)
    # a budget that fits about two of these requests at a time
    with Server(hbm_budget_bytes=25_000_000) as srv:
        ids = [srv.submit(inst, want_grad=g) for inst, g in reqs]
        for r in ids:
            assert srv.wait(r, 120)
        st = srv.stats
        assert st["completed"] == len(reqs)
        assert st["peak_running"] < len(reqs)
        for r in ids:
            srv.result(r)


def test_wait_is_bounded():
    inst = W.make_instance(128, 3000, seed=9, n_obstacles=5)
    with Server() as srv:
        rid = srv.submit(inst)
        t0 = time.perf_counter()
        done = srv.wait(rid, 1e-4)
        assert time.perf_counter() - t0 < 5.0
        assert done in (True, False)
        assert srv.wait(rid, 120)
        srv.result(rid)


def test_served_request_of_each_size_class_matches_the_oracle():
    """One request of each grid side of the served mix (128 .. 1024), submitted
    together so they share the batched launches, against the CPU oracle (a
    short horizon keeps the oracle's 1024^2 run to seconds): Lcost 1e-10 and
    gradE 1e-8 relative."""
    import oracle as O
    sides = (128, 256, 384, 512, 768, 1024)
    insts = [W.make_instance(n, 24, seed=500 + n, n_obstacles=max(1, round(3e-4 * n * n)), intervals=6,
                             wavefronts=4, objective="gradient", alpha=0.1) for n in sides]
    with Server() as srv:
        ids = [srv.submit(inst) for inst in insts]
        res = []
        for rid in ids:
            assert srv.wait(rid, 300)
            res.append(srv.result(rid))
    for inst, r in zip(insts, res):
        o = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
                   inst.active_index, O.Objective(inst.S, inst.gamma), inst.alpha, mode="ref")
        assert abs(r["Lcost"] - o["Lcost"]) <= 1e-10 * abs(o["Lcost"]), inst.nrows
        assert np.linalg.norm(r["gradE"] - o["gradE"]) <= 1e-8 * np.linalg.norm(o["gradE"]), inst.nrows

"""One-shot calls (fkadj_grad / fkadj_forward, the reference's drop-in) keep
their device memory (a per-device pool) and pinned staging for the next call.
Results must not depend on it: two cached calls in a row and a call with the
pool turned off (FKADJ_ONESHOT_POOL=0) give the same bits, and after
fkadj_release_cached_memory the memory is back on the device and the next call
still matches."""
import numpy as np
import pytest

from fkadj import _lib, api, workloads as W

pytestmark = pytest.mark.gpu


def _grad(inst):
    g, Lc, L0, LE, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                      inst.nrows, inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params,
                                      opts=api.options(ckpt_policy=_lib.CKPT_SQRT))
    return np.concatenate([g, [Lc, L0, LE]])


def _forward(inst):
    _, yf, _ = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                 inst.ghost, 0, params=inst.params)
    return yf


def _same(a, b):
    m = np.isnan(a)
    return np.array_equal(m, np.isnan(b)) and np.array_equal(a[~m], b[~m])


def test_cached_one_shot_calls_match_uncached_and_release_returns_memory(monkeypatch):
    import torch
    inst = W.plain_instance(n=128, nt=300, seed=4)
    monkeypatch.delenv("FKADJ_ONESHOT_POOL", raising=False)
    a, b = _grad(inst), _grad(inst)
    fa, fb = _forward(inst), _forward(inst)
    monkeypatch.setenv("FKADJ_ONESHOT_POOL", "0")
    c, fc = _grad(inst), _forward(inst)
    monkeypatch.delenv("FKADJ_ONESHOT_POOL")
    assert np.array_equal(a, b) and np.array_equal(a, c)
    assert _same(fa, fb) and _same(fa, fc)
    torch.cuda.synchronize()
    free_cached, _ = torch.cuda.mem_get_info()
    api.release_cached_memory()
    free_released, _ = torch.cuda.mem_get_info()
    assert free_released > free_cached          # the pool held the last call's buffers
    assert np.array_equal(a, _grad(inst))       # and the next call allocates afresh

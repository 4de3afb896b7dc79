"""Parity on the two standard single-instance workloads, at the horizons the
round-off growth allows (tests/chaos_horizon.py measures them).

  C1  fkadj.workloads.plain_instance(): 128^2, dx 0.025 cm, dt 0.02 ms,
      2000 RK4 steps, 20 holes r~U(0.02, 0.08) cm, one broken wavefront,
      E over 100 intervals, J = mean u(T)^2: the whole horizon.
  C2  fkadj.workloads.large_instance(): 512^2, 200 holes r~U(0.02, 0.1) cm,
      8 broken wavefronts, E over 400 intervals, 20000 steps: the forward
      states over the whole horizon against the reference binary; the gradient
      against the reference binary over its first 2500 steps (the longest its
      int trajectory offset allows) and against the oracle over the first
      C2_HORIZON steps (the oracle's run time).

Each is checked against the reference's own CUDA code compiled here
(oracle/_ref, skipped where absent) and against the CPU oracle: states
1e-10 relative (max-norm), Lcost 1e-10 and gradE 1e-8 relative (2-norm); and
the discrete-exact gradient of C2 against central finite differences
(h = 1e-6) on 10 seeded intervals."""
import copy

import numpy as np
import pytest

import oracle as O
import refbin
from fkadj import _lib, api, workloads as W

pytestmark = pytest.mark.gpu

# steps of the C2 instance the oracle comparisons run for (the oracle's 512^2
# gradient costs about 14 ms per step on 16 cores)
C2_HORIZON = 2000
# the reference binary's gradient addresses its host trajectory with a 32-bit
# int offset, (i+1)*3*n (src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1720, 1871),
# which overflows past 2729 steps at 512^2: its comparison runs to 2500 steps
C2_REF_GRAD_HORIZON = 2500


def _truncate(inst, T):
    """The first T steps of an instance: same geometry, initial state and
    pulse samples Et[0..T]."""
    c = copy.copy(inst)
    c.nt = int(T)
    c.Et = np.ascontiguousarray(inst.Et[:T + 1])
    c.interval_of_sample = inst.interval_of_sample[:T + 1]
    return c


def _rel(a, b):
    m = np.isfinite(b)
    assert np.array_equal(np.isfinite(a), m), "NaN pattern differs"
    return np.abs(a[m] - b[m]).max() / np.abs(b[m]).max()


def _rel2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def c1():
    return W.plain_instance()


@pytest.fixture(scope="module")
def c2():
    return _truncate(W.large_instance(), C2_HORIZON)


def _check_forward(inst, nstep):
    ys, yf, _ = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                  inst.ghost, nstep, params=inst.params)
    ns = api.compute_ns(inst.nt, nstep)
    ys_o, yf_o = O.forward(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid,
                           inst.gh_grid, nstep, ns)
    assert _rel(yf, yf_o) <= 1e-10
    for k in range(ns):
        assert _rel(ys[:, k], ys_o[k]) <= 1e-10
    if refbin.available():
        ys_r, yf_r = refbin.forward(inst.dt, inst.Et, inst.nt, inst.y0, inst.active_index, inst.nrows, inst.ncols,
                                    inst.ghost, nstep, ns)
        assert _rel(yf, yf_r) <= 1e-10
        for k in range(ns):
            assert _rel(ys[:, k], ys_r[k]) <= 1e-10


def _check_gradient(inst):
    g, Lc, L0, LE, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols,
                                      inst.nrows, inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params)
    o = O.grad(inst.params, inst.dt, inst.Et, inst.nt, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
               inst.active_index, O.Objective(inst.S, inst.gamma), inst.alpha, mode="ref")
    assert abs(Lc - o["Lcost"]) <= 1e-10 * abs(o["Lcost"])
    assert _rel2(g, o["gradE"]) <= 1e-8
    if refbin.available():
        r = refbin.grad(inst.dt, inst.Et, inst.nt, inst.y0, inst.active_index, inst.nrows, inst.ncols,
                        inst.ghost, inst.gamma, inst.S, inst.alpha)
        assert abs(Lc - r["Lcost"]) <= 1e-10 * abs(r["Lcost"])
        assert _rel2(g, r["gradE"]) <= 1e-8
        assert _rel2(o["gradE"], r["gradE"]) <= 1e-8


def test_c1_forward_states_over_the_whole_horizon(c1):
    assert (c1.nrows, c1.ncols, c1.nt, len(c1.amplitudes)) == (128, 128, 2000, 100)
    assert (~c1.mask).any()
    _check_forward(c1, 250)


def test_c1_gradient(c1):
    _check_gradient(c1)


def test_c2_forward_states_at_the_parity_horizon(c2):
    assert (c2.nrows, c2.ncols, len(c2.amplitudes)) == (512, 512, 400)
    _check_forward(c2, 500)


def test_c2_gradient_at_the_parity_horizon(c2):
    _check_gradient(c2)


@pytest.mark.skipif(not refbin.available(), reason="oracle/_ref not built")
def test_c2_forward_states_over_the_whole_horizon_against_the_reference_binary():
    """All 20000 steps of C2 against the reference's own CUDA forward: the
    measured round-off growth (tests/chaos_horizon.py: about 0.07 decades per
    1000 steps) keeps the states within 1e-10 at every snapshot."""
    inst = W.large_instance()
    nstep = 5000
    ns = api.compute_ns(inst.nt, nstep)
    ys, yf, _ = api.fk_forward_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                  inst.ghost, nstep, params=inst.params)
    ys_r, yf_r = refbin.forward(inst.dt, inst.Et, inst.nt, inst.y0, inst.active_index, inst.nrows, inst.ncols,
                                inst.ghost, nstep, ns)
    assert _rel(yf, yf_r) <= 1e-10
    for k in range(ns):
        assert _rel(ys[:, k], ys_r[k]) <= 1e-10


@pytest.mark.skipif(not refbin.available(), reason="oracle/_ref not built")
def test_c2_gradient_against_the_reference_binary_at_its_longest_horizon():
    inst = _truncate(W.large_instance(), C2_REF_GRAD_HORIZON)
    g, Lc, _, _, _ = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows,
                                    inst.ghost, inst.gamma, inst.S, inst.alpha, params=inst.params)
    r = refbin.grad(inst.dt, inst.Et, inst.nt, inst.y0, inst.active_index, inst.nrows, inst.ncols, inst.ghost,
                    inst.gamma, inst.S, inst.alpha)
    assert abs(Lc - r["Lcost"]) <= 1e-10 * abs(r["Lcost"])
    assert _rel2(g, r["gradE"]) <= 1e-8


def test_c2_exact_gradient_central_fd_on_10_seeded_intervals(c2):
    """dJ/dA_k of the piecewise-constant amplitudes by central differences
    (h = 1e-6) against dt * sum_{i in k} gradE[i] of the discrete-exact
    gradient, on 10 seeded intervals of those the horizon covers."""
    inst = c2
    amps, iv = inst.amplitudes, inst.interval_of_sample
    opts = api.options(grad_mode=_lib.GRAD_EXACT)
    g = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost,
                       inst.gamma, inst.S, inst.alpha, params=inst.params, opts=opts)[0]
    covered = np.unique(iv)
    dJdA = {int(k): inst.dt * g[iv == k].sum() for k in covered}
    scale = max(abs(v) for v in dJdA.values())
    rng = np.random.default_rng(2025)
    h = 1e-6
    full_nt = len(W.piecewise_constant(20000, amps)[0]) - 1

    def pulse(a):
        return np.ascontiguousarray(W.piecewise_constant(full_nt, a)[0][:inst.nt + 1])

    assert np.array_equal(pulse(amps), inst.Et)
    with api.Problem(inst, opts=opts) as pb:
        for k in rng.choice(covered, size=10, replace=False):
            Ap, Am = amps.copy(), amps.copy()
            Ap[k] += h
            Am[k] -= h
            Jp = pb.objective(pulse(Ap), inst.y0)["Lcost"]
            Jm = pb.objective(pulse(Am), inst.y0)["Lcost"]
            fd = (Jp - Jm) / (2 * h)
            assert abs(fd - dJdA[int(k)]) <= 1e-6 * scale + 1e-5 * abs(fd), (k, fd, dJdA[int(k)])

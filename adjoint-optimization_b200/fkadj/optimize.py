"""Gradient-descent drivers on top of the engine.

``simple_grad_desc`` is the reference's optimisation loop
(src/cuda/simple_grad_desc.m:78-107): each iteration takes
[gradE, Lcost, L0, LE] at the current pulse, records Lcost/L0/LE in
``Lcost_vec``/``L0_vec``/``LE_vec``, hands (Et, gradE) to ``on_save`` every
``nmod`` iterations *before* the update (as the script saves them, :93-101), and
steps ``Et <- Et - ds*gradE`` (:103).  The problem stays resident on the GPU
and later iterations re-use the resident initial state.

``armijo_descent`` optimises the interval amplitudes A of a piecewise-constant
pulse (E = P A) on the energy-penalised cost Lcost = L0/2 + alpha/2 dt sum E^2
with the discrete-exact gradient dLcost/dA_k = dt * sum_{i in k} gradE[i] and a
backtracking (Armijo) line search whose trial step sizes are evaluated together
as one batch of objective-only jobs.
"""
from __future__ import annotations

import numpy as np

from . import _lib, api
from .batch import Batch
from .workloads import piecewise_constant


def simple_grad_desc(inst, ns: int, ds: float, Et=None, nmod: int | None = None, on_save=None, opts=None):
    Et = np.array(inst.Et if Et is None else Et, dtype=np.float64)
    hist = {"Lcost_vec": [], "L0_vec": [], "LE_vec": []}
    gradE = None
    with api.Problem(inst, opts=opts) as pb:
        for i in range(1, ns + 1):
            r = pb.grad(Et, inst.y0 if i == 1 else None)
            gradE = r["gradE"]
            hist["Lcost_vec"].append(r["Lcost"])
            hist["L0_vec"].append(r["L0"])
            hist["LE_vec"].append(r["LE"])
            if nmod and i % nmod == 0 and on_save is not None:
                on_save(i, Et.copy(), gradE.copy(), r["Lcost"],
                        {k: np.array(v[-nmod:]) for k, v in hist.items()})
            Et = Et - ds * gradE
    out = {k: np.array(v) for k, v in hist.items()}
    out.update(Et=Et, gradE=gradE)
    return out


def interval_gradient(gradE_exact, dt, interval_of_sample, K):
    """dLcost/dA_k from the exact-mode gradient ((1/dt) dLcost/dEt)."""
    return dt * np.bincount(interval_of_sample, weights=gradE_exact, minlength=K)


def armijo_descent(inst, iters: int, probes: int = 6, s0: float | None = None, beta: float = 0.5,
                   c1: float = 1e-4, amplitudes=None, grow: float = 2.0, ckpt_policy: int = _lib.CKPT_AUTO,
                   ckpt_budget_bytes: int = 0):
    """Returns dict(A, J (per iteration, at the iterate), step, armijo_ok,
    probes, t_grad / t_probes: wall seconds per iteration of the gradient and
    of the probe batch, device_bytes of the gradient problem)."""
    import time
    K = len(inst.amplitudes)
    A = np.array(inst.amplitudes if amplitudes is None else amplitudes, dtype=np.float64)
    nt = inst.nt
    hist = {"J": [], "step": [], "armijo_ok": [], "probes": [], "t_grad": [], "t_probes": []}
    gopts = api.options(grad_mode=_lib.GRAD_EXACT, ckpt_policy=ckpt_policy, ckpt_budget_bytes=ckpt_budget_bytes)
    with api.Problem(inst, opts=gopts) as pb, Batch() as bt:
        pids = [bt.add_problem(inst) for _ in range(probes)]
        first = True
        for it in range(iters):
            E = piecewise_constant(nt, A)[0]
            t0 = time.perf_counter()
            r = pb.grad(E, inst.y0 if first else None)
            hist["t_grad"].append(time.perf_counter() - t0)
            first = False
            J0 = r["Lcost"]
            g = interval_gradient(r["gradE"], inst.dt, inst.interval_of_sample, K)
            d = -g
            slope = float(g @ d)
            if s0 is None:
                s0 = 0.1 * max(1.0, np.abs(A).max()) / max(np.abs(d).max(), 1e-300)
            steps = [s0 * beta ** k for k in range(probes)]
            t0 = time.perf_counter()
            jobs = [bt.submit(p, piecewise_constant(nt, A + s * d)[0], inst.y0, want_grad=False)
                    for p, s in zip(pids, steps)]
            bt.run()
            Js = [bt.result(j)["Lcost"] for j in jobs]
            hist["t_probes"].append(time.perf_counter() - t0)
            ok = [Jk <= J0 + c1 * s * slope for Jk, s in zip(Js, steps)]
            hist["J"].append(J0)
            hist["probes"].append(list(zip(steps, Js)))
            if any(ok):
                k = ok.index(True)  # largest step that satisfies Armijo
                A = A + steps[k] * d
                hist["step"].append(steps[k])
                hist["armijo_ok"].append(True)
                s0 = steps[k] * grow if k == 0 else steps[k]
            else:
                hist["step"].append(0.0)
                hist["armijo_ok"].append(False)
                s0 = steps[-1] * beta
        device_bytes = pb.device_bytes
    return dict(A=A, J=np.array(hist["J"]), step=np.array(hist["step"]), armijo_ok=hist["armijo_ok"],
                probes=hist["probes"], t_grad=hist["t_grad"], t_probes=hist["t_probes"], device_bytes=device_bytes)

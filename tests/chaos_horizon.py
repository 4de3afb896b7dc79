"""Round-off growth of the FK forward/adjoint on the two standard instances,
and the horizon up to which state and gradient parity can hold.

Test infrastructure (a measurement run by hand on a GPU box; its numbers are
the horizons the parity tests use).  For the 128^2 x 2000-step instance with
20 holes and one broken wavefront (fkadj.workloads.plain_instance) and the
first T steps of the 512^2 x 20000-step instance with 200 holes and 8 broken
wavefronts (large_instance), it measures against T:

  perturbation   libfkadj from y0 and from y0 * (1 + 1e-15 xi), xi ~ N(0, 1)
                 per value: max-norm relative state difference, and the
                 2-norm relative difference of the reference-mode gradient;
  reference      libfkadj against the reference's own CUDA code compiled
                 here (oracle/_ref): the same two differences, which is what
                 the parity tests bound (states 1e-10, gradients 1e-8).

The reference's gradient keeps the whole trajectory in host memory and
addresses it with a 32-bit int offset, (i+1)*3*n doubles
(src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1720 and :1871), which overflows past
2729 steps at 512^2: its horizons are capped (--ref-grad-cap, 2500).  One JSON
line per instance goes to --out (the reference's routines print to stdout).

    python tests/chaos_horizon.py [--which c1,c2] [--c2-steps 20000] [--out FILE]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (os.path.join(ROOT, "adjoint-optimization_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import refbin  # noqa: E402
from fkadj import api, workloads as W  # noqa: E402


OUT = "chaos_horizon.jsonl"


def rel_state(a, b):
    m = np.isfinite(b) & np.isfinite(a)
    return float(np.abs(a[m] - b[m]).max() / np.abs(b[m]).max())


def rel_grad(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def forward_snaps(inst, y0, nt, nstep, ref=False):
    Et = inst.Et[:nt + 1]
    ns = api.compute_ns(nt, nstep)
    if ref:
        ys, yf = refbin.forward(inst.dt, Et, nt, y0, inst.active_index, inst.nrows, inst.ncols, inst.ghost,
                                nstep, ns)
        snaps = [ys[k] for k in range(ns)]
    else:
        ys, yf, _ = api.fk_forward_Et(Et, inst.dt, nt, y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost,
                                      nstep, params=inst.params)
        snaps = [ys[:, k] for k in range(ns)]
    return snaps + [yf]


def grad(inst, y0, nt, ref=False):
    Et = inst.Et[:nt + 1]
    if ref:
        return refbin.grad(inst.dt, Et, nt, y0, inst.active_index, inst.nrows, inst.ncols, inst.ghost,
                           inst.gamma, inst.S, inst.alpha)["gradE"]
    return api.fk_grad_Et(Et, inst.dt, nt, y0, inst.active_index, inst.ncols, inst.nrows, inst.ghost, inst.gamma,
                          inst.S, inst.alpha, params=inst.params)[0]


def growth_rate(ts, errs, floor=1e-14):
    """Least-squares slope of log10(err) against T (decades per 1000 steps)
    over the points above the round-off floor."""
    pts = [(t, math.log10(e)) for t, e in zip(ts, errs) if e > floor]
    if len(pts) < 2:
        return None
    t = np.array([p[0] for p in pts], float)
    y = np.array([p[1] for p in pts], float)
    return float(np.polyfit(t, y, 1)[0] * 1000.0)


def horizon(ts, errs, tol):
    """Last T before the first T whose error exceeds tol (None: never within)."""
    last = None
    for t, e in zip(ts, errs):
        if e > tol:
            break
        last = t
    return last


def measure(name, inst, nt, nstep, grad_ts, ref_grad_cap, seed=11):
    rng = np.random.default_rng(seed)
    y0 = inst.y0
    y0p = y0 * (1.0 + 1e-15 * rng.standard_normal(y0.size))
    ts = [nstep * (k + 1) for k in range(api.compute_ns(nt, nstep))] + [nt]
    a = forward_snaps(inst, y0, nt, nstep)
    b = forward_snaps(inst, y0p, nt, nstep)
    r = forward_snaps(inst, y0, nt, nstep, ref=True)
    pert_state = [rel_state(x, y) for x, y in zip(b, a)]
    ref_state = [rel_state(x, y) for x, y in zip(a, r)]
    gts, pert_grad, ref_grad = [], [], []
    for T in grad_ts:
        if T > nt:
            continue
        g0 = grad(inst, y0, T)
        gts.append(T)
        pert_grad.append(rel_grad(grad(inst, y0p, T), g0))
        ref_grad.append(rel_grad(g0, grad(inst, y0, T, ref=True)) if T <= ref_grad_cap else None)
    rg = [(t, e) for t, e in zip(gts, ref_grad) if e is not None]
    out = {"instance": name, "grid": [inst.nrows, inst.ncols], "nt": nt, "dt_ms": inst.dt,
           "holes_seeded": name, "perturbation": 1e-15,
           "state_T": ts, "state_rel_perturbed": pert_state, "state_rel_vs_reference": ref_state,
           "grad_T": gts, "grad_rel_perturbed": pert_grad, "grad_rel_vs_reference": ref_grad,
           "state_growth_decades_per_1000_steps": growth_rate(ts, pert_state),
           "grad_growth_decades_per_1000_steps": growth_rate(gts, pert_grad),
           "state_horizon_1e-10_vs_reference": horizon(ts, ref_state, 1e-10),
           "grad_horizon_1e-8_vs_reference": horizon([t for t, _ in rg], [e for _, e in rg], 1e-8),
           "state_horizon_1e-10_perturbed": horizon(ts, pert_state, 1e-10),
           "grad_horizon_1e-8_perturbed": horizon(gts, pert_grad, 1e-8)}
    with open(OUT, "a") as f:
        f.write(json.dumps(out) + "\n")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", default="c1,c2")
    ap.add_argument("--c2-steps", type=int, default=20000)
    ap.add_argument("--ref-grad-cap", type=int, default=2500,
                    help="longest horizon of the reference binary's gradient at 512^2 (its int trajectory offset)")
    ap.add_argument("--out", default="chaos_horizon.jsonl")
    a = ap.parse_args()
    global OUT
    OUT = a.out
    which = a.which.split(",")
    if "c1" in which:
        inst = W.plain_instance()
        measure("plain_instance 128^2", inst, inst.nt, 100, [100, 250, 500, 1000, 1500, 2000], 2000)
    if "c2" in which:
        inst = W.large_instance()
        nt = min(a.c2_steps, inst.nt)
        measure("large_instance 512^2", inst, nt, 500,
                [250, 500, 1000, 1500, 2000, 2500, 3000, 4000, 6000, 8000, 12000, 16000, 20000], a.ref_grad_cap)


if __name__ == "__main__":
    main()

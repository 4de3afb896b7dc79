"""Workload measurements beyond the headline bench line (one JSON line each).

  python -m fkadj.suite ckpt   [--n 512 --nt 20000]
      one 512^2 x 20000-step gradient under FULL storage, sqrt checkpoints and
      a binomial schedule within a small budget (device time per gradient)
  python -m fkadj.suite batch  [--count 64 --max-side 1024 --nt-scale 1]
      uneven instances (sides {128..1024}, horizons U{1000..20000} x nt-scale,
      hole density 3e-4, 100-400 intervals): one resident problem at a time vs
      all of them in one batch; gradients/s and makespan
  python -m fkadj.suite serve  [--rates 10,50,200,500 --requests 48 --all-gradients ...]
      Poisson arrivals, half objective-only, half objective+gradient, sizes as
      above: served latency p50/p99 and throughput, against the same stream
      solved one request at a time (FIFO): as plain solves of new instances
      (set-up included) and as warm resident calls.  With --all-gradients and
      --rates inf it runs the 64-instance batched workload through the server,
      whose admission by device footprint lets it hold more instances than
      fit the GPU at once

  python -m fkadj.suite opt   [--n 2048 --nt 100000 --iters 1 --probes 4 --budget-gb 60]
      the optimisation loop at scale: Armijo descent on the interval
      amplitudes of the energy-penalised cost (discrete-exact gradient,
      checkpoints chosen within the HBM budget: binomial at 2048^2 x 1e5),
      trial steps batched; time per gradient and per probe batch, J history

Sizes can be scaled down (max side, horizon scale) to fit a time budget; the
line says which.  Inputs are seeded synthetic instances (fkadj.workloads).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _lib, api, workloads as W
from .batch import Batch
from .serve import Server


def _pct(x, q):
    return float(np.percentile(np.asarray(x), q)) if len(x) else None


def cmd_ckpt(a):
    inst = W.large_instance(n=a.n, nt=a.nt, seed=1)
    out = {"suite": "ckpt", "grid": a.n, "nt": a.nt}
    for name, pol, budget in (("full", _lib.CKPT_FULL, 0), ("sqrt", _lib.CKPT_SQRT, 0),
                              ("binomial", _lib.CKPT_BINOMIAL, a.binomial_gb * 2**30)):
        try:
            with api.Problem(inst, opts=api.options(ckpt_policy=pol, ckpt_budget_bytes=budget)) as pb:
                pb.grad(inst.Et, inst.y0)
                ms = []
                for _ in range(a.steps):
                    pb.grad(inst.Et)
                    ms.append(pb.last_timing["total_ms"])
                out[name] = {"ms_per_gradient": min(ms), "gradients_per_s": 1000.0 / min(ms),
                             "device_bytes": pb.device_bytes, "launches": pb.last_launches}
        except _lib.FkadjError as e:
            out[name] = {"unavailable": str(e)}
    print(json.dumps(out), flush=True)


def _batch_insts(a):
    if getattr(a, "side", 0) > 0:  # `count` instances of one size, each with its own seeded geometry and pulse
        return [W.make_instance(a.side, a.nt, seed=100 + k, n_obstacles=8, intervals=20) for k in range(a.count)]
    return W.batch_instances(count=a.count, seed=a.seed, max_side=a.max_side, nt_scale=a.nt_scale)


def batch_measure(insts):
    """Gradients of `insts` one resident problem at a time (created, warmed,
    timed, freed; the timed call replays the gradient's captured graph) and all
    of them as one batch; wall times and throughputs."""
    cells_steps = sum(i.nrows * i.ncols * i.nt for i in insts)
    seq = 0.0
    for inst in insts:
        with api.Problem(inst, opts=api.options(ckpt_policy=_lib.CKPT_SQRT)) as pb:
            pb.grad(inst.Et, inst.y0)
            pb.grad(inst.Et)
            t0 = time.perf_counter()
            pb.grad(inst.Et)
            seq += time.perf_counter() - t0
    with Batch() as b:
        pids = [b.add_problem(i, ckpt_policy=_lib.CKPT_SQRT) for i in insts]
        jobs = [b.submit(p, i.Et, i.y0) for p, i in zip(pids, insts)]
        b.run()
        [b.result(j) for j in jobs]
        t0 = time.perf_counter()
        jobs = [b.submit(p, i.Et) for p, i in zip(pids, insts)]
        b.run()
        [b.result(j) for j in jobs]
        bt = time.perf_counter() - t0
        st = b.stats
    n = len(insts)
    return {"count": n, "sides": sorted({i.nrows for i in insts}),
            "nt_range": [min(i.nt for i in insts), max(i.nt for i in insts)],
            "sequential_s": seq, "batched_s": bt, "speedup": seq / bt,
            "gradients_per_s_sequential": n / seq, "gradients_per_s_batched": n / bt,
            "cell_steps_per_s_batched": cells_steps / bt, "ticks": st["ticks"], "launches": st["launches"],
            "device_bytes": st["device_bytes"]}


def cmd_batch(a):
    out = batch_measure(_batch_insts(a))
    out.update({"suite": "batch", "max_side": a.max_side, "nt_scale": a.nt_scale, "uniform": getattr(a, "side", 0) > 0})
    print(json.dumps(out), flush=True)


def serve_measure(base, grads, rates, rng):
    """A stream of requests (instances `base`, objective+gradient where
    grads[k]) at each Poisson rate: latency p50/p99 and throughput served by
    the continuous-batching server, against the same arrivals solved one at a
    time in arrival order (FIFO) as plain solves of new instances (problem
    set-up, upload and the call: what a request costs without the server) and
    as warm resident calls (set-up excluded)."""
    # every grid shape tuned first (the autotuner's trials are cached per shape),
    # so that neither side's first request of a shape pays for them
    tuned = set()
    for inst in base:
        if (inst.nrows, inst.ncols) not in tuned:
            tuned.add((inst.nrows, inst.ncols))
            with api.Problem(inst, opts=api.options(ckpt_policy=_lib.CKPT_SQRT)) as pb:
                pb.grad(inst.Et, inst.y0)
    service, service_warm = [], []
    for inst, g in zip(base, grads):
        t0 = time.perf_counter()
        with api.Problem(inst, opts=api.options(ckpt_policy=_lib.CKPT_SQRT)) as pb:
            (pb.grad if g else pb.objective)(inst.Et, inst.y0)
            service.append(time.perf_counter() - t0)
            (pb.grad if g else pb.objective)(inst.Et)   # the gradient's graph is captured here
            t0 = time.perf_counter()
            (pb.grad if g else pb.objective)(inst.Et)
            service_warm.append(time.perf_counter() - t0)
    n = len(base)
    out = []
    for rate in rates:
        gaps = rng.exponential(1.0 / rate, size=n)
        arrive = np.cumsum(gaps) - gaps[0]
        with Server(opts=api.options(ckpt_policy=_lib.CKPT_SQRT)) as srv:
            t0 = time.perf_counter()
            ids = []
            for k, inst in enumerate(base):
                now = time.perf_counter() - t0
                if arrive[k] > now:
                    time.sleep(arrive[k] - now)
                ids.append(srv.submit(inst, want_grad=grads[k]))
            lat = []
            for rid in ids:
                srv.wait(rid, 3600)
                lat.append(srv.result(rid)["latency_s"])
            makespan = time.perf_counter() - t0
            peak = srv.stats["peak_running"]

        def fifo(svc):
            fin, res = 0.0, []
            for k in range(n):
                fin = max(arrive[k], fin) + svc[k]
                res.append(fin - arrive[k])
            return fin, res
        fin, seq_lat = fifo(service)
        fin_w, seq_w = fifo(service_warm)
        out.append({"rate_req_s": rate, "requests": n,
                    "served_p50_s": _pct(lat, 50), "served_p99_s": _pct(lat, 99),
                    "served_throughput_req_s": n / makespan,
                    "sequential_p50_s": _pct(seq_lat, 50), "sequential_p99_s": _pct(seq_lat, 99),
                    "sequential_throughput_req_s": n / fin,
                    "sequential_warm_p50_s": _pct(seq_w, 50), "sequential_warm_p99_s": _pct(seq_w, 99),
                    "sequential_warm_throughput_req_s": n / fin_w, "peak_running": peak})
    return out


def serve_requests(requests, seed, max_side, nt_scale, all_gradients=False):
    """The request mix of the served stream: sizes and horizons as the uneven
    batch (fkadj.workloads.batch_instances), half of them objective+gradient
    (all of them with all_gradients: the batched workload as a request stream)."""
    rng = np.random.default_rng(seed)
    base = _batch_insts(argparse.Namespace(count=requests, seed=seed, max_side=max_side, nt_scale=nt_scale))
    grads = [bool(x) for x in rng.integers(0, 2, size=requests)]
    if all_gradients:
        grads = [True] * requests
    return base, grads, rng


def cmd_serve(a):
    base, grads, rng = serve_requests(a.requests, a.seed, a.max_side, a.nt_scale, a.all_gradients)
    for r in serve_measure(base, grads, a.rates, rng):
        r.update({"suite": "serve", "max_side": a.max_side, "nt_scale": a.nt_scale,
                  "all_gradients": a.all_gradients, "sides": sorted({i.nrows for i in base}),
                  "nt_range": [min(i.nt for i in base), max(i.nt for i in base)],
                  "gradients": int(sum(grads))})
        print(json.dumps(r), flush=True)


def cmd_opt(a):
    from .optimize import armijo_descent
    inst = W.scale_instance(n=a.n, nt=a.nt, alpha=a.alpha)
    t0 = time.perf_counter()
    out = armijo_descent(inst, iters=a.iters, probes=a.probes, ckpt_budget_bytes=int(a.budget_gb * 1e9))
    wall = time.perf_counter() - t0
    state = 3 * (a.n + 72) * (a.n + 72) * 8
    print(json.dumps({"suite": "opt", "grid": a.n, "nt": a.nt, "holes": 3000, "wavefronts": 32, "intervals": 1000,
                      "alpha": a.alpha, "iters": a.iters, "probes": a.probes, "budget_gb": a.budget_gb,
                      "full_store_gb": (a.nt + 1) * state / 1e9, "device_bytes": out["device_bytes"],
                      "J": out["J"].tolist(), "step": out["step"].tolist(), "armijo_ok": out["armijo_ok"],
                      "t_grad_s": out["t_grad"], "t_probes_s": out["t_probes"], "wall_s": wall}), flush=True)


def main(argv=None):
    ap = argparse.ArgumentParser(prog="fkadj.suite")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("ckpt")
    c.add_argument("--n", type=int, default=512)
    c.add_argument("--nt", type=int, default=20000)
    c.add_argument("--steps", type=int, default=2)
    c.add_argument("--binomial-gb", type=float, default=0.5)
    for name in ("batch", "serve"):
        p = sub.add_parser(name)
        p.add_argument("--max-side", type=int, default=1024)
        p.add_argument("--nt-scale", type=float, default=1.0)
        p.add_argument("--seed", type=int, default=2)
        if name == "batch":
            p.add_argument("--count", type=int, default=64)
            p.add_argument("--side", type=int, default=0, help="uniform batch: grid side (0 = uneven mix)")
            p.add_argument("--nt", type=int, default=2000, help="uniform batch: steps")
        else:
            p.add_argument("--requests", type=int, default=48)
            p.add_argument("--rates", type=lambda s: [float(x) for x in s.split(",")], default=[10, 50, 200, 500],
                           help="Poisson arrival rates in req/s; inf = every request at once")
            p.add_argument("--all-gradients", action="store_true",
                           help="every request objective+gradient (the batched workload as a stream)")
    o = sub.add_parser("opt")
    o.add_argument("--n", type=int, default=2048)
    o.add_argument("--nt", type=int, default=100000)
    o.add_argument("--iters", type=int, default=1)
    o.add_argument("--probes", type=int, default=4)
    o.add_argument("--budget-gb", type=float, default=60.0)
    o.add_argument("--alpha", type=float, default=0.05)
    a = ap.parse_args(argv)
    {"ckpt": cmd_ckpt, "batch": cmd_batch, "serve": cmd_serve, "opt": cmd_opt}[a.cmd](a)


if __name__ == "__main__":
    main()

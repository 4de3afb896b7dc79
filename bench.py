#!/usr/bin/env python3
"""Benchmark: forward + adjoint gradients per second at 512^2 on B200.

Workload (one "step" = one gradient): 512 x 512 FK grid (fp64), dx 0.025 cm,
dt 0.02 ms, 20000 RK4 steps, 200 circular holes, 8 broken wavefronts, E(t)
piecewise constant over 400 intervals, J = mean u(T)^2, reference-mode
adjoint with sqrt(nt) checkpoints (142 stored states + 141-state segment
buffer recomputed backward).  Seeded synthetic inputs with the reference's
layouts (the reference publishes no benchmark).

  value   gradients/s with the inputs resident on the device, device time
          (CUDA events on the engine's stream), max over ranks, x ranks
  e2e     the same metric through the drop-in C-ABI call fkadj_grad with host
          buffers (pinned), host<->device copies inside the timed region
  roofline  the dominant kernel's algorithmic bytes (and FP64 flops) / its
          average launch time (CUDA events on the engine stream) against
          MEASURED_PEAKS.json's HBM copy bandwidth (and the FP64 peak); the
          roof with the larger fraction leads the block
  cpu_baseline  the CPU oracle (C, OpenMP, all host cores) on a bounded
          sample of the same workload, scaled to gradients/s

--impl reference times the reference algorithm on the host cores (the CPU
oracle port; the reference's own code runs through MATLAB, absent here), one
bounded sample of the workload per timed step.
Multi-GPU: independent replicas (one instance per rank, no collective on the
data path); torch.distributed/NCCL only for the barrier and the max.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "adjoint-optimization_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "fwd+adjoint gradients/s at 512^2"
UNIT = "gradients/s"

# bytes per dense cell per launch the kernels move as designed (one RK4 step)
BYTES_PER_CELL = {0: 56.0,    # forward step: read y (24) + gh (8), write y (24)
                  1: 160.0,   # adjoint midpoint: read y_{i-1}, y_i (48) + f(y_{i-1}), f(y_i) (48) + gh (8),
                              #   write J(yh) (56; yh itself is not stored while the J(yh) cache is read)
                  2: 249.0}   # adjoint step: read z (24) + J(y_i), J(yh) (112) + y_{i-1} (24) + gh (8)
                              #   + weight code (1), write z (24) + J(y_{i-1}) (56)
# DRAM bytes per cell of one k_fwd_step launch measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, caches flushed before the launch) at 512x512.  The reads
# (33 B/cell: y 24 + gh 8 + halo) reach DRAM; the 24 B/cell of writes stay in the
# 126 MB L2.
FWD_TRAFFIC_PER_CELL = 8654848 / 262144
KERNEL_NAMES = {0: "k_fwd_step", 1: "k_adj_mid", 2: "k_adj_step"}
# fused reference-adjoint step (midpoint + four stages in one launch): read z, y_{i-1}, y_i (72) + kept f(y_{i-1}),
# f(y_i) (48) + gh (8) + weight and stencil codes (2), write z (24); with the J_F(y)^T cache also read J(y_i) and
# write J(y_{i-1}) (56 each)
FUSED_BYTES_PER_CELL = {"fused": 266.0, "fused-recompute": 154.0}
# discrete-exact adjoint step (--mode exact): read lambda (24), y (24), the three stage states (72), gh (8),
# weight code (1); write lambda (24)
EXACT_BYTES_PER_CELL = 153.0
# FP64 flops per vector-field evaluation of the forward step (stage update included), counted by ncu
# (2 x DFMA + DMUL + DADD thread instructions) at 512x512: 585.1 per cell on 64x29 tiles of the
# 64x32/640 preset, whose launch makes 1216384 evaluations (fwd_evaluations)
FWD_FLOPS_PER_EVAL = 585.1 * 262144 / 1216384
# the same capture's FP64 pipe activity (sm__pipe_fp64_cycles_active, % of active cycles) and launch duration:
# DMUL, DADD and compare instructions occupy the pipe as a DFMA does, so the pipe is busier than the flop rate
# says; scaled to the live launch time it estimates the pipe's activity in the replayed graph
FWD_FP64_PIPE_NCU = (0.400, 0.019936)  # (fraction, ms of the serialised launch)


def fwd_evaluations(nrows, ncols, tx, ty):
    """Vector-field evaluations of one forward-step launch: stage s of a tile
    runs on the tile grown by 4 - s cells (temporal blocking); bottom-row tiles
    stop at the grid's edge."""
    n = 0
    for i0 in range(0, nrows, ty):
        rows = min(ty, nrows - i0)
        per = sum((tx + 2 * e) * (rows + 2 * e) for e in range(4))
        n += per * ((ncols + tx - 1) // tx)
    return n


def peaks():
    """HBM copy bandwidth (GB/s) for the roofline: MEASURED_PEAKS.json's when
    present (its first numeric entry whose key names HBM, searched depth-first;
    "hbm_gbs" preferred), else the pool's earlier measurement, 6.65 TB/s."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
    except (OSError, ValueError):
        return 6650.0, "fallback"

    def find(x):
        if isinstance(x, dict):
            if isinstance(x.get("hbm_gbs"), (int, float)):
                return float(x["hbm_gbs"])
            for k, v in x.items():
                if "hbm" in str(k).lower() and isinstance(v, (int, float)) and not isinstance(v, bool):
                    return float(v)
            for v in x.values():
                r = find(v)
                if r is not None:
                    return r
        return None

    v = find(d)
    return (v, "measured") if v and v > 0 else (6650.0, "fallback")


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def binding_roof(roof):
    """The roofline block led by the roof the kernel is nearer to: the HBM
    fraction (algorithmic bytes / copy bandwidth) and the FP64 fraction (flops /
    nominal FP64 peak) are both measured on the same launches; the larger one
    binds and takes the top-level fields, the other stays as a sub-block."""
    fp = roof.get("fp64")
    if not fp or fp["kernel"] != roof["kernel"] or fp["frac"] <= roof["frac"]:
        return roof
    hbm = {k: roof[k] for k in ("kernel", "achieved", "peak", "unit", "frac", "peak_source", "traffic",
                                "bytes_per_launch", "avg_launch_ms") if k in roof}
    out = {k: v for k, v in roof.items() if k not in hbm and k != "fp64"}
    out.update({"bound": "fp64", "kernel": fp["kernel"], "achieved": fp["achieved"], "peak": fp["peak"],
                "unit": fp["unit"], "frac": fp["frac"], "peak_source": fp["peak_source"],
                "traffic": roof.get("traffic"), "flops_per_launch": fp["flops_per_launch"],
                "avg_launch_ms": fp["avg_launch_ms"], "flops_source": fp["flops_source"], "hbm": hbm})
    if "traffic_source" in roof:
        out["traffic_source"] = roof["traffic_source"]
    return out


def workload(args):
    from fkadj import workloads as W
    inst = W.large_instance(n=args.n, nt=args.nt, seed=1)
    return inst


def workload_config(args, inst, ckpt):
    return {"workload": f"FK {args.n}x{args.n} fp64, {args.nt} RK4 steps, 200 holes, 8 wavefronts, "
                        f"400 E intervals, J=mean u^2, {args.mode}-mode adjoint, {ckpt} checkpoints",
            "grid": [args.n, args.n], "nt": args.nt, "dt_ms": inst.dt, "dx_cm": inst.dx,
            "active_cells": inst.n_num, "checkpoint": ckpt, "grad_mode": args.mode,
            "l2": "working set larger than L2 (checkpoint + segment store > 1 GB per gradient)",
            "parallelism": f"replicas x{args.gpus}"}


def cpu_sample(args, inst, steps=None):
    """CPU oracle (reference algorithm, FP64, OpenMP on all host cores) on a
    bounded sample: the same grid for args.cpu_steps steps (about 10 s on 16
    cores), scaled to nt."""
    import numpy as np
    import oracle as O
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    nts = steps or args.cpu_steps
    Et = np.ascontiguousarray(inst.Et[:nts + 1])
    obj = O.Objective(inst.S, inst.gamma)
    t0 = time.perf_counter()
    O.grad(inst.params, inst.dt, Et, nts, inst.nrows, inst.ncols, inst.y0_grid, inst.gh_grid,
           inst.active_index, obj, inst.alpha, mode="ref")
    dt = time.perf_counter() - t0
    per_grad = dt * inst.nt / nts
    return {"value": 1.0 / per_grad, "unit": UNIT, "cores": O.threads(), "kind": "port", "sample_s": dt,
            "sample": f"{inst.nrows}x{inst.ncols} grid, {nts} fwd+adjoint steps ({dt:.1f} s) scaled to "
                      f"{inst.nt} steps; C oracle, OpenMP"}


def run_reference(args):
    """The reference algorithm on the host cores.  Each of the K timed steps is
    one bounded sample of the workload: args.ref_sample_steps of its nt RK4
    steps, forward then adjoint, on the same grid (the full 20000-step gradient
    takes about five minutes on 16 cores).  ms_per_step is the wall time of one
    sample, so steps x ms_per_step is the timed run; value scales each sample to
    whole gradients (per-step cost does not depend on the horizon)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    inst = workload(args)
    for _ in range(args.warmup):
        cpu_sample(args, inst, steps=4)  # untimed: pages the oracle and its buffers in
    samples = [cpu_sample(args, inst, steps=args.ref_sample_steps) for _ in range(max(1, args.steps))]
    sample_s = [x["sample_s"] for x in samples]
    per_sample = statistics.median(sample_s)
    v = statistics.median([x["value"] for x in samples])
    cb = dict(samples[0])
    cb["value"] = v
    cb.pop("sample_s", None)
    config = workload_config(args, inst, "full (host)")
    config["timed_step"] = (f"one sample of {args.ref_sample_steps} of the {inst.nt} RK4 steps (forward + "
                            f"adjoint), scaled to whole gradients")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": len(samples), "warmup": args.warmup, "ms_per_step": 1000.0 * per_sample,
            "sample_steps": args.ref_sample_steps, "extrapolated_to": inst.nt,
            "timed_s": sum(sample_s), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config, "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


class Ranks:
    """One process per GPU (torchrun environment): instances are replicas, so
    the only collectives are the barrier around the timed region and the max
    of the per-rank times.  backend "nccl" on GPUs, "gloo" for the CPU tests."""

    def __init__(self, backend="nccl", timeout_s=300):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def gmax(self, x):
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def replica_value(world, steps, ms_max):
    """Whole-job throughput: every rank runs `steps` gradients of its own
    replica; the job takes the slowest rank's time."""
    return world * steps / (ms_max / 1000.0)


def run_ours(args):
    import numpy as np
    import torch
    from fkadj import _lib, api

    ranks = Ranks("nccl")
    rank, world, local = ranks.rank, ranks.world, ranks.local
    torch.cuda.set_device(local)
    barrier, gmax = ranks.barrier, ranks.gmax

    inst = workload(args)
    ckpt = {"sqrt": _lib.CKPT_SQRT, "full": _lib.CKPT_FULL, "auto": _lib.CKPT_AUTO}[args.ckpt]
    stream = torch.cuda.Stream()
    gmode = _lib.GRAD_EXACT if args.mode == "exact" else _lib.GRAD_REF
    opts = api.options(ckpt_policy=ckpt, stream=stream.cuda_stream, device=local, tile=args.tile, grad_mode=gmode)
    pb = api.Problem(inst, opts=opts)
    Et = np.ascontiguousarray(inst.Et)
    pb.grad(Et, inst.y0)                     # uploads the initial state (resident afterwards)
    for _ in range(max(0, args.warmup - 1)):
        pb.grad(Et)
    launches = 0
    clk = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        pb.grad(Et)
        launches += pb.last_launches
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    ms = gmax(ev0.elapsed_time(ev1))
    value = replica_value(world, args.steps, ms)
    # the last timed gradient's forward sweep: CUDA events on the engine stream around its nt back-to-back
    # k_fwd_step launches (recorded inside the replayed graph)
    fwd_sweep_ms = pb.last_timing["fwd_ms"]

    # roofline: sampled per-kernel device times in one more gradient
    pb.set_profiling(True)
    pb.grad(Et)
    pb.set_profiling(False)
    recompute = 0 if args.ckpt == "full" else inst.nt - (inst.nt + pb_stride(inst.nt) - 1) // pb_stride(inst.nt)
    names, nbytes = dict(KERNEL_NAMES), dict(BYTES_PER_CELL)
    if args.mode == "exact":
        # forward sweep + recompute + one stage replay per backward step; the
        # discrete adjoint step in the adjoint slot; no midpoint kernel
        per_grad = {0: 2 * inst.nt + recompute, 2: inst.nt}
        names[2], nbytes[2] = "k_adj_exact", EXACT_BYTES_PER_CELL
    else:
        per_grad = {0: inst.nt + recompute, 1: inst.nt, 2: inst.nt}
        adj = pb.adjoint_kernel
        if adj["path"] != "split":  # one fused launch per backward step: no midpoint kernel
            per_grad = {0: inst.nt + recompute, 2: inst.nt}
            names[2], nbytes[2] = "k_adj_fused", FUSED_BYTES_PER_CELL[adj["path"]]
    kt = {k: pb.kernel_time(k) for k in per_grad}
    tiles = pb.tiles
    share = {k: kt[k][0] * per_grad[k] for k in kt}
    dom = max(share, key=share.get)
    cells = inst.nrows * inst.ncols
    # the dominant kernel's live average launch: for the forward step, its sweep in the timed region / nt;
    # otherwise the sampled launches of the profiling gradient (each bracketed by its own events, which
    # adds the gap a graph replay hides: an upper bound)
    fwd_live_ms = fwd_sweep_ms / inst.nt
    avg_ms, avg_src = ((fwd_live_ms, "forward sweep of the last timed gradient / nt (CUDA events)") if dom == 0
                       else (kt[dom][0], "sampled launches, each bracketed by CUDA events"))
    achieved = nbytes[dom] * cells / (avg_ms / 1000.0) / 1e9
    peak, peak_kind = peaks()
    roof = {"bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": peak_kind, "traffic": args.traffic,
            "bytes_per_launch": nbytes[dom] * cells, "avg_launch_ms": avg_ms, "avg_launch_source": avg_src,
            "samples": kt[dom][1],
            "kernel_ms_bracketed": {names[k]: kt[k][0] for k in kt},
            "time_share": {names[k]: share[k] / sum(share.values()) for k in share},
            "tiles": {k: list(v) for k, v in tiles.items()
                      if (k == "adj_exact") == (args.mode == "exact") or k == "fwd_step"},
            "adjoint_path": pb.adjoint_kernel,
            "note": "FP64 bound: a vector-field evaluation costs 2 exp (table-driven, 11 FP64 "
                    "instructions each), 4 reciprocals (estimate + one cubic refinement) and ~50 "
                    "FMA-class operations, 126 FP64 flops, 4.6 evaluations per cell-step; the HBM fraction "
                    "is reported against the copy peak"}
    # the forward step against the FP64 roof (the bound it is nearer to)
    ftx, fty, _ = tiles["fwd_step"]
    fl = FWD_FLOPS_PER_EVAL * fwd_evaluations(inst.nrows, inst.ncols, ftx, fty)
    mhz = clocks.get("sm_mhz") or 1965.0
    fpeak = 148 * 128 * mhz * 1e6 / 1e12
    roof["fp64"] = {"kernel": "k_fwd_step", "achieved": fl / (fwd_live_ms / 1000.0) / 1e12, "peak": fpeak,
                    "unit": "TFLOP/s", "frac": fl / (fwd_live_ms / 1000.0) / 1e12 / fpeak, "avg_launch_ms": fwd_live_ms,
                    "flops_per_launch": fl, "peak_source": "148 SMs x 64 DFMA/clock x 2 at the sampled SM clock",
                    "flops_source": "ncu-counted FP64 instructions per evaluation at 512x512"}
    if inst.nrows == 512 and inst.ncols == 512 and (ftx, fty) == (64, 29):
        frac_ncu, ms_ncu = FWD_FP64_PIPE_NCU
        roof["fp64"]["pipe_active"] = {
            "ncu": frac_ncu, "ncu_launch_ms": ms_ncu, "live_estimate": min(1.0, frac_ncu * ms_ncu / fwd_live_ms),
            "what": "FP64 pipe busy fraction: ncu capture of one serialised launch of the same preset, and that "
                    "scaled to the live launch time"}
    if roof["traffic"] is None and dom == 0 and FWD_TRAFFIC_PER_CELL:
        roof["traffic"] = FWD_TRAFFIC_PER_CELL * cells
        roof["traffic_source"] = "ncu capture of one k_fwd_step launch at 512x512 (dram read + write)"
    roof = binding_roof(roof)
    sqrt_bytes = pb.device_bytes
    pb.close()

    # the other trajectory store of the configuration: the full trajectory on the device
    full = None
    if not args.no_full and args.ckpt != "full" and world == 1:
        try:
            fopts = api.options(ckpt_policy=_lib.CKPT_FULL, stream=stream.cuda_stream, device=local, tile=args.tile,
                                grad_mode=gmode)
            with api.Problem(inst, opts=fopts) as pf:
                pf.grad(Et, inst.y0)
                pf.grad(Et)  # the second call captures the gradient's graph: outside the timed region
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(args.full_steps):
                    pf.grad(Et)
                e1.record(stream)
                torch.cuda.synchronize()
                fms = e0.elapsed_time(e1) / args.full_steps
                full = {"value": 1000.0 / fms, "unit": UNIT, "ms_per_step": fms, "steps": args.full_steps,
                        "device_bytes": pf.device_bytes, "sqrt_device_bytes": sqrt_bytes}
        except _lib.FkadjError as e:
            full = {"unavailable": str(e)}

    # the same gradient with the store AUTO picks within the default budget (60% of free memory)
    auto = None
    if not args.no_auto and args.ckpt != "auto" and world == 1:
        try:
            aopts = api.options(ckpt_policy=_lib.CKPT_AUTO, stream=stream.cuda_stream, device=local, tile=args.tile,
                                grad_mode=gmode)
            with api.Problem(inst, opts=aopts) as pa:
                pa.grad(Et, inst.y0)
                pa.grad(Et)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record(stream)
                for _ in range(args.full_steps):
                    pa.grad(Et)
                e1.record(stream)
                torch.cuda.synchronize()
                ams = e0.elapsed_time(e1) / args.full_steps
                auto = {"value": 1000.0 / ams, "unit": UNIT, "ms_per_step": ams, "steps": args.full_steps,
                        "device_bytes": pa.device_bytes, **pa.last_plan}
        except _lib.FkadjError as e:
            auto = {"unavailable": str(e)}

    # e2e through the drop-in C ABI (fkadj_grad), host buffers in pinned memory
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    Et_h, y0_h = pin(inst.Et), pin(inst.y0)
    ai_h, gh_h = pin(inst.active_index.astype(np.int32)), pin(inst.ghost.astype(np.float64))
    import scipy.sparse as sp
    S = sp.csc_matrix(inst.S)
    h2d = Et_h.nbytes + y0_h.nbytes + ai_h.nbytes + gh_h.nbytes + 24 + S.indptr.size * 8 + S.indices.size * 8 \
        + S.data.size * 8
    d2h = (inst.nt + 1) * 8 + 3 * 8
    eopts = api.options(ckpt_policy=ckpt, device=local, tile=args.tile, grad_mode=gmode)
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    # one untimed call first, as every timed loop here has warm-up steps: a
    # process's first drop-in call also grows the one-shot memory pool and the
    # pinned staging (measured 50-270 ms more than the steady calls)
    api.fk_grad_Et(Et_h, inst.dt, inst.nt, y0_h, ai_h, inst.ncols, inst.nrows, gh_h, inst.gamma, S, inst.alpha,
                   params=inst.params, opts=eopts)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        api.fk_grad_Et(Et_h, inst.dt, inst.nt, y0_h, ai_h, inst.ncols, inst.nrows, gh_h, inst.gamma, S,
                       inst.alpha, params=inst.params, opts=eopts)
    torch.cuda.synchronize()
    e2e_s = gmax(time.perf_counter() - t0)
    e2e = {"value": replica_value(world, e2e_steps, e2e_s * 1000.0), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
           "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
           "path": "fkadj_grad (drop-in for fk_grad_Et_comp), one call per gradient incl. device setup, "
                   "after one untimed call"}

    # the metric's second half: served p50/p99 against plain solves, and the
    # batched uneven instances, at a stated scale-down of their workloads
    served = plain = batched = None
    if rank == 0 and world == 1 and not args.no_serve:
        served, plain, batched = serve_and_batch(args)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(args, inst)
        cpu.pop("sample_s", None)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(args, inst, args.ckpt), "roofline": roof, "cpu_baseline": cpu,
                "e2e": e2e, "gpu_launches": launches, "clocks": clocks}
        if full is not None:
            line["full_storage"] = full
        if auto is not None:
            line["auto_store"] = auto
        if served is not None:
            line["served"], line["plain_solve"], line["batched"] = served, plain, batched
        print(json.dumps(line), flush=True)
    ranks.close()
    return 0


def serve_and_batch(args):
    """Served stream and batched uneven instances (scaled down from the
    standard 128-1024 sides and 1000-20000 steps so the bench stays within
    minutes; the keys say how)."""
    import numpy as np
    from fkadj import suite
    from fkadj import workloads as W
    base, grads, rng = suite.serve_requests(args.serve_requests, 7, args.serve_max_side, args.serve_nt_scale)
    rows = suite.serve_measure(base, grads, args.serve_rates, rng)
    mix = {"requests": args.serve_requests, "objective_and_gradient": int(sum(grads)),
           "sides": sorted({i.nrows for i in base}), "nt_range": [min(i.nt for i in base), max(i.nt for i in base)],
           "arrivals": "Poisson", "scale": f"sides <= {args.serve_max_side}, horizons x{args.serve_nt_scale} of "
                                           f"the 128-1024 / 1000-20000-step mix", "timer": "host wall clock"}
    served = dict(mix, rates=[{"rate_req_s": r["rate_req_s"], "p50_s": r["served_p50_s"], "p99_s": r["served_p99_s"],
                               "throughput_req_s": r["served_throughput_req_s"], "peak_running": r["peak_running"]}
                              for r in rows])
    plain = dict(mix, what="the same arrivals solved one at a time in arrival order, each a plain "
                           "single-instance solve of a new problem (set-up, upload, call)",
                 rates=[{"rate_req_s": r["rate_req_s"], "p50_s": r["sequential_p50_s"], "p99_s": r["sequential_p99_s"],
                         "throughput_req_s": r["sequential_throughput_req_s"],
                         "warm_p50_s": r["sequential_warm_p50_s"], "warm_p99_s": r["sequential_warm_p99_s"]}
                        for r in rows])
    insts = W.batch_instances(count=args.batch_count, seed=2, max_side=args.serve_max_side,
                              nt_scale=args.serve_nt_scale)
    ticks = suite.batch_measure(insts)
    # the same gradients as one burst of requests to the server: its workers run
    # them concurrently through the single-instance path, one stream each
    stream_rows = suite.serve_measure(insts, [True] * len(insts), [float("inf")], np.random.default_rng(3))
    r = stream_rows[0]
    streams = {"gradients_per_s": len(insts) / (len(insts) / r["served_throughput_req_s"]),
               "makespan_s": len(insts) / r["served_throughput_req_s"],
               "speedup": r["served_throughput_req_s"] / r["sequential_warm_throughput_req_s"],
               "sequential_warm_gradients_per_s": r["sequential_warm_throughput_req_s"],
               "what": "every gradient submitted at once to the server (concurrent single-instance solves, one "
                       "stream each, admission by device footprint)"}
    ticks["what"] = "one BatchEngine: every tick's steps of all jobs in one persistent launch per kernel kind"
    best = max((streams, ticks), key=lambda x: x["speedup"])
    batched = {"count": len(insts), "sides": ticks["sides"], "nt_range": ticks["nt_range"],
               "scale": (f"{args.batch_count} of the 64 uneven instances, sides <= {args.serve_max_side}, "
                         f"horizons x{args.serve_nt_scale}"),
               "sequential": "one resident problem at a time, each gradient a replayed graph",
               "speedup": best["speedup"], "streams": streams, "persistent_kernels": ticks}
    return served, plain, batched


def pb_stride(nt):
    import math
    return max(2, int(math.ceil(math.sqrt(nt))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="fkadj", choices=["fkadj", "reference"])
    ap.add_argument("--n", type=int, default=512)
    ap.add_argument("--nt", type=int, default=20000)
    ap.add_argument("--ckpt", default="sqrt", choices=["sqrt", "full", "auto"])
    ap.add_argument("--mode", default="ref", choices=["ref", "exact"],
                    help="gradient mode: the reference's continuous adjoint (the headline) or the discrete-exact one")
    ap.add_argument("--tile", type=int, default=0)
    ap.add_argument("--cpu-steps", type=int, default=600)
    ap.add_argument("--ref-sample-steps", type=int, default=300,
                    help="reference arm: RK4 steps (forward + adjoint) timed per step of the run")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-full", action="store_true", help="skip the full-trajectory comparison")
    ap.add_argument("--full-steps", type=int, default=2)
    ap.add_argument("--no-auto", action="store_true", help="skip the AUTO-store comparison")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream and batched measurements")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-rates", type=lambda x: [float(v) for v in x.split(",")], default=[10.0, 50.0, 200.0])
    ap.add_argument("--serve-max-side", type=int, default=512)
    ap.add_argument("--serve-nt-scale", type=float, default=0.1)
    ap.add_argument("--batch-count", type=int, default=16)
    ap.add_argument("--traffic", type=float, default=None,
                    help="ncu dram bytes per launch of the dominant kernel, if captured")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

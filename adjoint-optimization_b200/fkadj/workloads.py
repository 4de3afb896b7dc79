"""Seeded synthetic FK problem instances.

The reference ships one pre-evolved 256^2 state (src/cuda/data/spirals.mat)
and no generator.  The instances here use the reference's layouts (compact
[u;v;w] states, 1-based ``active_index``, ``ghost_lr`` per active cell, one
E sample per step) with the sizes of the standard workloads:

* ``plain_instance``   128^2, dx 0.025 cm, dt 0.02 ms, 2000 steps,
                       20 circular holes r~U(0.02,0.08) cm, broken-wavefront
                       IC (u=1 lower-left quadrant, v=0 upper half, w=1,
                       N(0,0.01) noise), E piecewise constant over 100
                       intervals with amplitudes U(0,1), J = mean u(T)^2;
* ``large_instance``   512^2, 20000 steps, 200 holes r~U(0.02,0.1) cm,
                       8 random broken wavefronts, 400 intervals;
* ``batch_instances``  uneven sides {128..1024}, horizons U{1000..20000},
                       hole density 3e-4 per cell, 100-400 intervals;
* ``scale_instance``   2048^2, 1e5 steps, 3000 holes, 32 wavefronts,
                       1000 intervals (energy-penalised objective).
Every field has its own ``numpy.random.default_rng`` stream derived from the
instance seed, so geometry, IC and pulse are reproducible independently.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from . import geometry as G
from .params import FkParams


@dataclass
class Instance:
    nrows: int
    ncols: int
    dx: float
    dt: float
    nt: int
    params: FkParams
    mask: np.ndarray
    active_index: np.ndarray
    ghost: np.ndarray
    y0: np.ndarray            # compact [u;v;w]
    Et: np.ndarray            # nt+1 samples, Et[i] at t = i*dt
    amplitudes: np.ndarray    # piecewise-constant interval amplitudes
    interval_of_sample: np.ndarray
    S: sp.csc_matrix
    gamma: np.ndarray
    alpha: float
    seed: int
    name: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return self.nrows * self.ncols

    @property
    def n_num(self) -> int:
        return int(self.mask.sum())

    @property
    def y0_grid(self) -> np.ndarray:
        return G.nan_grid(self.y0, self.active_index)

    @property
    def gh_grid(self) -> np.ndarray:
        return G.gh_grid(self.ghost, self.active_index, self.params.Du, self.params.h)

    def with_Et(self, Et: np.ndarray) -> "Instance":
        import copy
        c = copy.copy(self)
        c.Et = np.ascontiguousarray(Et, dtype=np.float64)
        return c


def _streams(seed: int):
    ss = np.random.SeedSequence(seed)
    g, ic, e = ss.spawn(3)
    return np.random.default_rng(g), np.random.default_rng(ic), np.random.default_rng(e)


def piecewise_constant(nt: int, amplitudes: np.ndarray):
    """Samples Et[0..nt] of a pulse constant on len(amplitudes) equal intervals."""
    K = len(amplitudes)
    idx = np.minimum((np.arange(nt + 1) * K) // nt, K - 1)
    return np.asarray(amplitudes, dtype=np.float64)[idx], idx


def broken_wavefront_ic(mask, rng):
    nr, nc = mask.shape
    u = np.zeros((nr, nc))
    v = np.ones((nr, nc))
    w = np.ones((nr, nc))
    u[nr // 2:, :nc // 2] = 1.0      # excited lower-left quadrant
    v[:nr // 2, :] = 0.0             # refractory block, upper half
    for f in (u, v, w):
        f += rng.normal(0.0, 0.01, size=f.shape)
    return u, v, w


def multi_wavefront_ic(mask, rng, count: int):
    """``count`` random broken wavefronts: an excited band (u=1) with a
    refractory band (v=0) behind it, cut off at a free end."""
    nr, nc = mask.shape
    u = np.zeros((nr, nc))
    v = np.ones((nr, nc))
    w = np.ones((nr, nc))
    I, J = np.meshgrid(np.arange(nr), np.arange(nc), indexing="ij")
    width = max(3.0, 0.02 * min(nr, nc))
    for _ in range(count):
        ci, cj = rng.uniform(0, nr), rng.uniform(0, nc)
        th = rng.uniform(0, 2 * np.pi)
        length = rng.uniform(0.15, 0.4) * min(nr, nc)
        ti, tj = np.cos(th), np.sin(th)
        along = (I - ci) * ti + (J - cj) * tj
        across = -(I - ci) * tj + (J - cj) * ti
        seg = (along >= 0) & (along <= length)
        front = seg & (across >= 0) & (across < width)
        back = seg & (across < 0) & (across > -2.5 * width)
        u[front] = 1.0
        v[front] = 1.0
        v[back] = 0.0
        u[back] = 0.0
    for f in (u, v, w):
        f += rng.normal(0.0, 0.01, size=f.shape)
    return u, v, w


def make_instance(n, nt, *, dx=0.025, dt=0.02, n_obstacles=20, r_range=(0.02, 0.08),
                  intervals=100, wavefronts=0, seed=0, objective="mean_u2", alpha=0.0,
                  name="", ncols=None) -> Instance:
    nr, nc = int(n), int(ncols if ncols is not None else n)
    rg, ric, re = _streams(seed)
    centres = np.stack([rg.uniform(0, nr * dx, n_obstacles), rg.uniform(0, nc * dx, n_obstacles)], 1)
    radii = rg.uniform(r_range[0], r_range[1], n_obstacles)
    mask = G.circles_mask(nr, nc, dx, centres, radii)
    ai = G.active_index(mask)
    ghost = G.ghost_lr(mask)
    if wavefronts:
        u, v, w = multi_wavefront_ic(mask, ric, wavefronts)
    else:
        u, v, w = broken_wavefront_ic(mask, ric)
    y0 = np.concatenate([f[mask] for f in (u, v, w)])
    amps = re.uniform(0.0, 1.0, intervals)
    Et, iv = piecewise_constant(nt, amps)
    n_num = int(mask.sum())
    if objective == "mean_u2":
        S = G.mean_square_matrix(n_num)
        gamma = np.array([1.0, 0.0, 0.0])
    elif objective == "gradient":
        S = G.objective_matrix(mask)
        gamma = np.array([1.0, 0.2, 0.2])
    else:
        raise ValueError(objective)
    return Instance(nr, nc, dx, dt, nt, FkParams().with_h(dx), mask, ai, ghost, y0, Et, amps, iv,
                    S, gamma, float(alpha), int(seed), name)


def plain_instance(n=128, nt=2000, seed=0, n_obstacles=20, intervals=100, **kw) -> Instance:
    """128^2 x 2000 steps, 20 holes, one broken wavefront, J = mean u^2."""
    return make_instance(n, nt, n_obstacles=n_obstacles, intervals=intervals, seed=seed,
                         name=kw.pop("name", "plain128"), **kw)


def large_instance(n=512, nt=20000, seed=1, **kw) -> Instance:
    """512^2 x 20000 steps, 200 holes r~U(0.02,0.1), 8 wavefronts, 400 intervals."""
    kw.setdefault("n_obstacles", 200)
    kw.setdefault("r_range", (0.02, 0.1))
    kw.setdefault("intervals", 400)
    kw.setdefault("wavefronts", 8)
    return make_instance(n, nt, seed=seed, name=kw.pop("name", "large512"), **kw)


def batch_instances(count=64, seed=2, sides=(128, 256, 384, 512, 768, 1024),
                    nt_range=(1000, 20000), density=3e-4, max_side=None, nt_scale=1.0):
    """Uneven instances; ``max_side``/``nt_scale`` shrink them for tests."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(count):
        side = int(rng.choice(sides))
        if max_side:
            side = min(side, max_side)
        nt = max(4, int(round(int(rng.integers(nt_range[0], nt_range[1] + 1)) * nt_scale)))
        K = int(rng.integers(100, 401))
        K = min(K, nt)
        nob = max(1, int(round(density * side * side)))
        out.append(make_instance(side, nt, n_obstacles=nob, intervals=K, wavefronts=4,
                                 seed=seed * 100003 + b, name=f"batch{b}"))
    return out


def scale_instance(n=2048, nt=100000, seed=5, **kw) -> Instance:
    """2048^2 x 1e5 steps, 3000 holes, 32 wavefronts, 1000 intervals."""
    kw.setdefault("n_obstacles", 3000)
    kw.setdefault("intervals", 1000)
    kw.setdefault("wavefronts", 32)
    return make_instance(n, nt, seed=seed, name=kw.pop("name", "scale2048"), **kw)

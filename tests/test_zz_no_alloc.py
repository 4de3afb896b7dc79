"""The no-allocation z.gh entry point, fkadj_zgh_dot_noalloc, checked through
the C ABI against the existing gradient entry point fkadj_grad.

Some callers cannot allocate device memory: their GPU memory belongs to
another allocator or to a pool reserved up front (an extra cudaMalloc fails
or synchronises the device), or they must not call cudaMalloc/cudaFree inside
a timed loop.  For them this entry point keeps its partial sums in a fixed
device array inside the library.

With alpha = 0 the reference's gradient ends in gradE[nt] = -z(T).gh, with
z(T) = -gamma_u S u(T); the entry point applied to that z(T) must return
-gradE[nt].  Each grid is checked on two calls in a row, and grids of
different sizes follow each other (whole and ragged 16x16 sub-block lattices,
a smaller lattice after a larger one), so the shared scratch always holds the
previous call's values when a call starts.
"""
import ctypes as C

import numpy as np
import pytest

from fkadj import _lib, api, geometry as G, workloads as W

pytestmark = pytest.mark.gpu


def _entry():
    L = _lib.load()
    fn = L.fkadj_zgh_dot_noalloc
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    fn.restype = C.c_int
    return L, fn


def test_noalloc_zgh_matches_gradient_entry_point():
    import torch
    L, fn = _entry()
    stream = torch.cuda.current_stream()
    # 64x80 and 96x48 are whole 16x16 sub-blocks; 67x83 and 19x50 end in partial
    # ones at the right and bottom edges (the kernel's edge guards), and 19x50
    # (8 sub-blocks) follows 67x83 (30), so its call starts on stale partials
    for seed, (nr, nc) in ((71, (64, 80)), (72, (96, 48)), (73, (67, 83)), (74, (19, 50))):
        inst = W.make_instance(nr, 60, seed=seed, ncols=nc, n_obstacles=6, objective="gradient")
        gradE, Lc, L0, LE, _, yf = api.fk_grad_Et(inst.Et, inst.dt, inst.nt, inst.y0, inst.active_index,
                                                  inst.ncols, inst.nrows, inst.ghost, inst.gamma, inst.S, 0.0,
                                                  params=inst.params, return_yf=True)
        n_num = inst.n_num
        act = inst.active_index > 0
        uT = G.compact(yf, inst.active_index)[:n_num]
        zc = -(inst.gamma[0] * (inst.S @ uT))
        zu = np.full(inst.n, np.nan)
        zu[act] = zc[inst.active_index[act] - 1]
        d_zu = torch.tensor(zu, dtype=torch.float64, device="cuda")
        d_gh = torch.tensor(inst.gh_grid, dtype=torch.float64, device="cuda")
        d_out = torch.empty(1, dtype=torch.float64, device="cuda")
        want = -gradE[-1]
        for _ in range(2):
            d_out.fill_(float("nan"))
            rc = fn(d_zu.data_ptr(), d_gh.data_ptr(), inst.nrows, inst.ncols, d_out.data_ptr(),
                    stream.cuda_stream)
            assert rc == _lib.OK, L.fkadj_last_error().decode()
            torch.cuda.synchronize()
            got = float(d_out.item())
            assert abs(got - want) <= 1e-10 * abs(want), (got, want)


def test_noalloc_single_row_and_column_grids():
    """1 x N and N x 1 grids (every sub-block ragged in one direction), after a
    larger grid so the scratch holds stale partials, against the plain sum of
    the non-NaN products."""
    import torch
    L, fn = _entry()
    stream = torch.cuda.current_stream()
    rng = np.random.default_rng(75)
    d_out = torch.empty(1, dtype=torch.float64, device="cuda")
    for nr, nc in ((40, 70), (1, 200), (150, 1), (1, 1), (17, 1), (1, 33)):
        zu = rng.standard_normal(nr * nc)
        gh = rng.standard_normal(nr * nc)
        zu[rng.random(nr * nc) < 0.2] = np.nan  # holes
        t = zu * gh
        want = float(np.sum(t[~np.isnan(t)]))
        d_zu = torch.tensor(zu, dtype=torch.float64, device="cuda")
        d_gh = torch.tensor(gh, dtype=torch.float64, device="cuda")
        d_out.fill_(float("nan"))
        rc = fn(d_zu.data_ptr(), d_gh.data_ptr(), nr, nc, d_out.data_ptr(), stream.cuda_stream)
        assert rc == _lib.OK, L.fkadj_last_error().decode()
        torch.cuda.synchronize()
        got = float(d_out.item())
        scale = float(np.sum(np.abs(t[~np.isnan(t)]))) or 1.0
        assert abs(got - want) <= 1e-13 * scale, (nr, nc, got, want)


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    L, fn = _entry()
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    rc = fn(d.data_ptr(), d.data_ptr(), 4097, 4097, d.data_ptr(), None)
    assert rc == _lib.ERR_ARG
    assert b"sub-blocks" in L.fkadj_last_error()

"""Writes the golden fixtures used by the parity tests from the reference's
shipped data files (run once, in a container where the reference is mounted).

Source files (agarzon27/adjoint-optimization, src/cuda/data/):
  spirals.mat                                   forward state yf (3*65536, NaN holes)
  lap_Cfile_2nd_order_grad_dx_0p035_N_256_hole_dens_16.mat
                                                active_index (int32, 1-based),
                                                ghost_lr (double class), lap (CSC)
  S_1o4_N_256_hole_dens_16.mat                  objective matrix S (CSC)
  Et_pulse_N_1_E0_5.00_t0_20.0_300ms.mat        seed pulse Et (3001)
  simple_grad_desc_step_2024-nov-02-17-32-50_000001_{50,100,150,200}.mat
                                                Et at which gradE was taken,
                                                gradE, Lcost, L0_vec, LE_vec, Lcost_vec
(written by src/cuda/simple_grad_desc.m:93-101 with alpha=0.5, dt=0.1,
gamma=[1,.2,.2], final_time=300, h=0.035 (fk_parameters_00_05_alpha_0p8_dx_0p035.h)).

Output: tests/golden/ref256.npz (compressed).  Usage:
    python tests/golden/make_golden.py [/path/to/reference]
(default: FKADJ_REFERENCE_DIR, else the container's mount point)
"""
import os
import sys

import numpy as np
import scipy.io as sio

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FKADJ_REFERENCE_DIR", "/root/reference")
D = os.path.join(REF, "src", "cuda", "data")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref256.npz")


def load(name):
    return sio.loadmat(os.path.join(D, name), mat_dtype=True)


def main():
    g = load("lap_Cfile_2nd_order_grad_dx_0p035_N_256_hole_dens_16.mat")
    ai = g["active_index"].ravel().astype(np.int32)
    ghost = g["ghost_lr"].ravel()
    lap = g["lap"].tocsc()
    S = load("S_1o4_N_256_hole_dens_16.mat")["S"].tocsc()
    yf = load("spirals.mat")["yf"].ravel()
    bx3 = np.concatenate([ai > 0] * 3)
    y0 = yf[bx3]                       # simple_grad_desc.m:57-60
    seed = load("Et_pulse_N_1_E0_5.00_t0_20.0_300ms.mat")["Et"].ravel()
    its = [50, 100, 150, 200]
    recs = [load(f"simple_grad_desc_step_2024-nov-02-17-32-50_000001_{k}.mat") for k in its]
    for M in (lap, S):
        M.sort_indices()
    out = dict(
        nrows=256, ncols=256, h=0.035, dt=0.1, nt=3000, alpha=0.5,
        gamma=np.array([1.0, 0.2, 0.2]),
        active_index=ai, ghost_lr=ghost.astype(np.int8), y0=y0,
        Et_seed=seed,
        iters=np.array(its),
        Et=np.stack([r["Et"].ravel() for r in recs]),
        gradE=np.stack([r["gradE"].ravel() for r in recs]),
        Lcost=np.array([float(r["Lcost"].ravel()[0]) for r in recs]),
        Lcost_vec=np.stack([r["Lcost_vec"].ravel() for r in recs]),
        L0_vec=np.stack([r["L0_vec"].ravel() for r in recs]),
        LE_vec=np.stack([r["LE_vec"].ravel() for r in recs]),
        lap_indptr=lap.indptr.astype(np.int32), lap_indices=lap.indices.astype(np.int32),
        lap_data=lap.data.astype(np.int8),
        S_indptr=S.indptr.astype(np.int32), S_indices=S.indices.astype(np.int32),
        S_data4=np.round(S.data * 4).astype(np.int16),
    )
    assert np.array_equal(out["S_data4"] / 4.0, S.data), "S entries are not multiples of 1/4"
    assert np.array_equal(out["lap_data"].astype(float), lap.data)
    assert np.array_equal(out["ghost_lr"].astype(float), ghost)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()

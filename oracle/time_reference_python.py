"""Times the reference's own CPU code for the forward path: the vector field of
its Python prototype (src/scripting/python/fk_lap_ion_t.py:31-67, numpy and
scipy.sparse) inside the RK4 loop of its driver (fk_holes_Et_rk4.py:128-140:
four evaluations per step, E from a cubic spline), on the standard 128^2 and
512^2 instances with the CUDA code's default parameter set (h := dx).

Test infrastructure: it imports the reference tree, which exists only where
the reference is mounted (FKADJ_REFERENCE_DIR, or the first argument), so it
runs on this host, not on a GPU box.  The reference has no CPU adjoint; this
is the forward half of its CPU path.

    python oracle/time_reference_python.py [REFERENCE_DIR]
"""
import os
import sys
import time

import numpy as np
import scipy.interpolate
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "adjoint-optimization_b200"))

from fkadj import geometry as G, workloads as W  # noqa: E402


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FKADJ_REFERENCE_DIR", "/root/reference")
    sys.path.insert(0, os.path.join(ref, "src", "scripting", "python"))
    import fk_lap_ion_t as fk

    threads = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    print(f"host cores {os.cpu_count()}, thread env {threads}")
    for name, inst, steps in (("C1 128^2", W.plain_instance(nt=40), 20), ("C2 512^2", W.large_instance(nt=10), 5)):
        P = inst.params
        lap = sp.csr_matrix(G.laplacian(inst.mask))
        h2 = P.h * P.h
        tt = inst.dt * np.arange(inst.nt + 1)
        param = dict(u_c=P.u_c, u_v=P.u_v, tau_d=P.tau_d, tau_v1_minus=P.tau_v1_minus,
                     tau_v2_minus=P.tau_v2_minus, tau_v_plus=P.tau_v_plus, tau_0=P.tau_0, tau_r=P.tau_r,
                     tau_si=P.tau_si, u_csi=P.u_csi, k_fk=P.k_fk, tau_w_minus=P.tau_w_minus,
                     tau_w_plus=P.tau_w_plus, ksm=P.ksm, lap_u=P.Du / h2 * lap, lap_v=P.Dv / h2 * lap,
                     lap_w=P.Dw / h2 * lap, gh=P.Du * 2 / P.h * np.asarray(inst.ghost, dtype=float),
                     E_fun=scipy.interpolate.CubicSpline(tt, inst.Et))
        fk.set_parameters(param)
        y = np.array(inst.y0, dtype=np.float64)
        dt = inst.dt
        k1 = fk.fk_lap_ion_t(y, 0.0)  # warm-up evaluation
        t0 = time.perf_counter()
        for kt in range(steps):
            t = tt[kt]
            k1 = fk.fk_lap_ion_t(y, t)
            k2 = fk.fk_lap_ion_t(y + dt / 2 * k1, t + dt / 2)
            k3 = fk.fk_lap_ion_t(y + dt / 2 * k2, t + dt / 2)
            k4 = fk.fk_lap_ion_t(y + dt * k3, t + dt)
            y = y + dt / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        sec = (time.perf_counter() - t0) / steps
        cells = inst.nrows * inst.ncols
        print(f"{name}: {sec * 1e3:.2f} ms per RK4 step ({steps} steps), {cells / sec / 1e6:.2f} M cell-steps/s, "
              f"n_num {inst.n_num}")


if __name__ == "__main__":
    main()

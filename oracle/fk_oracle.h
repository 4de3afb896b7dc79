/*
 * fk_oracle.h -- CPU oracle for the Fenton-Karma forward / adjoint hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C (C99 + OpenMP, FP64, no FMA
 * contraction) restatement of the reference algorithm, used as the checker for
 * the CUDA library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product (libfkadj) never links or calls it.
 *
 * Layout conventions follow the reference (agarzon27/adjoint-optimization):
 *   - a state is three dense grids u, v, w stacked as y[0..3n), n = nrows*ncols,
 *     linear index k = i*ncols + j (i = row, slow; j = column, fast);
 *   - holes (non-conducting cells) hold NaN in every field
 *     (num2nan, src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1533-1541);
 *   - gh[k] = (Du*2/h) * ghost_lr[compact(k)], NaN at holes
 *     (src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1588-1595).
 */
#ifndef FK_ORACLE_H
#define FK_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* FK ionic constants + diffusivities + spacing.  Field order matches
 * src/cuda/fk_parameters_00_05_alpha_0p8_dx_0p035.h:2-23. */
typedef struct {
    double u_c, u_v, tau_d, tau_v1_minus, tau_v2_minus, tau_v_plus, tau_0, tau_r,
           tau_si, u_csi, k_fk, tau_w_minus, tau_w_plus, Du, Dv, Dw, ksm, h;
} ora_params;

/* Objective L0 = sum_v gamma[v] * y_v^T S y_v on compact (active-cell) vectors.
 * S is n_num x n_num in CSC form (Jc[n_num+1], Ir[nnz], Sv[nnz]). */
typedef struct {
    int n_num;
    const int64_t *Jc, *Ir;
    const double *Sv;
    double gamma[3];
} ora_objective;

/* One evaluation of the forward vector field f = L y + F_ion(y) + E*gh. */
void ora_rhs(const ora_params *p, int nrows, int ncols, const double *y,
             const double *gh, double E, double *f);

/* Adjoint vector field fz = L^T z + J_F(y)^T z (reference mode). */
void ora_adj_rhs(const ora_params *p, int nrows, int ncols, const double *z,
                 const double *y, double *fz);

/* Not-a-knot cubic spline through (i*dt, Et[i]), i = 0..n-1: second
 * derivatives ypp[n].  Returns 0, or -1 when n < 4. */
int ora_spline_ypp(int n, double dt, const double *Et, double *ypp);
/* Value of that spline at t. */
double ora_spline_val(int n, double dt, const double *Et, const double *ypp, double t);

/* Forward sweep, reference driver order (cu-F:766-815).  Snapshots every
 * nstep steps into ys[ns][3n] (ns may be 0), final state into yf[3n]. */
int ora_forward(const ora_params *p, double dt, const double *Et, int nt,
                int nrows, int ncols, const double *y0, const double *gh,
                int nstep, int ns, double *ys, double *yf);

/* Objective at a final state (NaN grid) -> L0 and z = -gamma*S*y (NaN grid). */
int ora_objective_eval(const ora_objective *obj, const int *active_index, int n,
                       const double *yT, double *L0, double *zT);

/* Reference-mode gradient (continuous adjoint with Hermite midpoint),
 * cu-G:1569-1938.  gradE[nt+1]; also L0, LE, Lcost.  Optionally returns
 * the forward final state yf[3n] (may be NULL). */
int ora_grad_ref(const ora_params *p, double dt, const double *Et, int nt,
                 int nrows, int ncols, const double *y0, const double *gh,
                 const int *active_index, const ora_objective *obj, double alpha,
                 double *gradE, double *L0, double *LE, double *Lcost, double *yf);

/* Exact-mode gradient: discrete adjoint of the RK4 forward and of the
 * not-a-knot spline.  gradE[i] = (1/dt) * dLcost/dEt[i]. */
int ora_grad_exact(const ora_params *p, double dt, const double *Et, int nt,
                   int nrows, int ncols, const double *y0, const double *gh,
                   const int *active_index, const ora_objective *obj, double alpha,
                   double *gradE, double *L0, double *LE, double *Lcost, double *yf);

/* Number of OpenMP threads the oracle uses (0 = library default). */
void ora_set_threads(int nthreads);
int ora_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif

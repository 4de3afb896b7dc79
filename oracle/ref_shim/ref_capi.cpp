/* C entry points around the reference's computational routines, compiled
 * together with the unmodified reference .cu file (test infrastructure).
 * fk_forward_Et_comp: src/cuda/fk_forward_Et_mono_PARAMETERS.cu:646-849
 * fk_grad_Et_comp:    src/cuda/fk_grad_Et_mono_PARAMETERS.cu:1569-1938 */
#include <stdint.h>
#include <stdlib.h>
#include <vector>

#include "matrix.h"

#ifdef FKREF_FORWARD
int fk_forward_Et_comp(const double dt, const double *Et, const int nt, const double *y_ini,
                       const int *active_index, const int nrows, const int ncols, const int n_num,
                       const double *gh_num, const int nstep, const int ns, double *ys, double *yf,
                       char **p_strPtr);

extern "C" int fkref_forward(double dt, const double *Et, int nt, const double *y_ini,
                             const int *active_index, int nrows, int ncols, int n_num,
                             const double *gh_num, int nstep, int ns, double *ys, double *yf) {
    char *p = nullptr;
    int rc = fk_forward_Et_comp(dt, Et, nt, y_ini, active_index, nrows, ncols, n_num, gh_num, nstep, ns,
                                ys, yf, &p);
    free(p);
    return rc;
}
#endif

#ifdef FKREF_GRAD
int fk_grad_Et_comp(const double dt, const double *Et, const int nt, const double *y_ini,
                    const int *active_index, const int nrows, const int ncols, const int n_num,
                    const double *gh_num, const double *gamma, const mxArray *SMx, const double alpha,
                    double *L0Ptr, double *LEPtr, double *LcostPtr, double *gradE, char **p_strPtr);

extern "C" int fkref_grad(double dt, const double *Et, int nt, const double *y_ini, const int *active_index,
                          int nrows, int ncols, int n_num, const double *gh_num, const double *gamma,
                          int64_t S_ncol, const int64_t *Jc, const int64_t *Ir, const double *Sv,
                          double alpha, double *L0, double *LE, double *Lcost, double *gradE) {
    std::vector<mwIndex> jc(Jc, Jc + S_ncol + 1), ir(Ir, Ir + Jc[S_ncol]);
    mxArray S;
    S.m = (size_t)S_ncol;
    S.n = (size_t)S_ncol;
    S.pr = const_cast<double *>(Sv);
    S.ir = ir.data();
    S.jc = jc.data();
    S.owns = 0;
    char *p = nullptr;
    int rc = fk_grad_Et_comp(dt, Et, nt, y_ini, active_index, nrows, ncols, n_num, gh_num, gamma, &S, alpha,
                             L0, LE, Lcost, gradE, &p);
    free(p);
    return rc;
}
#endif

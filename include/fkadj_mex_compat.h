/*
 * fkadj_mex_compat.h -- the reference's two computational routines, by name
 * and signature, implemented on libfkadj.  Include it in the unmodified MEX
 * gateways in place of their forward declarations:
 *
 *   src/cuda/fk_forward_Et_param_mex.cpp:27-29  declares fk_forward_Et_comp
 *   src/cuda/fk_grad_Et_param_mex.cpp:3-6       declares fk_grad_Et_comp
 *
 * after "mex.h" (which provides mxArray, mxGetN, mxGetIr, mxGetJc, mxGetPr,
 * mxMalloc), and link the gateway against libfkadj.so.  The FK parameter set is
 * the reference's default one with h = FKADJ_MEX_DX (0.035, the spacing of
 * src/cuda/fk_parameters_00_05_alpha_0p8_dx_0p035.h:23, unless defined before
 * the include).  C++ linkage, like the originals (cu-F:646, cu-G:1569).
 *
 * Differences from the originals: errors do not exit() the MATLAB process;
 * inside a MEX file (MATLAB_MEX_FILE defined) they raise a MATLAB error with
 * the library's message, elsewhere the routine returns the fkadj_status.  The
 * returned parameter string is NUL-terminated.
 */
#ifndef FKADJ_MEX_COMPAT_H
#define FKADJ_MEX_COMPAT_H

#include <cstdint>
#include <cstring>
#include <vector>

#include "fkadj.h"

#ifndef FKADJ_MEX_DX
#define FKADJ_MEX_DX 0.035
#endif

namespace fkadj_mex {
inline int finish(fkadj_status st, char **p_strPtr, const fkadj_params *p) {
    if (p_strPtr) {
        const char *s = fkadj_param_string(p);
        const size_t n = std::strlen(s);
        char *out = (char *)mxMalloc(n + 1);
        if (out) std::memcpy(out, s, n + 1);
        *p_strPtr = out;
    }
#ifdef MATLAB_MEX_FILE
    if (st != FKADJ_OK) mexErrMsgIdAndTxt("fkadj:error", "%s", fkadj_last_error());
#endif
    return (int)st;
}
}  // namespace fkadj_mex

inline int fk_forward_Et_comp(const double dt, const double *Et, const int nt, const double *y_ini,
                              const int *active_index, const int nrows, const int ncols, const int n_num,
                              const double *gh_num, const int nstep, const int ns, double *ys, double *yf,
                              char **p_strPtr) {
    fkadj_params p;
    fkadj_default_params(&p, FKADJ_MEX_DX);
    fkadj_status st = fkadj_forward(&p, dt, Et, nt, y_ini, active_index, nrows, ncols, n_num, gh_num, nstep, ns,
                                    ys, yf, nullptr);
    return fkadj_mex::finish(st, p_strPtr, &p);
}

inline int fk_grad_Et_comp(const double dt, const double *Et, const int nt, const double *y_ini,
                           const int *active_index, const int nrows, const int ncols, const int n_num,
                           const double *gh_num, const double *gamma, const mxArray *SMx, const double alpha,
                           double *L0Ptr, double *LEPtr, double *LcostPtr, double *gradE, char **p_strPtr) {
    fkadj_params p;
    fkadj_default_params(&p, FKADJ_MEX_DX);
    const int64_t ncol = (int64_t)mxGetN(SMx);
    const mwIndex *jc = mxGetJc(SMx);
    const mwIndex *ir = mxGetIr(SMx);
    std::vector<int64_t> Jc(jc, jc + ncol + 1), Ir(ir, ir + (ncol ? jc[ncol] : 0));
    fkadj_status st = fkadj_grad(&p, dt, Et, nt, y_ini, active_index, nrows, ncols, n_num, gh_num, gamma, ncol,
                                 Jc.data(), Ir.data(), mxGetPr(SMx), alpha, L0Ptr, LEPtr, LcostPtr, gradE,
                                 nullptr, nullptr);
    return fkadj_mex::finish(st, p_strPtr, &p);
}

#endif /* FKADJ_MEX_COMPAT_H */

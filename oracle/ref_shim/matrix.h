/* Minimal stand-in for the MATLAB MEX matrix API, enough to compile the
 * reference's computational routines outside MATLAB (test infrastructure).
 * Only the calls the reference makes are provided: mxCreateDoubleMatrix,
 * mxGetPr, mxGetN, mxGetIr, mxGetJc, mxDestroyArray, mxMalloc. */
#ifndef FKREF_MATRIX_STANDIN_H
#define FKREF_MATRIX_STANDIN_H
#include <stddef.h>
#include <stdlib.h>

typedef size_t mwSize;
typedef size_t mwIndex;
typedef enum { mxREAL = 0, mxCOMPLEX = 1 } mxComplexity;

typedef struct mxArray_tag {
    size_t m, n;
    double *pr;
    mwIndex *ir, *jc;
    int owns;
} mxArray;

static inline mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity c) {
    (void)c;
    mxArray *a = (mxArray *)calloc(1, sizeof(mxArray));
    a->m = m;
    a->n = n;
    a->pr = (double *)calloc(m * n ? m * n : 1, sizeof(double));
    a->owns = 1;
    return a;
}
static inline double *mxGetPr(const mxArray *a) { return a->pr; }
static inline size_t mxGetN(const mxArray *a) { return a->n; }
static inline size_t mxGetM(const mxArray *a) { return a->m; }
static inline mwIndex *mxGetIr(const mxArray *a) { return a->ir; }
static inline mwIndex *mxGetJc(const mxArray *a) { return a->jc; }
static inline void mxDestroyArray(mxArray *a) {
    if (!a) return;
    if (a->owns) free(a->pr);
    free(a);
}
static inline void *mxMalloc(size_t n) { return malloc(n ? n : 1); }
static inline void mxFree(void *p) { free(p); }
#endif

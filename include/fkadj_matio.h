/* fkadj_matio.h -- MAT-file (level 5) reader and writer for the engine's
 * inputs and outputs.
 *
 * The reference keeps every input and output of its hot path in MATLAB
 * level-5 MAT files: the grid file (active_index int32, ghost_lr double
 * stored as int16, lap sparse), the objective matrix S (sparse), the initial
 * state yf, the seed pulse Et, and the gradient-descent snapshots
 * simple_grad_desc_step_*.mat (src/cuda/simple_grad_desc.m:44-67, 93-96;
 * src/cuda/save_fk_forward_Et.m:80-117).  This module reads and writes that
 * format in C++ so the native drivers need neither MATLAB nor Python.
 *
 * Supported: little-endian level-5 files, compressed (zlib) and uncompressed
 * elements, real dense numeric arrays of every numeric class with any stored
 * type (MATLAB may store a double array as int16, as it does ghost_lr), char
 * arrays, logical arrays, and real sparse matrices.  Cells, structs, objects
 * and function handles are listed by name and class but not read.
 *
 * All functions return FKADJ_OK or an error status with the message in
 * fkadj_last_error().  Arrays are column-major as MATLAB stores them.
 */
#ifndef FKADJ_MATIO_H
#define FKADJ_MATIO_H

#include <stdint.h>

#include "fkadj.h"

#ifdef __cplusplus
extern "C" {
#endif

/* MATLAB array classes (mxClassID values of the level-5 format). */
enum {
    FKADJ_MX_CELL = 1, FKADJ_MX_STRUCT = 2, FKADJ_MX_OBJECT = 3, FKADJ_MX_CHAR = 4,
    FKADJ_MX_SPARSE = 5, FKADJ_MX_DOUBLE = 6, FKADJ_MX_SINGLE = 7, FKADJ_MX_INT8 = 8,
    FKADJ_MX_UINT8 = 9, FKADJ_MX_INT16 = 10, FKADJ_MX_UINT16 = 11, FKADJ_MX_INT32 = 12,
    FKADJ_MX_UINT32 = 13, FKADJ_MX_INT64 = 14, FKADJ_MX_UINT64 = 15, FKADJ_MX_FUNCTION = 16,
    FKADJ_MX_OPAQUE = 17
};

typedef struct fkadj_mat fkadj_mat;

/* Reads the whole file (inflating compressed elements) into memory. */
fkadj_status fkadj_mat_open(const char *path, fkadj_mat **out);
void fkadj_mat_close(fkadj_mat *m);

/* Variables in file order. */
int fkadj_mat_count(const fkadj_mat *m);
const char *fkadj_mat_name(const fkadj_mat *m, int i);

/* Class, dimensions (up to maxdims of them; *ndims receives the count), the
 * element count (product of the dimensions) and, for sparse matrices, nnz.
 * flags: bit 0 complex, bit 1 logical, bit 2 readable by this module. */
fkadj_status fkadj_mat_info(const fkadj_mat *m, const char *name, int *mx_class, int *ndims,
                            int64_t *dims, int maxdims, int64_t *numel, int64_t *nnz, int *flags);

/* Dense numeric or logical array as doubles (n = numel). */
fkadj_status fkadj_mat_read_double(const fkadj_mat *m, const char *name, double *out, int64_t n);
/* Dense array as int32; every value must be an integer in range. */
fkadj_status fkadj_mat_read_int32(const fkadj_mat *m, const char *name, int32_t *out, int64_t n);
/* Char array as a NUL-terminated string (rows concatenated column-major, as
 * MATLAB stores a 1-by-n char row); cap bytes including the NUL. */
fkadj_status fkadj_mat_read_string(const fkadj_mat *m, const char *name, char *out, int64_t cap);
/* Real sparse matrix in CSC: colptr[ncols+1], rowidx[nnz], val[nnz]. */
fkadj_status fkadj_mat_read_sparse(const fkadj_mat *m, const char *name, int64_t *colptr,
                                   int64_t *rowidx, double *val);

typedef struct fkadj_matw fkadj_matw;

/* Starts a level-5 file; compress != 0 writes every variable as a
 * zlib-compressed element (what MATLAB's save does by default). */
fkadj_status fkadj_matw_open(const char *path, int compress, fkadj_matw **out);
/* Dense rows-by-cols array of class FKADJ_MX_DOUBLE, _INT32, _INT16 or
 * _UINT8; data holds rows*cols elements of that class's C type. */
fkadj_status fkadj_matw_dense(fkadj_matw *w, const char *name, int mx_class, int64_t rows,
                              int64_t cols, const void *data);
/* 1-by-strlen(s) char array. */
fkadj_status fkadj_matw_string(fkadj_matw *w, const char *name, const char *s);
/* Real sparse rows-by-cols matrix from CSC arrays (nnz = colptr[cols]). */
fkadj_status fkadj_matw_sparse(fkadj_matw *w, const char *name, int64_t rows, int64_t cols,
                               const int64_t *colptr, const int64_t *rowidx, const double *val);
/* Writes the file and frees the writer (also on error). */
fkadj_status fkadj_matw_close(fkadj_matw *w);

#ifdef __cplusplus
}
#endif

#endif /* FKADJ_MATIO_H */

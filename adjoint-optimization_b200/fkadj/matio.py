"""MAT-file (level 5) access through libfkadj's native reader and writer
(include/fkadj_matio.h).

``loadmat(path)`` returns {name: value} for every variable the native reader
can read: dense numeric and logical arrays as numpy arrays of their MATLAB
shape (column-major data), char arrays as str, real sparse matrices as
scipy.sparse.csc_matrix.  Cells, structs, objects and function handles are
skipped.  ``savemat(path, variables)`` writes float64, int32, int16 and uint8
arrays (vectors as columns), str, and scipy sparse matrices.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.sparse as sp

from ._lib import check, load

MX_CHAR, MX_SPARSE, MX_DOUBLE, MX_INT16, MX_INT32, MX_UINT8 = 4, 5, 6, 10, 12, 9
_CLASS_OF = {np.dtype(np.float64): MX_DOUBLE, np.dtype(np.int32): MX_INT32,
             np.dtype(np.int16): MX_INT16, np.dtype(np.uint8): MX_UINT8}
_bound = False


def _lib():
    global _bound
    L = load()
    if _bound:
        return L
    vp, i64p = C.c_void_p, C.POINTER(C.c_int64)
    L.fkadj_mat_open.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.fkadj_mat_close.argtypes = [vp]
    L.fkadj_mat_count.argtypes = [vp]
    L.fkadj_mat_name.argtypes = [vp, C.c_int]
    L.fkadj_mat_name.restype = C.c_char_p
    L.fkadj_mat_info.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), i64p, C.c_int,
                                 i64p, i64p, C.POINTER(C.c_int)]
    L.fkadj_mat_read_double.argtypes = [vp, C.c_char_p, C.POINTER(C.c_double), C.c_int64]
    L.fkadj_mat_read_int32.argtypes = [vp, C.c_char_p, C.POINTER(C.c_int32), C.c_int64]
    L.fkadj_mat_read_string.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_int64]
    L.fkadj_mat_read_sparse.argtypes = [vp, C.c_char_p, i64p, i64p, C.POINTER(C.c_double)]
    L.fkadj_matw_open.argtypes = [C.c_char_p, C.c_int, C.POINTER(vp)]
    L.fkadj_matw_dense.argtypes = [vp, C.c_char_p, C.c_int, C.c_int64, C.c_int64, vp]
    L.fkadj_matw_string.argtypes = [vp, C.c_char_p, C.c_char_p]
    L.fkadj_matw_sparse.argtypes = [vp, C.c_char_p, C.c_int64, C.c_int64, i64p, i64p, C.POINTER(C.c_double)]
    L.fkadj_matw_close.argtypes = [vp]
    for n in ("fkadj_mat_open", "fkadj_mat_info", "fkadj_mat_read_double", "fkadj_mat_read_int32",
              "fkadj_mat_read_string", "fkadj_mat_read_sparse", "fkadj_matw_open", "fkadj_matw_dense",
              "fkadj_matw_string", "fkadj_matw_sparse", "fkadj_matw_close"):
        getattr(L, n).restype = C.c_int
    _bound = True
    return L


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def loadmat(path: str, integer_as_int32: bool = True) -> dict:
    """Variables of a level-5 MAT file.  Arrays of the classes int8 to int32
    come back as int32 when ``integer_as_int32``; every other numeric class
    (uint32, int64, uint64 included) as float64."""
    L = _lib()
    h = C.c_void_p()
    check(L.fkadj_mat_open(str(path).encode(), C.byref(h)))
    out = {}
    try:
        for i in range(L.fkadj_mat_count(h)):
            name = L.fkadj_mat_name(h, i)
            cls, nd, numel, nnz, flags = C.c_int(), C.c_int(), C.c_int64(), C.c_int64(), C.c_int()
            dims = (C.c_int64 * 8)()
            check(L.fkadj_mat_info(h, name, C.byref(cls), C.byref(nd), dims, 8, C.byref(numel),
                                   C.byref(nnz), C.byref(flags)))
            if not flags.value & 4:
                continue  # not readable here (cell, struct, object, function handle, complex)
            shape = tuple(dims[k] for k in range(min(nd.value, 8)))
            key = name.decode()
            if cls.value == MX_SPARSE:
                colptr = np.empty(shape[1] + 1, np.int64)
                rowidx = np.empty(nnz.value, np.int64)
                val = np.empty(nnz.value, np.float64)
                check(L.fkadj_mat_read_sparse(h, name, _ptr(colptr, C.c_int64), _ptr(rowidx, C.c_int64),
                                              _ptr(val, C.c_double)))
                out[key] = sp.csc_matrix((val, rowidx, colptr), shape=shape)
            elif cls.value == MX_CHAR:
                buf = C.create_string_buffer(numel.value + 1)
                check(L.fkadj_mat_read_string(h, name, buf, numel.value + 1))
                out[key] = buf.value.decode()
            elif integer_as_int32 and 8 <= cls.value <= 12:
                a = np.empty(numel.value, np.int32)
                check(L.fkadj_mat_read_int32(h, name, _ptr(a, C.c_int32), numel.value))
                out[key] = a.reshape(shape, order="F")
            else:
                a = np.empty(numel.value, np.float64)
                check(L.fkadj_mat_read_double(h, name, _ptr(a, C.c_double), numel.value))
                out[key] = a.reshape(shape, order="F")
    finally:
        L.fkadj_mat_close(h)
    return out


def savemat(path: str, variables: dict, compress: bool = True) -> None:
    L = _lib()
    w = C.c_void_p()
    check(L.fkadj_matw_open(str(path).encode(), int(compress), C.byref(w)))
    try:
        for name, v in variables.items():
            key = name.encode()
            if isinstance(v, str):
                check(L.fkadj_matw_string(w, key, v.encode()))
            elif sp.issparse(v):
                m = sp.csc_matrix(v, dtype=np.float64)
                m.sort_indices()
                colptr = np.ascontiguousarray(m.indptr, np.int64)
                rowidx = np.ascontiguousarray(m.indices, np.int64)
                val = np.ascontiguousarray(m.data, np.float64)
                check(L.fkadj_matw_sparse(w, key, m.shape[0], m.shape[1], _ptr(colptr, C.c_int64),
                                          _ptr(rowidx, C.c_int64), _ptr(val, C.c_double)))
            else:
                a = np.asarray(v)
                if a.dtype not in _CLASS_OF:
                    a = a.astype(np.float64)
                if a.ndim == 0:
                    a = a.reshape(1, 1)
                elif a.ndim == 1:
                    a = a.reshape(-1, 1)
                elif a.ndim > 2:
                    raise ValueError(f"{name}: only 2-D arrays are written")
                data = np.asfortranarray(a)
                check(L.fkadj_matw_dense(w, key, _CLASS_OF[a.dtype], a.shape[0], a.shape[1],
                                         data.ctypes.data_as(C.c_void_p)))
    except BaseException:
        L.fkadj_matw_close(w)
        raise
    check(L.fkadj_matw_close(w))

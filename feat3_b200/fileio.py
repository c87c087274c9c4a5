"""Container file I/O in FEAT3's formats, through the C-ABI (``fb_io_*``, host code).

``FileMode`` keeps the values of ``LAFEM::FileMode`` (kernel/lafem/base.hpp:31-46). Matrices are
returned as ``CsrFile`` (rows, columns, uint64 row pointers and column indices, float64 values:
the arrays FEAT3's ``SparseMatrixCSR<Mem::Main, double, Index>`` holds); vectors as float64 numpy
arrays. Errors raise ``FeatError`` with the library's status (FB_ERR_IO for an unreadable file,
FB_ERR_FORMAT for contents that do not match the mode), where the reference throws
``InternalError`` or fails an assertion.

    A = read_csr(FileMode.fm_csr, "level3.A.csr")       # SparseMatrixCSR::read_from
    write_csr(FileMode.fm_mtx, "level3.A.mtx", A)       # SparseMatrixCSR::write_out
    b = read_vector(FileMode.fm_dv, "rhs.dv")           # DenseVector::read_from
    n, dirichlet, _ = read_sparse_vector(FileMode.fm_mtx, "level3.filter.mtx")  # UnitFilter's list
"""
from __future__ import annotations

import ctypes as C
import os
from typing import NamedTuple

import numpy as np

from . import _lib


class FileMode:
    fm_exp = 0
    fm_dv = 1
    fm_mtx = 2
    fm_csr = 4
    fm_binary = 12


class CsrFile(NamedTuple):
    rows: int
    columns: int
    row_ptr: np.ndarray   # uint64, rows + 1
    col_ind: np.ndarray   # uint64, used_elements
    val: np.ndarray       # float64, used_elements

    @property
    def used_elements(self):
        return int(self.val.size)

    def arrays(self):
        """(row_ptr, col_ind, val), the form ``MultiGrid.from_csr`` takes"""
        return self.row_ptr, self.col_ind, self.val


def _path(filename):
    return os.fsencode(os.fspath(filename))


def _csr_host(m):
    rp = np.ascontiguousarray(m.row_ptr, dtype=np.uint64)
    ci = np.ascontiguousarray(m.col_ind, dtype=np.uint64)
    va = np.ascontiguousarray(m.val, dtype=np.float64)
    h = _lib.CsrHost(int(m.rows), int(m.columns), int(va.size), rp.ctypes.data, ci.ctypes.data, va.ctypes.data)
    return h, (rp, ci, va)


def _take_csr(h):
    """copy a library-allocated CsrHost into numpy and release it"""
    lib = _lib.load()
    try:
        rows, nnz = int(h.rows), int(h.nnz)

        def arr(ptr, n, ctype, dtype):
            if n == 0:
                return np.zeros(0, dtype=dtype)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).astype(dtype, copy=True)

        rp = arr(h.row_ptr, rows + 1, C.c_uint64, np.uint64)
        if rows == 0:
            rp = np.zeros(1, dtype=np.uint64)
        return CsrFile(rows, int(h.cols), rp, arr(h.col_ind, nnz, C.c_uint64, np.uint64),
                       arr(h.val, nnz, C.c_double, np.float64))
    finally:
        lib.fb_io_csr_release(C.byref(h))


def _take_vector(n, data):
    lib = _lib.load()
    try:
        if n.value == 0:
            return np.zeros(0)
        return np.ctypeslib.as_array(data, shape=(n.value,)).copy()
    finally:
        lib.fb_io_free(C.cast(data, C.c_void_p))


def read_csr(mode, filename) -> CsrFile:
    """SparseMatrixCSR::read_from (sparse_matrix_csr.hpp:1098-1246): fm_mtx, fm_csr, fm_binary"""
    h = _lib.CsrHost()
    _lib.call("fb_io_csr_read", _path(filename), int(mode), C.byref(h))
    return _take_csr(h)


def write_csr(mode, filename, m, symmetric=False):
    """SparseMatrixCSR::write_out (sparse_matrix_csr.hpp:1261-1343): fm_mtx (optionally the lower
    triangle as 'symmetric'), fm_csr, fm_binary. ``m`` is a CsrFile or any object with rows,
    columns, row_ptr, col_ind and val."""
    h, _keep = _csr_host(m)
    _lib.call("fb_io_csr_write", _path(filename), int(mode), C.byref(h), int(bool(symmetric)))


def serialise_csr(m) -> bytes:
    """SparseMatrixCSR::serialise (sparse_matrix_csr.hpp:1081-1090): the fm_csr byte layout"""
    h, _keep = _csr_host(m)
    size = C.c_uint64(0)
    _lib.call("fb_io_csr_serialised_size", C.byref(h), C.byref(size))
    buf = C.create_string_buffer(size.value)
    _lib.call("fb_io_csr_serialise", C.byref(h), C.cast(buf, C.c_void_p), size.value)
    return buf.raw


def deserialise_csr(data: bytes) -> CsrFile:
    """SparseMatrixCSR::deserialise (sparse_matrix_csr.hpp:1066-1077)"""
    buf = C.create_string_buffer(bytes(data), len(data))
    h = _lib.CsrHost()
    _lib.call("fb_io_csr_deserialise", C.cast(buf, C.c_void_p), len(data), C.byref(h))
    return _take_csr(h)


def read_vector(mode, filename) -> np.ndarray:
    """DenseVector::read_from (dense_vector.hpp:587-712): fm_exp, fm_mtx, fm_dv, fm_binary"""
    n, data = C.c_uint64(0), C.POINTER(C.c_double)()
    _lib.call("fb_io_vector_read", _path(filename), int(mode), C.byref(n), C.byref(data))
    return _take_vector(n, data)


def write_vector(mode, filename, v):
    """DenseVector::write_out (dense_vector.hpp:721-777): fm_exp, fm_mtx, fm_dv, fm_binary"""
    a = np.ascontiguousarray(v, dtype=np.float64)
    _lib.call("fb_io_vector_write", _path(filename), int(mode), a.ctypes.data if a.size else None, a.size)


def serialise_vector(v) -> bytes:
    """DenseVector::serialise (dense_vector.hpp:495-505): the fm_dv byte layout"""
    a = np.ascontiguousarray(v, dtype=np.float64)
    size = C.c_uint64(0)
    _lib.call("fb_io_vector_serialised_size", a.size, C.byref(size))
    buf = C.create_string_buffer(size.value)
    _lib.call("fb_io_vector_serialise", a.ctypes.data if a.size else None, a.size, C.cast(buf, C.c_void_p),
              size.value)
    return buf.raw


def deserialise_vector(data: bytes) -> np.ndarray:
    """DenseVector::deserialise (dense_vector.hpp:480-490)"""
    buf = C.create_string_buffer(bytes(data), len(data))
    n, out = C.c_uint64(0), C.POINTER(C.c_double)()
    _lib.call("fb_io_vector_deserialise", C.cast(buf, C.c_void_p), len(data), C.byref(n), C.byref(out))
    return _take_vector(n, out)


def read_sparse_vector(mode, filename):
    """SparseVector::read_from (sparse_vector.hpp:517-630), fm_mtx: (size, indices, values) with
    0-based indices sorted ascending (a repeated index keeps its last value)"""
    size, nnz = C.c_uint64(0), C.c_uint64(0)
    idx, val = C.POINTER(C.c_uint64)(), C.POINTER(C.c_double)()
    _lib.call("fb_io_sparse_vector_read", _path(filename), int(mode), C.byref(size), C.byref(nnz), C.byref(idx),
              C.byref(val))
    lib = _lib.load()
    try:
        n = nnz.value
        i = np.ctypeslib.as_array(idx, shape=(n,)).copy() if n else np.zeros(0, np.uint64)
        v = np.ctypeslib.as_array(val, shape=(n,)).copy() if n else np.zeros(0)
    finally:
        lib.fb_io_free(C.cast(idx, C.c_void_p))
        lib.fb_io_free(C.cast(val, C.c_void_p))
    return size.value, i.astype(np.uint64), v


def write_sparse_vector(mode, filename, size, indices, values=None):
    """SparseVector::write_out (sparse_vector.hpp:639-680), fm_mtx; values default to 0 (a
    homogeneous Dirichlet list)"""
    i = np.ascontiguousarray(indices, dtype=np.uint64)
    v = np.zeros(i.size) if values is None else np.ascontiguousarray(values, dtype=np.float64)
    _lib.call("fb_io_sparse_vector_write", _path(filename), int(mode), int(size), i.size,
              i.ctypes.data if i.size else None, v.ctypes.data if v.size else None)


def read_hierarchy(files):
    """Levels for ``MultiGrid.from_csr`` from FEAT3 matrix files, finest level first. ``files``
    holds one dict per level with the paths (or CsrFile objects) of 'A' and, except on the
    coarsest level, 'P' and 'R', plus the Dirichlet DOF list 'filter' (an index array, or the path
    of the filter's sparse vector in fm_mtx); a matrix path ending in '.mtx' is read as fm_mtx,
    any other as fm_binary."""
    def load(x):
        if isinstance(x, CsrFile):
            return x
        mode = FileMode.fm_mtx if os.fspath(x).endswith(".mtx") else FileMode.fm_binary
        return read_csr(mode, x)

    levels = []
    for f in files:
        flt = f["filter"]
        if isinstance(flt, (str, bytes, os.PathLike)):
            flt = read_sparse_vector(FileMode.fm_mtx, flt)[1]
        d = {"A": load(f["A"]).arrays(), "filter": np.asarray(flt, dtype=np.uint64)}
        for key in ("P", "R"):
            if key in f:
                d[key] = load(f[key]).arrays()
        levels.append(d)
    return levels

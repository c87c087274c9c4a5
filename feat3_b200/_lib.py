"""ctypes binding of ``libfeat3_b200.so`` (the C-ABI declared in ``include/feat3_b200.h``).

The library is the only compute path: if it is missing it is built in-tree with nvcc, and
if that fails the import fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

from . import build as _build

HERE = os.path.dirname(os.path.abspath(__file__))
HEADER = os.path.join(os.path.dirname(HERE), "include", "feat3_b200.h")

(FB_OK, FB_ERR_INVALID, FB_ERR_CUDA, FB_ERR_ALLOC, FB_ERR_UNSUPPORTED, FB_ERR_NOT_READY, FB_ERR_TOO_LARGE,
 FB_ERR_TIMEOUT, FB_ERR_IO, FB_ERR_FORMAT) = range(10)
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "allocation failed", 4: "unsupported", 5: "not ready",
          6: "exceeds a fixed capacity", 7: "bounded wait in a kernel expired", 8: "file I/O error",
          9: "contents do not match the file format"}


class FeatError(RuntimeError):
    def __init__(self, fn, code):
        super().__init__(f"{fn} failed: {ERRORS.get(code, code)} (status {code})")
        self.code = code


vp, u64, u32, i32, dbl, flt = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int, C.c_double, C.c_float


class StructuredDesc(C.Structure):
    _fields_ = [("dim", i32), ("degree", i32), ("level", i32), ("level_min", i32),
                ("k", vp), ("k_on_device", i32), ("sell_sigma", i32), ("numbering", i32)]


class CsrHost(C.Structure):
    _fields_ = [("rows", u64), ("cols", u64), ("nnz", u64), ("row_ptr", vp), ("col_ind", vp), ("val", vp)]


class SolverCfg(C.Structure):
    _fields_ = [("outer", i32), ("nu", i32), ("omega_jac", dbl), ("omega_rich", dbl), ("omega_outer", dbl),
                ("coarse", i32), ("tol_rel", dbl), ("max_iter", i32), ("precision", i32), ("use_graphs", i32), ("format", i32),
                ("flags", i32), ("cycle", i32), ("adapt_cgc", i32)]


class SolveInfo(C.Structure):
    _fields_ = [("status", i32), ("iters", i32), ("def_init", dbl), ("def_final", dbl),
                ("solve_ms", dbl), ("kernel_launches", i32)]


_SIGS = {
    # operator layer
    "fb_csr_apply_f64": [vp, dbl, vp, dbl, vp, vp, vp, vp, u64, u64, u64, i32, vp],
    "fb_csr_apply_f32": [vp, flt, vp, flt, vp, vp, vp, vp, u64, u64, u64, i32, vp],
    "fb_ell_apply_f64": [vp, dbl, vp, dbl, vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_ell_apply_f32": [vp, flt, vp, flt, vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_csr_apply_f64_u64": [vp, dbl, vp, dbl, vp, vp, vp, vp, u64, u64, u64, i32, vp],
    "fb_csr_apply_f32_u64": [vp, flt, vp, flt, vp, vp, vp, vp, u64, u64, u64, i32, vp],
    "fb_ell_apply_f64_u64": [vp, dbl, vp, dbl, vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_ell_apply_f32_u64": [vp, flt, vp, flt, vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_axpy_f64": [vp, dbl, vp, vp, u64, vp],
    "fb_axpy_f32": [vp, flt, vp, vp, u64, vp],
    "fb_dot_f64": [vp, vp, u64, vp, vp],
    "fb_dot_f32": [vp, vp, u64, vp, vp],
    "fb_dot_f64_sync": [vp, vp, u64, vp, vp],
    "fb_dot_f32_sync": [vp, vp, u64, vp, vp],
    "fb_dot_f64_noalloc": [vp, vp, u64, vp, vp],
    "fb_norm2_f64": [vp, u64, vp, vp],
    "fb_norm2_f32": [vp, u64, vp, vp],
    "fb_norm2_f64_sync": [vp, u64, vp, vp],
    "fb_norm2_f32_sync": [vp, u64, vp, vp],
    "fb_component_product_f64": [vp, vp, vp, u64, vp],
    "fb_component_product_f32": [vp, vp, vp, u64, vp],
    "fb_component_invert_f64": [vp, vp, dbl, u64, vp],
    "fb_component_invert_f32": [vp, vp, flt, u64, vp],
    "fb_scale_f64": [vp, vp, dbl, u64, vp],
    "fb_scale_f32": [vp, vp, flt, u64, vp],
    "fb_diagonal_csr_f64": [vp, vp, vp, vp, u64, vp],
    "fb_diagonal_csr_f32": [vp, vp, vp, vp, u64, vp],
    "fb_diagonal_ell_f64": [vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_diagonal_ell_f32": [vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_diagonal_csr_f64_u64": [vp, vp, vp, vp, u64, vp],
    "fb_diagonal_csr_f32_u64": [vp, vp, vp, vp, u64, vp],
    "fb_diagonal_ell_f64_u64": [vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_diagonal_ell_f32_u64": [vp, vp, vp, vp, vp, u64, u64, vp],
    "fb_unit_filter_rhs_f64": [vp, vp, vp, u64, vp],
    "fb_unit_filter_def_f64": [vp, vp, u64, vp],
    "fb_unit_filter_rhs_f32": [vp, vp, vp, u64, vp],
    "fb_unit_filter_def_f32": [vp, vp, u64, vp],
    "fb_unit_filter_rhs_f64_u64": [vp, vp, vp, u64, vp],
    "fb_unit_filter_def_f64_u64": [vp, vp, u64, vp],
    "fb_unit_filter_rhs_f32_u64": [vp, vp, vp, u64, vp],
    "fb_unit_filter_def_f32_u64": [vp, vp, u64, vp],
    "fb_convert_f64_to_f32": [vp, vp, u64, vp],
    "fb_convert_f32_to_f64": [vp, vp, u64, vp],
    "fb_set_f64": [vp, dbl, u64, vp],
    "fb_set_f32": [vp, flt, u64, vp],
    # solver layer
    "fb_mg_create_structured": [C.POINTER(vp), C.POINTER(StructuredDesc)],
    "fb_feat_numbering": [i32, i32, i32, vp, vp, vp],
    "fb_mg_create_csr": [C.POINTER(vp), i32, vp, vp, vp, vp, vp, i32],
    "fb_mg_destroy": [vp],
    "fb_solver_cfg_default": [C.POINTER(SolverCfg)],
    "fb_mg_configure": [vp, C.POINTER(SolverCfg)],
    "fb_mg_solve": [vp, vp, vp, vp, C.POINTER(SolveInfo)],
    "fb_mg_solve_host": [vp, vp, vp, vp, C.POINTER(SolveInfo)],
    "fb_mg_solve_host_zero": [vp, vp, vp, vp, C.POINTER(SolveInfo)],
    "fb_mg_vcycle": [vp, vp, vp],
    "fb_mg_assemble_rhs": [vp, i32, vp],
    "fb_mg_num_dofs": [vp, i32],
    "fb_mg_num_levels": [vp],
    "fb_mg_nnz": [vp, i32],
    "fb_mg_export_csr": [vp, i32, vp, vp, vp],
    "fb_mg_adjoint_grad": [vp, vp, vp, vp, vp, C.POINTER(SolveInfo)],
    "fb_mg_element_grad": [vp, vp, vp, vp],
    "fb_mg_time_spmv": [vp, i32, i32, i32, i32, C.POINTER(dbl)],
    "fb_mg_test_expire_wait": [vp],
    # container file I/O
    "fb_io_csr_read": [C.c_char_p, i32, C.POINTER(CsrHost)],
    "fb_io_csr_write": [C.c_char_p, i32, C.POINTER(CsrHost), i32],
    "fb_io_csr_serialised_size": [C.POINTER(CsrHost), C.POINTER(u64)],
    "fb_io_csr_serialise": [C.POINTER(CsrHost), vp, u64],
    "fb_io_csr_deserialise": [vp, u64, C.POINTER(CsrHost)],
    "fb_io_csr_release": [C.POINTER(CsrHost)],
    "fb_io_vector_read": [C.c_char_p, i32, C.POINTER(u64), C.POINTER(C.POINTER(dbl))],
    "fb_io_vector_write": [C.c_char_p, i32, vp, u64],
    "fb_io_vector_serialised_size": [u64, C.POINTER(u64)],
    "fb_io_vector_serialise": [vp, u64, vp, u64],
    "fb_io_vector_deserialise": [vp, u64, C.POINTER(u64), C.POINTER(C.POINTER(dbl))],
    "fb_io_sparse_vector_read": [C.c_char_p, i32, C.POINTER(u64), C.POINTER(u64), C.POINTER(C.POINTER(u64)),
                                 C.POINTER(C.POINTER(dbl))],
    "fb_io_sparse_vector_write": [C.c_char_p, i32, u64, u64, vp, vp],
    "fb_io_free": [vp],
    "fb_version": [],
}
_RESTYPE = {"fb_mg_destroy": None, "fb_io_csr_release": None, "fb_io_free": None, "fb_solver_cfg_default": None, "fb_mg_num_dofs": u64,
            "fb_mg_nnz": u64, "fb_version": C.c_char_p}

_lib = None


def header_symbols():
    """Every function name declared in include/feat3_b200.h."""
    with open(HEADER) as f:
        txt = f.read()
    return sorted(set(re.findall(r"^FB_API\s+[\w\s\*]+?\b(fb_\w+)\s*\(", txt, flags=re.M)))


def load(build_if_missing=True):
    global _lib
    if _lib is not None:
        return _lib
    if build_if_missing and not _build.up_to_date():
        _build.build()
    if not os.path.exists(_build.LIB):
        raise ImportError(f"feat3_b200: native library {_build.LIB} is missing and could not be built")
    lib = C.CDLL(_build.LIB)
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, i32)
    _lib = lib
    return lib


def check(name, code):
    if code != FB_OK:
        raise FeatError(name, code)


def call(name, *args):
    lib = load()
    rc = getattr(lib, name)(*args)
    check(name, rc)
    return rc

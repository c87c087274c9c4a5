"""ctypes front-end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may use
this module. It wraps

* ``oracle/build/liboracle.so`` -- this project's C++ restatement of the reference multigrid
  path (see ``oracle/feat_oracle.h`` for the reference files it follows; independent loops on
  OpenMP threads, reductions sequential), and
* ``oracle/_ref/feat_ref`` -- the reference's own CPU solver (FEAT3 compiled from its
  sources by ``oracle/Makefile``), driven through files, when that binary exists.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "feat_ref")

STATUS = {0: "undefined", 1: "progress", 2: "success", 3: "aborted", 4: "diverged", 5: "max_iter", 6: "stagnated"}
RHS_KIND = {"sine": 0, "one": 1, "expbubble": 2}
COARSE = {"direct": 0, "pcg": 1, "smoother": 2, "none": 3}
INNER = {"f64": 0, "f32": 1, "f16": 2}


def build():
    """Compile the restatement library (g++ only; no GPU or reference sources needed)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i64, i32, d = C.c_void_p, C.c_int64, C.c_int, C.c_double
        P = C.POINTER
        L.or_hier_create.restype = vp
        L.or_hier_create.argtypes = [i32, i32, i32, i32, vp]
        L.or_hier_destroy.argtypes = [vp]
        for fn in ("or_level_ndofs", "or_level_nnz", "or_level_pnnz", "or_level_nfilter"):
            getattr(L, fn).restype = i64
            getattr(L, fn).argtypes = [vp, i32]
        for fn in ("or_level_csr", "or_level_p", "or_level_r"):
            getattr(L, fn).argtypes = [vp, i32, vp, vp, vp]
        L.or_level_filter.argtypes = [vp, i32, vp]
        L.or_element_matrix.restype = i32
        L.or_element_matrix.argtypes = [vp, i32, vp]
        L.or_rhs.argtypes = [vp, i32, vp]
        L.or_solve.restype = i32
        L.or_solve.argtypes = [vp, vp, vp, vp, vp, P(i32)]
        L.or_vcycle.argtypes = [vp, vp, vp, vp]
        L.or_element_grad.argtypes = [vp, vp, vp, vp]
        L.or_csr_apply.argtypes = [vp, d, vp, d, vp, vp, vp, vp, i64, i64, i32]
        L.or_feat_numbering.restype = i32
        L.or_feat_numbering.argtypes = [i32, i32, i32, vp, vp]
        L.or_threads.restype = i32
        L.or_threads.argtypes = []
        _lib = L
    return _lib


class Cfg(C.Structure):
    _fields_ = [("solver", C.c_int), ("nu", C.c_int), ("omega_jac", C.c_double),
                ("omega_rich", C.c_double), ("omega_outer", C.c_double), ("coarse", C.c_int),
                ("tol_rel", C.c_double), ("max_iter", C.c_int), ("inner", C.c_int), ("cycle", C.c_int),
                ("cgc", C.c_int)]


CYCLE = {"v": 0, "f": 1, "w": 2}
CGC = {"fixed": 0, "energy": 1, "defect": 2}


def make_cfg(solver="pcg", nu=4, omega_jac=0.5, omega_rich=1.0, omega_outer=1.0, coarse="direct",
             tol=1e-8, max_iter=1000, inner="f64", cycle="v", cgc="fixed"):
    return Cfg(0 if solver == "pcg" else 1, nu, omega_jac, omega_rich, omega_outer, COARSE[coarse],
               tol, max_iter, INNER[inner], CYCLE[cycle], CGC[cgc])


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class Hierarchy:
    """Structured level hierarchy of the restatement (lexicographic lattice numbering)."""

    def __init__(self, dim, degree, level, level_min=1, k=None):
        self.dim, self.degree, self.level, self.level_min = dim, degree, level, level_min
        self._k = None if k is None else np.ascontiguousarray(k, dtype=np.float64)
        self.h = lib().or_hier_create(dim, degree, level, level_min,
                                      None if self._k is None else _p(self._k))
        if not self.h:
            raise ValueError("invalid hierarchy parameters")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_hier_destroy(self.h)
            self.h = None

    def ndofs(self, l=None):
        return int(lib().or_level_ndofs(self.h, self.level if l is None else l))

    def csr(self, l=None):
        l = self.level if l is None else l
        n, nnz = self.ndofs(l), int(lib().or_level_nnz(self.h, l))
        rp, ci, va = np.zeros(n + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
        lib().or_level_csr(self.h, l, _p(rp), _p(ci), _p(va))
        return rp, ci, va

    def prol(self, l):
        n, nnz = self.ndofs(l), int(lib().or_level_pnnz(self.h, l))
        rp, ci, va = np.zeros(n + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
        lib().or_level_p(self.h, l, _p(rp), _p(ci), _p(va))
        return rp, ci, va

    def rest(self, l):
        nc, nnz = self.ndofs(l - 1), int(lib().or_level_pnnz(self.h, l))
        rp, ci, va = np.zeros(nc + 1, np.int64), np.zeros(nnz, np.int32), np.zeros(nnz)
        lib().or_level_r(self.h, l, _p(rp), _p(ci), _p(va))
        return rp, ci, va

    def filter(self, l=None):
        l = self.level if l is None else l
        idx = np.zeros(int(lib().or_level_nfilter(self.h, l)), np.int32)
        lib().or_level_filter(self.h, l, _p(idx))
        return idx

    def element_matrix(self, l=None):
        nloc = (self.degree + 1) ** self.dim
        out = np.zeros(nloc * nloc)
        lib().or_element_matrix(self.h, self.level if l is None else l, _p(out))
        return out.reshape(nloc, nloc)

    def rhs(self, kind="sine"):
        out = np.zeros(self.ndofs())
        lib().or_rhs(self.h, RHS_KIND[kind], _p(out))
        return out

    def solve(self, rhs, sol=None, **kw):
        cfg = make_cfg(**kw)
        sol = np.zeros(self.ndofs()) if sol is None else np.array(sol, dtype=np.float64, copy=True)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        hist = np.zeros(cfg.max_iter + 1)
        it = C.c_int(0)
        st = lib().or_solve(self.h, C.byref(cfg), _p(rhs), _p(sol), _p(hist), C.byref(it))
        return {"status": STATUS[st], "iters": it.value, "hist": hist[: it.value + 1].copy(), "u": sol}

    def vcycle(self, d, **kw):
        cfg = make_cfg(**kw)
        d = np.ascontiguousarray(d, dtype=np.float64)
        out = np.zeros_like(d)
        lib().or_vcycle(self.h, C.byref(cfg), _p(d), _p(out))
        return out

    def element_grad(self, u, lam):
        N = 1 << self.level
        out = np.zeros(N ** self.dim)
        u = np.ascontiguousarray(u, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        lib().or_element_grad(self.h, _p(u), _p(lam), _p(out))
        return out


def threads():
    """threads the restatement's parallel loops use (1 without OpenMP)"""
    return int(lib().or_threads())


def csr_apply(a, x, b, y, rp, ci, va, rows, cols, transposed=False):
    """r = b*y + a*A*x with the reference's CSR loop (apply_generic.hpp:25-70)."""
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    r = np.zeros(cols if transposed else rows)
    lib().or_csr_apply(_p(r), a, _p(x), b, _p(y), _p(np.ascontiguousarray(va, np.float64)),
                       _p(np.ascontiguousarray(ci, np.int32)), _p(np.ascontiguousarray(rp, np.int64)),
                       rows, cols, 1 if transposed else 0)
    return r


# ---------------------------------------------------------------------------------------
# the reference's own solver (oracle/_ref/feat_ref), when built
def feat_numbering(dim, degree, level):
    """(dof_lex, cell_lex): lexicographic index of each FEAT DOF / cell of the unit square or
    cube refined `level` times (or_feat_numbering)"""
    n = degree * (1 << level) + 1
    dofs = np.zeros(n ** dim, dtype=np.uint32)
    cells = np.zeros((1 << level) ** dim, dtype=np.uint32)
    if lib().or_feat_numbering(dim, degree, level, _p(dofs), _p(cells)) != 0:
        raise ValueError("unsupported numbering arguments")
    return dofs, cells


def have_ref():
    return os.path.exists(REF_BIN)


def _read_info(fn):
    info = {}
    with open(fn) as f:
        for line in f:
            parts = line.split()
            if not parts:
                continue
            if parts[0] in ("hist", "solve_times"):
                info[parts[0]] = np.array([float(v) for v in parts[1:]])
            else:
                v = parts[1]
                try:
                    info[parts[0]] = int(v)
                except ValueError:
                    info[parts[0]] = float(v)
    return info


def run_ref(dim, degree, level, level_min=1, rhs="sine", k=None, solver="pcg", nu=4, omega_jac=0.5,
            omega_rich=1.0, omega_outer=1.0, coarse="direct", tol=1e-8, max_iter=1000, inner="f64",
            target=None, dump_matrices=False, workdir=None, cycle="v", cgc="fixed", feat_files=False,
            repeat=1, budget_s=0.0, warmup=0, outputs=True):
    """Run the reference's own FP64/mixed MG solver; returns info and arrays in lattice order.
    repeat / budget_s / warmup: timed solves from a zero initial guess after `warmup` untimed
    one-iteration solves, stopping early when the next solve would end past budget_s seconds of
    timed solving (info["solve_times"]). outputs=False skips reading the solution files back."""
    if not have_ref():
        raise FileNotFoundError(REF_BIN)
    wd = workdir or tempfile.mkdtemp(prefix="feat_ref_")
    out = os.path.join(wd, "r")
    cmd = [REF_BIN, "--dim", str(dim), "--degree", str(degree), "--level", str(level),
           "--level-min", str(level_min), "--rhs", rhs, "--solver", solver, "--nu", str(nu),
           "--omega-jac", repr(omega_jac), "--omega-rich", repr(omega_rich),
           "--omega-outer", repr(omega_outer), "--coarse", coarse, "--tol", repr(tol),
           "--maxit", str(max_iter), "--inner", inner, "--out", out, "--quiet", "--cycle", cycle,
           "--cgc", cgc, "--repeat", str(repeat), "--budget-s", repr(float(budget_s)), "--warmup", str(warmup)]
    if k is not None:
        kf = os.path.join(wd, "k.bin")
        np.ascontiguousarray(k, np.float64).tofile(kf)
        cmd += ["--kfile", kf]
    if target is not None:
        tf = os.path.join(wd, "t.bin")
        np.ascontiguousarray(target, np.float64).tofile(tf)
        cmd += ["--target", tf]
    if dump_matrices:
        cmd += ["--dump-matrices"]
    if feat_files:
        cmd += ["--feat-files"]
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    info = _read_info(out + ".info")
    if not outputs:
        return {"info": info, "workdir": wd, "prefix": out}
    lat = np.fromfile(out + ".lattice", dtype=np.uint64).astype(np.int64)
    n = lat.size
    res = {"info": info, "lattice": lat, "workdir": wd, "prefix": out}
    for key in ("u", "rhs", "lambda"):
        fn = out + "." + key
        if os.path.exists(fn):
            v = np.fromfile(fn, dtype=np.float64)
            lexv = np.zeros(n)
            lexv[lat] = v
            res[key] = lexv
    if os.path.exists(out + ".grad"):
        res["grad"] = np.fromfile(out + ".grad", dtype=np.float64)
    return res

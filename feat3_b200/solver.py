"""Python face of the native multigrid driver (solver layer of the C-ABI).

The composition mirrors the reference's solver trees: ``PCG(MultiGrid(V; Richardson(Jacobi)
smoothers; coarse solver))`` of applications/poisson_dirichlet.cpp:152-190 and
``Richardson(MultiGrid)`` of tutorials/tutorial_05_multigrid.cpp:373-449, with the mixed
form ``Richardson/PCG(ConvertPrecond(MultiGrid<float>))`` of
kernel/solver/convert_precond.hpp:41-120. The status codes are the reference's
``Solver::Status`` (kernel/solver/base.hpp:48-64).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib

STATUS = {0: "undefined", 1: "progress", 2: "success", 3: "aborted", 4: "diverged", 5: "max_iter", 6: "stagnated"}
OUTER = {"pcg": 0, "richardson": 1}
COARSE = {"direct": 0, "pcg": 1, "smoother": 2, "none": 3}
PRECISION = {"f64": 0, "f32": 1, "f16": 2}
FORMAT = {"sell": 0, "stencil": 1, "matfree": 2}
CYCLE = {"v": 0, "f": 1, "w": 2}
CGC = {"fixed": 0, "energy": 1, "defect": 2}
NUMBERING = {"lattice": 0, "feat": 1}


def feat_numbering(dim, degree, level, device="cuda"):
    """(dof_lex, cell_lex) as int64 CUDA tensors: the lexicographic lattice index of each FEAT3
    DOF / cell of the unit square or cube refined `level` times (fb_feat_numbering)"""
    n = (degree * (1 << level) + 1) ** dim
    ne = (1 << level) ** dim
    dofs = torch.empty(n, dtype=torch.int32, device=device)
    cells = torch.empty(ne, dtype=torch.int32, device=device)
    _lib.call("fb_feat_numbering", dim, degree, level, dofs.data_ptr(), cells.data_ptr(),
              torch.cuda.current_stream().cuda_stream)
    torch.cuda.current_stream().synchronize()
    mask = (1 << 32) - 1
    return dofs.to(torch.int64) & mask, cells.to(torch.int64) & mask
RHS = {"sine": 0, "one": 1, "expbubble": 2}


def _torch_sync():
    """The library runs on its own non-blocking stream: finish torch's pending work on the
    tensors handed over (and on memory torch may recycle) before every call."""
    torch.cuda.current_stream().synchronize()


class MultiGrid:
    """A device multigrid hierarchy plus its outer solver."""

    def __init__(self, handle, structured):
        self.h = handle
        self.structured = structured
        self.cfg = None

    # ---------------------------------------------------------------- construction
    @classmethod
    def structured(cls, dim, degree, level, level_min=1, k=None, sell_sigma=1, numbering="lattice"):
        """Structured unit-square/cube hierarchy assembled on the device. numbering="feat" makes
        every finest-level vector (rhs, solution, V-cycle, adjoint) and the coefficient / gradient
        per cell use FEAT3's numbering of the refined unit cube instead of the lexicographic lattice."""
        lib = _lib.load()
        karr = None
        if numbering not in NUMBERING:
            raise ValueError(f"numbering must be one of {sorted(NUMBERING)}")
        desc = _lib.StructuredDesc(dim, degree, level, level_min, None, 0, sell_sigma, NUMBERING[numbering])
        if k is not None:
            if isinstance(k, torch.Tensor) and k.is_cuda:
                karr = k.contiguous().to(torch.float64)
                desc.k, desc.k_on_device = karr.data_ptr(), 1
                _torch_sync()
            else:
                karr = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
                desc.k = karr.ctypes.data
        h = C.c_void_p()
        _lib.check("fb_mg_create_structured", lib.fb_mg_create_structured(C.byref(h), C.byref(desc)))
        mg = cls(h, True)
        mg.dim, mg.degree, mg.level, mg.level_min = dim, degree, level, level_min
        mg.numbering = numbering
        return mg

    @classmethod
    def from_csr(cls, levels, sell_sigma=1):
        """levels: finest first; each a dict with A=(row_ptr, col_ind, val), filter=indices and,
        except on the coarsest level, P=(...) mapping the next level onto this one and R=(...)."""
        lib = _lib.load()
        nl = len(levels)
        keep = []

        def csr(t, rows, cols):
            rp = np.ascontiguousarray(np.asarray(t[0], dtype=np.uint64))
            ci = np.ascontiguousarray(np.asarray(t[1], dtype=np.uint64))
            va = np.ascontiguousarray(np.asarray(t[2], dtype=np.float64))
            keep.extend([rp, ci, va])
            return _lib.CsrHost(rows, cols, int(rp[-1]), rp.ctypes.data, ci.ctypes.data, va.ctypes.data)

        n = [len(l["A"][0]) - 1 for l in levels]
        A = (_lib.CsrHost * nl)(*[csr(l["A"], n[i], n[i]) for i, l in enumerate(levels)])
        P = (_lib.CsrHost * max(nl - 1, 1))()
        R = (_lib.CsrHost * max(nl - 1, 1))()
        for i in range(nl - 1):
            P[i] = csr(levels[i]["P"], n[i], n[i + 1])
            R[i] = csr(levels[i]["R"], n[i + 1], n[i])
        filt = [np.ascontiguousarray(np.asarray(l["filter"], dtype=np.uint64)) for l in levels]
        fptr = (C.c_void_p * nl)(*[f.ctypes.data if f.size else None for f in filt])
        fsz = (C.c_uint64 * nl)(*[f.size for f in filt])
        h = C.c_void_p()
        rc = lib.fb_mg_create_csr(C.byref(h), nl, C.cast(A, C.c_void_p), C.cast(P, C.c_void_p),
                                  C.cast(R, C.c_void_p), C.cast(fptr, C.c_void_p), C.cast(fsz, C.c_void_p),
                                  sell_sigma)
        _lib.check("fb_mg_create_csr", rc)
        return cls(h, False)

    def close(self):
        if getattr(self, "h", None):
            _lib.load().fb_mg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- configuration
    def configure(self, outer="pcg", nu=4, omega_jac=0.5, omega_rich=1.0, omega_outer=1.0, coarse="direct",
                  tol=1e-8, max_iter=1000, precision="f64", graphs=True, format="sell", fuse_coarse=True,
                  fuse_dot=True, tiled=True, stream=True, cycle="v", cgc="fixed"):
        """Solver configuration (fb_solver_cfg). cycle: "v", "f" or "w" (Solver::MultiGridCycle);
        cgc: "fixed", "energy" or "defect" (Solver::MultiGridAdaptCGC). fuse_coarse / fuse_dot /
        tiled / stream switch individual fusions and kernels of the matrix-free form off
        (FB_FLAG_*), for comparisons."""
        flags = (0 if fuse_coarse else 1) | (0 if fuse_dot else 2) | (0 if tiled else 4) | (0 if stream else 8)
        cfg = _lib.SolverCfg(OUTER[outer], nu, omega_jac, omega_rich, omega_outer, COARSE[coarse], tol, max_iter,
                             PRECISION[precision], 1 if graphs else 0, FORMAT[format], flags, CYCLE[cycle], CGC[cgc])
        _lib.check("fb_mg_configure", _lib.load().fb_mg_configure(self.h, C.byref(cfg)))
        self.cfg = cfg
        return self

    # ---------------------------------------------------------------- queries
    def num_levels(self):
        return _lib.load().fb_mg_num_levels(self.h)

    def ndofs(self, level=0):
        return int(_lib.load().fb_mg_num_dofs(self.h, level))

    def nnz(self, level=0):
        return int(_lib.load().fb_mg_nnz(self.h, level))

    def export_csr(self, level=0):
        n, nnz = self.ndofs(level), self.nnz(level)
        rp = np.zeros(n + 1, np.uint64)
        ci = np.zeros(nnz, np.uint32)
        va = np.zeros(nnz)
        _lib.call("fb_mg_export_csr", self.h, level, rp.ctypes.data, ci.ctypes.data, va.ctypes.data)
        return rp.astype(np.int64), ci.astype(np.int64), va

    # ---------------------------------------------------------------- work
    def assemble_rhs(self, kind="sine"):
        b = torch.empty(self.ndofs(), dtype=torch.float64, device="cuda")
        _torch_sync()
        _lib.call("fb_mg_assemble_rhs", self.h, RHS[kind], b.data_ptr())
        return b

    def _info(self, info, hist):
        it = info.iters
        return {"status": STATUS.get(info.status, info.status), "iters": it, "def_init": info.def_init,
                "def_final": info.def_final, "solve_ms": info.solve_ms, "kernel_launches": info.kernel_launches,
                "hist": None if hist is None else hist[: it + 1].copy()}

    def solve(self, rhs, sol=None, record=True):
        """Solver::solve(solver, sol, rhs) on device tensors; sol is updated in place."""
        if self.cfg is None:
            self.configure()
        if sol is None:
            sol = torch.zeros_like(rhs)
        hist = np.zeros(self.cfg.max_iter + 1) if record else None
        info = _lib.SolveInfo()
        _torch_sync()
        _lib.call("fb_mg_solve", self.h, rhs.data_ptr(), sol.data_ptr(),
                  None if hist is None else hist.ctypes.data, C.byref(info))
        out = self._info(info, hist)
        out["u"] = sol
        return out

    def solve_host(self, rhs, sol=None, record=True, zero_init=False):
        """End-to-end: host buffers in, host solution out (copies inside the timed region).
        zero_init: solve from a zero initial guess; sol is then output only and is not copied
        to the device (fb_mg_solve_host_zero)."""
        if self.cfg is None:
            self.configure()
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        sol = np.zeros_like(rhs) if sol is None else np.ascontiguousarray(sol, dtype=np.float64)
        hist = np.zeros(self.cfg.max_iter + 1) if record else None
        info = _lib.SolveInfo()
        _lib.call("fb_mg_solve_host_zero" if zero_init else "fb_mg_solve_host", self.h, rhs.ctypes.data,
                  sol.ctypes.data, None if hist is None else hist.ctypes.data, C.byref(info))
        out = self._info(info, hist)
        out["u"] = sol
        return out

    def vcycle(self, d):
        cor = torch.empty_like(d)
        _torch_sync()
        _lib.call("fb_mg_vcycle", self.h, d.data_ptr(), cor.data_ptr())
        return cor

    def element_grad(self, u, lam):
        ne = (1 << self.level) ** self.dim
        g = torch.empty(ne, dtype=torch.float64, device="cuda")
        _torch_sync()
        _lib.call("fb_mg_element_grad", self.h, u.data_ptr(), lam.data_ptr(), g.data_ptr())
        return g

    def adjoint_grad(self, u, u_target):
        """lambda = (A^T)^-1 filter(u - u_target) by the configured MG solver; dJ/dk per element."""
        ne = (1 << self.level) ** self.dim
        lam = torch.empty_like(u)
        g = torch.empty(ne, dtype=torch.float64, device="cuda")
        info = _lib.SolveInfo()
        _torch_sync()
        _lib.call("fb_mg_adjoint_grad", self.h, u.data_ptr(), u_target.data_ptr(), lam.data_ptr(), g.data_ptr(),
                  C.byref(info))
        return lam, g, self._info(info, None)

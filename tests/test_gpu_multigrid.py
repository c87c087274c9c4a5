"""Solver-layer parity on the GPU against the oracle restatement (itself pinned to the
reference's own solver by tests/test_oracle_golden.py): identical iteration counts and the
solution within 1e-10 relative for the FP64 drop-in; error <= 1e-8 against the FP64 oracle
for the mixed forms."""
import numpy as np
import pytest
import torch

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

TOL_U = 1e-10


def relerr(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def lognormal_k(dim, level, sigma=1.0, seed=0):
    n = (1 << level) ** dim
    return np.exp(sigma * np.random.default_rng(seed).standard_normal(n))


CASES = [
    # dim, degree, level, level_min, rhs, k-sigma, nu, omega_jac, coarse
    (2, 1, 7, 1, "sine", None, 4, 0.5, "direct"),        # C1
    (3, 1, 4, 1, "sine", None, 2, 0.5, "direct"),        # C2 shape, smaller
    (2, 2, 5, 1, "one", 1.0, 2, 0.5, "direct"),          # C3 shape, smaller
    (2, 1, 6, 1, "one", 0.5, 2, 0.5, "direct"),          # C4 shape, smaller
    (3, 1, 4, 1, "one", 1.0, 2, 0.5, "direct"),          # C5 shape, smaller
    (3, 2, 3, 1, "one", 1.0, 2, 0.5, "direct"),          # 3D Q2
    (2, 1, 5, 0, "expbubble", None, 4, 0.7, "smoother"),  # poisson_dirichlet composition
    (2, 1, 6, 2, "sine", None, 1, 0.5, "none"),          # nu = 1 paths, identity coarse solver
    (2, 1, 6, 2, "sine", None, 3, 0.5, "smoother"),      # odd nu, smoother coarse solver
]


@pytest.mark.parametrize("case", CASES, ids=[f"d{c[0]}q{c[1]}L{c[2]}-{c[4]}-k{c[5]}-nu{c[6]}-{c[8]}" for c in CASES])
@pytest.mark.parametrize("graphs,fmt", [(True, "sell"), (False, "sell"), (True, "stencil"), (False, "stencil"),
                                        (True, "matfree"), (False, "matfree")])
def test_structured_pcg_matches_oracle(case, graphs, fmt):
    from feat3_b200.solver import MultiGrid
    dim, deg, lvl, lmin, rhs, ks, nu, wj, coarse = case
    k = None if ks is None else lognormal_k(dim, lvl, ks, seed=lvl)
    H = po.Hierarchy(dim, deg, lvl, lmin, k)
    b = H.rhs(rhs)
    ref = H.solve(b, nu=nu, omega_jac=wj, coarse=coarse)
    mg = MultiGrid.structured(dim, deg, lvl, lmin, k)
    mg.configure(nu=nu, omega_jac=wj, coarse=coarse, graphs=graphs, format=fmt)
    bg = mg.assemble_rhs(rhs)
    np.testing.assert_allclose(bg.cpu().numpy(), b, rtol=1e-12, atol=1e-15 * np.abs(b).max())
    res = mg.solve(torch.tensor(b).cuda())
    assert res["status"] == ref["status"] == "success"
    assert res["iters"] == ref["iters"]
    np.testing.assert_allclose(res["hist"], ref["hist"], rtol=1e-6)
    assert relerr(res["u"].cpu().numpy(), ref["u"]) <= TOL_U


@pytest.mark.parametrize("dim,deg,lvl", [(2, 1, 5), (2, 2, 4), (3, 1, 3), (3, 2, 2)])
def test_structured_assembly_bitwise(dim, deg, lvl):
    """device assembly reproduces the cell-wise scatter assembly entry for entry"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(dim, lvl, 1.0, seed=7)
    H = po.Hierarchy(dim, deg, lvl, 1, k)
    mg = MultiGrid.structured(dim, deg, lvl, 1, k)
    for l in range(mg.num_levels()):
        rp, ci, va = mg.export_csr(l)
        orp, oci, ova = H.csr(lvl - l)
        np.testing.assert_array_equal(rp, orp)
        np.testing.assert_array_equal(ci, oci)
        np.testing.assert_array_equal(va, ova)


@pytest.mark.parametrize("sigma", [1, 256])
def test_csr_hierarchy_dropin(sigma):
    """a hierarchy handed over as CSR matrices (push_level semantics), SELL-C-sigma inside"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(2, 6, 1.0, seed=3)
    H = po.Hierarchy(2, 2, 6, 2, k)
    levels = []
    for l in range(6, 1, -1):
        d = {"A": H.csr(l), "filter": H.filter(l)}
        if l > 2:
            d["P"], d["R"] = H.prol(l), H.rest(l)
        levels.append(d)
    b = H.rhs("one")
    ref = H.solve(b, nu=2)
    mg = MultiGrid.from_csr(levels, sell_sigma=sigma)
    mg.configure(nu=2)
    res = mg.solve(torch.tensor(b).cuda())
    assert res["iters"] == ref["iters"]
    assert relerr(res["u"].cpu().numpy(), ref["u"]) <= TOL_U


@pytest.mark.parametrize("outer", ["richardson", "pcg"])
@pytest.mark.parametrize("graphs", [False, True])
def test_richardson_outer(outer, graphs):
    from feat3_b200.solver import MultiGrid
    H = po.Hierarchy(2, 1, 7, 1)
    b = H.rhs("sine")
    kw = dict(nu=4, omega_jac=1.0, omega_rich=0.8, coarse="direct")
    ref = H.solve(b, solver=outer, **kw)
    mg = MultiGrid.structured(2, 1, 7, 1)
    mg.configure(outer=outer, graphs=graphs, **kw)
    res = mg.solve(torch.tensor(b).cuda())
    assert res["iters"] == ref["iters"]
    assert relerr(res["u"].cpu().numpy(), ref["u"]) <= TOL_U


@pytest.mark.parametrize("prec", ["f32", "f16"])
@pytest.mark.parametrize("outer", ["richardson", "pcg"])
@pytest.mark.parametrize("fmt", ["sell", "stencil", "matfree"])
def test_mixed_precision_error(prec, outer, fmt):
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(3, 5, 1.0, seed=5)
    H = po.Hierarchy(3, 1, 5, 1, k)
    b = H.rhs("one")
    ref = H.solve(b, nu=2, tol=1e-12)
    mg = MultiGrid.structured(3, 1, 5, 1, k)
    mg.configure(nu=2, precision=prec, outer=outer, format=fmt)
    res = mg.solve(torch.tensor(b).cuda())
    assert res["status"] == "success"
    assert res["hist"][-1] <= 1e-8 * res["hist"][0]
    assert relerr(res["u"].cpu().numpy(), ref["u"]) <= 1e-8


def test_host_buffer_solve_matches_device_solve():
    from feat3_b200.solver import MultiGrid
    mg = MultiGrid.structured(2, 1, 6, 1).configure(nu=2)
    b = mg.assemble_rhs("sine")
    r1 = mg.solve(b)
    r2 = mg.solve_host(b.cpu().numpy())
    assert r1["iters"] == r2["iters"]
    np.testing.assert_array_equal(r1["u"].cpu().numpy(), r2["u"])
    # zero initial guess: whatever the output buffer holds is ignored
    junk = np.full(b.numel(), np.nan)
    r3 = mg.solve_host(b.cpu().numpy(), junk, zero_init=True)
    assert r3["iters"] == r1["iters"]
    np.testing.assert_array_equal(r1["u"].cpu().numpy(), r3["u"])


def test_zero_rhs_and_nan_status():
    """initial defect <= eps^2 -> success at once; a NaN defect -> aborted (iterative.hpp:744-766)"""
    from feat3_b200.solver import MultiGrid
    mg = MultiGrid.structured(2, 1, 5, 1).configure(nu=2)
    z = torch.zeros(mg.ndofs(), dtype=torch.float64, device="cuda")
    r = mg.solve(z)
    assert r["status"] == "success" and r["iters"] == 0
    b = mg.assemble_rhs("sine")
    b[100] = float("nan")
    r = mg.solve(b)
    assert r["status"] == "aborted"


@pytest.mark.parametrize("lvl", [4, 5, 6])
@pytest.mark.parametrize("fmt", ["sell", "stencil", "matfree"])
def test_vcycle_matches_oracle(fmt, lvl):
    """one V(2,2) cycle against the oracle's; from level 5 on the restriction onto the 17^3 and
    33^3 levels runs as the bulk-staged kernel, whose terms and order are those of R"""
    from feat3_b200.solver import MultiGrid
    H = po.Hierarchy(3, 1, lvl, 1, lognormal_k(3, lvl, 1.0, 11))
    d = H.rhs("one")
    ref = H.vcycle(d, nu=2)
    mg = MultiGrid.structured(3, 1, lvl, 1, lognormal_k(3, lvl, 1.0, 11)).configure(nu=2, format=fmt)
    cor = mg.vcycle(torch.tensor(d).cuda()).cpu().numpy()
    assert relerr(cor, ref) <= 1e-13
    mg.close()


def test_adjoint_gradient_matches_oracle():
    from feat3_b200.solver import MultiGrid
    lvl = 6
    k = lognormal_k(2, lvl, 0.5, seed=21)
    H = po.Hierarchy(2, 1, lvl, 1, k)
    b = H.rhs("one")
    u = H.solve(b, nu=2, tol=1e-14)["u"]
    ut = H.solve(b * 0 + H.rhs("one"), nu=2, tol=1e-14)["u"] * 0.9
    g = u - ut
    g[H.filter()] = 0.0
    lam = H.solve(g, nu=2, tol=1e-14)["u"]
    gref = H.element_grad(u, lam)
    mg = MultiGrid.structured(2, 1, lvl, 1, k).configure(nu=2, tol=1e-14)
    ud = mg.solve(torch.tensor(b).cuda())["u"]
    lam_d, gd, info = mg.adjoint_grad(ud, torch.tensor(ut).cuda())
    assert info["status"] == "success"
    assert relerr(lam_d.cpu().numpy(), lam) <= 1e-10
    assert relerr(gd.cpu().numpy(), gref) <= 1e-10


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("dim,lvl", [(3, 5), (2, 7)])
def test_matfree_fusions_match_unfused(prec, dim, lvl):
    """the fused coarse cycle, the r.z fused into the last smoothing step and the tiled
    operator kernel against the level-by-level, separate-reduction, simple-kernel path"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(dim, lvl, 1.0, seed=9)
    mg = MultiGrid.structured(dim, 1, lvl, 1, k)
    b = mg.assemble_rhs("one")
    mg.configure(nu=2, precision=prec, format="matfree")
    fused = mg.solve(b)
    mg.configure(nu=2, precision=prec, format="matfree", fuse_coarse=False, fuse_dot=False, tiled=False)
    plain = mg.solve(b)
    assert fused["status"] == plain["status"] == "success"
    assert abs(fused["iters"] - plain["iters"]) <= (0 if prec == "f64" else 1)
    tol = 1e-10 if prec == "f64" else 1e-8
    assert relerr(fused["u"].cpu().numpy(), plain["u"].cpu().numpy()) <= tol
    # fused forms launch fewer kernels
    assert fused["kernel_launches"] < plain["kernel_launches"]


def test_matfree_operator_matches_assembled():
    """one Jacobi step of the matrix-free form equals the assembled (stencil) form on every
    level, through the V-cycle API: same corrections to FP64 rounding"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(3, 5, 1.0, 13)
    mg = MultiGrid.structured(3, 1, 5, 1, k)
    d = mg.assemble_rhs("one")
    mg.configure(nu=3, format="stencil")
    a = mg.vcycle(d).cpu().numpy()
    mg.configure(nu=3, format="matfree")
    b = mg.vcycle(d).cpu().numpy()
    mg.configure(nu=3, format="matfree", tiled=False, fuse_coarse=False)
    c = mg.vcycle(d).cpu().numpy()
    assert relerr(b, a) <= 1e-13
    assert relerr(c, a) <= 1e-13


def test_full_size_forms_agree():
    """the bench problem at full size (3D Q1, 257^3 = 16,974,593 DOFs, k = exp(N(0,1))): the FP64
    drop-in on assembled SELL-C-sigma matrices and the FP64 matrix-free form take the same
    iterations and agree to 1e-10; the mixed matrix-free form (the headline) reaches 1e-8 with
    its error against the FP64 solution <= 1e-8 (size-independent checks where the oracle would
    take minutes)"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(3, 8, 1.0, seed=2026)
    mg = MultiGrid.structured(3, 1, 8, 1, k, sell_sigma=256)
    b = mg.assemble_rhs("one")
    common = dict(nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    ref = mg.configure(format="sell", **common).solve(b)
    u64 = ref["u"].clone()
    mf = mg.configure(format="matfree", **common).solve(b)
    mix = mg.configure(format="matfree", precision="f32", **common).solve(b)
    assert ref["status"] == mf["status"] == mix["status"] == "success"
    assert ref["iters"] == mf["iters"]
    assert abs(mix["iters"] - ref["iters"]) <= 1
    assert float(torch.linalg.norm(mf["u"] - u64) / torch.linalg.norm(u64)) <= 1e-10
    assert float(torch.linalg.norm(mix["u"] - u64) / torch.linalg.norm(u64)) <= 1e-8
    assert mix["hist"][-1] <= 1e-8 * mix["hist"][0]
    mg.close()


def test_c3_full_size_fp16_storage():
    """2D Q2, 1 quad refined 9 times (1,050,625 DOFs), k = exp(N(0,1)) per element, f = 1: the
    FP16-storage mixed form (per-level FP32 scale) against the plain FP64 MG-PCG, error <= 1e-8"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(2, 9, 1.0, seed=3)
    mg = MultiGrid.structured(2, 2, 9, 1, k)
    b = mg.assemble_rhs("one")
    common = dict(nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
    ref = mg.configure(format="sell", **common).solve(b)
    u64 = ref["u"].clone()
    for fmt in ("sell", "stencil"):
        mix = mg.configure(format=fmt, precision="f16", **common).solve(b)
        assert mix["status"] == "success" and abs(mix["iters"] - ref["iters"]) <= 1
        assert float(torch.linalg.norm(mix["u"] - u64) / torch.linalg.norm(u64)) <= 1e-8
    mg.close()


@pytest.mark.parametrize("lvl", [7, 8])
def test_stream_kernel_matches_tiled(lvl):
    """the streaming kernel of the 129^3 and 257^3 matrix-free levels forms each row from the
    tiled kernel's terms in the tiled kernel's order: one FP32 V-cycle is bit-identical with either
    kernel; mixed PCG solves (whose q . p sums its CTAs' partials in another grouping) take the
    same iterations and agree to rounding"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(3, lvl, 1.0, seed=17)
    mg = MultiGrid.structured(3, 1, lvl, 1, k)
    d = mg.assemble_rhs("one")
    common = dict(nu=2, precision="f32", format="matfree")
    a = mg.configure(**common).vcycle(d).cpu().numpy()
    b = mg.configure(stream=False, **common).vcycle(d).cpu().numpy()
    np.testing.assert_array_equal(a, b)
    s1 = mg.configure(**common).solve(d)
    s2 = mg.configure(stream=False, **common).solve(d)
    assert s1["status"] == s2["status"] == "success" and s1["iters"] == s2["iters"]
    assert relerr(s1["u"].cpu().numpy(), s2["u"].cpu().numpy()) <= 1e-12
    mg.close()


def test_unknown_flags_are_rejected():
    """fb_mg_configure refuses flag bits it does not define (FB_ERR_INVALID), and keeps the previous
    configuration usable"""
    import ctypes
    from feat3_b200 import _lib
    from feat3_b200.solver import MultiGrid
    mg = MultiGrid.structured(3, 1, 3, 1).configure(nu=2, format="matfree")
    cfg = _lib.SolverCfg()
    _lib.load().fb_solver_cfg_default(ctypes.byref(cfg))
    for bad in (16, 1 << 20, -1):
        cfg.flags = bad
        assert _lib.load().fb_mg_configure(mg.h, ctypes.byref(cfg)) == _lib.FB_ERR_INVALID
    assert mg.solve(mg.assemble_rhs("one"))["status"] == "success"
    mg.close()


@pytest.mark.parametrize("dim,lvl,prec", [(3, 6, "f32"), (2, 9, "f32"), (3, 5, "f64"), (2, 8, "f64")])
def test_coarse_cluster_matches_level_kernels(dim, lvl, prec):
    """the fused coarse cycle (one cluster, levels up to 5,000 rows) runs each row's arithmetic of
    the level-by-level kernels in the same order, and its reductions feed only the smoothers' skip
    tests: one V-cycle is bit-identical with the coarse end fused or level by level"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(dim, lvl, 1.0, seed=19)
    mg = MultiGrid.structured(dim, 1, lvl, 1, k)
    d = mg.assemble_rhs("one")
    a = mg.configure(nu=2, precision=prec, format="matfree").vcycle(d).cpu().numpy()
    b = mg.configure(nu=2, precision=prec, format="matfree", fuse_coarse=False).vcycle(d).cpu().numpy()
    np.testing.assert_array_equal(a, b)
    mg.close()


@pytest.mark.parametrize("prec", ["f16", "f32"])
def test_stencil_stream_matches_packed(prec):
    """the streaming stencil SpMV of the 257^3 level (x staged once per run, register window; FP16
    values) sums each row's 27 products in the packed kernel's slot order: one V-cycle on the FP16
    stencil values is bit-identical with either kernel (FP32 values take the packed kernel either
    way); mixed PCG solves (whose r . z groups its partial sums differently) take the same
    iterations and agree to rounding"""
    from feat3_b200.solver import MultiGrid
    k = lognormal_k(3, 8, 1.0, seed=23)
    mg = MultiGrid.structured(3, 1, 8, 1, k)
    d = mg.assemble_rhs("one")
    common = dict(nu=2, precision=prec, format="stencil")
    a = mg.configure(**common).vcycle(d).cpu().numpy()
    b = mg.configure(stream=False, **common).vcycle(d).cpu().numpy()
    np.testing.assert_array_equal(a, b)
    s1 = mg.configure(**common).solve(d)
    s2 = mg.configure(stream=False, **common).solve(d)
    assert s1["status"] == s2["status"] == "success" and s1["iters"] == s2["iters"]
    assert relerr(s1["u"].cpu().numpy(), s2["u"].cpu().numpy()) <= 1e-12
    mg.close()


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_pcg_deferred_x_updates_match_the_defect(prec):
    """PCG defers x += alpha p over two iterations (held in even iterations, applied in odd ones,
    the rest after the last): stopped after every count of 1 to 5 iterations, the returned
    iterate's true defect ||filter(b - A u)|| equals the defect the iteration carried (||r||),
    so no pending step is lost or applied twice at either parity"""
    import scipy.sparse as sp
    from feat3_b200.solver import MultiGrid
    lvl = 5
    k = lognormal_k(3, lvl, 1.0, seed=29)
    mg = MultiGrid.structured(3, 1, lvl, 1, k)
    b = mg.assemble_rhs("one")
    rp, ci, va = mg.export_csr(0)
    A = sp.csr_matrix((va, ci, rp), shape=(len(rp) - 1, len(rp) - 1))
    bc = po.Hierarchy(3, 1, lvl, lvl).filter()
    bh = b.cpu().numpy()
    for its in range(1, 6):
        out = mg.configure(nu=2, precision=prec, format="matfree", tol=1e-30, max_iter=its).solve(b)
        assert out["iters"] == its
        r = bh - A @ out["u"].cpu().numpy()
        r[bc] = 0.0
        assert abs(np.linalg.norm(r) - out["def_final"]) <= 1e-11 * np.linalg.norm(bh), (its, np.linalg.norm(r), out["def_final"])
    mg.close()

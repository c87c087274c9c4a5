"""GPU parity against the reference's own outputs (tests/golden/, made by the reference's
FEAT3 solver) and against the known answers of the reference's solver tests
(kernel/solver/basic_solver-test.cpp:69-143, 380-390), all through the C-ABI."""
import ast
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    d = np.load(os.path.join(GOLD, name + ".npz"), allow_pickle=False)
    out = {k: d[k] for k in d.files}
    out["cfg"] = ast.literal_eval(str(out["cfg"]))
    return out


def relerr(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def gpu_solve(fx, fmt="sell", precision="f64", outer=None):
    from feat3_b200.solver import MultiGrid
    cfg = fx["cfg"]
    mg = MultiGrid.structured(int(fx["dim"]), int(fx["degree"]), int(fx["level"]), int(fx["level_min"]), fx.get("k"))
    mg.configure(outer=outer or cfg.get("solver", "pcg"), nu=cfg.get("nu", 4), omega_jac=cfg.get("omega_jac", 0.5),
                 omega_rich=cfg.get("omega_rich", 1.0), coarse=cfg.get("coarse", "direct"), tol=cfg.get("tol", 1e-8),
                 max_iter=cfg.get("max_iter", 1000), precision=precision, format=fmt,
                 cycle=cfg.get("cycle", "v"), cgc=cfg.get("cgc", "fixed"))
    b = mg.assemble_rhs(str(fx["rhs_kind"]))
    return mg, mg.solve(b)


@pytest.mark.parametrize("name", ["ref_poisson_dirichlet_L5", "ref_c1_q1_2d_L7", "ref_c2_q1_3d_L4",
                                  "ref_c3_q2_2d_L5", "ref_c5_q1_3d_L4", "ref_q2_3d_L3"])
@pytest.mark.parametrize("fmt", ["sell", "stencil"])
def test_fp64_solve_matches_reference_solver(name, fmt):
    fx = load(name)
    _, res = gpu_solve(fx, fmt)
    assert res["status"] == "success"
    assert res["iters"] == int(fx["iters"])
    np.testing.assert_allclose(res["hist"], fx["hist"], rtol=1e-5)
    assert relerr(res["u"].cpu().numpy(), fx["u"]) <= 1e-10


CYCLE_FIXTURES = ["ref_cycle_f_q1_2d_L6", "ref_cycle_w_q1_3d_L4", "ref_cgc_energy_q1_2d_L6",
                  "ref_cgc_defect_f_q1_2d_L6", "ref_cycle_w_richardson_q1_2d_L5"]


@pytest.mark.parametrize("name", CYCLE_FIXTURES)
@pytest.mark.parametrize("fmt", ["sell", "stencil", "matfree"])
def test_fw_cycles_and_adaptive_cgc_match_reference(name, fmt):
    """F and W cycles, MinEnergy / MinDefect coarse-grid corrections (multigrid.hpp:1354-1519,
    1898-1925) against the reference solver's own outputs"""
    fx = load(name)
    _, res = gpu_solve(fx, fmt)
    assert res["status"] == "success"
    assert res["iters"] == int(fx["iters"])
    np.testing.assert_allclose(res["hist"], fx["hist"], rtol=1e-5)
    assert relerr(res["u"].cpu().numpy(), fx["u"]) <= 1e-10


@pytest.mark.parametrize("name", ["ref_cycle_w_q1_3d_L4", "ref_cgc_defect_f_q1_2d_L6"])
@pytest.mark.parametrize("precision", ["f32", "f16"])
def test_fw_cycles_mixed_precision(name, precision):
    """mixed forms of the F/W-cycle compositions: error against the FP64 oracle solution
    (same composition, converged to 1e-12) within 1e-8"""
    from oracle import pyoracle as po
    fx = load(name)
    cfg = fx["cfg"]
    H = po.Hierarchy(int(fx["dim"]), int(fx["degree"]), int(fx["level"]), int(fx["level_min"]), fx.get("k"))
    ref = H.solve(H.rhs(str(fx["rhs_kind"])), nu=cfg["nu"], omega_jac=cfg["omega_jac"], coarse=cfg["coarse"],
                  tol=1e-12, cycle=cfg.get("cycle", "v"), cgc=cfg.get("cgc", "fixed"))
    _, res = gpu_solve(fx, "matfree", precision=precision)
    assert res["status"] == "success"
    assert abs(res["iters"] - int(fx["iters"])) <= 1
    assert relerr(res["u"].cpu().numpy(), ref["u"]) <= 1e-8


@pytest.mark.parametrize("fmt", ["sell", "stencil"])
def test_tutorial05_composition(fmt):
    """Richardson(MultiGrid V(4,4), Richardson(0.8)+Jacobi(1.0) smoothers, unpreconditioned CG
    coarse solver with default settings) -- tutorials/tutorial_05_multigrid.cpp:373-449"""
    fx = load("ref_tutorial05_L7")
    _, res = gpu_solve(fx, fmt)
    assert res["status"] == "success"
    assert res["iters"] == int(fx["iters"]) == 6
    np.testing.assert_allclose(res["hist"], fx["hist"], rtol=1e-4)


@pytest.mark.parametrize("inner", ["f32", "f16"])
@pytest.mark.parametrize("fmt", ["sell", "stencil"])
def test_mixed_solve_matches_reference_solver(inner, fmt):
    fx = load(f"ref_mixed_{inner}_q1_3d_L4")
    _, res = gpu_solve(fx, fmt, precision=inner)
    assert res["status"] == "success"
    assert abs(res["iters"] - int(fx["iters"])) <= 1
    assert relerr(res["u"].cpu().numpy(), fx["u"]) <= 1e-7
    assert relerr(res["u"].cpu().numpy(), load("ref_c5_q1_3d_L4")["u"]) <= 1e-7


@pytest.mark.parametrize("sigma", [1, 256])
def test_dropin_on_reference_matrices(sigma):
    """The reference's own assembled hierarchy in its own numbering (push_level semantics)."""
    from feat3_b200.solver import MultiGrid
    fx = np.load(os.path.join(GOLD, "ref_matrices_q1_2d_L3.npz"))
    levels = []
    for l in (3, 2, 1):
        d = {"A": (fx[f"L{l}_A_rowptr"], fx[f"L{l}_A_col"], fx[f"L{l}_A_val"]), "filter": fx[f"L{l}_filter"]}
        if l > 1:
            d["P"] = (fx[f"L{l}_P_rowptr"], fx[f"L{l}_P_col"], fx[f"L{l}_P_val"])
            d["R"] = (fx[f"L{l}_R_rowptr"], fx[f"L{l}_R_col"], fx[f"L{l}_R_val"])
        levels.append(d)
    mg = MultiGrid.from_csr(levels, sell_sigma=sigma).configure(nu=2, omega_jac=0.5, coarse="direct")
    res = mg.solve(torch.tensor(fx["rhs_feat_order"]).cuda())
    assert res["iters"] == int(fx["iters"])
    assert relerr(res["u"].cpu().numpy(), fx["u_feat_order"]) <= 1e-10


def pointstar_fd(m, d=2):
    """restatement of PointstarFactoryFD(m, d) (kernel/lafem/pointstar_factory.hpp:181-330):
    the 2d-point FD star on m^d inner nodes, diagonal 2d, off-diagonals -1, and the Q2
    bubble vector prod 4x(1-x), x = (i+1)/(m+1) (pointstar_factory.hpp:125-151)"""
    n = m ** d
    rp, ci, va = [0], [], []
    for i in range(n):
        c = [(i // m ** a) % m for a in range(d)]
        cols = []
        for a in range(d):
            for s in (-1, 1):
                if 0 <= c[a] + s < m:
                    cols.append((i + s * m ** a, -1.0))
        cols.append((i, 2.0 * d))
        for j, v in sorted(cols):
            ci.append(j)
            va.append(v)
        rp.append(len(ci))
    q2 = np.ones(n)
    for i in range(n):
        for a in range(d):
            x = ((i // m ** a) % m + 1) / (m + 1)
            q2[i] *= 4.0 * x * (1.0 - x)
    return np.array(rp), np.array(ci), np.array(va), q2


@pytest.mark.parametrize("name,outer,coarse,ref_iters,max_iter", [
    ("CG", "pcg", "none", 28, 100),                 # basic_solver-test.cpp:130-134
    ("PCG-JAC", "pcg", "smoother", 28, 100),        # :136-141
    ("Richardson-JAC", "richardson", "smoother", 1175, 1500),  # :383-389
])
def test_basic_solver_known_answers(name, outer, coarse, ref_iters, max_iter):
    """One-level hierarchy: the coarse 'solver' is the identity (CG) or one Jacobi step
    (JacobiPrecond, omega = 1), so the driver runs the reference's CG / PCG-JAC / Richardson-JAC."""
    from feat3_b200.solver import MultiGrid
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    rp, ci, va, xref = pointstar_fd(17, 2)
    A = SparseMatrixCSR(rp, ci, va)
    rhs = DenseVector.zeros(xref.size)
    A.apply(rhs, DenseVector(torch.tensor(xref).cuda()))
    mg = MultiGrid.from_csr([{"A": (rp, ci, va), "filter": np.zeros(0, np.int64)}])
    mg.configure(outer=outer, nu=1, omega_jac=1.0, omega_rich=1.0, coarse=coarse,
                 tol=float(np.sqrt(np.finfo(np.float64).eps)), max_iter=max_iter)
    res = mg.solve(rhs.t)
    assert res["status"] == "success"
    d = float(np.sum((res["u"].cpu().numpy() - xref) ** 2))
    assert d <= np.sqrt(np.finfo(np.float64).eps)
    assert abs(res["iters"] - ref_iters) <= 2, res["iters"]


def test_adjoint_gradient_matches_reference():
    from feat3_b200.solver import MultiGrid
    fx = load("ref_adjoint_q1_2d_L6")
    mg, res = gpu_solve(fx)
    u = res["u"]
    assert relerr(u.cpu().numpy(), fx["u"]) <= 1e-10
    lam, g, info = mg.adjoint_grad(u, torch.tensor(fx["target"]).cuda())
    assert info["status"] == "success"
    assert relerr(lam.cpu().numpy(), fx["lambda"]) <= 1e-9
    assert relerr(g.cpu().numpy(), fx["grad"]) <= 1e-9


@pytest.mark.parametrize("precision", ["f64", "f16"])
def test_adjoint_gradient_finite_differences(precision):
    """dJ/dg . d against central differences (h = 1e-6) along 16 seeded directions in g-space
    (k = exp(g)), unit in the max norm (entries +-1). J(g+hd) - J(g-hd) is evaluated as
    1/2 sum (u+ - u-)(u+ + u- - 2 u_t). To keep the FP64 round-off of the two solves out of
    the difference, u+ - u- is obtained from the exact identity
        A(g+hd) (u+ - u-) = (A(g-hd) - A(g+hd)) u-,   A(g-hd) - A(g+hd) = A(-2 k sinh(h d)),
    solved with the FP64 solver. The gradient under test comes from solves in `precision`
    (the mixed form stops at 1e-12, its outer FP64 PCG's attainable accuracy with an FP16/FP32
    V-cycle). Tolerance 1e-6 relative."""
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    from feat3_b200.solver import MultiGrid
    from oracle import pyoracle as po
    fx = load("ref_adjoint_q1_2d_L6")
    lvl = int(fx["level"])
    g0 = np.log(fx["k"])
    target = torch.tensor(fx["target"]).cuda()
    kw = dict(nu=2, omega_jac=0.5, coarse="direct", tol=1e-14, max_iter=100, precision="f64")

    def hierarchy(g, **over):
        return MultiGrid.structured(2, 1, lvl, 1, np.exp(g)).configure(**{**kw, **over})

    mg = hierarchy(g0, precision=precision, tol=1e-14 if precision == "f64" else 1e-12)
    u = mg.solve(mg.assemble_rhs("one"))["u"]
    _, gk, _ = mg.adjoint_grad(u, target)
    grad_g = gk.cpu().numpy() * np.exp(g0)
    dirichlet = po.Hierarchy(2, 1, lvl, lvl).filter()
    rng = np.random.default_rng(16)
    h = 1e-6
    worst = 0.0
    for _ in range(16):
        d = rng.choice([-1.0, 1.0], size=g0.size)
        mp, mm = hierarchy(g0 + h * d), hierarchy(g0 - h * d)
        up = mp.solve(mp.assemble_rhs("one"))["u"]
        um = mm.solve(mm.assemble_rhs("one"))["u"]
        # (A(g-hd) - A(g+hd)) u- with the per-element coefficient difference -2 k sinh(h d)
        w = -2.0 * np.exp(g0) * np.sinh(h * d)
        rp, ci, va = po.Hierarchy(2, 1, lvl, lvl, w).csr()
        Aw = SparseMatrixCSR(rp, ci, va)
        rhs_d = DenseVector.zeros(um.numel())
        Aw.apply(rhs_d, DenseVector(um))
        rhs_d.t[torch.tensor(dirichlet, dtype=torch.long, device="cuda")] = 0.0
        du = mp.solve(rhs_d.t)["u"]
        dJ = 0.5 * torch.sum(du * (up + um - 2.0 * target)).item()
        fd = dJ / (2.0 * h)
        an = float(grad_g @ d)
        worst = max(worst, abs(fd - an) / abs(an))
    assert worst <= 1e-6, worst

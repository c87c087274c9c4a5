"""GPU parity at the full sizes of the measured configurations, against the oracle run on the
same seeded inputs in the same process, and against the reference's own solver at the same sizes
(tests/golden/ref_c*_full_*.npz, made by ``tests/golden/gen_golden.py --full``; they hold the
reference's iteration counts, defect histories and every 7th/97th/997th solution entry, and
tests/test_oracle_golden.py pins the oracle to them):

* 3D Q1 on 65^3 (274,625 DOFs), f = 3 pi^2 prod sin(pi x_i): the FP64 SELL-C-sigma (C = 32,
  sigma = 256) MG-PCG V(2,2) drop-in, and the mixed form FP64 Richardson around an FP32 V-cycle
  (kernel/solver/convert_precond.hpp:41-120);
* 2D Q2 on 1025^2 (1,050,625 DOFs), k = exp(N(0,1)) per element, f = 1: FP64 (structured and
  CSR hierarchies), and FP32 V-cycles on FP16 matrix values behind a per-level scale;
* 2D Q1 on 513^2 (263,169 DOFs), k = exp(g), g ~ N(0, 0.25): the adjoint gradient against the
  oracle's and the reference's FP64 adjoint, and against central differences;
* 3D Q1 on 257^3 (16,974,593 DOFs), k = exp(N(0,1)), f = 1: every storage form and precision,
  and one adjoint gradient.

Bars: the FP64 forms take the oracle's (= the reference's) iteration count and stay within 1e-10
of its solution; the mixed forms reach a relative residual of 1e-8 with an error of at most 1e-8
against the FP64 oracle solution; FP64 gradients within 1e-9 of the oracle's, and every
gradient within 1e-6 of central differences."""
import os

import numpy as np
import pytest
import torch

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PCG = dict(nu=2, omega_jac=0.5, coarse="direct", tol=1e-8)
TOL_U = 1e-10
TOL_MIXED = 1e-8


def load(name):
    d = np.load(os.path.join(GOLD, name + ".npz"), allow_pickle=False)
    return {k: d[k] for k in d.files}


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def lognormal(n, sigma, seed):
    return np.exp(sigma * np.random.default_rng(seed).standard_normal(n))


def sample_err(u, fx, key="u"):
    s = int(fx[key + "_stride"] if key + "_stride" in fx else fx["u_stride"])
    return relerr(np.asarray(u)[::s], fx[key + "_sample"])


def structured(dim, degree, level, k=None, sigma=1):
    from feat3_b200.solver import MultiGrid
    return MultiGrid.structured(dim, degree, level, 1, k, sell_sigma=sigma)


# ------------------------------------------------------------------------------- 3D Q1, 65^3
@pytest.fixture(scope="module")
def cube65():
    H = po.Hierarchy(3, 1, 6, 1)
    b = H.rhs("sine")
    return {"b": b, "ref": H.solve(b, **PCG)}


@pytest.mark.parametrize("fmt", ["sell", "stencil", "matfree"])
def test_cube65_fp64(cube65, fmt):
    ref, fx = cube65["ref"], load("ref_c2_full_q1_3d_L6")
    mg = structured(3, 1, 6, sigma=256).configure(format=fmt, **PCG)
    b = mg.assemble_rhs("sine")
    np.testing.assert_allclose(b.cpu().numpy(), cube65["b"], rtol=1e-12, atol=1e-15 * np.abs(cube65["b"]).max())
    res = mg.solve(b)
    u = res["u"].cpu().numpy()
    assert res["status"] == ref["status"] == "success"
    assert res["iters"] == ref["iters"] == int(fx["iters"])
    np.testing.assert_allclose(res["hist"], fx["hist"], rtol=1e-6)
    assert relerr(u, ref["u"]) <= TOL_U
    assert sample_err(u, fx) <= TOL_U
    mg.close()


@pytest.mark.parametrize("fmt", ["sell", "stencil", "matfree"])
def test_cube65_mixed_richardson(cube65, fmt):
    """FP64 Richardson around ConvertPrecond(FP32 MG), the reference's own mixed composition"""
    fx = load("ref_c2_full_mixed_richardson_q1_3d_L6")
    mg = structured(3, 1, 6, sigma=256).configure(format=fmt, outer="richardson", precision="f32", **PCG)
    res = mg.solve(mg.assemble_rhs("sine"))
    assert res["status"] == "success"
    assert abs(res["iters"] - int(fx["iters"])) <= 1
    assert res["hist"][-1] <= 1e-8 * res["hist"][0]
    assert relerr(res["u"].cpu().numpy(), cube65["ref"]["u"]) <= TOL_MIXED
    mg.close()


# ------------------------------------------------------------------------------- 2D Q2, 1025^2
@pytest.fixture(scope="module")
def q2_1025():
    k = lognormal(512 * 512, 1.0, 3)
    H = po.Hierarchy(2, 2, 9, 1, k)
    b = H.rhs("one")
    return {"k": k, "H": H, "b": b, "ref": H.solve(b, **PCG)}


@pytest.mark.parametrize("fmt", ["sell", "stencil", "csr"])
def test_q2_1025_fp64(q2_1025, fmt):
    from feat3_b200.solver import MultiGrid
    ref, fx, H = q2_1025["ref"], load("ref_c3_full_q2_2d_L9"), q2_1025["H"]
    np.testing.assert_allclose(q2_1025["k"].sum(), fx["k_checksum"][0], rtol=1e-12)
    if fmt == "csr":
        # the hierarchy handed over as CSR matrices (push_level semantics), as a FEAT3 build would
        levels = []
        for l in range(9, 0, -1):
            d = {"A": H.csr(l), "filter": H.filter(l)}
            if l > 1:
                d["P"], d["R"] = H.prol(l), H.rest(l)
            levels.append(d)
        mg = MultiGrid.from_csr(levels).configure(**PCG)
        b = torch.tensor(q2_1025["b"]).cuda()
    else:
        mg = structured(2, 2, 9, q2_1025["k"]).configure(format=fmt, **PCG)
        b = mg.assemble_rhs("one")
    res = mg.solve(b)
    u = res["u"].cpu().numpy()
    assert res["status"] == "success"
    assert res["iters"] == ref["iters"] == int(fx["iters"])
    np.testing.assert_allclose(res["hist"], fx["hist"], rtol=1e-6)
    assert relerr(u, ref["u"]) <= TOL_U
    assert sample_err(u, fx) <= TOL_U
    mg.close()


@pytest.mark.parametrize("fmt", ["sell", "stencil"])
def test_q2_1025_fp16_storage(q2_1025, fmt):
    """FP32 V-cycle on FP16 matrix values (one FP32 scale per level), FP64 outer PCG: error
    against the FP64 oracle solution"""
    fx = load("ref_c3_full_f16_q2_2d_L9")
    mg = structured(2, 2, 9, q2_1025["k"]).configure(format=fmt, precision="f16", **PCG)
    res = mg.solve(mg.assemble_rhs("one"))
    assert res["status"] == "success"
    assert abs(res["iters"] - int(fx["iters"])) <= 1
    assert res["hist"][-1] <= 1e-8 * res["hist"][0]
    assert relerr(res["u"].cpu().numpy(), q2_1025["ref"]["u"]) <= TOL_MIXED
    mg.close()


# ------------------------------------------------------------------------------- adjoint, 2D Q1, 513^2
ADJ_TOL = 1e-14


@pytest.fixture(scope="module")
def adj513():
    """J(k) = 1/2 ||u(k) - u_t||^2, k = exp(g), g ~ N(0, 0.25) (sigma 0.5, seed 21),
    u_t = u(k = 1) + N(0, 1e-2) noise (sigma 1e-2, seed 22); the oracle's FP64 adjoint"""
    lvl = 9
    H1 = po.Hierarchy(2, 1, lvl, 1)
    u1 = H1.solve(H1.rhs("one"), **dict(PCG, tol=ADJ_TOL))["u"]
    target = u1 + 1e-2 * np.random.default_rng(22).standard_normal(u1.size)
    g = np.log(lognormal(512 * 512, 0.5, 21))
    H = po.Hierarchy(2, 1, lvl, 1, np.exp(g))
    u = H.solve(H.rhs("one"), **dict(PCG, tol=ADJ_TOL))["u"]
    d = u - target
    d[H.filter()] = 0.0
    lam = H.solve(d, **dict(PCG, tol=ADJ_TOL))["u"]
    return {"g": g, "target": target, "u": u, "lam": lam, "grad": H.element_grad(u, lam), "level": lvl,
            "dirichlet": H.filter()}


FORMS = [("f64", "sell"), ("f64", "matfree"), ("f32", "matfree")]


def form_tol(precision):
    """solver tolerance of the gradient's solves: the mixed forms stop at 1e-12, their outer
    FP64 PCG's attainable accuracy with an FP32 V-cycle"""
    return ADJ_TOL if precision == "f64" else 1e-12


def adjoint(adj, precision, fmt):
    mg = structured(2, 1, adj["level"], np.exp(adj["g"]))
    mg.configure(format=fmt, precision=precision, **dict(PCG, tol=form_tol(precision)))
    u = mg.solve(mg.assemble_rhs("one"))["u"]
    lam, grad, info = mg.adjoint_grad(u, torch.tensor(adj["target"]).cuda())
    return mg, u, lam, grad, info


@pytest.mark.parametrize("precision,fmt", FORMS)
def test_adj513_gradient_matches_oracle_and_reference(adj513, precision, fmt):
    fx = load("ref_c4_full_adjoint_q1_2d_L9")
    np.testing.assert_allclose(adj513["target"].sum(), fx["target_checksum"][0], rtol=1e-10)
    mg, u, lam, grad, info = adjoint(adj513, precision, fmt)
    assert info["status"] == "success"
    tol = 1e-9 if precision == "f64" else TOL_MIXED
    assert relerr(u.cpu().numpy(), adj513["u"]) <= tol
    assert relerr(lam.cpu().numpy(), adj513["lam"]) <= tol
    assert relerr(grad.cpu().numpy(), adj513["grad"]) <= tol
    assert sample_err(grad.cpu().numpy(), fx, "grad") <= tol
    assert sample_err(lam.cpu().numpy(), fx, "lambda") <= tol
    mg.close()


@pytest.mark.parametrize("precision,fmt", FORMS)
def test_adj513_gradient_finite_differences(adj513, precision, fmt):
    """dJ/dg . d against central differences (h = 1e-6) along 16 seeded directions in g-space
    (k = exp(g)), entries +-1. J(g+hd) - J(g-hd) = 1/2 sum (u+ - u-)(u+ + u- - 2 u_t), with
    u+ - u- from the exact identity A(g+hd)(u+ - u-) = (A(g-hd) - A(g+hd)) u-, where
    A(g-hd) - A(g+hd) = A(-2 k sinh(h d)), solved in FP64 so the round-off of the two solves
    stays out of the difference. Tolerance 1e-6 relative."""
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    lvl, g0 = adj513["level"], adj513["g"]
    target = torch.tensor(adj513["target"]).cuda()
    mg, _, _, gk, _ = adjoint(adj513, precision, fmt)
    grad_g = gk.cpu().numpy() * np.exp(g0)
    mg.close()
    fd64 = dict(PCG, tol=ADJ_TOL, max_iter=100)
    dirichlet = torch.tensor(adj513["dirichlet"], dtype=torch.long, device="cuda")
    rng = np.random.default_rng(16)
    h = 1e-6
    worst = 0.0
    for _ in range(16):
        d = rng.choice([-1.0, 1.0], size=g0.size)
        mp = structured(2, 1, lvl, np.exp(g0 + h * d)).configure(**fd64)
        mm = structured(2, 1, lvl, np.exp(g0 - h * d)).configure(**fd64)
        up = mp.solve(mp.assemble_rhs("one"))["u"]
        um = mm.solve(mm.assemble_rhs("one"))["u"]
        rp, ci, va = po.Hierarchy(2, 1, lvl, lvl, -2.0 * np.exp(g0) * np.sinh(h * d)).csr()
        rhs_d = DenseVector.zeros(um.numel())
        SparseMatrixCSR(rp, ci, va).apply(rhs_d, DenseVector(um))
        rhs_d.t[dirichlet] = 0.0
        du = mp.solve(rhs_d.t)["u"]
        fd = 0.5 * torch.sum(du * (up + um - 2.0 * target)).item() / (2.0 * h)
        an = float(grad_g @ d)
        worst = max(worst, abs(fd - an) / abs(an))
        mp.close()
        mm.close()
    assert worst <= 1e-6, worst


# ------------------------------------------------------------------------------- 3D Q1, 257^3
ADJ257_TOL = 1e-12


@pytest.fixture(scope="module")
def cube257():
    k = lognormal(256 ** 3, 1.0, 2026)
    H = po.Hierarchy(3, 1, 8, 1, k)
    b = H.rhs("one")
    ref = H.solve(b, **PCG)
    # one adjoint solve: u_t = u + N(0, 1e-2 max|u|) noise (seed 23), J = 1/2 ||u - u_t||^2, on the
    # oracle's solution u. lambda = A^-1 (u - u_t) amplifies smooth changes of u against the rough
    # noise (two solutions that agree to 1e-11 give lambdas 1e-7 apart), so the GPU adjoint gets the
    # same u, and both adjoint solves stop at 1e-12 (lambda within ~4e-13 of the exact one)
    u = ref["u"]
    target = u + 1e-2 * np.abs(u).max() * np.random.default_rng(23).standard_normal(u.size)
    d = u - target
    d[H.filter()] = 0.0
    lam = H.solve(d, **dict(PCG, tol=ADJ257_TOL))["u"]
    grad = H.element_grad(u, lam)
    mg = structured(3, 1, 8, k, sigma=256)
    yield {"k": k, "ref": ref, "target": target, "lam": lam, "grad": grad, "mg": mg}
    mg.close()


FORMS257 = [("f64", "sell"), ("f64", "stencil"), ("f64", "matfree"), ("f32", "matfree"), ("f32", "sell"),
            ("f16", "stencil"), ("f16", "sell")]


@pytest.mark.parametrize("precision,fmt", FORMS257)
def test_cube257_solve_matches_oracle(cube257, precision, fmt):
    ref, fx, mg = cube257["ref"], load("ref_c5_full_q1_3d_L8"), cube257["mg"]
    np.testing.assert_allclose(cube257["k"].sum(), fx["k_checksum"][0], rtol=1e-12)
    mg.configure(format=fmt, precision=precision, **PCG)
    res = mg.solve(mg.assemble_rhs("one"))
    u = res["u"].cpu().numpy()
    assert res["status"] == "success"
    assert res["hist"][-1] <= 1e-8 * res["hist"][0]
    if precision == "f64":
        assert res["iters"] == ref["iters"] == int(fx["iters"])
        np.testing.assert_allclose(res["hist"], fx["hist"], rtol=1e-6)
        assert relerr(u, ref["u"]) <= TOL_U
        assert sample_err(u, fx) <= TOL_U
    else:
        assert abs(res["iters"] - ref["iters"]) <= 1
        assert relerr(u, ref["u"]) <= TOL_MIXED


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_cube257_adjoint_matches_oracle(cube257, precision):
    """the transposed MG-PCG solve and the element gradient on the matrix-free form, against the
    oracle's FP64 adjoint, both from the oracle's solution u and stopping at 1e-12"""
    mg = cube257["mg"]
    mg.configure(format="matfree", precision=precision, **dict(PCG, tol=ADJ257_TOL))
    u = torch.tensor(cube257["ref"]["u"]).cuda()
    lam, grad, info = mg.adjoint_grad(u, torch.tensor(cube257["target"]).cuda())
    assert info["status"] == "success"
    tol = 1e-9 if precision == "f64" else TOL_MIXED
    assert relerr(lam.cpu().numpy(), cube257["lam"]) <= tol
    assert relerr(grad.cpu().numpy(), cube257["grad"]) <= tol

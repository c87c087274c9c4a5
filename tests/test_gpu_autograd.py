"""The torch.autograd binding of the hand-written adjoint (feat3_b200/adjoint.py) on the 2D Q1
problem of 513^2 DOFs: k = exp(g), g ~ N(0, 0.25) per element, J = 1/2 ||u(k) - u_t||^2.
torch.autograd.grad of J through PoissonObjective (forward: MG-PCG solve; backward:
fb_mg_adjoint_grad, the transposed MG-PCG solve plus the element gradient) must equal the
oracle's FP64 adjoint gradient, and its directional derivatives must match central finite
differences of J (h = 1e-6) computed with the same binding's forward passes."""
import numpy as np
import pytest
import torch

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

LEVEL = 9
KW = dict(nu=2, omega_jac=0.5, coarse="direct", tol=1e-14)


def factory(k):
    from feat3_b200.solver import MultiGrid
    return MultiGrid.structured(2, 1, LEVEL, 1, k).configure(**KW)


@pytest.fixture(scope="module")
def problem():
    H1 = po.Hierarchy(2, 1, LEVEL, 1)
    u1 = H1.solve(H1.rhs("one"), **KW)["u"]
    target = u1 + 1e-2 * np.random.default_rng(22).standard_normal(u1.size)
    g = 0.5 * np.random.default_rng(21).standard_normal((1 << LEVEL) ** 2)
    H = po.Hierarchy(2, 1, LEVEL, 1, np.exp(g))
    u = H.solve(H.rhs("one"), **KW)["u"]
    d = u - target
    d[H.filter()] = 0.0
    lam = H.solve(d, **KW)["u"]
    return {"g": g, "target": target, "grad_k": H.element_grad(u, lam), "J": 0.5 * float(np.sum((u - target) ** 2))}


def objective(g, target):
    from feat3_b200.adjoint import PoissonObjective
    return PoissonObjective.apply(torch.exp(g), factory, "one", target)


def test_autograd_gradient_matches_oracle_adjoint(problem):
    g = torch.tensor(problem["g"], device="cuda", requires_grad=True)
    target = torch.tensor(problem["target"], device="cuda")
    J = objective(g, target)
    np.testing.assert_allclose(J.item(), problem["J"], rtol=1e-10)
    (dg,) = torch.autograd.grad(J, g)
    # chain rule through k = exp(g), done by torch: dJ/dg = dJ/dk * k
    ref = problem["grad_k"] * np.exp(problem["g"])
    err = np.linalg.norm(dg.cpu().numpy() - ref) / np.linalg.norm(ref)
    assert err <= 1e-9, err


def test_autograd_gradient_finite_differences(problem):
    """the autograd gradient's directional derivatives against central differences of J
    (h = 1e-6) along 4 seeded directions, entries +-1. J(g+hd) - J(g-hd) = 1/2 sum (u+ - u-)
    (u+ + u- - 2 u_t), with u+ - u- from the exact identity A(g+hd)(u+ - u-) = A(-2 k sinh(h d)) u-,
    so the round-off of two separate solves stays out of the difference"""
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    g0 = torch.tensor(problem["g"], device="cuda", requires_grad=True)
    target = torch.tensor(problem["target"], device="cuda")
    (dg,) = torch.autograd.grad(objective(g0, target), g0)
    g = problem["g"]
    dirichlet = torch.tensor(po.Hierarchy(2, 1, LEVEL, LEVEL).filter(), dtype=torch.long, device="cuda")
    rng = np.random.default_rng(16)
    h = 1e-6
    worst = 0.0
    for _ in range(4):
        d = rng.choice([-1.0, 1.0], size=g.size)
        mp, mm = factory(np.exp(g + h * d)), factory(np.exp(g - h * d))
        up = mp.solve(mp.assemble_rhs("one"))["u"]
        um = mm.solve(mm.assemble_rhs("one"))["u"]
        rp, ci, va = po.Hierarchy(2, 1, LEVEL, LEVEL, -2.0 * np.exp(g) * np.sinh(h * d)).csr()
        rhs_d = DenseVector.zeros(um.numel())
        SparseMatrixCSR(rp, ci, va).apply(rhs_d, DenseVector(um))
        rhs_d.t[dirichlet] = 0.0
        du = mp.solve(rhs_d.t)["u"]
        fd = 0.5 * torch.sum(du * (up + um - 2.0 * target)).item() / (2.0 * h)
        an = float(torch.dot(dg, torch.tensor(d, device="cuda")))
        worst = max(worst, abs(fd - an) / abs(an))
        mp.close()
        mm.close()
    assert worst <= 1e-6, worst

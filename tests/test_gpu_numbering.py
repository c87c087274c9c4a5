"""FEAT3 numbering on the device (fb_feat_numbering) and the solver layer in FEAT numbering.

The device descent is checked bit for bit against the oracle's entity-by-entity refinement
(itself pinned to the reference's numbering in tests/test_oracle_golden.py) and against the
reference's own numbering fixtures; at the full 3D level-8 size through size-independent
properties. A structured hierarchy created with numbering="feat" must give, in FEAT order, the
very numbers the lattice-numbered hierarchy gives, and the reference's own solution.
"""
import os

import numpy as np
import pytest
import torch

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def numbering(dim, degree, level):
    from feat3_b200.solver import feat_numbering
    d, c = feat_numbering(dim, degree, level)
    return d.cpu().numpy(), c.cpu().numpy()


@pytest.mark.parametrize("dim,degree,level", [(2, 1, 0), (2, 1, 1), (2, 1, 9), (2, 2, 8), (3, 1, 0), (3, 1, 5),
                                              (3, 2, 4)])
def test_device_numbering_matches_oracle(dim, degree, level):
    d, c = numbering(dim, degree, level)
    od, oc = po.feat_numbering(dim, degree, level)
    np.testing.assert_array_equal(d, od)
    np.testing.assert_array_equal(c, oc)


def test_device_numbering_matches_reference_fixtures():
    fx = np.load(os.path.join(GOLD, "ref_numbering.npz"))
    for key in fx.files:
        if key.endswith("_dofs"):
            dd, q, lv = key.split("_")[:3]
            d, c = numbering(int(dd[1]), int(q[1]), int(lv[1:]))
            np.testing.assert_array_equal(d, fx[key])
            np.testing.assert_array_equal(c, fx[key.replace("_dofs", "_cells")])


def test_device_numbering_full_size_properties():
    """3D Q1 level 8 (16,974,593 DOFs): a permutation, nested in level 7, equal to Q2 on level 7,
    cells grouped child by child"""
    d8, c8 = numbering(3, 1, 8)
    d7, c7 = numbering(3, 1, 7)
    q7, _ = numbering(3, 2, 7)
    m8, m7 = 257, 129
    assert np.array_equal(np.bincount(d8, minlength=m8 ** 3), np.ones(m8 ** 3, np.int64))
    assert np.array_equal(q7, d8)
    fine = np.stack(np.unravel_index(d8[:d7.size], (m8,) * 3, order="F"))
    coarse = np.stack(np.unravel_index(d7, (m7,) * 3, order="F"))
    assert np.array_equal(fine, 2 * coarse)
    parents = np.stack(np.unravel_index(c8, (256,) * 3, order="F")) // 2
    assert np.array_equal(np.ravel_multi_index(tuple(parents), (128,) * 3, order="F"), np.repeat(c7, 8))


def test_structured_solve_in_feat_numbering_matches_reference():
    """the structured device hierarchy, addressed in FEAT's numbering, against the reference's own
    solution in its own numbering (2D Q1 level 3, PCG + V(2,2), direct coarse solver)"""
    from feat3_b200.solver import MultiGrid
    fx = np.load(os.path.join(GOLD, "ref_matrices_q1_2d_L3.npz"))
    mg = MultiGrid.structured(2, 1, 3, 1, numbering="feat").configure(nu=2, omega_jac=0.5, coarse="direct")
    rhs = mg.assemble_rhs("sine")
    assert torch.allclose(rhs.cpu(), torch.tensor(fx["rhs_feat_order"]), rtol=1e-13, atol=1e-15)
    res = mg.solve(torch.tensor(fx["rhs_feat_order"]).cuda())
    assert res["status"] == "success" and res["iters"] == int(fx["iters"])
    u = res["u"].cpu().numpy()
    assert np.linalg.norm(u - fx["u_feat_order"]) <= 1e-10 * np.linalg.norm(fx["u_feat_order"])
    # the finest matrix in FEAT numbering is the reference's matrix
    rp, ci, va = mg.export_csr(0)
    np.testing.assert_array_equal(rp, fx["L3_A_rowptr"].astype(np.int64))
    np.testing.assert_array_equal(ci, fx["L3_A_col"].astype(np.int64))
    np.testing.assert_allclose(va, fx["L3_A_val"], rtol=0, atol=1e-14 * np.abs(fx["L3_A_val"]).max())
    mg.close()


@pytest.mark.parametrize("dim,degree,level,fmt,prec", [(2, 1, 6, "sell", "f64"), (3, 1, 5, "matfree", "f32"),
                                                       (3, 2, 3, "stencil", "f64")])
def test_feat_numbering_is_a_relabelling(dim, degree, level, fmt, prec):
    """same coefficient field, same right-hand side: the FEAT-numbered hierarchy returns the
    lattice-numbered results permuted, bit for bit"""
    from feat3_b200.solver import MultiGrid
    d, c = numbering(dim, degree, level)
    rng = np.random.default_rng(5)
    k_lat = np.exp(rng.standard_normal((1 << level) ** dim))
    lat = MultiGrid.structured(dim, degree, level, 1, k=k_lat).configure(nu=2, format=fmt, precision=prec)
    feat = MultiGrid.structured(dim, degree, level, 1, k=k_lat[c], numbering="feat").configure(
        nu=2, format=fmt, precision=prec)
    dd = torch.tensor(d, device="cuda")
    b_lat = lat.assemble_rhs("one")
    b_feat = feat.assemble_rhs("one")
    assert torch.equal(b_feat, b_lat[dd])
    r_lat, r_feat = lat.solve(b_lat), feat.solve(b_feat)
    assert r_lat["iters"] == r_feat["iters"]
    assert torch.equal(r_feat["u"], r_lat["u"][dd])
    h = feat.solve_host(b_feat.cpu().numpy(), zero_init=True)
    assert np.array_equal(h["u"], r_feat["u"].cpu().numpy())
    assert torch.equal(feat.vcycle(b_feat), lat.vcycle(b_lat)[dd])
    if degree == 1:
        ut_lat = 0.9 * r_lat["u"]
        lam_l, g_l, _ = lat.adjoint_grad(r_lat["u"], ut_lat)
        lam_f, g_f, _ = feat.adjoint_grad(r_feat["u"], ut_lat[dd])
        assert torch.equal(lam_f, lam_l[dd])
        assert torch.equal(g_f, g_l[torch.tensor(c, device="cuda")])
    lat.close()
    feat.close()

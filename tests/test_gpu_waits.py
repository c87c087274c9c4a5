"""The bounded waits of the bulk-staged matrix-free kernel (k_mf_q1_tiled). The test hook
fb_mg_test_expire_wait leaves one stage of the next launch unfilled: nothing arrives on it and no
copy is issued for it, so the consumers' bounded wait expires (about one second), the producer's
waits on the released stage and on its own copies expire or complete, and the kernel returns with
the event recorded. The solve must stop and return FB_ERR_TIMEOUT, and the same handle must then
solve normally, matching the oracle."""
import numpy as np
import pytest
import torch

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu

FB_ERR_TIMEOUT = 7


def relerr(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.mark.parametrize("precision,graphs", [("f64", True), ("f32", True), ("f64", False)])
def test_expired_wait_returns_timeout_and_handle_recovers(precision, graphs):
    from feat3_b200 import _lib
    from feat3_b200.solver import MultiGrid
    k = np.exp(np.random.default_rng(31).standard_normal(64 ** 3))
    H = po.Hierarchy(3, 1, 6, 1, k)
    b = H.rhs("one")
    ref = H.solve(b, nu=2, tol=1e-8)
    mg = MultiGrid.structured(3, 1, 6, 1, k).configure(nu=2, precision=precision, format="matfree", graphs=graphs)
    bg = torch.tensor(b).cuda()
    before = mg.solve(bg)
    _lib.call("fb_mg_test_expire_wait", mg.h)
    with pytest.raises(_lib.FeatError) as err:
        mg.solve(bg)
    assert err.value.code == FB_ERR_TIMEOUT
    after = mg.solve(bg)
    assert after["status"] == "success"
    assert after["iters"] == before["iters"]
    np.testing.assert_array_equal(after["u"].cpu().numpy(), before["u"].cpu().numpy())
    tol = 1e-10 if precision == "f64" else 1e-8
    if precision == "f64":
        assert after["iters"] == ref["iters"]
    assert relerr(after["u"].cpu().numpy(), ref["u"]) <= tol
    mg.close()


def test_expired_wait_in_the_streaming_kernel():
    """the same through the streaming kernel of the 129^3 level: one FP32 V-cycle, whose first
    staged launch is the streaming smoother step; the V-cycle returns FB_ERR_TIMEOUT and the next
    one on the same handle is bit-identical to one before the expiry"""
    from feat3_b200 import _lib
    from feat3_b200.solver import MultiGrid
    k = np.exp(np.random.default_rng(33).standard_normal(128 ** 3))
    mg = MultiGrid.structured(3, 1, 7, 1, k).configure(nu=2, precision="f32", format="matfree")
    d = mg.assemble_rhs("one")
    before = mg.vcycle(d).cpu().numpy()
    _lib.call("fb_mg_test_expire_wait", mg.h)
    with pytest.raises(_lib.FeatError) as err:
        mg.vcycle(d)
    assert err.value.code == FB_ERR_TIMEOUT
    after = mg.vcycle(d).cpu().numpy()
    np.testing.assert_array_equal(after, before)
    mg.close()


def test_expired_wait_in_the_stencil_stream_kernel():
    """the same through the streaming FP16 stencil SpMV of the 257^3 level: one V-cycle on the
    FP16 stencil values, whose first staged launch is that kernel's smoothing step, returns
    FB_ERR_TIMEOUT, and the next one on the same handle is bit-identical to one before the expiry"""
    from feat3_b200 import _lib
    from feat3_b200.solver import MultiGrid
    k = np.exp(np.random.default_rng(35).standard_normal(256 ** 3))
    mg = MultiGrid.structured(3, 1, 8, 1, k).configure(nu=2, precision="f16", format="stencil")
    d = mg.assemble_rhs("one")
    before = mg.vcycle(d).cpu().numpy()
    _lib.call("fb_mg_test_expire_wait", mg.h)
    with pytest.raises(_lib.FeatError) as err:
        mg.vcycle(d)
    assert err.value.code == FB_ERR_TIMEOUT
    after = mg.vcycle(d).cpu().numpy()
    np.testing.assert_array_equal(after, before)
    mg.close()

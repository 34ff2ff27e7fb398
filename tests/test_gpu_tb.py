"""GPU: temporally blocked sweep pairs (rb_tb2_kernel) against the one-colour-per-launch
sweeps. The update order inside a colour does not matter, so the two must agree bit
for bit; the residual they report must agree to rounding."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx_tb(pkg):
    old = os.environ.get("IM3D_TB")
    os.environ["IM3D_TB"] = "1"
    try:
        c = pkg.Context(0)
    finally:
        if old is None:
            del os.environ["IM3D_TB"]
        else:
            os.environ["IM3D_TB"] = old
    yield c
    c.close()


@pytest.mark.parametrize("shape", [(37, 29, 23), (64, 48, 40), (20, 70, 9), (33, 33, 66)])
@pytest.mark.parametrize("bc_type", [1, 2])
def test_blocked_pairs_bit_identical(ctx_tb, ctx, shape, bc_type):
    rng = np.random.default_rng(7)
    u = rng.random(shape, dtype=np.float32)
    b = (rng.random(shape, dtype=np.float32) - 0.5).astype(np.float32)
    a = u.copy()
    sa, ra, _ = ctx_tb.poisson_solve(a, b, bc=0.0, bc_type=bc_type, tol=0.0, max_sweeps=10,
                                  check_every=2)
    p = u.copy()
    sp, rp, _ = ctx.poisson_solve(p, b, bc=0.0, bc_type=bc_type, tol=0.0, max_sweeps=10,
                                        check_every=2)
    assert sa == sp == 10
    assert np.array_equal(a, p)
    assert abs(ra - rp) <= 1e-9 * rp


def test_blocked_solve_converges_like_plain(ctx_tb, ctx, O):
    rng = np.random.default_rng(8)
    shape = (48, 40, 36)
    u = rng.random(shape, dtype=np.float32)
    b = (rng.random(shape, dtype=np.float32) - 0.5).astype(np.float32)
    a = u.copy()
    sa, ra, ca = ctx_tb.poisson_solve(a, b, tol=1e-6)
    p = u.copy()
    sp, rp, cp = ctx.poisson_solve(p, b, tol=1e-6)
    assert ca and cp and ra <= 1e-6 and rp <= 1e-6
    assert abs(sa - sp) <= 2
    want, _, _, _ = O.poisson_solve(u, b, tol=1e-6)
    assert np.linalg.norm(a - want) / np.linalg.norm(want) < 1e-5

"""GPU: the FP32 Heaviside pass with TMA-moved rows (conv_k_heav_tma_kernel) against the
register-window kernel (IM3D_OPT_TILE_LOADS 0): the same operations on every cell, so
whole segmentations must agree bit for bit, with 19 and 25 taps, zero and periodic
halos, Dirichlet and Neumann conditions, partial row blocks, a box wider than the row,
and rows the TMA pass does not take (nz above 256 or not a multiple of 8)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BASE = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, epsilon=1e-3, lamda=0.5, bc=2, tol=0.0,
            gs_rel_res_tol=1e-6, gs_max_sweeps=400)


def _run(ctx, pkg, u0, phi0, tile, **kw):
    ctx.set_option(pkg.OPT_TILE_LOADS, tile)
    try:
        return ctx.rsfe_apply(u0, phi0, pkg.default_params(**{**BASE, **kw}), want_u=True, want_f=True)
    finally:
        ctx.set_option(pkg.OPT_TILE_LOADS, 1)


@pytest.mark.parametrize("shape, kw", [
    ((24, 20, 64), dict(maxiter=4)),
    ((13, 11, 256), dict(maxiter=3)),                      # 143 rows: a partial row block
    ((10, 9, 320), dict(maxiter=3, sigma=4.0)),            # rows the TMA pass does not take
    ((7, 6, 256), dict(maxiter=3, sigma=4.0)),             # 25 taps
    ((9, 8, 200), dict(maxiter=3)),                        # a box wider than the row (208)
    ((12, 10, 96), dict(maxiter=3, conv_cyclic=1)),        # periodic halo
    ((12, 10, 128), dict(maxiter=2, conv_cyclic=1, sigma=4.0)),
    ((14, 12, 64), dict(maxiter=3, bc=1)),                 # Neumann
    ((11, 9, 8), dict(maxiter=3)),                         # rows shorter than the halo
    ((12, 10, 70), dict(maxiter=3)),                       # not taken by the TMA pass
])
def test_tma_pass_is_bit_identical(ctx, pkg, shape, kw):
    u0 = pkg.synth.ellipsoids(shape, 3, n=2, semi_axes=(2, max(3, min(shape) // 3))).astype(np.float32)
    phi0 = pkg.synth.sphere_phi0(shape, min(shape) / 3).astype(np.float32)
    a = _run(ctx, pkg, u0, phi0, 1, **kw)
    b = _run(ctx, pkg, u0, phi0, 0, **kw)
    for key in ("phi", "u", "f1", "f2"):
        assert np.array_equal(a[key], b[key]), key
    for key in ("iterations", "total_sweeps", "residual_checks"):
        assert a["stats"][key] == b["stats"][key], key


def test_tma_pass_at_256_cube(ctx, pkg):
    u0, phi0 = pkg.synth.config_volume("c2", seed=0, dtype=np.float32)
    a = _run(ctx, pkg, u0, phi0, 1, maxiter=3, gs_max_sweeps=1000)
    b = _run(ctx, pkg, u0, phi0, 0, maxiter=3, gs_max_sweeps=1000)
    for key in ("phi", "u", "f1", "f2"):
        assert np.array_equal(a[key], b[key]), key


def test_tile_loads_option_is_checked(ctx, pkg):
    with pytest.raises(pkg.Im3dError):
        ctx.set_option(pkg.OPT_TILE_LOADS, 2)
    ctx.set_option(pkg.OPT_TILE_LOADS, 1)

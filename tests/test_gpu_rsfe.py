"""GPU: segm::rsfe_splitbregman<T>::apply through the C ABI against the CPU checker.

FP64 runs follow the reference's operations and are compared at 1e-9 relative L2
(the only differences are the convolution's rounding, direct vs FFT, and atan);
FP32 runs are compared with the FP64 checker at the acceptance bars of the
workload: u, f1, f2 relative L2 <= 1e-5, sign(phi - alpha) agreement >= 99.9%,
Dice >= 0.999."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

BASE = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, epsilon=1e-3, lamda=0.5, ls_steps=1, tol=0.0)


def _case(pkg, shape=(32, 30, 28), seed=1, r=8.0):
    u0 = pkg.synth.ellipsoids(shape, seed, n=2, semi_axes=(4, 8))
    return u0, pkg.synth.sphere_phi0(shape, r)


def _both(ctx, pkg, O, u0, phi0, dtype=np.float64, **kw):
    kw = {**BASE, **kw}
    got = ctx.rsfe_apply(u0.astype(dtype), None if phi0 is None else phi0.astype(dtype),
                         pkg.default_params(**kw), want_u=True, want_f=True)
    want = O.rsfe_apply(u0, phi0, O.default_params(**kw))
    return got, want


@pytest.mark.parametrize("mode", [
    dict(bc=2), dict(bc=1), dict(), dict(bc=2, sweep=1), dict(bc=1, sweep=1),
    dict(bc=2, ls_steps=3), dict(bc=2, ls_steps=2, ls_tol=1e-3),
    dict(bc=2, gs_rel_res_tol=1e-6), dict(bc=1, gs_rel_res_tol=1e-6, omega=1.3),
    dict(bc=2, gs_rel_res_tol=1e-6, maxiter=20),
    dict(bc=2, init_variables=1), dict(bc=2, lamda1=1.0, lamda2=2.0),
    dict(bc=2, edge_detector_sigma=1.0), dict(bc=2, gaussian_pixel_approach=1),
    dict(bc=2, conv_cyclic=1), dict(bc=1, conv_cyclic=1, edge_detector_sigma=1.0),
    dict(bc=2, conv_cyclic=1, gs_rel_res_tol=1e-6),
])
def test_apply_fp64_matches_checker(ctx, pkg, O, mode):
    u0, phi0 = _case(pkg)
    got, want = _both(ctx, pkg, O, u0, phi0, **{"maxiter": 6, **mode})
    for key in ("phi", "u", "f1", "f2"):
        assert rel(got[key], want[key]) < 1e-9, key
    for key in ("iterations", "total_sweeps", "last_sweeps", "residual_checks"):
        assert got["stats"][key] == want["stats"][key], key
    if mode.get("gs_rel_res_tol"):
        # the residual schedule carries over between solves: after the first solve,
        # most solves need one or two residual evaluations
        assert want["stats"]["residual_checks"] <= 3 * want["stats"]["iterations"]


def test_apply_cube_init_and_spacing(ctx, pkg, O):
    u0, _ = _case(pkg, (20, 24, 18))
    kw = {**BASE, "maxiter": 4, "bc": 2}
    h = (0.9, 1.0, 1.2)
    got = ctx.rsfe_apply(u0, None, pkg.default_params(**kw), h=h, want_u=True)
    want = O.rsfe_apply(u0, None, O.default_params(**kw), h=h)
    assert rel(got["phi"], want["phi"]) < 1e-9
    assert rel(got["u"], want["u"]) < 1e-9


def test_apply_tolerance_stops_like_checker(ctx, pkg, O):
    u0, phi0 = _case(pkg, (24, 24, 24))
    got, want = _both(ctx, pkg, O, u0, phi0, maxiter=200, tol=2e-3, bc=2)
    assert got["stats"]["iterations"] == want["stats"]["iterations"] < 200
    assert rel(got["phi"], want["phi"]) < 1e-9


def test_config1_fp64_64cube(ctx, pkg, O):
    """64^3 float64, 2 ellipsoids, sigma 3, 20 outer iterations, 1 sweep each."""
    u0, phi0 = pkg.synth.config_volume("c1", seed=0)
    got, want = _both(ctx, pkg, O, u0, -(-phi0), maxiter=20, bc=2)
    for key in ("phi", "u", "f1", "f2"):
        assert rel(got[key], want[key]) < 1e-9, key


@pytest.mark.parametrize("sweep", [0, 1])
def test_config1_fp32_acceptance(ctx, pkg, O, sweep):
    u0, phi0 = pkg.synth.config_volume("c1", seed=0)
    got, want = _both(ctx, pkg, O, u0, phi0, dtype=np.float32, maxiter=20, bc=2, sweep=sweep)
    for key in ("u", "f1", "f2"):
        assert rel(got[key], want[key]) <= 1e-5, key
    alpha = 0.5
    agree = np.mean((got["phi"] > alpha) == (want["phi"] > alpha))
    assert agree >= 0.999
    assert pkg.synth.dice(got["phi"], want["phi"], alpha) >= 0.999


def test_solve_mode_fp32_acceptance(ctx, pkg, O):
    u0, phi0 = _case(pkg, (48, 44, 40), seed=5, r=12.0)
    got, want = _both(ctx, pkg, O, u0, phi0, dtype=np.float32, maxiter=15, bc=2,
                      gs_rel_res_tol=1e-6)
    assert rel(got["u"], want["u"]) <= 1e-5
    assert pkg.synth.dice(got["phi"], want["phi"]) >= 0.999


@pytest.mark.parametrize("shape,extra", [
    ((37, 29, 45), dict(bc=2)),
    ((70, 33, 21), dict(bc=1)),
    ((45, 38, 52), dict(bc=2, sigma=4.0)),
    ((33, 27, 30), dict(bc=2, conv_cyclic=1)),
    ((26, 20, 36), dict(bc=1, conv_cyclic=1, sigma=4.0)),
    ((40, 36, 34), dict(bc=2, lamda1=1.0, lamda2=2.0)),
])
def test_fp32_fit_stage_shapes(ctx, pkg, O, shape, extra):
    """FP32 fitting stage (the i-axis march over chunks of planes) on ragged shapes,
    both kernel widths and both convolution boundaries, against the FP64 checker."""
    u0, phi0 = _case(pkg, shape, seed=3, r=min(shape) / 3.0)
    got, want = _both(ctx, pkg, O, u0, phi0, dtype=np.float32, **{"maxiter": 4, **extra})
    for key in ("u", "f1", "f2"):
        assert rel(got[key], want[key]) <= 1e-5, key
    assert pkg.synth.dice(got["phi"], want["phi"]) >= 0.999


def test_fp32_fit_stage_chunking_bit_identical(pkg):
    """The i-axis march gives every output cell the same operations whatever the chunk
    count, so the results are bit-identical for 1, 3 and 7 chunks and the cost model's
    choice (context option IM3D_OPT_FIT_CHUNKS)."""
    u0, phi0 = _case(pkg, (75, 34, 40), seed=9, r=12.0)
    params = pkg.default_params(**{**BASE, "maxiter": 3, "bc": 2})
    outs = []
    for chunks in (1, 3, 7, 0):
        c = pkg.Context(0)
        try:
            c.set_option(pkg.OPT_FIT_CHUNKS, chunks)
            outs.append(c.rsfe_apply(u0.astype(np.float32), phi0.astype(np.float32), params,
                                     want_u=True, want_f=True))
        finally:
            c.close()
    for o in outs[1:]:
        for key in ("phi", "u", "f1", "f2"):
            assert np.array_equal(o[key], outs[0][key]), key


def test_invalid_parameters_rejected(ctx, pkg):
    u0, phi0 = _case(pkg, (8, 8, 8))
    for bad in (dict(sigma=0.0), dict(lamda=-1.0), dict(dt=0.0), dict(epsilon=0.0),
                dict(ls_steps=0), dict(bc=7), dict(a0=1.0, b0=0.0)):
        with pytest.raises(pkg.Im3dError) as e:
            ctx.rsfe_apply(u0, phi0, pkg.default_params(**bad))
        assert e.value.status == 1, bad
    with pytest.raises(pkg.Im3dError) as e:
        ctx.rsfe_apply(np.zeros((8, 8, 1)), None)
    assert e.value.status == 2

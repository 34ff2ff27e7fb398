"""GPU: the batched entry point (uneven volumes, several streams) against single-volume
runs and the CPU checker."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

SHAPES = [(20, 18, 16), (24, 22, 20), (16, 16, 16), (30, 20, 12), (12, 14, 22)]
KW = dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=5, tol=0.0, bc=2,
          gs_rel_res_tol=1e-6)


def _volumes(pkg, dtype):
    vols = [pkg.synth.ellipsoids(s, 100 + q, n=2, semi_axes=(3, 5)).astype(dtype)
            for q, s in enumerate(SHAPES)]
    inits = [pkg.synth.sphere_phi0(s, 4.0, dtype=dtype) for s in SHAPES]
    return vols, inits


@pytest.mark.parametrize("streams", [1, 3])
def test_batch_fp64_matches_checker(ctx, pkg, O, streams):
    vols, inits = _volumes(pkg, np.float64)
    phis, stats, lat = ctx.rsfe_apply_batched(vols, inits, pkg.default_params(**KW), streams=streams)
    for v, i0, phi, st in zip(vols, inits, phis, stats):
        want = O.rsfe_apply(v, i0, O.default_params(**KW))
        assert rel(phi, want["phi"]) < 1e-9
        assert st["iterations"] == 5 and st["total_sweeps"] == want["stats"]["total_sweeps"]
    assert len(lat) == len(vols) and all(x > 0 for x in lat)


def test_batch_fp32_equals_single_runs(ctx, pkg):
    vols, inits = _volumes(pkg, np.float32)
    p = pkg.default_params(**KW)
    phis, _, _ = ctx.rsfe_apply_batched(vols, inits, p, streams=4)
    for v, i0, phi in zip(vols, inits, phis):
        single = ctx.rsfe_apply(v, i0, p)["phi"]
        assert np.array_equal(phi, single)


def test_batch_reports_a_bad_volume_and_runs_the_rest(ctx, pkg):
    vols, inits = _volumes(pkg, np.float64)
    vols.append(np.zeros((8, 8, 1)))
    inits.append(None)
    with pytest.raises(pkg.Im3dError) as e:
        ctx.rsfe_apply_batched(vols, inits, pkg.default_params(**KW), streams=2)
    assert e.value.status == 2


# ------------------------------------------------------------------ work-list batches
# sigma 3 (19 taps) and 4 (25 taps) run as a work list; nz of 12, 14, 16, 22 and 20 mix
# the vectorised (nz % 4 == 0) and the column kernels of the clamp, Bregman and div stages
WL_SHAPES = [(20, 18, 16), (24, 22, 20), (16, 16, 12), (30, 20, 14), (12, 14, 22), (9, 11, 13)]
WL_KW = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, tol=0.0, bc=2,
             gs_rel_res_tol=1e-6)


def _wl_volumes(pkg, dtype, shapes=WL_SHAPES):
    vols = [pkg.synth.ellipsoids(s, 200 + q, n=2, semi_axes=(3, 5)).astype(dtype)
            for q, s in enumerate(shapes)]
    inits = [pkg.synth.sphere_phi0(s, 4.0, dtype=dtype) for s in shapes]
    return vols, inits


def _same_as_single(ctx, pkg, vols, inits, p):
    phis, stats, lat = ctx.rsfe_apply_batched(vols, inits, p)
    for v, i0, phi, st in zip(vols, inits, phis, stats):
        single = ctx.rsfe_apply(v, i0, p)
        assert np.array_equal(phi, single["phi"])
        for key in ("iterations", "total_sweeps", "residual_checks", "last_sweeps", "not_converged"):
            assert st[key] == single["stats"][key], key
        assert st["last_tol"] == single["stats"]["last_tol"]
        assert st["last_rel_res"] == single["stats"]["last_rel_res"]
    assert len(lat) == len(vols) and all(x > 0 for x in lat)
    return phis, stats


@pytest.fixture
def wl_ctx(pkg):
    with pkg.Context(0) as c:
        c.set_option(pkg.OPT_BATCH_MODE, pkg.BATCH_WORKLIST)
        yield c


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("extra", [{}, dict(bc=1), dict(sigma=4.0), dict(lamda1=1.5, maxiter=4),
                                   dict(init_variables=1, maxiter=3)])
def test_worklist_equals_single_runs(wl_ctx, pkg, dtype, extra):
    """Every volume of a work-list batch gets its own single-volume result bit for bit:
    level set, iteration, sweep and residual-check counts, last tolerance and residual."""
    vols, inits = _wl_volumes(pkg, dtype)
    _same_as_single(wl_ctx, pkg, vols, inits, pkg.default_params(**{**WL_KW, **extra}))


def test_worklist_volumes_stop_at_their_own_iteration(wl_ctx, pkg):
    """With a tolerance the volumes leave the group at different outer iterations."""
    vols, inits = _wl_volumes(pkg, np.float32)
    _, stats = _same_as_single(wl_ctx, pkg, vols, inits,
                               pkg.default_params(**{**WL_KW, "tol": 2e-3, "maxiter": 40}))
    assert len({st["iterations"] for st in stats}) > 1


def test_worklist_matches_the_checker(wl_ctx, pkg, O):
    vols, inits = _wl_volumes(pkg, np.float64, WL_SHAPES[:3])
    p = pkg.default_params(**WL_KW)
    phis, stats, _ = wl_ctx.rsfe_apply_batched(vols, inits, p)
    for v, i0, phi, st in zip(vols, inits, phis, stats):
        want = O.rsfe_apply(v, i0, O.default_params(**WL_KW))
        assert rel(phi, want["phi"]) < 1e-9
        assert st["total_sweeps"] == want["stats"]["total_sweeps"]


def test_worklist_groups_of_more_than_64_volumes(wl_ctx, pkg):
    shapes = [(8 + q % 5, 9 + q % 3, 7 + q % 4) for q in range(70)]
    vols, inits = _wl_volumes(pkg, np.float32, shapes)
    _same_as_single(wl_ctx, pkg, vols, inits, pkg.default_params(**{**WL_KW, "maxiter": 3}))


def test_worklist_and_stream_queue_agree(ctx, pkg):
    vols, inits = _wl_volumes(pkg, np.float32)
    p = pkg.default_params(**WL_KW)
    ctx.set_option(pkg.OPT_BATCH_MODE, pkg.BATCH_STREAMS)
    a, sa, _ = ctx.rsfe_apply_batched(vols, inits, p, streams=3)
    ctx.set_option(pkg.OPT_BATCH_MODE, pkg.BATCH_WORKLIST)
    b, sb, _ = ctx.rsfe_apply_batched(vols, inits, p)
    ctx.set_option(pkg.OPT_BATCH_MODE, pkg.BATCH_AUTO)
    for x, y, u, w in zip(a, b, sa, sb):
        assert np.array_equal(x, y)
        assert u["total_sweeps"] == w["total_sweeps"]


def test_worklist_refuses_what_it_cannot_run(wl_ctx, pkg):
    vols, inits = _wl_volumes(pkg, np.float32, WL_SHAPES[:2])
    for extra in (dict(gs_rel_res_tol=0.0), dict(sigma=2.0), dict(omega=1.5)):
        with pytest.raises(pkg.Im3dError) as e:
            wl_ctx.rsfe_apply_batched(vols, inits, pkg.default_params(**{**WL_KW, **extra}))
        assert e.value.status == pkg._abi.ERR_UNSUPPORTED


def test_worklist_memory_budget_covers_the_group(pkg):
    vols, inits = _wl_volumes(pkg, np.float32, [(40, 40, 40)] * 4)
    with pkg.Context(0) as c:
        c.set_option(pkg.OPT_BATCH_MODE, pkg.BATCH_WORKLIST)
        # one volume's buffers fit, four do not
        c.set_option(pkg.OPT_DEVICE_MEMORY_LIMIT, 40 ** 3 * 4 * 40)
        with pytest.raises(pkg.Im3dError) as e:
            c.rsfe_apply_batched(vols, inits, pkg.default_params(**WL_KW))
        assert e.value.status == pkg._abi.ERR_OOM

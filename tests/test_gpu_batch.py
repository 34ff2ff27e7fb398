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

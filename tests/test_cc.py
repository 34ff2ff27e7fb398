"""Connected-component extraction (image3d<T>::connected_component,
image3d_imp.hxx:1592-2120, and the automatic extraction inside the loop,
rsfe_splitbregman_imp.hxx:448-536, 1809).

CPU: the restatement (oracle/) against the reference's own code (oracle/_ref), bit for
bit, over seeded and init-mask variants, both connectivities, binary and non-binary
output, 2-D images, seeds on faces and seeds in the dark (negative) part.
GPU: the CUDA path through the C ABI against the restatement, bit for bit in FP64,
and as the same 0/1 component in FP32 on images kept away from the pivot."""
import numpy as np
import pytest

from conftest import rel

SHAPES = [(12, 11, 10), (9, 14, 7), (5, 5, 5), (13, 12, 1), (2, 6, 5), (40, 33, 29)]


def _blobs(O, shape, seed):
    """Random noise (many small components) or, for odd seeds, a smoothed field (few
    large ones)."""
    x = np.random.default_rng(seed).random(shape)
    if seed % 2 and shape[2] > 1 and min(shape) >= 3:
        x = O.gauss_filter(x, 1.2)
    return x


def _seeds(shape, seed):
    rng = np.random.default_rng(seed)
    pts = [tuple(int(rng.integers(0, s)) for s in shape) for _ in range(4)]
    pts += [(0, 0, 0), tuple(s - 1 for s in shape), (-3, 1, 2)]
    return pts


def _need_ref(O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")


@pytest.mark.parametrize("shape", SHAPES[:5])
@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("binary", [True, False])
@pytest.mark.parametrize("field", [1, 2])
def test_oracle_seeded_matches_reference(O, shape, full, binary, field):
    _need_ref(O)
    x = _blobs(O, shape, field)
    for ijk in _seeds(shape, 2):
        for thr in (0.5, 0.3, 1.7):
            want = O.connected_component(x, ijk, threshold=thr, full_connected=full,
                                         binary_output=binary, use_reference=True)
            got = O.connected_component(x, ijk, threshold=thr, full_connected=full,
                                        binary_output=binary)
            assert np.array_equal(got, want), (ijk, thr)


@pytest.mark.parametrize("shape", SHAPES[:5])
@pytest.mark.parametrize("full", [False, True])
def test_oracle_init_matches_reference(O, shape, full):
    _need_ref(O)
    x = _blobs(O, shape, 3)
    init = (np.random.default_rng(4).random(shape) < 0.05).astype(np.float64)
    for binary in (True, False):
        want = O.connected_component(x, init=init, threshold=0.45, full_connected=full,
                                     binary_output=binary, use_reference=True)
        got = O.connected_component(x, init=init, threshold=0.45, full_connected=full,
                                    binary_output=binary)
        assert np.array_equal(got, want)


def test_components_are_not_trivial(O):
    # the fixtures above do exercise growth: a component bigger than its seed and
    # smaller than the white part
    x = np.random.default_rng(1).random((12, 11, 10))
    bw = x >= x.min() + (x.max() - x.min()) * 0.5
    for ijk in [(6, 5, 5), (3, 3, 3)]:
        cc = O.connected_component(x, ijk, threshold=0.5)
        white = bw if bw[ijk] else ~bw
        assert 1 < cc.sum() < white.sum()
        full = O.connected_component(x, ijk, threshold=0.5, full_connected=True)
        assert cc.sum() < full.sum() <= white.sum()


def _cc_params(O_or_pkg, **kw):
    base = dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=2,
                auto_extract_conn_comp=1, auto_extract_conn_comp_freq=2,
                cc_init_pixel_x=9.0, cc_init_pixel_y=8.0, cc_init_pixel_z=7.0)
    base.update(kw)
    return O_or_pkg.default_params(**base)


def _loop_volume(pkg):
    shape = (18, 16, 14)
    u0 = pkg.synth.ellipsoids(shape, seed=7, n=2, semi_axes=(3.0, 5.0))
    phi0 = pkg.synth.sphere_phi0(shape, radius=5.0)
    return u0, phi0


LOOP_MODES = [dict(), dict(cc_binary_output=0), dict(cc_init_variables=0),
              dict(auto_extract_conn_comp_freq=1, bc=1), dict(cc_init_pixel_x=0.2, alpha=0.3),
              dict(cc_init_pixel_x=-5.0)]


@pytest.mark.parametrize("mode", range(len(LOOP_MODES)))
def test_oracle_loop_with_extraction_matches_reference(O, pkg, mode):
    _need_ref(O)
    u0, phi0 = _loop_volume(pkg)
    p = _cc_params(O, **LOOP_MODES[mode])
    want = O.rsfe_apply(u0, phi0, p, use_reference=True)
    got = O.rsfe_apply(u0, phi0, p)
    assert got["stats"]["iterations"] == want["stats"]["iterations"]
    for f in ("phi", "u", "f1", "f2"):
        assert rel(got[f], want[f]) < 1e-12, f


# ------------------------------------------------------------------ CUDA path

@pytest.mark.gpu
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("field", [1, 2])
def test_gpu_seeded_matches_checker(ctx, O, shape, full, field):
    x = _blobs(O, shape, field)
    for ijk in _seeds(shape, 2):
        for binary in (True, False):
            want = O.connected_component(x, ijk, threshold=0.5, full_connected=full,
                                         binary_output=binary)
            got = ctx.connected_component(x, ijk, threshold=0.5, full_connected=full,
                                          binary_output=binary)
            assert np.array_equal(got, want), (ijk, binary)


@pytest.mark.gpu
@pytest.mark.parametrize("full", [False, True])
def test_gpu_init_matches_checker(ctx, O, full):
    shape = (40, 33, 29)
    x = _blobs(O, shape, 3)
    init = (np.random.default_rng(4).random(shape) < 0.01).astype(np.float64)
    for binary in (True, False):
        want = O.connected_component(x, init=init, threshold=0.45, full_connected=full,
                                     binary_output=binary)
        got = ctx.connected_component(x, init=init, threshold=0.45, full_connected=full,
                                      binary_output=binary)
        assert np.array_equal(got, want)


@pytest.mark.gpu
def test_gpu_fp32_and_long_component(ctx, O):
    # a serpentine corridor: the component is much longer than a tile, so the growth
    # needs many passes between tiles
    shape = (24, 64, 64)
    x = np.zeros(shape)
    for j in range(1, 63, 4):
        x[1:23, j:j + 2, 1:63] = 1.0
        kk = 1 if (j // 4) % 2 else 61
        x[1:23, j:j + 5, kk:kk + 2] = 1.0
    x = x * 0.8 + 0.1
    want = O.connected_component(x, (12, 1, 1))
    got, passes = ctx.connected_component(x, (12, 1, 1), return_passes=True)
    assert np.array_equal(got, want)
    assert passes > 2
    got32 = ctx.connected_component(x.astype(np.float32), (12, 1, 1))
    assert got32.dtype == np.float32 and np.array_equal(got32, want.astype(np.float32))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", range(len(LOOP_MODES)))
def test_gpu_loop_with_extraction_matches_checker(ctx, pkg, O, mode):
    u0, phi0 = _loop_volume(pkg)
    want = O.rsfe_apply(u0, phi0, _cc_params(O, **LOOP_MODES[mode]))
    got = ctx.rsfe_apply(u0, phi0, _cc_params(pkg, **LOOP_MODES[mode]), want_u=True, want_f=True)
    assert got["stats"]["iterations"] == want["stats"]["iterations"]
    for f in ("phi", "u", "f1", "f2"):
        assert rel(got[f], want[f]) < 1e-9, f

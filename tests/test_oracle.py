"""CPU: the C restatement of the oracle against the reference compiled from its own
headers (oracle/_ref), against numpy.fft, and against the reference's known answers
(examples/test.cxx)."""
import numpy as np
import pytest

from conftest import rel


def _need_ref(O):
    if not O.ref_available():
        pytest.skip("reference build (oracle/_ref) not present")


def test_fft_shim_matches_numpy(O):
    _need_ref(O)
    rng = np.random.default_rng(0)
    for shape in [(8, 6, 5), (14, 12, 11), (30, 7, 9), (20, 19, 13), (17, 1, 4)]:
        x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
        assert rel(O.ref_fft3d(x, -1), np.fft.fftn(x)) < 1e-14
        assert rel(O.ref_fft3d(x, +1), np.fft.ifftn(x) * x.size) < 1e-14


def test_pocketfft_behind_the_shim_matches(O):
    """The CPU baseline serves the reference's FFTW calls with scipy's pocketfft: the
    same transforms (and the same reference convolution) as the in-tree FFT."""
    _need_ref(O)
    pytest.importorskip("scipy")
    rng = np.random.default_rng(2)
    x = rng.standard_normal((20, 19, 13)) + 1j * rng.standard_normal((20, 19, 13))
    v = rng.random((18, 20, 22))
    a_fwd, a_bwd = O.ref_fft3d(x, -1), O.ref_fft3d(x, +1)
    a_conv = O.ref_gauss_filter(v, 2.0)
    try:
        assert O.use_pocketfft(2)
        assert rel(O.ref_fft3d(x, -1), a_fwd) < 1e-14
        assert rel(O.ref_fft3d(x, +1), a_bwd) < 1e-14
        assert rel(O.ref_gauss_filter(v, 2.0), a_conv) < 1e-13
    finally:
        O.use_pocketfft(None)
    assert np.array_equal(O.ref_fft3d(x, -1), a_fwd)


@pytest.mark.parametrize("h", [(1.0, 1.0, 1.0), (0.8, 1.1, 1.3)])
@pytest.mark.parametrize("gpa", [False, True])
def test_separable_conv_equals_reference_fft_and_direct(O, h, gpa):
    _need_ref(O)
    x = np.random.default_rng(1).random((20, 22, 24))
    a = O.gauss_filter(x, 2.0, h=h, pixel_approach=gpa)
    fft = O.ref_gauss_filter(x, 2.0, h=h, pixel_approach=gpa)
    direct = O.ref_gauss_filter(x, 2.0, h=h, pixel_approach=gpa, direct=True)
    assert np.abs(a - fft).max() < 1e-14
    assert np.abs(a - direct).max() < 1e-14


@pytest.mark.parametrize("case", [((20, 22, 24), (1.0, 1.0, 1.0), False, 2.0),
                                  ((9, 14, 11), (0.8, 1.1, 1.3), True, 1.5),
                                  ((7, 5, 30), (1.0, 1.0, 1.0), False, 3.0),
                                  ((12, 10, 8), (1.0, 0.9, 1.2), False, 2.5)])
def test_cyclic_conv_equals_reference(O, case):
    # cyclic_fftw_convolution: periodic boundary, also on axes shorter than the kernel
    _need_ref(O)
    shape, h, gpa, sigma = case
    x = np.random.default_rng(5).random(shape)
    a = O.gauss_filter(x, sigma, h=h, pixel_approach=gpa, cyclic=True)
    b = O.ref_gauss_filter(x, sigma, h=h, pixel_approach=gpa, cyclic=True)
    assert np.abs(a - b).max() < 1e-14
    assert not np.allclose(a, O.gauss_filter(x, sigma, h=h, pixel_approach=gpa))


@pytest.mark.parametrize("shape", [(7, 9, 11), (3, 3, 3), (5, 4, 3)])
@pytest.mark.parametrize("h", [(1.0, 1.0, 1.0), (0.8, 1.1, 1.3)])
def test_grad_div_bit_exact_vs_reference(O, shape, h):
    _need_ref(O)
    rng = np.random.default_rng(2)
    x = rng.random(shape)
    assert np.array_equal(O.grad(x, h), O.ref_grad(x, h))
    v = rng.random((3,) + shape)
    assert np.array_equal(O.div(v, h), O.ref_div(v, h))


@pytest.mark.parametrize("neu", [False, True])
@pytest.mark.parametrize("h", [(1.0, 1.0, 1.0), (0.8, 1.1, 1.3)])
def test_gauss_seidel_bit_exact_vs_reference(O, neu, h):
    _need_ref(O)
    rng = np.random.default_rng(3)
    r0 = rng.random((9, 8, 10))
    b = rng.random((9, 8, 10))
    a = O.ref_gs(r0, b, dt=0.7, bc=0.3, neu=neu, sweeps=3, h=h)
    c = O.poisson_sweeps(r0, b, dt=0.7, bc=0.3, bc_type=O.BC_NEU if neu else O.BC_DIR, sweeps=3, h=h)
    assert np.array_equal(a, c)


def test_change_range_matches_reference(O):
    _need_ref(O)
    x = np.random.default_rng(4).random((5, 6, 7)) * 3 - 1
    got = O.ref_change_range(x, 1.0, 0.0)
    want = (x - x.min()) / ((x - x.min()).max() / 1.0) + 0.0
    assert np.array_equal(got, want)


@pytest.mark.parametrize("mode", ["lex-dir", "lex-neu", "default", "rb", "solve", "cyclic",
                                  "cyclic-neu-edge"])
def test_full_loop_restatement_vs_reference(O, pkg, mode):
    _need_ref(O)
    shape = (20, 18, 16)
    u0 = pkg.synth.ellipsoids(shape, 1, n=2, semi_axes=(3, 6))
    phi0 = pkg.synth.sphere_phi0(shape, 5.0)
    kw = dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=5, ls_steps=1, tol=0.0)
    kw.update({"lex-dir": dict(bc=O.BC_DIR), "lex-neu": dict(bc=O.BC_NEU), "default": {},
               "rb": dict(bc=O.BC_DIR, sweep=O.SWEEP_RB),
               "solve": dict(bc=O.BC_DIR, gs_rel_res_tol=1e-6),
               "cyclic": dict(bc=O.BC_DIR, conv_cyclic=1),
               "cyclic-neu-edge": dict(bc=O.BC_NEU, conv_cyclic=1, edge_detector_sigma=1.0)}[mode])
    p = O.default_params(**kw)
    a = O.rsfe_apply(u0, phi0, p)
    b = O.rsfe_apply(u0, phi0, p, use_reference=True)
    for key in ("phi", "u", "f1", "f2"):
        assert rel(a[key], b[key]) < 1e-12, key
    assert a["stats"]["iterations"] == b["stats"]["iterations"] == 5
    assert a["stats"]["total_sweeps"] == b["stats"]["total_sweeps"]
    assert a["stats"]["residual_checks"] == b["stats"]["residual_checks"]


def test_known_answers_of_reference_examples(O):
    """examples/test.cxx:226-252: grad of enumerate (i + 3j + 9k on 3x3x3) is
    (1, 3, 9) everywhere and div(grad) is 0."""
    i, j, k = np.meshgrid(np.arange(3), np.arange(3), np.arange(3), indexing="ij")
    e = (i + 3 * j + 9 * k).astype(np.float64)
    g = O.grad(e)
    assert np.all(g[0] == 1) and np.all(g[1] == 3) and np.all(g[2] == 9)
    assert np.all(O.div(g) == 0)
    # norm1 = normL1 = 351, max = 26, min = 0 (:245-252)
    assert e.sum() == 351 and e.max() == 26 and e.min() == 0

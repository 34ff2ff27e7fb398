"""GPU: each operator of the path through the C ABI against the CPU checker.

Bars: FP64 stencils and Gauss-Seidel sweeps are bit-exact against the restatement
(which is bit-exact against the reference); FP64 convolution within 1e-13 relative
(the reference's own FFT differs from its direct convolution by ~1e-15); FP32
within 2e-6 relative L2 (a few ulp of float accumulated over 19-tap sums)."""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

SHAPES = [(20, 22, 24), (7, 9, 11), (3, 3, 3), (33, 17, 5)]
SPACINGS = [(1.0, 1.0, 1.0), (0.8, 1.1, 1.3)]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("h", SPACINGS)
def test_gauss_filter(ctx, O, shape, h):
    x = np.random.default_rng(10).random(shape)
    want = O.gauss_filter(x, 2.0, h=h)
    got64 = ctx.gauss_filter(x, 2.0, h=h)
    assert rel(got64, want) < 1e-13
    got32 = ctx.gauss_filter(x.astype(np.float32), 2.0, h=h)
    assert got32.dtype == np.float32
    assert rel(got32, want) < 2e-6


@pytest.mark.parametrize("case", [((20, 22, 24), (1.0, 1.0, 1.0), 2.0), ((9, 14, 11), (0.8, 1.1, 1.3), 1.5),
                                  ((7, 5, 30), (1.0, 1.0, 1.0), 3.0), ((40, 36, 33), (1.0, 1.0, 1.0), 3.0)])
def test_gauss_filter_cyclic(ctx, O, case):
    shape, h, sigma = case
    x = np.random.default_rng(12).random(shape)
    want = O.gauss_filter(x, sigma, h=h, cyclic=True)
    assert rel(ctx.gauss_filter(x, sigma, h=h, cyclic=True), want) < 1e-13
    got32 = ctx.gauss_filter(x.astype(np.float32), sigma, h=h, cyclic=True)
    assert rel(got32, want) < 2e-6


def test_gauss_filter_pixel_approach_and_radius(ctx, O):
    x = np.random.default_rng(11).random((16, 15, 14))
    for gpa in (False, True):
        for radius in (2.0, 3.0):
            want = O.gauss_filter(x, 1.5, h=(0.7, 1.0, 1.4), radius=radius, pixel_approach=gpa)
            got = ctx.gauss_filter(x, 1.5, h=(0.7, 1.0, 1.4), radius=radius, pixel_approach=gpa)
            assert rel(got, want) < 1e-13


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("h", SPACINGS)
def test_grad_div_fp64_bit_exact(ctx, O, shape, h):
    rng = np.random.default_rng(12)
    x = rng.random(shape)
    assert np.array_equal(ctx.grad(x, h), O.grad(x, h))
    v = rng.random((3,) + shape)
    assert np.array_equal(ctx.div(v, h), O.div(v, h))
    g32 = ctx.grad(x.astype(np.float32), h)
    assert rel(g32, O.grad(x, h)) < 1e-6


@pytest.mark.parametrize("bc_type", ["dir", "neu"])
@pytest.mark.parametrize("shape", [(9, 8, 10), (3, 3, 3), (12, 5, 7)])
@pytest.mark.parametrize("h", SPACINGS)
def test_lexicographic_sweep_fp64_bit_exact(ctx, O, bc_type, shape, h):
    rng = np.random.default_rng(13)
    r0 = rng.random(shape)
    b = rng.random(shape)
    t = O.BC_NEU if bc_type == "neu" else O.BC_DIR
    want = O.poisson_sweeps(r0, b, dt=0.7, bc=0.3, bc_type=t, sweeps=3, h=h)
    got = ctx.poisson_sweeps(r0.copy(), b, dt=0.7, bc=0.3, bc_type=t, sweeps=3, h=h)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("bc_type", ["dir", "neu"])
@pytest.mark.parametrize("shape", [(9, 8, 10), (12, 5, 7), (4, 4, 3)])
def test_red_black_sweep_fp64_bit_exact(ctx, O, bc_type, shape):
    rng = np.random.default_rng(14)
    r0 = rng.random(shape)
    b = rng.random(shape)
    t = O.BC_NEU if bc_type == "neu" else O.BC_DIR
    want = O.poisson_sweeps(r0, b, dt=1.0, bc=0.2, bc_type=t, order=O.SWEEP_RB, sweeps=4)
    got = ctx.poisson_sweeps(r0.copy(), b, dt=1.0, bc=0.2, bc_type=t, order=O.SWEEP_RB, sweeps=4)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("bc_type", ["dir", "neu"])
@pytest.mark.parametrize("omega", [1.0, 1.3])
def test_poisson_solve_matches_oracle(ctx, O, bc_type, omega):
    rng = np.random.default_rng(15)
    shape = (18, 16, 14)
    u = rng.random(shape)
    b = rng.random(shape) - 0.5
    t = O.BC_NEU if bc_type == "neu" else O.BC_DIR
    want, sw_w, rel_w, st = O.poisson_solve(u, b, dt=1.0, bc=0.0, bc_type=t, tol=1e-8,
                                            check_every=2, omega=omega)
    assert st == 0
    got = u.copy()
    sw, rr, conv = ctx.poisson_solve(got, b, dt=1.0, bc=0.0, bc_type=t, tol=1e-8, check_every=2,
                                     omega=omega)
    assert conv and sw == sw_w
    assert abs(rr - rel_w) <= 1e-6 * rel_w + 1e-15
    assert rel(got, want) < 1e-12
    got32 = u.astype(np.float32)
    sw32, rr32, conv32 = ctx.poisson_solve(got32, b.astype(np.float32), bc_type=t, tol=1e-6,
                                           check_every=2, omega=omega)
    assert conv32 and rr32 <= 1e-6
    want6, _, _, _ = O.poisson_solve(u, b, bc_type=t, tol=1e-6, check_every=2, omega=omega)
    assert rel(got32, want6) < 1e-5


def test_poisson_solve_reports_not_converged(ctx, pkg):
    rng = np.random.default_rng(16)
    u = rng.random((10, 10, 10))
    b = rng.random((10, 10, 10))
    sw, rr, conv = ctx.poisson_solve(u, b, tol=1e-30, max_sweeps=3, check_every=1)
    assert not conv and sw == 3 and rr > 0


@pytest.mark.parametrize("shape,status", [((8, 8, 1), 2), ((2, 8, 8), 2), ((8, 0, 8), 1)])
def test_unsupported_and_invalid_sizes(ctx, pkg, shape, status):
    with pytest.raises(pkg.Im3dError) as e:
        ctx.gauss_filter(np.zeros(shape), 1.0)
    assert e.value.status == status


def test_invalid_sigma(ctx, pkg):
    with pytest.raises(pkg.Im3dError) as e:
        ctx.gauss_filter(np.zeros((4, 4, 4)), 0.0)
    assert e.value.status == 1


def test_device_tensors_in_place(ctx, O):
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(17).random((12, 13, 14))
    xt = torch.from_numpy(x).cuda()
    out = ctx.gauss_filter(xt, 2.0)
    assert out.is_cuda
    assert rel(out.cpu().numpy(), O.gauss_filter(x, 2.0)) < 1e-13

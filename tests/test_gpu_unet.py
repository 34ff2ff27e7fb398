"""GPU: the learned warm start's network on the tensor cores, against the CPU checker
(tests/unet_ref.py: the same network in torch FP32 on the CPU, with the GPU path's BF16
roundings emulated where it rounds).

* im3d_conv3d_bf16 (one tcgen05 implicit-GEMM 3x3x3 convolution, FP32 output) against
  an FP64 convolution of the same BF16 inputs and filter: relative L2 <= 1e-5 (only the
  order of the FP32 sums differs), over every (cin, cout) pair the network uses, the
  tile widths 16..128 and a 256-wide volume, ragged D and H, a channel offset into a
  wider tensor and two samples.
* The network's forward pass: every layer rounds its output to BF16, so a sum whose
  order differs lands on the other side of a rounding now and then, and the flips
  compound over the 13 layers. The GPU output must lie within 1e-2 of the FP64-summed
  checker with the BF16 roundings, and nearer to it than the checker without them is.
* Its gradients (the tcgen05 data- and weight-gradient kernels, the pooling, transposed
  convolution and output-layer kernels): per parameter tensor relative L2 <= 3e-2 and
  cosine >= 0.999 against torch autograd; the loss to 1e-3.
* Training reduces the loss; the warm start inside the segmentation loop leaves the
  result unchanged when the network predicts nothing, and training during a
  segmentation does not change the segmentation.
"""
import numpy as np
import pytest

from conftest import rel

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _bf16_tensor(shape, gen):
    return torch.randn(shape, generator=gen).to(torch.bfloat16)


@pytest.mark.parametrize("cin, cout, dims, nsamp, pitch, coff", [
    (16, 16, (4, 6, 16), 1, 16, 0),
    (16, 32, (5, 7, 32), 1, 16, 0),
    (32, 16, (3, 5, 64), 2, 48, 16),
    (32, 32, (4, 4, 128), 1, 32, 0),
    (64, 16, (3, 3, 128), 1, 64, 0),
    (64, 32, (2, 6, 64), 1, 64, 0),
    (32, 64, (3, 4, 32), 1, 32, 0),
    (64, 64, (2, 3, 16), 1, 64, 0),
    (16, 16, (2, 3, 256), 1, 16, 0),
])
def test_conv3d_matches_fp64(ctx, cin, cout, dims, nsamp, pitch, coff):
    gen = torch.Generator().manual_seed(cin * 7 + cout + dims[2])
    x = _bf16_tensor((nsamp,) + dims + (pitch,), gen)
    # the filter the kernel multiplies is BF16: give the checker the same values
    w = (_bf16_tensor((cout, cin, 3, 3, 3), gen).float() * 0.2).to(torch.bfloat16).float()
    b = torch.randn(cout, generator=gen)
    got = ctx.conv3d_bf16(x.cuda(), w, b, cin=cin, c_off=coff).cpu().double()
    xin = x[..., coff:coff + cin].double().permute(0, 4, 1, 2, 3)
    want = torch.nn.functional.conv3d(xin, w.double(), b.double(), padding=1).permute(0, 2, 3, 4, 1)
    assert rel(got.numpy(), want.numpy()) <= 1e-5


def _net_case(pkg, ctx, shape, nsamp, seed):
    import unet_ref as R

    net = pkg.UNet(ctx, seed=seed)
    flat = net.get_params()
    lay, _ = R.layout()
    rng = np.random.default_rng(seed)
    o, _ = lay["out.w"]
    flat[o:o + 16] = rng.standard_normal(16) * 0.3  # the output layer starts at zero
    ob, _ = lay["up2.b"]
    flat[ob:ob + 32] = rng.standard_normal(32) * 0.1
    net.set_params(flat)
    x = rng.standard_normal((nsamp, 4) + shape).astype(np.float32)
    t = rng.standard_normal((nsamp,) + shape).astype(np.float32)
    return net, flat, x, t


@pytest.mark.parametrize("shape, nsamp", [((8, 8, 64), 1), ((4, 8, 128), 2), ((4, 4, 256), 1)])
def test_network_forward_matches_cpu(pkg, ctx, shape, nsamp):
    import unet_ref as R

    net, flat, x, _ = _net_case(pkg, ctx, shape, nsamp, seed=11)
    with net:
        y = net.forward(x)
    ps = R.unflatten(flat)
    ps64 = {k: v.double() for k, v in ps.items()}
    x64 = torch.tensor(x, dtype=torch.float64)
    want = R.forward(x64, ps64, emulate_bf16=True)[:, 0].detach().numpy()
    plain = R.forward(x64, ps64, emulate_bf16=False)[:, 0].detach().numpy()
    # Each BF16 rounding of an activation near a rounding boundary flips with the order
    # of the FP32 sums before it (one BF16 ulp, 0.4 %), and the flips propagate through
    # the layers, so the GPU and the checker differ by a fraction of the BF16 effect
    # itself (measured on B200: 0.02-0.63 %, against a BF16 effect of 0.8-0.9 %).
    got = rel(y, want)
    assert got <= 1e-2, got
    assert got < rel(plain, want), (got, rel(plain, want))


@pytest.mark.parametrize("shape, nsamp", [((8, 8, 64), 1), ((4, 4, 128), 2)])
def test_network_gradients_match_cpu(pkg, ctx, shape, nsamp):
    import unet_ref as R

    net, flat, x, t = _net_case(pkg, ctx, shape, nsamp, seed=5)
    with net:
        loss, g = net.train_step(x, t, lr=0.0, want_grads=True)
        after = net.get_params()
    assert np.array_equal(after, flat)  # lr = 0: no update
    want_loss, want_g, _ = R.loss_and_grads(x, t, flat)
    assert abs(loss - want_loss) <= 1e-3 * abs(want_loss)
    lay, _ = R.layout()
    for k, (o, shp) in lay.items():
        n = int(np.prod(shp))
        a = g[o:o + n].astype(np.float64)
        b = want_g[o:o + n]
        if k == "e1a.w":  # the 12 padding input channels see zeros: compare the 4 used
            a = a.reshape(shp)[:, :4].ravel()
            b = b.reshape(shp)[:, :4].ravel()
        nb = np.linalg.norm(b)
        assert nb > 0, k
        assert np.linalg.norm(a - b) / nb <= 3e-2, (k, np.linalg.norm(a - b) / nb)
        assert a @ b / (np.linalg.norm(a) * nb) >= 0.999, k


def test_training_reduces_the_loss(pkg, ctx):
    net, _, x, _ = _net_case(pkg, ctx, (8, 8, 64), 1, seed=3)
    # a smooth target the network can fit: a weighted sum of the inputs
    t = (0.5 * x[:, 0] - 0.25 * x[:, 3]).astype(np.float32)
    with net:
        first = net.train_step(x, t, lr=2e-3)
        for _ in range(60):
            last = net.train_step(x, t, lr=2e-3)
    assert last < 0.5 * first, (first, last)


BASE = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, epsilon=1e-3, lamda=0.5, tol=0.0, bc=2,
            gs_rel_res_tol=1e-6, maxiter=6)


def _seg_case(pkg, shape=(32, 32, 64), seed=2):
    u0 = pkg.synth.ellipsoids(shape, seed, n=2, semi_axes=(5, 10)).astype(np.float32)
    return u0, pkg.synth.sphere_phi0(shape, 10.0).astype(np.float32)


def test_untrained_warm_start_changes_nothing(pkg):
    u0, phi0 = _seg_case(pkg)
    params = pkg.default_params(**BASE)
    with pkg.Context(0) as c:
        plain = c.rsfe_apply(u0, phi0, params, want_u=True, want_f=True)
        with pkg.UNet(c, seed=1) as net:  # output layer zero: it predicts no correction
            c.set_warm_start(net, pkg.WS_PREDICT)
            ws = c.rsfe_apply(u0, phi0, params, want_u=True, want_f=True)
            c.set_warm_start(None, pkg.WS_OFF)
    for key in ("phi", "u", "f1", "f2"):
        assert np.array_equal(ws[key], plain[key]), key
    assert ws["stats"]["ws_used"] == 0
    assert ws["stats"]["ws_rejected"] == BASE["maxiter"]
    assert ws["stats"]["total_sweeps"] == plain["stats"]["total_sweeps"]


def test_training_during_a_segmentation_leaves_it_unchanged(pkg):
    u0, phi0 = _seg_case(pkg, seed=4)
    params = pkg.default_params(**BASE)
    with pkg.Context(0) as c:
        plain = c.rsfe_apply(u0, phi0, params, want_u=True)
        with pkg.UNet(c, seed=2) as net:
            before = net.get_params()
            c.set_warm_start(net, pkg.WS_TRAIN, lr=1e-3)
            tr = c.rsfe_apply(u0, phi0, params, want_u=True)
            c.set_warm_start(None, pkg.WS_OFF)
            after = net.get_params()
            # the trained network then starts solves of another volume; every solve still
            # reaches the tolerance
            c.set_warm_start(net, pkg.WS_PREDICT)
            u1, p1 = _seg_case(pkg, seed=9)
            pr = c.rsfe_apply(u1, p1, params, want_u=True)
            c.set_warm_start(None, pkg.WS_OFF)
            ref = c.rsfe_apply(u1, p1, params, want_u=True)
    assert np.array_equal(tr["phi"], plain["phi"]) and np.array_equal(tr["u"], plain["u"])
    assert tr["stats"]["ws_loss"] > 0
    assert not np.array_equal(before, after)
    assert pr["stats"]["not_converged"] == 0 and pr["stats"]["last_rel_res"] <= 1e-6
    assert pr["stats"]["ws_used"] + pr["stats"]["ws_rejected"] == BASE["maxiter"]
    assert pkg.synth.dice(pr["phi"], ref["phi"]) >= 0.999

"""CPU checker of the learned warm start's network (TEST INFRASTRUCTURE ONLY).

The same 3-level U-Net as 3dimagetoolkit_b200/csrc/unet.cu, written with torch.nn.functional
on the CPU in FP32, reading the flat parameter vector in the library's order
(include/im3d_b200.h, im3d_unet_param_count). With emulate_bf16 the BF16 roundings of the
GPU path are applied at the same points: the filters, every layer's output after its
ReLU, the transposed convolutions' outputs, and (through gradient hooks) every gradient
the GPU stores in BF16. What is left between the two is the order of the FP32 sums.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

CONV = [("e1a", 16, 16), ("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32), ("e3a", 32, 64),
        ("e3b", 64, 64), ("d2a", 64, 32), ("d2b", 32, 32), ("d1a", 32, 16), ("d1b", 16, 16)]


def layout():
    """name -> (offset, shape) of every parameter tensor in the flat vector."""
    off = 0
    out = {}
    for name, cin, cout in CONV:
        out[name + ".w"] = (off, (cout, cin, 3, 3, 3))
        off += cout * cin * 27
        out[name + ".b"] = (off, (cout,))
        off += cout
    for name, cin, cout in (("up2", 64, 32), ("up1", 32, 16)):
        out[name + ".w"] = (off, (8, cin, cout))
        off += 8 * cin * cout
        out[name + ".b"] = (off, (cout,))
        off += cout
    out["out.w"] = (off, (16,))
    off += 16
    out["out.b"] = (off, (1,))
    off += 1
    return out, off


def bf16(t):
    return t.to(torch.bfloat16).to(t.dtype)


def round_st(t):
    """The value rounded to BF16, the gradient passed through unrounded (the GPU rounds
    stored values; the gradients it stores are rounded by the hooks instead)."""
    return t + (bf16(t.detach()) - t.detach())


def unflatten(flat, requires_grad=False):
    lay, total = layout()
    assert flat.size == total, (flat.size, total)
    ps = {}
    for k, (o, shp) in lay.items():
        n = int(np.prod(shp))
        ps[k] = torch.tensor(flat[o:o + n].reshape(shp), dtype=torch.float32, requires_grad=requires_grad)
    return ps


def flatten_grads(ps):
    lay, total = layout()
    out = np.zeros(total, dtype=np.float64)
    for k, (o, shp) in lay.items():
        g = ps[k].grad
        out[o:o + int(np.prod(shp))] = 0 if g is None else g.detach().numpy().ravel()
    return out


def _upconv(x, w, b, emulate):
    # w[o][ci][co], child o = 4 di + 2 dj + dk -> conv_transpose3d weight [ci][co][2][2][2]
    wt = w.permute(1, 2, 0).reshape(w.shape[1], w.shape[2], 2, 2, 2)
    if emulate:
        wt = round_st(wt)
    return F.conv_transpose3d(x, wt, b, stride=2)


def forward(x, ps, emulate_bf16=True, hooks=False):
    """x: [N, 4, D, H, W] FP32 -> y [N, 1, D, H, W]."""
    rd = round_st if emulate_bf16 else (lambda t: t)

    def gh(t):
        if hooks and emulate_bf16 and t.requires_grad:
            t.register_hook(lambda g: bf16(g))
        return t

    def conv(t, name):
        w = ps[name + ".w"]
        z = gh(F.conv3d(t, rd(w), ps[name + ".b"], padding=1))  # its gradient: stored in BF16
        return rd(F.relu(z))

    x0 = rd(torch.cat([x, torch.zeros((x.shape[0], 12) + tuple(x.shape[2:]), dtype=x.dtype)], 1))
    a1 = conv(x0, "e1a")
    a = conv(a1, "e1b")
    p1 = gh(F.max_pool3d(a, 2))
    b1 = conv(p1, "e2a")
    b = conv(b1, "e2b")
    p2 = gh(F.max_pool3d(b, 2))
    c1 = conv(p2, "e3a")
    c = conv(c1, "e3b")
    u2 = rd(_upconv(c, ps["up2.w"], ps["up2.b"], emulate_bf16))
    cat2 = gh(torch.cat([u2, b], 1))
    d2a = conv(cat2, "d2a")
    d2 = conv(d2a, "d2b")
    u1 = rd(_upconv(d2, ps["up1.w"], ps["up1.b"], emulate_bf16))
    cat1 = gh(torch.cat([u1, a], 1))
    d1a = conv(cat1, "d1a")
    d1 = gh(conv(d1a, "d1b"))
    y = torch.einsum("ncdhw,c->ndhw", d1, ps["out.w"]) + ps["out.b"]
    return y[:, None]


def loss_and_grads(x, target, flat, emulate_bf16=True):
    """Mean squared error and the FP32 gradient of every parameter (flat order)."""
    ps = unflatten(flat, requires_grad=True)
    y = forward(torch.tensor(x), ps, emulate_bf16, hooks=True)
    t = torch.tensor(target)[:, None]
    loss = ((y - t) ** 2).mean()
    loss.backward()
    return float(loss), flatten_grads(ps), y.detach().numpy()[:, 0]

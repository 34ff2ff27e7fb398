"""Seeded synthetic volumes for the segmentation workloads.

The reference ships no image data (its examples read user files), so every workload
here is generated. Volumes use the reference's image3d layout ``v[i, j, k]`` with k
the contiguous axis and unit spacing; "along z" means along k.

Generators (all intensities before bias and noise):

* ``ellipsoids``: background ~ N(bg_mean, bg_std^2) per voxel; ``n`` ellipsoids with
  semi-axes ~ U(lo, hi) and centres ~ U(inside the volume); inside ellipsoid e each
  voxel ~ N(mu_e, fg_std^2) with mu_e fixed (``fg_mean``) or ~ U(fg_range); a
  multiplicative bias ramping linearly along k from ``bias[0]`` to ``bias[1]``;
  additive noise ~ N(0, noise^2).
* ``ct_like``: background ~ N(0.1, 0.02^2), a body ellipsoid at 0.4, ``n`` organ
  ellipsoids inside it with means ~ U(0.55, 0.9); multiplicative bias
  1 + sum of 3 random low-frequency cosines of amplitude 0.15; noise ~ N(0, 0.04^2).
* ``sphere_phi0``: the initial level set, the signed distance to a sphere at the
  volume centre, positive inside (r - |x - c|).
"""
from __future__ import annotations

import numpy as np


def _grid(shape):
    X, Y, Z = shape
    return (np.arange(X, dtype=np.float64)[:, None, None],
            np.arange(Y, dtype=np.float64)[None, :, None],
            np.arange(Z, dtype=np.float64)[None, None, :])


def ellipsoids(shape, seed, n=2, semi_axes=(8.0, 16.0), bg_mean=0.2, bg_std=0.03,
               fg_mean=0.8, fg_range=None, fg_std=0.03, bias=(0.8, 1.2), noise=0.05,
               dtype=np.float64):
    """Background plus ``n`` textured ellipsoids, linear bias along k, Gaussian noise."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    X, Y, Z = shape
    dims = np.array(shape, dtype=np.float64)
    vol = bg_mean + bg_std * rng.standard_normal(shape)
    gi, gj, gk = _grid(shape)
    for _ in range(n):
        semi = rng.uniform(semi_axes[0], semi_axes[1], 3)
        semi = np.minimum(semi, (dims - 1) / 2.0)
        centre = rng.uniform(semi, dims - 1 - semi)
        mu = fg_mean if fg_range is None else rng.uniform(fg_range[0], fg_range[1])
        inside = (((gi - centre[0]) / semi[0]) ** 2 + ((gj - centre[1]) / semi[1]) ** 2 +
                  ((gk - centre[2]) / semi[2]) ** 2) <= 1.0
        tex = mu + fg_std * rng.standard_normal(shape)
        vol = np.where(inside, tex, vol)
    ramp = bias[0] + (bias[1] - bias[0]) * (gk / max(Z - 1, 1))
    vol = vol * ramp + noise * rng.standard_normal(shape)
    return vol.astype(dtype, copy=False)


def ct_like(shape, seed, n=20, noise=0.04, dtype=np.float32):
    """Body ellipsoid with embedded organs and a smooth cosine bias (built per i-slab)."""
    rng = np.random.default_rng(seed)
    shape = tuple(int(s) for s in shape)
    X, Y, Z = shape
    dims = np.array(shape, dtype=np.float64)
    c_body = (dims - 1) / 2.0
    a_body = 0.45 * dims
    organs = []
    for _ in range(n):
        semi = rng.uniform(0.04, 0.10, 3) * dims
        # centre inside the body ellipsoid, shrunk so the organ stays inside it
        while True:
            u = rng.uniform(-1, 1, 3)
            if (u ** 2).sum() <= 1:
                break
        centre = c_body + u * np.maximum(a_body - semi, 1.0) * 0.9
        organs.append((centre, semi, rng.uniform(0.55, 0.9)))
    waves = []
    for _ in range(3):
        freq = rng.uniform(0.5, 2.0, 3) * 2 * np.pi / dims
        phase = rng.uniform(0, 2 * np.pi)
        waves.append((freq, phase))
    out = np.empty(shape, dtype=dtype)
    gj = np.arange(Y, dtype=np.float64)[:, None]
    gk = np.arange(Z, dtype=np.float64)[None, :]
    for i in range(X):
        sl = 0.1 + 0.02 * rng.standard_normal((Y, Z))
        body = (((i - c_body[0]) / a_body[0]) ** 2 + ((gj - c_body[1]) / a_body[1]) ** 2 +
                ((gk - c_body[2]) / a_body[2]) ** 2) <= 1.0
        sl = np.where(body, 0.4, sl)
        for centre, semi, mu in organs:
            ins = (((i - centre[0]) / semi[0]) ** 2 + ((gj - centre[1]) / semi[1]) ** 2 +
                   ((gk - centre[2]) / semi[2]) ** 2) <= 1.0
            sl = np.where(ins, mu, sl)
        b = 1.0
        for freq, phase in waves:
            b = b + 0.15 * np.cos(freq[0] * i + freq[1] * gj + freq[2] * gk + phase)
        out[i] = (sl * b + noise * rng.standard_normal((Y, Z))).astype(dtype)
    return out


def sphere_phi0(shape, radius=20.0, dtype=np.float64):
    """Signed distance to a sphere at the volume centre, positive inside."""
    shape = tuple(int(s) for s in shape)
    gi, gj, gk = _grid(shape)
    c = [(s - 1) / 2.0 for s in shape]
    d = np.sqrt((gi - c[0]) ** 2 + (gj - c[1]) ** 2 + (gk - c[2]) ** 2)
    return (radius - d).astype(dtype)


def config_volume(name, seed=0, dtype=np.float64):
    """(u0, phi0) of a named workload: 'c1' 64^3, 'c2' 256^3, 'c3' 512x512x320."""
    if name == "c1":
        shape = (64, 64, 64)
        u0 = ellipsoids(shape, seed, n=2, semi_axes=(8, 16), fg_mean=0.8, bias=(0.8, 1.2),
                        noise=0.05, dtype=dtype)
    elif name == "c2":
        shape = (256, 256, 256)
        u0 = ellipsoids(shape, seed, n=8, semi_axes=(10, 40), fg_range=(0.6, 0.9),
                        bias=(0.7, 1.3), noise=0.05, dtype=dtype)
    elif name == "c3":
        shape = (512, 512, 320)
        u0 = ct_like(shape, seed, n=20, noise=0.04, dtype=dtype)
    else:
        raise ValueError(name)
    return u0, sphere_phi0(shape, 20.0, dtype=dtype)


def batch_shapes(count=48, seed=0):
    """Uneven volume sizes between 96x96x64 and 256x256x192."""
    rng = np.random.default_rng(seed)
    return [(int(rng.integers(96, 257)), int(rng.integers(96, 257)), int(rng.integers(64, 193)))
            for _ in range(count)]


def dice(a, b, alpha=0.5):
    """Dice overlap of the regions {a > alpha} and {b > alpha}."""
    A = a > alpha
    B = b > alpha
    s = A.sum() + B.sum()
    return 1.0 if s == 0 else 2.0 * np.logical_and(A, B).sum() / s

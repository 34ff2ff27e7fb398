"""Writes the golden vectors of this directory by running the REFERENCE's own code:
oracle/_ref/libim3d_ref.so, the reference headers compiled in place by oracle/Makefile
(headless interface, GetPot subset and the FFTW3 API over an in-tree FFT as shims).

Run from the repository root after `make -C oracle ref` (which needs the reference
tree); the .npz files it writes are committed, so the tests that read them need
neither the reference tree nor its build.

    python tests/golden/make_golden.py
"""
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as O  # noqa: E402

synth = importlib.import_module("3dimagetoolkit_b200.synth")

ANISO = (0.8, 1.1, 1.3)


def ops():
    rng = np.random.default_rng(2024)
    out = {}
    x = rng.random((16, 14, 12))
    out["conv_x"] = x
    out["conv_iso"] = O.ref_gauss_filter(x, 2.0)
    out["conv_aniso_gpa"] = O.ref_gauss_filter(x, 1.5, h=ANISO, pixel_approach=True)
    out["conv_cyclic"] = O.ref_gauss_filter(x, 2.0, h=ANISO, cyclic=True)
    g = rng.random((7, 9, 11))
    out["grad_x"] = g
    out["grad"] = O.ref_grad(g, ANISO)
    v = rng.random((3, 7, 9, 11))
    out["div_v"] = v
    out["div"] = O.ref_div(v, ANISO)
    r0 = rng.random((9, 8, 10))
    b = rng.random((9, 8, 10))
    out["gs_r0"] = r0
    out["gs_b"] = b
    out["gs_dir"] = O.ref_gs(r0, b, dt=0.7, bc=0.3, neu=False, sweeps=3, h=ANISO)
    out["gs_neu"] = O.ref_gs(r0, b, dt=0.7, bc=0.3, neu=True, sweeps=3, h=ANISO)
    c = rng.random((10, 9, 8))
    out["cc_x"] = c
    out["cc_seeded"] = O.connected_component(c, (4, 4, 4), use_reference=True)
    out["cc_seeded_full_nonbinary"] = O.connected_component(c, (2, 3, 5), full_connected=True,
                                                           binary_output=False,
                                                           use_reference=True)
    init = (rng.random((10, 9, 8)) < 0.05).astype(np.float64)
    out["cc_init"] = init
    out["cc_from_init"] = O.connected_component(c, init=init, threshold=0.4, use_reference=True)
    np.savez_compressed(os.path.join(HERE, "ops_f64.npz"), **out)


RSFE_MODES = {
    # name: parameters on top of the reference constructor's defaults
    "dir": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=2),
    "neu": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=1),
    "default": dict(maxiter=4),
    "cyclic": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=1,
                   conv_cyclic=1),
    "cc": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=2,
               auto_extract_conn_comp=1, auto_extract_conn_comp_freq=2, cc_init_pixel_x=9.0,
               cc_init_pixel_y=8.0, cc_init_pixel_z=7.0),
}


def rsfe():
    shape = (18, 16, 14)
    u0 = synth.ellipsoids(shape, seed=7, n=2, semi_axes=(3.0, 5.0))
    phi0 = synth.sphere_phi0(shape, radius=5.0)
    out = {"u0": u0, "phi0": phi0}
    for name, kw in RSFE_MODES.items():
        r = O.rsfe_apply(u0, phi0, O.default_params(**kw), use_reference=True)
        for f in ("phi", "u", "f1", "f2"):
            out[f"{name}_{f}"] = r[f]
        out[f"{name}_iterations"] = np.array(r["stats"]["iterations"])
    np.savez_compressed(os.path.join(HERE, "rsfe_f64.npz"), **out)


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/libim3d_ref.so is missing: run `make -C oracle ref` first")
    ops()
    rsfe()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)), "bytes")

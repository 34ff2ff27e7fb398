"""Golden vectors written by the reference's own code (tests/golden/make_golden.py
runs oracle/_ref, the reference headers compiled in place): the CPU restatement
(oracle/) and the CUDA path (C ABI) are both checked against them, so neither check
needs the reference tree at run time.

Bars: stencils and Gauss-Seidel sweeps bit-exact in FP64; the convolution within
1e-14 (CPU) / 1e-13 (GPU) relative, the reference's FFT against a separable direct
sum; the whole RSFE loop within 1e-12 (CPU) / 1e-9 (GPU) relative L2 with the same
number of outer iterations."""
import os

import numpy as np
import pytest

from conftest import rel

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ANISO = (0.8, 1.1, 1.3)
MODES = {
    "dir": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=2),
    "neu": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=1),
    "default": dict(maxiter=4),
    "cyclic": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=1,
                   conv_cyclic=1),
    "cc": dict(sigma=2.0, lamda1=1.0, lamda2=1.0, lamda=0.5, maxiter=6, ls_steps=1, bc=2,
               auto_extract_conn_comp=1, auto_extract_conn_comp_freq=2, cc_init_pixel_x=9.0,
               cc_init_pixel_y=8.0, cc_init_pixel_z=7.0),
}


@pytest.fixture(scope="module")
def ops():
    return np.load(os.path.join(GOLD, "ops_f64.npz"))


@pytest.fixture(scope="module")
def loop():
    return np.load(os.path.join(GOLD, "rsfe_f64.npz"))


# ------------------------------------------------------------------ CPU checker

def test_oracle_ops_match_golden(O, ops):
    assert rel(O.gauss_filter(ops["conv_x"], 2.0), ops["conv_iso"]) < 1e-14
    assert rel(O.gauss_filter(ops["conv_x"], 1.5, h=ANISO, pixel_approach=True),
               ops["conv_aniso_gpa"]) < 1e-14
    assert rel(O.gauss_filter(ops["conv_x"], 2.0, h=ANISO, cyclic=True), ops["conv_cyclic"]) < 1e-14
    assert np.array_equal(O.grad(ops["grad_x"], ANISO), ops["grad"])
    assert np.array_equal(O.div(ops["div_v"], ANISO), ops["div"])
    for name, bct in (("gs_dir", O.BC_DIR), ("gs_neu", O.BC_NEU)):
        got = O.poisson_sweeps(ops["gs_r0"], ops["gs_b"], dt=0.7, bc=0.3, bc_type=bct, sweeps=3,
                               h=ANISO)
        assert np.array_equal(got, ops[name]), name
    assert np.array_equal(O.connected_component(ops["cc_x"], (4, 4, 4)), ops["cc_seeded"])
    assert np.array_equal(O.connected_component(ops["cc_x"], (2, 3, 5), full_connected=True,
                                                binary_output=False),
                          ops["cc_seeded_full_nonbinary"])
    assert np.array_equal(O.connected_component(ops["cc_x"], init=ops["cc_init"], threshold=0.4),
                          ops["cc_from_init"])


@pytest.mark.parametrize("mode", list(MODES))
def test_oracle_loop_matches_golden(O, loop, mode):
    r = O.rsfe_apply(loop["u0"], loop["phi0"], O.default_params(**MODES[mode]))
    assert r["stats"]["iterations"] == int(loop[f"{mode}_iterations"])
    for f in ("phi", "u", "f1", "f2"):
        assert rel(r[f], loop[f"{mode}_{f}"]) < 1e-12, f
    # the fixture is not the initial state: the loop moved phi
    assert rel(loop[f"{mode}_phi"], loop["phi0"]) > 1e-3


# ------------------------------------------------------------------ CUDA path

@pytest.mark.gpu
def test_gpu_ops_match_golden(ctx, ops):
    assert rel(ctx.gauss_filter(ops["conv_x"], 2.0), ops["conv_iso"]) < 1e-13
    assert rel(ctx.gauss_filter(ops["conv_x"], 1.5, h=ANISO, pixel_approach=True),
               ops["conv_aniso_gpa"]) < 1e-13
    assert rel(ctx.gauss_filter(ops["conv_x"], 2.0, h=ANISO, cyclic=True), ops["conv_cyclic"]) < 1e-13
    assert np.array_equal(ctx.grad(ops["grad_x"], ANISO), ops["grad"])
    assert np.array_equal(ctx.div(ops["div_v"], ANISO), ops["div"])
    for name, bct in (("gs_dir", 2), ("gs_neu", 1)):
        got = ctx.poisson_sweeps(ops["gs_r0"].copy(), ops["gs_b"], dt=0.7, bc=0.3, bc_type=bct,
                                 sweeps=3, h=ANISO)
        assert np.array_equal(got, ops[name]), name
    assert np.array_equal(ctx.connected_component(ops["cc_x"], (4, 4, 4)), ops["cc_seeded"])
    assert np.array_equal(ctx.connected_component(ops["cc_x"], (2, 3, 5), full_connected=True,
                                                  binary_output=False),
                          ops["cc_seeded_full_nonbinary"])
    assert np.array_equal(ctx.connected_component(ops["cc_x"], init=ops["cc_init"], threshold=0.4),
                          ops["cc_from_init"])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", list(MODES))
def test_gpu_loop_matches_golden(ctx, pkg, loop, mode):
    r = ctx.rsfe_apply(loop["u0"], loop["phi0"], pkg.default_params(**MODES[mode]),
                       want_u=True, want_f=True)
    assert r["stats"]["iterations"] == int(loop[f"{mode}_iterations"])
    for f in ("phi", "u", "f1", "f2"):
        assert rel(r[f], loop[f"{mode}_{f}"]) < 1e-9, f

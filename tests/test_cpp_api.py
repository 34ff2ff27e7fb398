"""The header-only C++ API (include/im3d/) and the command-line driver.

CPU: both compile against the headers and link against libim3d_b200.so.
GPU: tests/cpp/api_check.cpp runs the reference's known answers (examples/test.cxx)
through the C++ classes, filters and sweeps a volume read from a MetaImage file, and
segments it with rsfe_splitbregman<double> configured by a GetPot file; the results
are compared with the CPU checker. The CLI segments a MetaImage volume end to end.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, rel

INC = os.path.join(ROOT, "include")
PKGDIR = os.path.join(ROOT, "3dimagetoolkit_b200")


def _compile(src, out):
    cmd = ["g++", "-std=c++14", "-O2", "-Wall", "-Werror", "-I", INC, src, "-L", PKGDIR,
           "-lim3d_b200", f"-Wl,-rpath,{PKGDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_cpp_api_and_cli_compile(tmp_path):
    _compile(os.path.join(ROOT, "tests", "cpp", "api_check.cpp"), str(tmp_path / "api_check"))
    _compile(os.path.join(PKGDIR, "cli", "rsfe_splitbregman.cpp"), str(tmp_path / "cli"))


def test_mhd_roundtrip(tmp_path, pkg):
    mhd = pkg.mhd if hasattr(pkg, "mhd") else __import__("importlib").import_module(
        "3dimagetoolkit_b200.mhd")
    v = np.random.default_rng(0).random((5, 6, 7))
    p = mhd.write(str(tmp_path / "v"), v, (0.5, 1.0, 2.0))
    w, sp = mhd.read(p)
    assert np.array_equal(v, w) and sp == (0.5, 1.0, 2.0)


PARAMS_POT = """[splitbregman]
    [./init]
    verbosity = 0
    maxiter = 6
    sigma = 2
    lamda = 0.5
    lamda1 = 1
    lamda2 = 1
    epsilon = 1.e-3
    bc = 2          # DIR
    ls_steps = 1
    tol = 0
    [../]
[../]
"""


@pytest.mark.gpu
def test_cpp_api_on_gpu(tmp_path, pkg, O):
    import importlib

    mhd = importlib.import_module("3dimagetoolkit_b200.mhd")
    shape = (20, 18, 16)
    u0 = pkg.synth.ellipsoids(shape, 4, n=2, semi_axes=(3, 6))
    phi0 = pkg.synth.sphere_phi0(shape, 5.0)
    mhd.write(str(tmp_path / "vol"), u0)
    mhd.write(str(tmp_path / "init"), phi0)
    (tmp_path / "params.pot").write_text(PARAMS_POT)
    exe = str(tmp_path / "api_check")
    _compile(os.path.join(ROOT, "tests", "cpp", "api_check.cpp"), exe)
    r = subprocess.run([exe, str(tmp_path)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "FAIL" not in r.stdout
    conv, _ = mhd.read(str(tmp_path / "conv_out.mhd"))
    assert rel(conv, O.gauss_filter(u0, 2.0)) < 1e-13
    gs, _ = mhd.read(str(tmp_path / "gs_out.mhd"))
    assert np.array_equal(gs, O.poisson_sweeps(u0, 0.5 * u0, dt=0.7, bc=0.25, sweeps=2))
    phi, _ = mhd.read(str(tmp_path / "phi_out.mhd"))
    want = O.rsfe_apply(u0, phi0, O.default_params(maxiter=6, sigma=2.0, lamda=0.5, lamda1=1.0,
                                                   lamda2=1.0, bc=O.BC_DIR, ls_steps=1, tol=0.0))
    assert rel(phi, want["phi"]) < 1e-9
    cc, _ = mhd.read(str(tmp_path / "cc_out.mhd"))
    assert np.array_equal(cc, O.connected_component(u0, (10, 9, 8), full_connected=True))
    phi_cc, _ = mhd.read(str(tmp_path / "phi_cc_out.mhd"))
    want = O.rsfe_apply(u0, phi0, O.default_params(
        maxiter=6, sigma=2.0, lamda=0.5, lamda1=1.0, lamda2=1.0, bc=O.BC_DIR, ls_steps=1, tol=0.0,
        auto_extract_conn_comp=1, auto_extract_conn_comp_freq=2, cc_init_pixel_x=10.0,
        cc_init_pixel_y=9.0, cc_init_pixel_z=8.0))
    assert rel(phi_cc, want["phi"]) < 1e-9


@pytest.mark.gpu
def test_cli_segments_a_metaimage(tmp_path, pkg, O):
    import importlib

    mhd = importlib.import_module("3dimagetoolkit_b200.mhd")
    shape = (24, 22, 20)
    u0 = pkg.synth.ellipsoids(shape, 5, n=2, semi_axes=(4, 7))
    mhd.write(str(tmp_path / "vol"), u0.astype(np.float32))
    pot = PARAMS_POT.replace("tol = 0", f"tol = 0\n    dumpfrequency = 1\n    outputname = {tmp_path}/res")
    (tmp_path / "data").write_text(pot)
    exe = os.path.join(PKGDIR, "bin", "rsfe_splitbregman")
    if not os.path.exists(exe):
        exe = str(tmp_path / "cli")
        _compile(os.path.join(PKGDIR, "cli", "rsfe_splitbregman.cpp"), exe)
    r = subprocess.run([exe, str(tmp_path / "vol.mhd"), str(tmp_path / "data")],
                       capture_output=True, text=True, timeout=300, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout + r.stderr
    phi, _ = mhd.read(str(tmp_path / "res_6_final.mhd"))
    # the driver rescales the image to [0, 255] (examples/rsfe_splitbregman.cxx:86)
    x = u0.astype(np.float32).astype(np.float64)
    x = (x - x.min()) / ((x - x.min()).max() / 255.0)
    kw = dict(sigma=2.0, lamda=0.5, lamda1=1.0, lamda2=1.0, bc=O.BC_DIR, ls_steps=1, tol=0.0)
    want = O.rsfe_apply(x, None, O.default_params(maxiter=6, **kw))
    assert rel(phi, want["phi"]) < 1e-9
    # the per-iteration dumps of the reference's loop: every iteration but the last
    names = sorted(f for f in os.listdir(tmp_path) if f.startswith("res_") and f.endswith(".mhd"))
    assert names == ["res_1.mhd", "res_2.mhd", "res_3.mhd", "res_4.mhd", "res_5.mhd", "res_6_final.mhd"]
    phi3, _ = mhd.read(str(tmp_path / "res_3.mhd"))
    want3 = O.rsfe_apply(x, None, O.default_params(maxiter=3, **kw))
    assert rel(phi3, want3["phi"]) < 1e-9

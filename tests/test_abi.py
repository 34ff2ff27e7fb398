"""CPU: the C ABI library loads and exports every symbol include/im3d_b200.h
declares; the parameter defaults are the reference constructor's. No compute."""
import ctypes as C

import pytest


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    names = pkg._abi.header_symbols()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_struct_layouts_match_oracle(pkg, O):
    assert C.sizeof(pkg.RsfeParams) == C.sizeof(O.RsfeParams)
    assert [f for f, _ in pkg.RsfeParams._fields_] == [f for f, _ in O.RsfeParams._fields_]
    assert C.sizeof(pkg.RsfeStats) == C.sizeof(O.RsfeStats)


def test_defaults_are_reference_constructor(pkg, O):
    # rsfe_splitbregman_imp.hxx:25-41
    p = pkg.default_params()
    assert (p.maxiter, p.ls_steps, p.bc) == (100, 5, pkg.BC_DEFAULT)
    assert (p.sigma, p.lamda, p.lamda1, p.lamda2) == (3, 5e-2, 1e-5, 1e-5)
    assert (p.beta, p.nu, p.dt, p.epsilon, p.a0, p.b0, p.tol) == (100, 1, 1, 1e-3, 0, 1, 1e-5)
    q = O.default_params()
    for f, _ in pkg.RsfeParams._fields_:
        assert getattr(p, f) == getattr(q, f), f


def test_no_device_is_reported_not_faked(pkg):
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(pkg.Im3dError) as e:
        pkg.Context(0)
    assert e.value.status == 6


def test_python_constants_match_the_header(pkg):
    """Every IM3D_ status, option, batch-mode, boundary, sweep and warm-start constant of
    include/im3d_b200.h has the same value in the Python binding."""
    import os
    import re

    hdr = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "im3d_b200.h")).read()
    defs = dict(re.findall(r"#define IM3D_([A-Z0-9_]+) \(?(-?\d+)\)?", hdr))
    prefixes = ("ERR_", "OPT_", "BATCH_", "BC_", "SWEEP_", "WS_")
    checked = 0
    for name, value in defs.items():
        if name.startswith(prefixes) and hasattr(pkg._abi, name):
            assert getattr(pkg._abi, name) == int(value), name
            checked += 1
    for must in ("OPT_BATCH_MODE", "OPT_TILE_LOADS", "BATCH_AUTO", "BATCH_STREAMS", "BATCH_WORKLIST", "ERR_NONFINITE"):
        assert must in defs and hasattr(pkg._abi, must), must
    assert checked >= 20

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

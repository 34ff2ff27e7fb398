"""ctypes bindings of the CPU checker.  TEST INFRASTRUCTURE ONLY.

Loads two libraries built by oracle/Makefile:

* ``oracle/liboracle.so`` -- the FP64 C restatement (``im3d_oracle.c``);
* ``oracle/_ref/libim3d_ref.so`` -- the reference's own headers compiled with the
  headless shims (``ref/``), exposing the reference's templates through C entry
  points (``ref/ref_capi.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import this module. Arrays are numpy float64 in the reference's image3d layout
(``a[i, j, k]``, k contiguous).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libim3d_ref.so")

BC_DEFAULT, BC_NEU, BC_DIR = 0, 1, 2
SWEEP_LEX, SWEEP_RB = 0, 1


class RsfeParams(C.Structure):
    """Mirror of ``im3d_rsfe_params`` (include/im3d_b200.h)."""

    _fields_ = [
        ("tol", C.c_double), ("sigma", C.c_double), ("lamda", C.c_double),
        ("lamda1", C.c_double), ("lamda2", C.c_double), ("beta", C.c_double),
        ("nu", C.c_double), ("dt", C.c_double), ("epsilon", C.c_double),
        ("a0", C.c_double), ("b0", C.c_double), ("ls_tol", C.c_double),
        ("edge_detector_sigma", C.c_double), ("gs_rel_res_tol", C.c_double),
        ("omega", C.c_double),
        ("maxiter", C.c_int32), ("ls_steps", C.c_int32), ("bc", C.c_int32),
        ("gaussian_pixel_approach", C.c_int32), ("init_variables", C.c_int32),
        ("sweep", C.c_int32), ("gs_max_sweeps", C.c_int32), ("gs_check_every", C.c_int32),
        ("cc_init_pixel_x", C.c_double), ("cc_init_pixel_y", C.c_double),
        ("cc_init_pixel_z", C.c_double), ("alpha", C.c_double),
        ("auto_extract_conn_comp", C.c_int32), ("auto_extract_conn_comp_freq", C.c_int32),
        ("cc_binary_output", C.c_int32), ("cc_init_variables", C.c_int32),
        ("conv_cyclic", C.c_int32), ("reserved_", C.c_int32),
    ]


class RsfeStats(C.Structure):
    """Mirror of ``im3d_rsfe_stats`` (include/im3d_b200.h)."""

    _fields_ = [
        ("last_tol", C.c_double), ("last_rel_res", C.c_double), ("last_ls_err", C.c_double),
        ("setup_ms", C.c_double), ("loop_ms", C.c_double), ("total_sweeps", C.c_int64),
        ("iterations", C.c_int32), ("last_sweeps", C.c_int32), ("not_converged", C.c_int32),
        ("residual_checks", C.c_int32), ("ws_used", C.c_int32), ("ws_rejected", C.c_int32),
        ("ws_loss", C.c_double),
    ]


def default_params(**kw) -> RsfeParams:
    """The reference constructor's values (rsfe_splitbregman_imp.hxx:25-41)."""
    p = RsfeParams(tol=1e-5, sigma=3.0, lamda=5e-2, lamda1=1e-5, lamda2=1e-5, beta=100.0,
                   nu=1.0, dt=1.0, epsilon=1e-3, a0=0.0, b0=1.0, ls_tol=0.0,
                   edge_detector_sigma=0.0, gs_rel_res_tol=0.0, omega=1.0, maxiter=100,
                   ls_steps=5, bc=BC_DEFAULT, gaussian_pixel_approach=0, init_variables=0,
                   sweep=SWEEP_LEX, gs_max_sweeps=1000, gs_check_every=0,
                   cc_init_pixel_x=-1.0, cc_init_pixel_y=-1.0, cc_init_pixel_z=-1.0, alpha=0.5,
                   auto_extract_conn_comp=0, auto_extract_conn_comp_freq=0, cc_binary_output=1,
                   cc_init_variables=1, conv_cyclic=0, reserved_=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


_D = C.POINTER(C.c_double)
_lib_cache: dict[str, C.CDLL] = {}


def _load(path: str) -> C.CDLL:
    if path not in _lib_cache:
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
        _lib_cache[path] = C.CDLL(path)
    return _lib_cache[path]


def oracle_lib() -> C.CDLL:
    return _load(ORACLE_SO)


def ref_lib() -> C.CDLL:
    return _load(REF_SO)


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def _p(a):
    return None if a is None else a.ctypes.data_as(_D)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ----------------------------------------------------------------- restatement

def gauss_filter(x, sigma, h=(1.0, 1.0, 1.0), radius=3.0, pixel_approach=False, lib=None,
                 cyclic=False):
    x = _f64(x)
    out = np.empty_like(x)
    L = lib or oracle_lib()
    if cyclic:
        fn = L.orc_gauss_filter_cyclic if lib is None else L.ref_gauss_filter_cyclic
    else:
        fn = L.orc_gauss_filter if lib is None else L.ref_gauss_filter
    fn(_p(x), _p(out), *map(C.c_int, x.shape), *map(C.c_double, h), C.c_double(sigma),
       C.c_double(radius), C.c_int(int(pixel_approach)))
    return out


def gauss_taps(sigma, h=1.0, radius=3.0):
    buf = np.zeros(4096)
    nh = oracle_lib().orc_gauss_taps(C.c_double(sigma), C.c_double(radius), C.c_double(h),
                                     _p(buf), C.c_int(4096))
    return buf[:nh].copy()


def grad(x, h=(1.0, 1.0, 1.0)):
    x = _f64(x)
    out = np.empty((3,) + x.shape)
    oracle_lib().orc_grad(_p(x), _p(out), *map(C.c_int, x.shape), *map(C.c_double, h))
    return out


def div(v, h=(1.0, 1.0, 1.0)):
    v = _f64(v)
    out = np.empty(v.shape[1:])
    oracle_lib().orc_div(_p(v), _p(out), *map(C.c_int, out.shape), *map(C.c_double, h))
    return out


def poisson_sweeps(res, b, dt=1.0, bc=0.0, bc_type=BC_DIR, order=SWEEP_LEX, sweeps=1,
                   h=(1.0, 1.0, 1.0)):
    r = _f64(res).copy()
    b = _f64(b)
    oracle_lib().orc_poisson_sweeps(_p(r), _p(b), *map(C.c_int, r.shape), *map(C.c_double, h),
                                    C.c_double(dt), C.c_double(bc), C.c_int(bc_type),
                                    C.c_int(order), C.c_int(sweeps))
    return r


def poisson_solve(u, b, dt=1.0, bc=0.0, bc_type=BC_DIR, tol=1e-6, max_sweeps=1000,
                  check_every=0, omega=1.0, h=(1.0, 1.0, 1.0)):
    u = _f64(u).copy()
    b = _f64(b)
    sw = C.c_int(0)
    rel = C.c_double(0)
    st = oracle_lib().orc_poisson_solve(_p(u), _p(b), *map(C.c_int, u.shape),
                                        *map(C.c_double, h), C.c_double(dt), C.c_double(bc),
                                        C.c_int(bc_type), C.c_double(tol), C.c_int(max_sweeps),
                                        C.c_int(check_every), C.c_double(omega), C.byref(sw),
                                        C.byref(rel))
    return u, int(sw.value), float(rel.value), int(st)


def rsfe_apply(myim, init=None, params=None, h=(1.0, 1.0, 1.0), use_reference=False,
               verbosity=False):
    """rsfe_splitbregman<double>::apply; returns dict(phi, u, f1, f2, stats)."""
    u0 = _f64(myim)
    ini = None if init is None else _f64(init)
    p = params or default_params()
    phi = np.empty_like(u0)
    u = np.empty_like(u0)
    f1 = np.empty_like(u0)
    f2 = np.empty_like(u0)
    st = RsfeStats()
    args = [_p(u0), _p(ini), *map(C.c_int, u0.shape), *map(C.c_double, h), C.byref(p),
            _p(phi), _p(u), _p(f1), _p(f2), C.byref(st)]
    if use_reference:
        rc = ref_lib().ref_rsfe_apply(*args, C.c_int(int(verbosity)))
    else:
        rc = oracle_lib().orc_rsfe_apply(*args)
    if rc != 0:
        raise RuntimeError(f"rsfe_apply failed with status {rc}")
    return dict(phi=phi, u=u, f1=f1, f2=f2, stats={f: getattr(st, f) for f, _ in st._fields_})


def connected_component(img, ijk=(0, 0, 0), init=None, threshold=0.5, full_connected=False,
                        binary_output=True, use_reference=False):
    """image3d<double>::connected_component (seeded when init is None)."""
    x = _f64(img)
    out = np.empty_like(x)
    ini = None if init is None else _f64(init)
    lib = ref_lib().ref_connected_component if use_reference else oracle_lib().orc_connected_component
    lib(_p(x), _p(out), *map(C.c_int, x.shape), _p(ini), *map(C.c_int, ijk), C.c_double(threshold),
        C.c_int(int(full_connected)), C.c_int(int(binary_output)))
    return out


# -------------------------------------------------------------- reference entry

def ref_gauss_filter(x, sigma, h=(1.0, 1.0, 1.0), radius=3.0, pixel_approach=False,
                     direct=False, cyclic=False):
    x = _f64(x)
    out = np.empty_like(x)
    L = ref_lib()
    fn = (L.ref_gauss_filter_cyclic if cyclic else
          (L.ref_gauss_filter_direct if direct else L.ref_gauss_filter))
    fn(_p(x), _p(out), *map(C.c_int, x.shape), *map(C.c_double, h), C.c_double(sigma),
       C.c_double(radius), C.c_int(int(pixel_approach)))
    return out


def ref_grad(x, h=(1.0, 1.0, 1.0)):
    x = _f64(x)
    out = np.empty((3,) + x.shape)
    ref_lib().ref_grad(_p(x), _p(out), *map(C.c_int, x.shape), *map(C.c_double, h))
    return out


def ref_div(v, h=(1.0, 1.0, 1.0)):
    v = _f64(v)
    out = np.empty(v.shape[1:])
    ref_lib().ref_div(_p(v), _p(out), *map(C.c_int, out.shape), *map(C.c_double, h))
    return out


def ref_gs(res, b, dt=1.0, bc=0.0, neu=False, sweeps=1, h=(1.0, 1.0, 1.0)):
    r = _f64(res).copy()
    b = _f64(b)
    ref_lib().ref_gs(_p(r), _p(b), *map(C.c_int, r.shape), *map(C.c_double, h), C.c_double(dt),
                     C.c_double(bc), C.c_int(int(neu)), C.c_int(sweeps))
    return r


def ref_fft3d(x, sign=-1):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    out = np.empty_like(x)
    ref_lib().ref_fft3d(x.ctypes.data_as(_D), out.ctypes.data_as(_D), *map(C.c_int, x.shape),
                        C.c_int(sign))
    return out


def ref_change_range(x, mx, mn):
    r = _f64(x).copy()
    ref_lib().ref_change_range(_p(r), *map(C.c_int, r.shape), C.c_double(mx), C.c_double(mn))
    return r


def ref_last_timeline():
    """[apply start, end of each outer iteration's Poisson step..., apply end] (s)."""
    buf = np.zeros(100000)
    n = ref_lib().ref_last_timeline(_p(buf), C.c_int(buf.size))
    return buf[:n].copy()


def ref_last_sweep_marks():
    """Sweeps run up to the end of each outer iteration's Poisson step (last run)."""
    buf = np.zeros(100000)
    n = ref_lib().ref_last_sweep_marks(_p(buf), C.c_int(buf.size))
    return buf[:n].copy()


def ref_last_step_profile():
    """(solve, fft) per outer iteration of the last run: wall seconds inside its Poisson
    step, and FFT wall seconds accumulated up to the end of that step."""
    solve = np.zeros(100000)
    fft = np.zeros(100000)
    n = ref_lib().ref_last_step_profile(_p(solve), _p(fft), C.c_int(solve.size))
    return solve[:n].copy(), fft[:n].copy()


def ref_fft_totals():
    """(seconds, calls) spent in the FFT shim's fftw_execute since the library loaded."""
    s = C.c_double(0)
    n = C.c_longlong(0)
    ref_lib().im3d_fft_shim_totals(C.byref(s), C.byref(n))
    return s.value, n.value


_EXT_FFT = None  # the registered callback (kept alive while it is in use)


def use_pocketfft(threads: int | None) -> bool:
    """Serves the reference's fftw_execute calls with scipy's pocketfft (multi-threaded,
    in place on the plan's output array) instead of the in-tree FFT; threads=None goes
    back to the in-tree FFT. Returns False when scipy is missing. For timing the
    reference: the checker's results use the in-tree FFT."""
    global _EXT_FFT
    L = ref_lib()
    proto = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int)
    L.im3d_fft_shim_set_external.argtypes = [proto]
    if threads is None:
        L.im3d_fft_shim_set_external(proto())
        _EXT_FFT = None
        return True
    try:
        import scipy.fft
    except ImportError:
        return False

    def run(n0, n1, n2, data, sign):
        n = n0 * n1 * n2
        buf = (C.c_double * (2 * n)).from_address(data)
        x = np.frombuffer(buf, dtype=np.complex128).reshape(n0, n1, n2)
        if sign < 0:
            y = scipy.fft.fftn(x, workers=threads, overwrite_x=True)
        else:
            y = scipy.fft.ifftn(x, norm="forward", workers=threads, overwrite_x=True)
        if not np.shares_memory(x, y):
            x[...] = y
        return 0

    _EXT_FFT = proto(run)
    L.im3d_fft_shim_set_external(_EXT_FFT)
    return True


def set_threads(n: int) -> None:
    """OpenMP threads of the checker's and the reference's parallel regions started from
    the calling thread (omp_set_num_threads of the libgomp both libraries use)."""
    ref_lib()
    C.CDLL("libgomp.so.1").omp_set_num_threads(C.c_int(int(n)))

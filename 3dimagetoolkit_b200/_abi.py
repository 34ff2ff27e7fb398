"""ctypes binding of the C ABI in include/im3d_b200.h (libim3d_b200.so).

The shared library is built in-tree by ``__graft_entry__.build()`` (nvcc, sm_100a).
There is no CPU fallback: if the library or a CUDA device is missing, every entry
point raises.

Arrays may be numpy arrays (host memory; the library stages them through its own
device buffers) or CUDA torch tensors (device memory, used in place). float32 calls
the ``_f32`` entry points, float64 the ``_f64`` ones.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libim3d_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "im3d_b200.h")

OK = 0
ERR_INVALID_ARG = 1
ERR_UNSUPPORTED = 2
ERR_NOT_CONVERGED = 3
ERR_CUDA = 4
ERR_OOM = 5
ERR_NO_DEVICE = 6
ERR_TOO_LARGE = 7
ERR_NONFINITE = 8

BC_DEFAULT, BC_NEU, BC_DIR = 0, 1, 2
SWEEP_LEXICOGRAPHIC, SWEEP_REDBLACK = 0, 1
OPT_FIT_CHUNKS, OPT_DEVICE_MEMORY_LIMIT, OPT_BATCH_MODE, OPT_TILE_LOADS = 1, 2, 3, 4
BATCH_AUTO, BATCH_STREAMS, BATCH_WORKLIST = 0, 1, 2
WS_OFF, WS_PREDICT, WS_TRAIN = 0, 1, 2

_STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "NOT_CONVERGED", 4: "CUDA",
                 5: "OOM", 6: "NO_DEVICE", 7: "TOO_LARGE", 8: "NONFINITE"}


class Im3dError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class RsfeParams(C.Structure):
    """``im3d_rsfe_params``: the parameters of segm::rsfe_splitbregman<T>."""

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

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class RsfeStats(C.Structure):
    _fields_ = [
        ("last_tol", C.c_double), ("last_rel_res", C.c_double), ("last_ls_err", C.c_double),
        ("setup_ms", C.c_double), ("loop_ms", C.c_double), ("total_sweeps", C.c_int64),
        ("iterations", C.c_int32), ("last_sweeps", C.c_int32), ("not_converged", C.c_int32),
        ("residual_checks", C.c_int32), ("ws_used", C.c_int32), ("ws_rejected", C.c_int32),
        ("ws_loss", C.c_double),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Checkpoint(C.Structure):
    """``im3d_rsfe_checkpoint``: the loop's state after outer iteration t."""

    _fields_ = [("t", C.c_int32), ("init_variables", C.c_int32), ("sched_first", C.c_int32),
                ("reserved", C.c_int32), ("sched_rate", C.c_double), ("tollerance", C.c_double),
                ("phi", C.c_void_p), ("b", C.c_void_p), ("divdb", C.c_void_p)]


OBSERVER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(Checkpoint))


class VolumeDesc(C.Structure):
    """``im3d_volume_desc``: one volume of a batch."""

    _fields_ = [("myim", C.c_void_p), ("init", C.c_void_p), ("phi_out", C.c_void_p),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("reserved", C.c_int32),
                ("hx", C.c_double), ("hy", C.c_double), ("hz", C.c_double)]


_lib = None


def lib() -> C.CDLL:
    """The loaded libim3d_b200.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        L.im3d_ctx_last_error.restype = C.c_char_p
        L.im3d_ctx_launch_count.restype = C.c_int64
        L.im3d_rsfe_params_default.restype = None
        L.im3d_unet_param_count.restype = C.c_int64
        _lib = L
    return _lib


def header_symbols(path: str = HEADER) -> list[str]:
    """Names of the functions declared in include/im3d_b200.h."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(im3d_[a-z0-9_]+)\s*\(", text)))


def default_params(**overrides) -> RsfeParams:
    """Reference constructor defaults (rsfe_splitbregman_imp.hxx:25-41), then overrides."""
    p = RsfeParams()
    lib().im3d_rsfe_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _is_torch(a) -> bool:
    return type(a).__module__.startswith("torch")


def _ptr(a):
    """(void*, dtype) of a numpy array or a CUDA torch tensor; None passes NULL."""
    if a is None:
        return None, None
    if _is_torch(a):
        import torch

        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        dt = {torch.float32: np.float32, torch.float64: np.float64}[a.dtype]
        return C.c_void_p(a.data_ptr()), dt
    if not isinstance(a, np.ndarray) or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous numpy array or a CUDA tensor")
    return C.c_void_p(a.ctypes.data), a.dtype.type


def _suffix(dt) -> str:
    if dt == np.float32:
        return "f32"
    if dt == np.float64:
        return "f64"
    raise TypeError(f"unsupported dtype {dt}")


def _empty_like(a, shape=None):
    shape = tuple(a.shape) if shape is None else tuple(shape)
    if _is_torch(a):
        import torch

        return torch.empty(shape, dtype=a.dtype, device=a.device)
    return np.empty(shape, dtype=a.dtype)


class Context:
    """One im3d_ctx: a CUDA stream, device buffers reused across calls."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        st = lib().im3d_ctx_create(C.c_int(device), C.byref(self._h))
        if st != OK:
            raise Im3dError(st, f"im3d_ctx_create(device={device}) failed")
        self.device = device
        self._obs = None
        self._obs_shape = ()
        self._resume_keep = None
        self._ws = None

    def close(self):
        if self._h:
            lib().im3d_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    @property
    def launches(self) -> int:
        return int(lib().im3d_ctx_launch_count(self._h))

    def last_error(self) -> str:
        return lib().im3d_ctx_last_error(self._h).decode()

    def _check(self, st: int, allow=()):
        if st != OK and st not in allow:
            raise Im3dError(st, self.last_error())
        return st

    def set_profiling(self, on: int = 1):
        """1 (True): every stage; 2: the Poisson solves as a whole only; 0: off."""
        self._check(lib().im3d_ctx_set_profiling(self._h, C.c_int(int(on))))

    def profile(self, reset: bool = True) -> dict:
        """{stage: (total_ms, launches)} accumulated since the last reset."""
        names = C.create_string_buffer(8192)
        ms = (C.c_double * 64)()
        cnt = (C.c_int64 * 64)()
        n = lib().im3d_ctx_profile(self._h, names, 8192, ms, cnt, 64, int(reset))
        if n < 0:
            raise Im3dError(-n, self.last_error())
        keys = names.value.decode().split("\n")[:n]
        return {k: (ms[i], int(cnt[i])) for i, k in enumerate(keys)}

    def set_stream(self, stream_handle: int | None):
        self._check(lib().im3d_ctx_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def set_option(self, option: int, value: int):
        """im3d_ctx_set_option: OPT_FIT_CHUNKS, OPT_DEVICE_MEMORY_LIMIT (bytes),
        OPT_BATCH_MODE (BATCH_AUTO, BATCH_STREAMS, BATCH_WORKLIST) or OPT_TILE_LOADS (0, 1)."""
        self._check(lib().im3d_ctx_set_option(self._h, C.c_int(option), C.c_int64(value)))

    def set_observer(self, every: int, fn=None, with_state: bool = False, dtype=np.float64):
        """Calls fn(state) after every ``every``-th outer iteration (not the last one) of
        the next segmentations; state is a dict (t, tollerance, sched_first, sched_rate,
        init_variables, phi[, b, divdb]) of numpy copies. fn returning True ends the
        loop after that iteration. fn=None removes the observer. ``dtype`` is the
        element type of the segmentations that follow."""
        if fn is None:
            self._obs = None
            self._check(lib().im3d_ctx_set_observer(self._h, 0, 0, None, None))
            return
        dt = np.dtype(dtype)

        def cb(_user, ck):
            c = ck.contents
            n = int(np.prod(self._obs_shape))

            def arr(ptr, count, shape):
                buf = (C.c_char * (count * dt.itemsize)).from_address(ptr)
                return np.frombuffer(buf, dtype=dt, count=count).reshape(shape).copy()

            st = dict(t=c.t, tollerance=c.tollerance, sched_first=c.sched_first,
                      sched_rate=c.sched_rate, init_variables=c.init_variables,
                      phi=arr(c.phi, n, self._obs_shape))
            if c.b:
                st["b"] = arr(c.b, 3 * n, (3,) + tuple(self._obs_shape))
                st["divdb"] = arr(c.divdb, n, self._obs_shape)
            try:
                return 1 if fn(st) else 0
            except Exception:  # an exception must not cross the C frame
                return 1

        self._obs = OBSERVER(cb)
        self._check(lib().im3d_ctx_set_observer(self._h, C.c_int(every), C.c_int(int(with_state)),
                                                self._obs, None))

    def set_warm_start(self, net: "UNet | None", mode: int = WS_PREDICT, lr: float = 0.0):
        """Learned warm start of the FP32 residual solves (WS_PREDICT, WS_TRAIN, WS_OFF)."""
        self._ws = net
        self._check(lib().im3d_ctx_set_warm_start(self._h, net.handle if net else None, C.c_int(mode),
                                                  C.c_double(lr)))

    def conv3d_bf16(self, x, w, bias=None, cin=None, c_off=0):
        """One 3x3x3 convolution on the tensor cores: x a CUDA bfloat16 tensor
        [N, D, H, W, C_pitch] (channels last), w FP32 [cout, cin, 3, 3, 3], bias FP32
        [cout]; returns FP32 [N, D, H, W, cout]."""
        import torch

        nsamp, D, H, W, pitch = (int(v) for v in x.shape)
        cout = int(w.shape[0])
        cin = int(w.shape[1]) if cin is None else cin
        w = w.to(device=x.device, dtype=torch.float32).contiguous()
        b = None if bias is None else bias.to(device=x.device, dtype=torch.float32).contiguous()
        out = torch.empty((nsamp, D, H, W, cout), dtype=torch.float32, device=x.device)
        self._check(lib().im3d_conv3d_bf16(self._h, C.c_void_p(x.data_ptr()), C.c_int(pitch), C.c_int(c_off),
                                           C.c_int(cin), C.c_void_p(w.data_ptr()),
                                           C.c_void_p(b.data_ptr() if b is not None else 0), C.c_int(cout),
                                           C.c_int(nsamp), C.c_int(D), C.c_int(H), C.c_int(W),
                                           C.c_void_p(out.data_ptr())))
        return out

    def set_resume(self, state: dict | None):
        """The next rsfe_apply starts from a state dict of set_observer(with_state=True)."""
        if state is None:
            self._check(lib().im3d_ctx_set_resume(self._h, None, C.c_int(0)))
            self._resume_keep = None
            return
        phi = np.ascontiguousarray(state["phi"])
        b = np.ascontiguousarray(state["b"], dtype=phi.dtype)
        dv = np.ascontiguousarray(state["divdb"], dtype=phi.dtype)
        ck = Checkpoint(t=state["t"], init_variables=state["init_variables"],
                        sched_first=state["sched_first"], reserved=0,
                        sched_rate=state["sched_rate"], tollerance=state["tollerance"],
                        phi=phi.ctypes.data, b=b.ctypes.data, divdb=dv.ctypes.data)
        self._resume_keep = (phi, b, dv)  # the arrays must live until the next apply
        self._check(lib().im3d_ctx_set_resume(self._h, C.byref(ck), C.c_int(phi.dtype.itemsize)))

    # -- operators -----------------------------------------------------------
    def gauss_filter(self, x, sigma, h=(1.0, 1.0, 1.0), radius=3.0, pixel_approach=False, out=None,
                     cyclic=False):
        """acyclic_fftw_convolution (zero boundary) or, with cyclic, cyclic_fftw_convolution
        (periodic boundary) with the normalised Gaussian."""
        px, dt = _ptr(x)
        out = _empty_like(x) if out is None else out
        po, _ = _ptr(out)
        name = "im3d_gauss_filter_cyclic_" if cyclic else "im3d_gauss_filter_"
        fn = getattr(lib(), name + _suffix(dt))
        self._check(fn(self._h, px, po, *map(C.c_int, x.shape), *map(C.c_double, h),
                       C.c_double(sigma), C.c_double(radius), C.c_int(int(pixel_approach))))
        return out

    def grad(self, x, h=(1.0, 1.0, 1.0)):
        px, dt = _ptr(x)
        out = _empty_like(x, (3,) + tuple(x.shape))
        po, _ = _ptr(out)
        fn = getattr(lib(), "im3d_grad_" + _suffix(dt))
        self._check(fn(self._h, px, po, *map(C.c_int, x.shape), *map(C.c_double, h)))
        return out

    def div(self, v, h=(1.0, 1.0, 1.0)):
        pv, dt = _ptr(v)
        out = _empty_like(v, tuple(v.shape[1:]))
        po, _ = _ptr(out)
        fn = getattr(lib(), "im3d_div_" + _suffix(dt))
        self._check(fn(self._h, pv, po, *map(C.c_int, out.shape), *map(C.c_double, h)))
        return out

    def connected_component(self, img, ijk=(0, 0, 0), init=None, threshold=0.5,
                            full_connected=False, binary_output=True, out=None,
                            return_passes=False):
        """image3d<T>::connected_component: seeded by cell ``ijk`` (init None) or by the
        cells where ``init`` != 0; returns the result (and the growth passes)."""
        pi, dtp = _ptr(img)
        pinit, _ = _ptr(init)
        res = _empty_like(img) if out is None else out
        passes = C.c_int(0)
        fn = getattr(lib(), "im3d_connected_component_" + _suffix(dtp))
        self._check(fn(self._h, pi, _ptr(res)[0], *map(C.c_int, img.shape), pinit,
                       *map(C.c_int, ijk), C.c_double(threshold), C.c_int(int(full_connected)),
                       C.c_int(int(binary_output)), C.byref(passes)))
        return (res, int(passes.value)) if return_passes else res

    def poisson_sweeps(self, res, b, dt=1.0, bc=0.0, bc_type=BC_DIR, order=SWEEP_LEXICOGRAPHIC,
                       sweeps=1, h=(1.0, 1.0, 1.0)):
        """In place on ``res``: DirGaussSeidel / NeuGaussSeidel called ``sweeps`` times."""
        pr, dtp = _ptr(res)
        pb, _ = _ptr(b)
        fn = getattr(lib(), "im3d_poisson_sweeps_" + _suffix(dtp))
        self._check(fn(self._h, pr, pb, *map(C.c_int, res.shape), *map(C.c_double, h),
                       C.c_double(dt), C.c_double(bc), C.c_int(bc_type), C.c_int(order),
                       C.c_int(sweeps)))
        return res

    def poisson_solve(self, u, b, dt=1.0, bc=0.0, bc_type=BC_DIR, tol=1e-6, max_sweeps=1000,
                      check_every=0, omega=1.0, h=(1.0, 1.0, 1.0)):
        """In place on ``u``; returns (sweeps, relative residual, converged)."""
        pu, dtp = _ptr(u)
        pb, _ = _ptr(b)
        sw = C.c_int(0)
        rel = C.c_double(0)
        fn = getattr(lib(), "im3d_poisson_solve_" + _suffix(dtp))
        st = self._check(fn(self._h, pu, pb, *map(C.c_int, u.shape), *map(C.c_double, h),
                            C.c_double(dt), C.c_double(bc), C.c_int(bc_type), C.c_double(tol),
                            C.c_int(max_sweeps), C.c_int(check_every), C.c_double(omega),
                            C.byref(sw), C.byref(rel)), allow=(ERR_NOT_CONVERGED,))
        return int(sw.value), float(rel.value), st == OK

    def rsfe_apply_batched(self, volumes, inits=None, params: RsfeParams | None = None,
                           streams: int = 4, outs=None, h=(1.0, 1.0, 1.0)):
        """Segments a list of volumes (same dtype); returns (phis, stats, latency_ms)."""
        p = params if params is not None else default_params()
        n = len(volumes)
        inits = inits if inits is not None else [None] * n
        outs = outs if outs is not None else [_empty_like(v) for v in volumes]
        descs = (VolumeDesc * n)()
        dt = None
        for q, (v, i0, o) in enumerate(zip(volumes, inits, outs)):
            pv, dt = _ptr(v)
            descs[q].myim = pv
            descs[q].init = _ptr(i0)[0]
            descs[q].phi_out = _ptr(o)[0]
            descs[q].nx, descs[q].ny, descs[q].nz = (int(s) for s in v.shape)
            descs[q].hx, descs[q].hy, descs[q].hz = h
        stats = (RsfeStats * n)()
        lat = (C.c_double * n)()
        fn = getattr(lib(), "im3d_rsfe_apply_batched_" + _suffix(dt))
        self._check(fn(self._h, C.c_int(n), descs, C.byref(p), C.c_int(streams), stats, lat))
        return outs, [s.as_dict() for s in stats], list(lat)

    def rsfe_apply(self, myim, init=None, params: RsfeParams | None = None, h=(1.0, 1.0, 1.0),
                   want_u=False, want_f=False, phi_out=None):
        """segm::rsfe_splitbregman<T>::apply; returns dict(phi, u, f1, f2, stats)."""
        p = params if params is not None else default_params()
        pm, dt = _ptr(myim)
        pi, _ = _ptr(init)
        phi = _empty_like(myim) if phi_out is None else phi_out
        u = _empty_like(myim) if want_u else None
        f1 = _empty_like(myim) if want_f else None
        f2 = _empty_like(myim) if want_f else None
        st = RsfeStats()
        self._obs_shape = tuple(int(x) for x in myim.shape)
        fn = getattr(lib(), "im3d_rsfe_apply_" + _suffix(dt))
        try:
            self._check(fn(self._h, pm, pi, *map(C.c_int, myim.shape), *map(C.c_double, h),
                           C.byref(p), _ptr(phi)[0], _ptr(u)[0], _ptr(f1)[0], _ptr(f2)[0],
                           C.byref(st)))
        finally:
            self._resume_keep = None
        return dict(phi=phi, u=u, f1=f1, f2=f2, stats=st.as_dict())


class UNet:
    """The learned warm start's network (im3d_unet_*): a 3-level 3-D U-Net whose
    forward and backward passes run on the library's tensor-core kernels."""

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        self._h = C.c_void_p()
        ctx._check(lib().im3d_unet_create(ctx.handle, C.c_uint64(seed), C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().im3d_unet_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def param_count(self) -> int:
        return int(lib().im3d_unet_param_count(self._h))

    def get_params(self) -> np.ndarray:
        out = np.empty(self.param_count, dtype=np.float32)
        self.ctx._check(lib().im3d_unet_get_params(self.ctx.handle, self._h, out.ctypes.data_as(C.c_void_p),
                                                   C.c_int64(out.size)))
        return out

    def set_params(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.float32)
        self.ctx._check(lib().im3d_unet_set_params(self.ctx.handle, self._h, flat.ctypes.data_as(C.c_void_p),
                                                   C.c_int64(flat.size)))

    def forward(self, x):
        """x: [nsamp, 4, nx, ny, nz] FP32 (numpy or CUDA tensor) -> y [nsamp, nx, ny, nz]."""
        px, dt = _ptr(x)
        ns, _, nx, ny, nz = (int(v) for v in x.shape)
        y = _empty_like(x, (ns, nx, ny, nz))
        self.ctx._check(lib().im3d_unet_forward(self.ctx.handle, self._h, px, C.c_int(ns), C.c_int(nx),
                                                C.c_int(ny), C.c_int(nz), _ptr(y)[0]))
        return y

    def train_step(self, x, target, lr: float, want_grads: bool = False):
        """One Adam step on (x, target); returns the loss (and the FP32 gradients)."""
        px, _ = _ptr(x)
        pt, _ = _ptr(target)
        ns, _, nx, ny, nz = (int(v) for v in x.shape)
        loss = C.c_double(0)
        g = np.empty(self.param_count, dtype=np.float32) if want_grads else None
        self.ctx._check(lib().im3d_unet_train_step(self.ctx.handle, self._h, px, pt, C.c_int(ns), C.c_int(nx),
                                                   C.c_int(ny), C.c_int(nz), C.c_double(lr), C.byref(loss),
                                                   g.ctypes.data_as(C.c_void_p) if g is not None else None))
        return (float(loss.value), g) if want_grads else float(loss.value)

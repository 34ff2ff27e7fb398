"""GPU: the Gaussian filter entry point that allocates nothing.

im3d_gauss_filter_f32_noalloc serves callers that cannot call cudaMalloc (a host
framework that owns all device memory through its own pool, a hard memory budget,
code that must not make allocation calls that can synchronise the device). It keeps
its intermediate volumes in a fixed __device__ array instead of context buffers.
This test calls it through the C ABI twice in a row, on two different volumes, and
checks each result against the allocating entry point im3d_gauss_filter_f32, with
the FP32 tolerance the other filter tests use; then on a stream the caller owns, with
inputs written on that stream, and on a small odd volume whose axes are shorter than
the Gaussian's support. It also checks that a volume above the fixed capacity, and
one whose launch geometry does not fit, are refused before anything runs. It sits in
its own file named to be collected last, and builds everything it needs itself, so
it passes alone in a fresh process as well as after the other tests.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_VOXELS = 1 << 21


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _noalloc(lib, x, out, sigma, h, stream=None):
    return lib.im3d_gauss_filter_f32_noalloc(
        C.c_void_p(x.data_ptr()), C.c_void_p(out.data_ptr()), *map(C.c_int, x.shape),
        *map(C.c_double, h), C.c_double(sigma), C.c_double(3.0), C.c_int(0),
        C.c_void_p(stream or 0))


def test_noalloc_filter_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    pkg = importlib.import_module("3dimagetoolkit_b200")
    lib = pkg.lib()
    rng = np.random.default_rng(123)
    cases = [((40, 36, 33), 2.0, (1.0, 1.0, 1.0)), ((128, 128, 128), 3.0, (0.9, 1.0, 1.1))]
    with pkg.Context(0) as ctx:
        for shape, sigma, h in cases:
            x_np = rng.random(shape, dtype=np.float32)
            x = torch.from_numpy(x_np).cuda()
            out = torch.empty_like(x)
            st = _noalloc(lib, x, out, sigma, h)
            assert st == 0, st
            want = ctx.gauss_filter(x_np, sigma, h=h)
            got = out.cpu().numpy()
            assert _rel(got, want) < 2e-6


def test_noalloc_filter_refuses_volumes_above_its_scratch():
    torch = pytest.importorskip("torch")
    pkg = importlib.import_module("3dimagetoolkit_b200")
    x = torch.zeros((129, 128, 128), dtype=torch.float32, device="cuda")
    assert x.numel() > MAX_VOXELS
    out = torch.empty_like(x)
    assert _noalloc(pkg.lib(), x, out, 2.0, (1.0, 1.0, 1.0)) == 7


def test_noalloc_filter_on_a_caller_stream_and_a_small_odd_volume():
    torch = pytest.importorskip("torch")
    pkg = importlib.import_module("3dimagetoolkit_b200")
    lib = pkg.lib()
    stream = torch.cuda.Stream()
    with pkg.Context(0) as ctx:
        for shape, sigma in (((96, 80, 72), 3.0), ((7, 9, 11), 2.0)):
            with torch.cuda.stream(stream):
                g = torch.Generator(device="cuda")
                g.manual_seed(7)
                x = torch.rand(shape, device="cuda", generator=g)
                out = torch.full_like(x, float("nan"))
            st = _noalloc(lib, x, out, sigma, (1.0, 1.0, 1.0), stream=stream.cuda_stream)
            assert st == 0, st
            got = out.cpu().numpy()  # the call returned after its stream finished
            want = ctx.gauss_filter(x.cpu().numpy(), sigma)
            assert np.isfinite(got).all()
            assert _rel(got, want) < 2e-6, shape


def test_noalloc_filter_refuses_a_launch_geometry_that_does_not_fit():
    torch = pytest.importorskip("torch")
    pkg = importlib.import_module("3dimagetoolkit_b200")
    x = torch.zeros((70000, 3, 3), dtype=torch.float32, device="cuda")
    assert x.numel() <= MAX_VOXELS
    out = torch.full_like(x, 5.0)
    assert _noalloc(pkg.lib(), x, out, 1.0, (1.0, 1.0, 1.0)) == 1
    assert bool((out == 5.0).all())  # nothing was written


def test_noalloc_filter_captured_in_a_cuda_graph():
    # the first call (outside any capture) looks the scratch up; a later call captured
    # into a graph neither waits nor fails, and each replay filters the current input
    torch = pytest.importorskip("torch")
    pkg = importlib.import_module("3dimagetoolkit_b200")
    lib = pkg.lib()
    shape = (40, 36, 32)
    x = torch.rand(shape, device="cuda")
    out = torch.empty_like(x)
    assert _noalloc(lib, x, out, 2.0, (1.0, 1.0, 1.0)) == 0
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        st = _noalloc(lib, x, out, 2.0, (1.0, 1.0, 1.0), stream=torch.cuda.current_stream().cuda_stream)
    assert st == 0, st
    with pkg.Context(0) as ctx:
        for seed in (1, 2):
            g = torch.Generator(device="cuda")
            g.manual_seed(seed)
            x.copy_(torch.rand(shape, device="cuda", generator=g))
            out.fill_(float("nan"))
            graph.replay()
            torch.cuda.synchronize()
            want = ctx.gauss_filter(x.cpu().numpy(), 2.0)
            assert _rel(out.cpu().numpy(), want) < 2e-6, seed
    del graph

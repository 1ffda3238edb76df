"""kw_gradient_noalloc: the allocation-free gradient entry point.

Callers such as a MATLAB MEX function on gpuArray data, a PyTorch extension
bound to the framework's caching allocator, or a service that forbids device
allocation after start-up cannot let the library call cudaMalloc.  This test
gives the entry point device buffers owned by PyTorch and checks two calls in
a row against the existing allocating path: with p0 = f and Nt = 1 the
reference loop sets u_i = dt / (2 rho0) real(ifftn(ddi_k_shift_pos kappa
fftn(f))) (kspaceFirstOrder3D.m:1023-1037), which kspaceFirstOrder2D/3D
return through kw_run when sensor.record = {'u'} covers every cell.

This file is collected last so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

TOL = 1e-4


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a, np.float64) - b).ravel()) / np.linalg.norm(np.ravel(b)))


def _reference_gradients(kw, f, dx, dt, c, rho):
    dim = f.ndim
    args = []
    for s in f.shape:
        args += [s, dx]
    g = kw.kWaveGrid(*args)
    g.setTime(1, dt)
    run = kw.kspaceFirstOrder2D if dim == 2 else kw.kspaceFirstOrder3D
    out = run(g, {"sound_speed": c, "density": rho}, {"p0": f},
              {"mask": np.ones(f.shape), "record": ["u"]}, Smooth=False, PMLSize=2)
    comps = ["ux", "uy", "uz"][:dim]
    # u = dt / (2 rho) * gradient, recorded at t = 1 in find(mask) order
    return [out[n][:, 0].reshape(f.shape, order="F") * (2.0 * rho / dt) for n in comps]


def _noalloc(lib, f_dev, out_dev, shape, dx, axis, c, dt):
    dim = len(shape)
    shp = (C.c_uint64 * 3)(*(list(shape) + [1] * (3 - dim)))
    sp = (C.c_double * 3)(*([dx] * 3))
    return lib.kw_gradient_noalloc(dim, shp, sp, axis, 1, c, dt, 1, C.c_void_p(f_dev.data_ptr()),
                                   C.c_void_p(out_dev.data_ptr()), None)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 48), (24, 20, 30), (64, 64), (32, 64, 64)])
def test_noalloc_gradient_matches_allocating_path(shape):
    torch = pytest.importorskip("torch")
    import kwave_b200 as kw
    from kwave_b200 import _abi
    lib = _abi.load_library()
    dx, c, rho = 1e-4, 1500.0, 1000.0
    dt = 0.3 * dx / c
    rng = np.random.default_rng(7)
    fields = [rng.standard_normal(shape), np.cos(np.linspace(0, 9, int(np.prod(shape)))).reshape(shape)]
    for f in fields:          # two calls in a row share the scratch array
        ref = _reference_gradients(kw, f, dx, dt, c, rho)
        f_dev = torch.tensor(f.ravel(order="F"), dtype=torch.float32, device="cuda")
        for axis in range(len(shape)):
            out_dev = torch.full_like(f_dev, float("nan"))
            torch.cuda.synchronize()
            st = _noalloc(lib, f_dev, out_dev, shape, dx, axis, c, dt)
            assert st == 0, lib.kw_last_error()
            got = out_dev.cpu().numpy().reshape(shape, order="F")
            e = _rel(got, ref[axis])
            assert e <= TOL, "axis %d rel-L2 %.3e" % (axis, e)


@pytest.mark.gpu
def test_noalloc_at_the_scratch_limit():
    """200^3 (a 32.3 MB half spectrum) is the largest cube that fits the
    32 MiB scratch: the spectrum's end and the operator tables sit at the top
    of the array.  Checked against the allocating path on a smooth field."""
    torch = pytest.importorskip("torch")
    import kwave_b200 as kw
    from kwave_b200 import _abi
    lib = _abi.load_library()
    shape = (200, 200, 200)
    dx, c, rho = 1e-4, 1500.0, 1000.0
    dt = 0.3 * dx / c
    ax = [np.arange(n) - n / 2 for n in shape]
    f = np.exp(-(ax[0][:, None, None] ** 2 + ax[1][None, :, None] ** 2 + ax[2][None, None, :] ** 2) / (2 * 12.0 ** 2))
    ref = _reference_gradients(kw, f, dx, dt, c, rho)
    f_dev = torch.tensor(f.ravel(order="F"), dtype=torch.float32, device="cuda")
    for axis in (0, 2):
        out_dev = torch.full_like(f_dev, float("nan"))
        torch.cuda.synchronize()
        assert _noalloc(lib, f_dev, out_dev, shape, dx, axis, c, dt) == 0, lib.kw_last_error()
        got = out_dev.cpu().numpy().reshape(shape, order="F")
        e = _rel(got, ref[axis])
        assert e <= TOL, "axis %d rel-L2 %.3e" % (axis, e)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(256, 256, 256), (256, 256, 128)])
def test_noalloc_rejects_grids_above_the_scratch_limit(shape):
    """256 x 256 x 128 (a 34.1 MB half spectrum) is the first such shape
    rejected; nothing is launched for it."""
    torch = pytest.importorskip("torch")
    from kwave_b200 import _abi
    lib = _abi.load_library()
    f = torch.zeros(8, device="cuda")
    shp = (C.c_uint64 * 3)(*shape)
    sp = (C.c_double * 3)(1e-4, 1e-4, 1e-4)
    st = lib.kw_gradient_noalloc(3, shp, sp, 0, 1, 1500.0, 1e-8, 1, C.c_void_p(f.data_ptr()),
                                 C.c_void_p(f.data_ptr()), None)
    assert st == _abi.KW_ERR_UNSUPPORTED
    assert b"limited to" in lib.kw_last_error()


@pytest.mark.gpu
def test_noalloc_refuses_a_capturing_stream():
    """A call on a stream under capture returns KW_ERR_UNSUPPORTED and
    enqueues nothing, so the capture stays valid; the same call then runs
    once the capture has ended."""
    torch = pytest.importorskip("torch")
    from kwave_b200 import _abi
    lib = _abi.load_library()
    shape = (64, 64)
    f_dev = torch.ones(int(np.prod(shape)), device="cuda")
    out_dev = torch.zeros_like(f_dev)
    shp = (C.c_uint64 * 3)(64, 64, 1)
    sp = (C.c_double * 3)(1e-4, 1e-4, 1e-4)
    graph = torch.cuda.CUDAGraph()
    torch.cuda.synchronize()
    with torch.cuda.graph(graph):
        handle = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        st = lib.kw_gradient_noalloc(2, shp, sp, 0, 1, 1500.0, 2e-8, 1, C.c_void_p(f_dev.data_ptr()),
                                     C.c_void_p(out_dev.data_ptr()), handle)
        out_dev.add_(1.0)     # something for the graph to hold
    assert st == _abi.KW_ERR_UNSUPPORTED
    assert b"captured" in lib.kw_last_error()
    del graph
    st = lib.kw_gradient_noalloc(2, shp, sp, 0, 1, 1500.0, 2e-8, 1, C.c_void_p(f_dev.data_ptr()),
                                 C.c_void_p(out_dev.data_ptr()), None)
    assert st == 0, lib.kw_last_error()
    torch.cuda.synchronize()
    # the gradient of a constant field is zero
    assert float(out_dev.abs().max()) < 1e-3

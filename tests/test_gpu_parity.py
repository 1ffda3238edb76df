"""GPU parity: the CUDA path through the C ABI against the FP64 CPU oracle.

Tolerance: relative L2 error <= 1e-4 on every recorded output (the bound the
FP32 loop must meet against an FP64 restatement of the reference solver).
"""
import numpy as np
import pytest

from cases import CASES, make_case

TOL = 1e-4


def _grid(mod, shape, dx, Nt, dt):
    args = []
    for s in shape:
        args += [s, dx]
    g = (mod.kWaveGrid if hasattr(mod, "kWaveGrid") else mod.KWaveGrid)(*args)
    g.setTime(Nt, dt)
    return g


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (d if d > 0 else 1.0))


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_parity(name):
    import kwave_b200 as kw
    from oracle import kspace as oracle
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    run = kw.kspaceFirstOrder2D if dim == 2 else kw.kspaceFirstOrder3D
    gpu = run(_grid(kw, shape, dx, Nt, dt), med, src, sen, **opts)
    ref = oracle.kspace_first_order(_grid(oracle, shape, dx, Nt, dt), med, src, sen, **opts)
    _compare_outputs(name, gpu, ref)


def _compare_outputs(name, gpu, ref):
    """Same output structure (matrix, dict of outputs, or one dict per
    cuboid) and every output within TOL."""
    if isinstance(ref, list):
        assert isinstance(gpu, list) and len(gpu) == len(ref)
        for i, (g, r) in enumerate(zip(gpu, ref)):
            _compare_outputs("%s[cuboid %d]" % (name, i), g, r)
    elif isinstance(ref, dict):
        assert set(gpu) == set(ref), (sorted(gpu), sorted(ref))
        for k in ref:
            assert gpu[k].shape == ref[k].shape, k
            e = _rel(gpu[k], ref[k])
            assert e <= TOL, "%s: %s rel-L2 %.3e" % (name, k, e)
    else:
        assert gpu.shape == ref.shape
        e = _rel(gpu, ref)
        assert e <= TOL, "%s rel-L2 %.3e" % (name, e)


GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden")


@pytest.mark.gpu
def test_golden_cfg1_small():
    """Config 1 recipe at 64^2 (Cartesian circle sensor, nearest) against the fixture."""
    import kwave_b200 as kw
    g = np.load(GOLDEN + "/cfg1_small.npz")
    N, dx = int(g["N"]), float(g["dx"])
    kg = kw.kWaveGrid(N, dx, N, dx)
    kg.setTime(int(g["Nt"]), float(g["dt"]))
    out = kw.kspaceFirstOrder2D(kg, {"sound_speed": float(g["c"]), "density": 1000.0}, {"p0": g["p0"]},
                                {"mask": g["sensor_mask"]}, PMLSize=10, CartInterp="nearest")
    assert _rel(out, g["p"]) <= TOL


@pytest.mark.gpu
def test_golden_absorbing_3d():
    import kwave_b200 as kw
    g = np.load(GOLDEN + "/absorbing_3d.npz")
    shape = tuple(int(v) for v in g["shape"])
    dx = float(g["dx"])
    kg = kw.kWaveGrid(shape[0], dx, shape[1], dx, shape[2], dx)
    kg.setTime(int(g["Nt"]), float(g["dt"]))
    med = {"sound_speed": g["c"], "density": g["rho"], "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
    out = kw.kspaceFirstOrder3D(kg, med, {"p_mask": g["p_mask"], "p": g["sig"]},
                                {"mask": g["sensor_mask"], "record": ["p", "p_max", "p_final"]}, PMLSize=4)
    for k in ("p", "p_max", "p_final"):
        assert _rel(out[k], g["out_" + k]) <= TOL, k


@pytest.mark.gpu
def test_golden_time_reversal_2d():
    import kwave_b200 as kw
    g = np.load(GOLDEN + "/time_reversal_2d.npz")
    N, dx = int(g["N"]), float(g["dx"])
    kg = kw.kWaveGrid(N, dx, N, dx)
    kg.setTime(int(g["Nt"]), float(g["dt"]))
    p = kw.kspaceFirstOrder2D(kg, {"sound_speed": float(g["c"]), "density": 1000.0}, {},
                              {"mask": g["sensor_mask"], "time_reversal_boundary_data": g["data"]}, PMLSize=8)
    assert _rel(p, g["p_final"]) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["2d_hetero_abs_nl", "3d_hetero_abs_nl_plane"])
def test_column_major_abi_matches_row_major(name):
    """The MATLAB-side form of the C ABI (column-major grid arrays, host-formed
    rho0_sg{x,y,z}) gives the results of the row-major form with staggered
    densities formed on the device."""
    import ctypes as C
    import kwave_b200 as kw
    from kwave_b200 import _abi
    from kwave_b200.solver import Simulation
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    row = Simulation.from_prepared(kw.Server.prepare(dim, _grid(kw, shape, dx, Nt, dt), med, src, sen, **opts))
    ref = row.run()
    row.close()
    prep = kw.Server.prepare(dim, _grid(kw, shape, dx, Nt, dt), med, src, sen, **opts)
    pr = prep.problem
    assert pr.array_order == _abi.KW_ROW_MAJOR and pr.derive_rho0_sg == 1
    N = int(np.prod(shape))
    keep = []

    def colmajor(ptr):
        a = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_float)), shape=(N,)).reshape(shape)
        x = np.ascontiguousarray(a.ravel(order="F"))
        keep.append(x)
        return x

    for f in ("c0", "rho0", "BonA", "alpha_coeff", "p0_source_input"):
        if getattr(pr, f):
            setattr(pr, f, _abi.fptr(colmajor(getattr(pr, f))))
    rho = np.asarray(med["density"], dtype=np.float64)
    for a, f in enumerate(("rho0_sgx", "rho0_sgy", "rho0_sgz")[:dim]):
        r = rho.copy()
        lo = [slice(None)] * dim
        hi = [slice(None)] * dim
        lo[a], hi[a] = slice(0, shape[a] - 1), slice(1, shape[a])
        r[tuple(lo)] = 0.5 * (rho[tuple(lo)] + rho[tuple(hi)])
        x = np.ascontiguousarray(r.ravel(order="F"), dtype=np.float32)
        keep.append(x)
        setattr(pr, f, _abi.fptr(x))
    pr.array_order = _abi.KW_COLUMN_MAJOR
    pr.derive_rho0_sg = 0
    col = Simulation.from_prepared(prep)
    out = col.run()
    col.close()
    ref = ref if isinstance(ref, dict) else {"p": ref}
    out = out if isinstance(out, dict) else {"p": out}
    for k in ref:
        assert _rel(out[k], ref[k]) <= 1e-5, (k, _rel(out[k], ref[k]))


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["3d_intensity_static", "3d_static_mixed_radix", "2d_homog_p0"])
def test_tile_widths_do_not_change_results(name):
    """Every choice of full, half or quarter tiles the autotuner may make gives
    bit-identical outputs (tile widths group lines into blocks; the
    arithmetic of a line does not depend on them)."""
    import itertools
    import kwave_b200 as kw
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case(name)
    sim = kw.Simulation(dim, _grid(kw, shape, dx, Nt, dt), med, src, sen, **opts)
    chosen = sim.tiles()
    ref = sim.run()
    ref = ref if isinstance(ref, dict) else {"p": ref}
    options = []
    for t, n in zip(chosen, (shape[-1], shape[1] if dim == 3 else 1, shape[0])):
        if t == 0:
            options.append([0])
        else:
            full = min(64, 1 << int(np.floor(np.log2(4096 // n))))
            options.append([full, full // 2, full // 4])
    for tiles in itertools.product(*options):
        sim.set_tiles(tiles)
        out = sim.run()
        out = out if isinstance(out, dict) else {"p": out}
        for k in ref:
            assert np.array_equal(out[k], ref[k]), (name, tiles, k)
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("N", [256, 512])
def test_full_size_homogeneous_is_exact(N):
    """At the full sizes, where the FP64 oracle is too slow, a size-independent
    check: in a homogeneous lossless medium with PMLAlpha = 0 the k-space
    scheme is exact (kspaceFirstOrder3D.m:23-25), so p_final after Nt steps is
    IFFT(FFT(p0) cos(c |k| (Nt - 1) dt)), evaluated here with an FP64 real FFT.
    Tolerance: 1e-4 relative L2, as for every parity test."""
    import scipy.fft as sfft
    import kwave_b200 as kw
    dx, c, Nt = 1e-4, 1500.0, 20
    dt = 0.3 * dx / c
    ax = np.arange(N) - N / 2
    r2 = ax[:, None, None] ** 2 + ax[None, :, None] ** 2 + ax[None, None, :] ** 2
    p0 = np.exp(-r2 / (2 * 6.0 ** 2))
    kg = kw.kWaveGrid(N, dx, N, dx, N, dx)
    kg.setTime(Nt, dt)
    out = kw.kspaceFirstOrder3D(kg, {"sound_speed": c, "density": 1000.0}, {"p0": p0}, {"record": ["p_final"]},
                                PMLAlpha=0.0, PMLSize=10, Smooth=False)
    k = 2 * np.pi * sfft.fftfreq(N, dx)
    kz = 2 * np.pi * sfft.rfftfreq(N, dx)
    kmag = np.sqrt(k[:, None, None] ** 2 + k[None, :, None] ** 2 + kz[None, None, :] ** 2)
    spec = sfft.rfftn(p0, workers=-1)
    spec *= np.cos(c * kmag * (Nt - 1) * dt)
    exact = sfft.irfftn(spec, s=p0.shape, workers=-1)
    err = float(np.linalg.norm((out["p_final"] - exact).ravel()) / np.linalg.norm(exact.ravel()))
    assert err <= TOL, "N=%d rel-L2 %.3e" % (N, err)

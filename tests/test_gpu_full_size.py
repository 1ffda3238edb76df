"""Full-size parity: the benchmark workloads themselves against the FP64 oracle.

At these sizes the NumPy oracle would take hours, so the oracle's time loop
runs on torch.float64 tensors on the GPU (``Device="cuda"``).  That backend
executes the same statements as the NumPy oracle and agrees with it to
<= 1e-12 (tests/test_oracle_backends.py); it uses torch.fft, never this
library's kernels.

Tolerance: relative L2 error <= 1e-4 on every compared output, as for every
parity test.
"""
import numpy as np
import pytest

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


def _run_both(w):
    import torch
    import kwave_b200 as kw
    from oracle import kspace as oracle
    gpu = kw.kspaceFirstOrder3D(_grid(kw, w["shape"], w["dx"], w["Nt"], w["dt"]), w["medium"], w["source"],
                                w["sensor"], **w["options"])
    ref = oracle.kspace_first_order(_grid(oracle, w["shape"], w["dx"], w["Nt"], w["dt"]), w["medium"],
                                    w["source"], w["sensor"], Device="cuda", **w["options"])
    torch.cuda.empty_cache()
    return gpu, ref


@pytest.mark.gpu
def test_headline_256_nt1000():
    """The headline workload exactly as benchmarked: 256^3, 8-blob medium,
    absorbing (y = 1.5), BonA 6, 64 x 64 additive plane source, PML 10,
    Nt = 1000; p on the central xy-plane and the 256-point line, p_max on both."""
    import bench
    w = bench.workload(seed=0)
    gpu, ref = _run_both(w)
    assert set(gpu) == set(ref) == {"p", "p_max"}
    # rows of the union mask in find() order: split the line from the plane
    N = w["shape"][0]
    lin = np.flatnonzero(w["sensor"]["mask"].ravel(order="F"))
    x, y, z = np.unravel_index(lin, w["shape"], order="F")
    on_line = (x == 3 * N // 4) & (y == N // 2)
    on_plane = z == N // 2
    assert on_line.sum() == N and on_plane.sum() == N * N
    errs = {
        "p plane": _rel(gpu["p"][on_plane], ref["p"][on_plane]),
        "p line": _rel(gpu["p"][on_line], ref["p"][on_line]),
        "p_max plane": _rel(gpu["p_max"][on_plane], ref["p_max"][on_plane]),
        "p_max line": _rel(gpu["p_max"][on_line], ref["p_max"][on_line]),
    }
    print("headline 256^3 Nt=1000 rel-L2:", {k: "%.2e" % v for k, v in errs.items()})
    for k, e in errs.items():
        assert e <= TOL, "%s rel-L2 %.3e" % (k, e)


@pytest.mark.gpu
def test_layered_512_full_volume():
    """The large layered 512^3 workload (rough interfaces, per-layer alpha and
    B/A, 128 x 128 focused plane source of 16 384 signals, PML 20) for its
    first 200 steps, p_max and p_rms over every cell."""
    import bench
    w = bench.layered_workload(seed=11, N=512, Nt=200)
    gpu, ref = _run_both(w)
    assert set(gpu) == set(ref) == {"p_max", "p_rms"}
    errs = {k: _rel(gpu[k], ref[k]) for k in ("p_max", "p_rms")}
    print("layered 512^3 Nt=200 rel-L2:", {k: "%.2e" % v for k, v in errs.items()})
    for k, e in errs.items():
        assert e <= TOL, "%s rel-L2 %.3e" % (k, e)


@pytest.mark.gpu
def test_cfg1_as_stated():
    """The 2-D homogeneous lossless case as specified: 128^2, dx = 0.1 mm,
    c = 1500, rho = 1000, p0 = makeDisc(128, 128, 65, 65, 5) (smoothed by
    default), PML 20 with alpha 2, CFL 0.3 and t_end = 1.2 x diagonal / c
    (Nt = 725), 64 points on a circle of radius 40 cells mapped to the grid
    by nearest neighbour, recording p."""
    import kwave_b200 as kw
    from oracle import kspace as oracle
    N, dx, c = 128, 1e-4, 1500.0
    t_end = 1.2 * np.sqrt(2) * N * dx / c
    p0 = kw.makeDisc(N, N, 65, 65, 5)
    cart = kw.makeCartCircle(40 * dx, 64)
    med = {"sound_speed": c, "density": 1000.0}
    kg = kw.kWaveGrid(N, dx, N, dx)
    kg.makeTime(c, 0.3, t_end)
    assert kg.Nt == 725
    gpu = kw.kspaceFirstOrder2D(kg, med, {"p0": p0}, {"mask": cart}, PMLSize=20, PMLAlpha=2.0,
                                CartInterp="nearest")
    okg = oracle.KWaveGrid(N, dx, N, dx)
    okg.makeTime(c, 0.3, t_end)
    ref = oracle.kspace_first_order(okg, med, {"p0": p0}, {"mask": cart}, PMLSize=20, PMLAlpha=2.0,
                                    CartInterp="nearest")
    assert gpu.shape == ref.shape == (64, 725)
    e = _rel(gpu, ref)
    print("cfg1 128^2 Nt=725 rel-L2 %.2e" % e)
    assert e <= TOL


@pytest.mark.gpu
def test_fast_oracle_on_cuda_matches_numpy():
    """The torch.float64 CUDA oracle against the NumPy oracle on a small
    heterogeneous absorbing nonlinear 3-D case with a plane source."""
    from cases import make_case
    from oracle import kspace as oracle
    dim, shape, dx, Nt, dt, med, src, sen, opts = make_case("3d_hetero_abs_nl_plane")
    a = oracle.kspace_first_order(_grid(oracle, shape, dx, Nt, dt), med, src, sen, **opts)
    b = oracle.kspace_first_order(_grid(oracle, shape, dx, Nt, dt), med, src, sen, Device="cuda", **opts)
    for k in a:
        assert _rel(b[k], a[k]) <= 1e-12, k

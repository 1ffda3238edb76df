"""Host-side setup of the drop-in (CPU only, no device calls).

The product's restatements of the reference helpers are checked against the
oracle's independent ones, and the setup that precedes the C ABI
(private/kspaceFirstOrder_inputChecking.m, scaleSourceTerms.m, the staggered
density of kspaceFirstOrder3D.m:585-607) is checked for the values it hands
over and for the errors the reference raises.
"""
import ctypes as C

import numpy as np
import pytest

import kwave_b200 as kw
from kwave_b200 import _abi
from kwave_b200.solver import KWaveInputError, _prepare
from oracle import kspace as ks


def _arr(ptr, n, dtype=np.float32):
    ctype = C.c_float if dtype == np.float32 else C.c_uint64
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).copy()


def _grids(shape, dx):
    a = []
    for s in shape:
        a += [s, dx]
    return kw.kWaveGrid(*a), ks.KWaveGrid(*a)


@pytest.mark.parametrize("n,d", [(64, 1e-3), (45, 2e-4)])
def test_kgrid_matches_oracle(n, d):
    g, o = _grids((n, n + 3, n - 1), d)
    for a in range(3):
        assert np.array_equal(g.k_vec(a), o.k_vecs()[a])
        assert np.allclose(g.grid_vec(a), o.vec(a), rtol=0, atol=1e-15)
    g.makeTime(np.array([1480.0, 1620.0]))
    o.makeTime(np.array([1480.0, 1620.0]))
    assert (g.Nt, g.dt) == (o.Nt, o.dt)


def test_shape_helpers_match_oracle():
    assert np.array_equal(kw.makeDisc(64, 48, 20, 30, 6), ks.make_disc(64, 48, 20, 30, 6))
    assert np.array_equal(kw.makeDisc(63, 47, 0, 0, 9), ks.make_disc(63, 47, 0, 0, 9))
    assert np.array_equal(kw.makeBall(20, 22, 24, 9, 10, 12, 5), ks.make_ball(20, 22, 24, 9, 10, 12, 5))
    assert np.allclose(kw.makeCartCircle(4e-3, 33, (1e-3, -2e-3)), ks.make_cart_circle(4e-3, 33, (1e-3, -2e-3)),
                       rtol=0, atol=1e-15)
    g, o = _grids((40, 40), 2e-4)
    pts = ks.make_cart_circle(3e-3, 50)
    m1, o1, r1 = kw.cart2grid(g, pts)
    m2, o2, r2 = ks.cart2grid(o, pts)
    assert np.array_equal(m1, m2) and np.array_equal(o1, o2) and np.array_equal(r1, r2)


@pytest.mark.parametrize("shape", [(64, 64), (45, 36), (20, 22, 17)])
def test_smooth_matches_oracle(shape):
    rng = np.random.default_rng(3)
    f = rng.random(shape)
    assert np.allclose(kw.smooth(f, True), ks.smooth(f, True), rtol=1e-12, atol=1e-12)
    assert np.allclose(kw.getWin(shape, "Blackman", Rotation=True, Symmetric=[s % 2 == 1 for s in shape]),
                       ks.get_win(list(shape), "Blackman", rotation=True, symmetric=[s % 2 == 1 for s in shape]))


def test_problem_contents_heterogeneous_absorbing_source():
    shape = (24, 20, 16)
    g, o = _grids(shape, 1e-4)
    g.setTime(30, 2e-8)
    rng = np.random.default_rng(5)
    c = 1500 + 100 * rng.random(shape)
    rho = 1000 + 50 * rng.random(shape)
    pm = np.zeros(shape)
    pm[3, 4:8, 5:9] = 1
    sig = np.sin(np.arange(12.0))
    sensor = np.zeros(shape)
    sensor[10, :, 3] = 1
    P = _prepare(3, g, {"sound_speed": c, "density": rho, "alpha_coeff": 0.5, "alpha_power": 1.3, "BonA": 4.0},
                 {"p_mask": pm, "p": sig}, {"mask": sensor, "record": ["p", "p_rms"]}, {"PMLSize": 3})
    pr = P.problem
    N = int(np.prod(shape))
    assert (pr.dim, pr.Nx, pr.Ny, pr.Nz, pr.Nt) == (3, 24, 20, 16, 30)
    assert pr.c_ref == pytest.approx(c.max())
    assert pr.absorbing_flag == _abi.KW_ABSORBING and pr.nonlinear_flag == 1
    # grid arrays go over in row-major order; the library transposes them
    assert pr.array_order == _abi.KW_ROW_MAJOR
    assert np.array_equal(_arr(pr.c0, N), c.ravel().astype(np.float32))
    assert np.array_equal(_arr(pr.rho0, N), rho.ravel().astype(np.float32))
    # staggered densities (kspaceFirstOrder3D.m:590-601) are formed on the device
    assert pr.derive_rho0_sg == 1 and not pr.rho0_sgx and not pr.rho0_sgy and not pr.rho0_sgz
    # source: find(mask) order, one signal scaled by 2 dt / (N c0(first point) dx) (scaleSourceTerms.m)
    pos = np.flatnonzero(pm.ravel(order="F"))
    assert np.array_equal(_arr(pr.p_source.index, pos.size, np.uint64), pos + 1)
    scale = 2 * 2e-8 / (3 * c.ravel(order="F")[pos[0]] * 1e-4)
    assert np.allclose(_arr(pr.p_source.input, 12), (sig * scale).astype(np.float32), rtol=1e-6)
    assert pr.p_source.mode == _abi.SOURCE_MODES["additive"]
    idx = np.flatnonzero(sensor.ravel(order="F"))
    assert np.array_equal(_arr(pr.sensor_mask_index, idx.size, np.uint64), idx + 1)
    assert pr.record == (1 << _abi.REC_BITS["p"]) | (1 << _abi.REC_BITS["p_rms"])


def test_pml_outside_expands_grid():
    g, _ = _grids((30, 26), 1e-4)
    g.setTime(10, 2e-8)
    mask = np.zeros((30, 26))
    mask[5, :] = 1
    P = _prepare(2, g, {"sound_speed": 1500.0, "density": 1000.0}, {"p0": np.ones((30, 26))},
                 {"mask": mask, "record": ["p_final"]}, {"PMLSize": [4, 6], "PMLInside": False})
    assert (P.problem.Nx, P.problem.Ny) == (38, 38)
    assert list(P.problem.inside_lo)[:2] == [5, 7] and list(P.problem.inside_hi)[:2] == [34, 32]


@pytest.mark.parametrize("medium,source,sensor,opts,msg", [
    ({}, {}, None, {}, "sound_speed"),
    ({"sound_speed": 1500.0, "alpha_coeff": 0.5, "alpha_power": 3.2}, {}, None, {}, "between 0 and 3"),
    ({"sound_speed": 1500.0, "alpha_coeff": 0.5, "alpha_power": 1.0}, {}, None, {}, "alpha_power = 1"),
    ({"sound_speed": 1500.0, "BonA": 5.0}, {"p0": np.ones((16, 16))}, None, {}, "density must be explicitly"),
    ({"sound_speed": 1500.0, "density": 1.0}, {"p0": np.ones((16, 16)), "p": np.ones(4), "p_mask": np.ones((16, 16))},
     None, {}, "can't be defined in the same"),
    ({"sound_speed": 1500.0}, {"p0": np.ones((16, 16))}, {"mask": np.ones((16, 16)), "record": ["q"]}, {},
     "not a valid input"),
    ({"sound_speed": 1500.0}, {"p0": np.ones((16, 16))}, {"mask": np.ones((16, 16))}, {"PMLSize": 9},
     "PML must be smaller"),
    ({"sound_speed": 1500.0}, {"p0": np.ones((16, 16))}, {"mask": np.ones((16, 16)), "record_start_index": 99}, {},
     "record_start_index"),
    ({"sound_speed": 1500.0}, {"p0": np.ones((16, 16))}, {"mask": 2 * np.ones((16, 16))}, {}, "binary grid"),
    ({"sound_speed": 1500.0}, {"p0": np.ones((16, 16))}, None, {"Smooth": [True, 1]}, "Boolean"),
    ({"sound_speed": 1500.0}, {"p0": np.ones((16, 16))}, None, {"NoSuchOption": 1}, "Unknown optional input"),
])
def test_setup_errors_mirror_reference(medium, source, sensor, opts, msg):
    g = kw.kWaveGrid(16, 1e-4, 16, 1e-4)
    g.setTime(10, 2e-8)
    with pytest.raises(KWaveInputError, match=msg):
        _prepare(2, g, medium, source, sensor, opts)


def test_time_varying_source_needs_explicit_time():
    g = kw.kWaveGrid(16, 1e-4, 16, 1e-4)
    pm = np.zeros((16, 16))
    pm[4, 4] = 1
    with pytest.raises(KWaveInputError, match="defined explicitly"):
        _prepare(2, g, {"sound_speed": 1500.0}, {"p": np.ones(5), "p_mask": pm}, None, {})


def test_labelled_source_rows():
    g = kw.kWaveGrid(16, 1e-4, 16, 1e-4)
    g.setTime(10, 2e-8)
    pm = np.zeros((16, 16))
    pm[2, 3] = 2
    pm[5, 3] = 1
    pm[7, 9] = 2
    P = _prepare(2, g, {"sound_speed": 1500.0}, {"p": np.ones((2, 5)), "p_mask": pm, "p_mode": "dirichlet"}, None,
                 {"PMLSize": 4})
    src = P.problem.p_source
    assert src.num_signals == 2 and src.num_points == 3
    assert list(_arr(src.signal_index, 3, np.uint64)) == [2, 1, 2]
    with pytest.raises(KWaveInputError, match="labelled"):
        _prepare(2, g, {"sound_speed": 1500.0}, {"p": np.ones((3, 5)), "p_mask": pm}, None, {"PMLSize": 4})


@pytest.mark.parametrize("shape", [(17, 12), (9, 11, 7), (64,)])
def test_find_is_matlab_find(shape):
    """find(mask) in column-major order, for C- and Fortran-ordered masks."""
    from kwave_b200.solver import _at, _find
    rng = np.random.default_rng(11)
    m = (rng.random(shape) < 0.3) * rng.integers(1, 4, shape)
    ref = np.flatnonzero(m.ravel(order="F"))
    for a in (m, np.asfortranarray(m)):
        assert np.array_equal(_find(a), ref)
        assert np.array_equal(_at(a, ref), m.ravel(order="F")[ref])


@pytest.mark.parametrize("shape", [(40, 36), (20, 22, 18), (41, 17)])
def test_cart_linear_weights(shape):
    """Barycentric weights of Cartesian points (CartInterp 'linear'): they are
    non-negative, sum to 1, reproduce every affine field exactly (true for
    any triangulation, so also for MATLAB's), and match the oracle's."""
    from kwave_b200.helpers import cartLinearWeights
    g, o = _grids(shape, 1e-4)
    rng = np.random.default_rng(4)
    dim = len(shape)
    half = np.array([(s // 2 - 1) * 1e-4 for s in shape])
    pts = (rng.random((dim, 50)) * 2 - 1) * half[:, None]
    pts[:, 0] = 0.0                                    # a grid node
    tri, bc = cartLinearWeights(shape, [1e-4] * dim, pts)
    assert bc.min() >= -1e-12 and np.allclose(bc.sum(axis=1), 1.0)
    coef = rng.standard_normal(dim + 1)
    grid = np.meshgrid(*[g.grid_vec(a) for a in range(dim)], indexing="ij")
    field = coef[0] + sum(coef[a + 1] * grid[a] for a in range(dim))
    interp = (field.ravel(order="F")[tri] * bc).sum(axis=1)
    exact = coef[0] + sum(coef[a + 1] * pts[a] for a in range(dim))
    assert np.allclose(interp, exact, rtol=0, atol=1e-12 * np.abs(coef).sum())
    assert np.isclose(bc[0].max(), 1.0)
    t2, b2 = ks.cart_linear(o, pts)
    assert np.array_equal(tri, t2) and np.allclose(bc, b2, rtol=0, atol=1e-15)
    with pytest.raises(ValueError, match="within the k-space grid"):
        cartLinearWeights(shape, [1e-4] * dim, pts + 1.0)


def test_layered_workload_recipe():
    """The large layered benchmark's inputs (built at 64^3): four layers
    along x at the recipe's speeds, rough interfaces of 3-cell RMS, B/A in
    5..9 per layer, one delayed burst per plane-source point (the element
    farthest from the focus fires first, delay 0) and every cell a sensor."""
    import bench
    rng = np.random.default_rng(0)
    h = bench.rough_surface(128, 96, rng)
    assert h.shape == (128, 96) and np.isclose(h.std(), 3.0) and abs(h.mean()) < 1.0
    w = bench.layered_workload(seed=3, N=64, Nt=60, pml=6, f0=2e6, cycles=3, focus=20, src=16, amp=1e5)
    med = w["medium"]
    assert set(np.unique(med["sound_speed"])) <= set(bench.LAYER_C)
    assert np.allclose(med["density"], 1000.0 + 0.6 * (med["sound_speed"] - 1500.0))
    assert med["BonA"].min() >= 5 and med["BonA"].max() <= 9 and med["alpha_power"] == 1.1
    # the first layer fills the x = 0 plane, the last the far plane
    assert np.all(med["sound_speed"][0] == bench.LAYER_C[0]) and np.all(med["sound_speed"][-1] == bench.LAYER_C[3])
    pm, sig = w["source"]["p_mask"], w["source"]["p"]
    assert pm.sum() == 16 * 16 and pm[6].sum() == 16 * 16          # every source point on the plane x = 6
    assert sig.shape == (256, w["src_len"]) and w["src_len"] <= w["Nt"]
    # corner elements are farthest from the focus: they start first (nonzero at sample 1)
    first = (np.abs(sig) > 0).argmax(axis=1)
    assert first.min() <= 1 and first[0] == first.min() and np.all(first >= 0)
    assert w["sensor"]["mask"].all() and w["sensor"]["record"] == ["p_max", "p_rms"]
    assert w["dt"] == pytest.approx(0.3 * 1e-4 / 2800.0)


def test_stream_to_disk_setup():
    """StreamToDisk (checkOptionalInputs.m:353-374, inputChecking.m:1369-1375):
    3-D only, p only; true means 200 steps; the series file is the
    reference's temp_sensor_data.bin."""
    g3 = kw.kWaveGrid(16, 1e-4, 16, 1e-4, 16, 1e-4)
    g3.setTime(10, 2e-8)
    med = {"sound_speed": 1500.0}
    src = {"p0": np.ones((16, 16, 16))}
    mask = np.zeros((16, 16, 16))
    mask[4, :, :] = 1
    P = _prepare(3, g3, med, src, {"mask": mask}, {"StreamToDisk": True, "PMLSize": 4})
    assert P.problem.stream_to_disk == 200 and P.problem.stream_to_disk_file == b"temp_sensor_data.bin"
    assert _prepare(3, g3, med, src, {"mask": mask}, {"StreamToDisk": 7, "PMLSize": 4}).problem.stream_to_disk == 7
    assert _prepare(3, g3, med, src, {"mask": mask}, {"PMLSize": 4}).problem.stream_to_disk == 0
    with pytest.raises(KWaveInputError, match="sensor.record"):
        _prepare(3, g3, med, src, {"mask": mask, "record": ["p", "p_max"]}, {"StreamToDisk": 5, "PMLSize": 4})
    g2 = kw.kWaveGrid(16, 1e-4, 16, 1e-4)
    g2.setTime(10, 2e-8)
    with pytest.raises(KWaveInputError, match="3D fluid"):
        _prepare(2, g2, med, {"p0": np.ones((16, 16))}, {"mask": np.ones((16, 16))}, {"StreamToDisk": True})

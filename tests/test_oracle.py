"""Pins of the FP64 oracle (CPU only).

The reference stores no golden vectors and its MATLAB cannot run here, so
the oracle is pinned against the known answers its own tests use:
closed-form homogeneous propagation (the exactness claim of
kspaceFirstOrder3D.m:23-25), the wavenumber formula (TestGrid.m:135-194),
analytic spectral derivatives (TestFourierCollocation.m:47-300), plane-wave
dimension invariance (TestAcousticSolver.m:49-316), PML interior
invariance (TestSplitFieldPML.m:74-106); plus the committed fixtures in
tests/golden/ (made by tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from oracle import kspace as ks

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _grid(shape, dx):
    args = []
    for s in shape:
        args += [s, dx]
    return ks.KWaveGrid(*args)


@pytest.mark.parametrize("shape", [(64, 48), (24, 20, 28), (45, 33)])
def test_homogeneous_lossless_is_exact(shape):
    """p(t) = IFFT(FFT(p0) cos(c |k| t)) for a homogeneous lossless medium
    without PML absorption (the k-space scheme is exact there)."""
    dx, c = 1e-4, 1500.0
    kg = _grid(shape, dx)
    kg.setTime(37, 0.3 * dx / c)
    rng = np.random.default_rng(1)
    p0 = np.zeros(shape)
    sl = tuple(slice(s // 2 - 3, s // 2 + 3) for s in shape)
    p0[sl] = rng.random(p0[sl].shape)
    out = ks.kspace_first_order(kg, {"sound_speed": c, "density": 1000.0}, {"p0": p0}, {"record": ["p_final"]},
                                PMLAlpha=0.0, Smooth=False)
    t = (kg.Nt - 1) * kg.dt
    exact = np.real(np.fft.ifftn(np.fft.fftn(p0) * np.fft.ifftshift(np.cos(c * kg.k * t))))
    assert ks.rel_l2(out["p_final"], exact) < 1e-12


def test_wavenumber_formula():
    """kx = 2 pi / dx * (-N/2 : N/2-1) / N (even) and the odd analogue."""
    for n, d in ((64, 1e-3), (63, 2e-4), (7, 0.5), (8, 0.25)):
        k = ks.make_dim(n, d)
        if n % 2 == 0:
            ref = 2 * np.pi / d * np.arange(-n // 2, n // 2) / n
        else:
            ref = 2 * np.pi / d * np.arange(-(n - 1) // 2, (n - 1) // 2 + 1) / n
        assert np.allclose(k, ref, rtol=1e-15, atol=0)
        assert k[n // 2] == 0.0


@pytest.mark.parametrize("shift", [1, -1, 0])
def test_spectral_derivative_of_periodic_function(shift):
    """d/dx sin(m x 2 pi / L) evaluated at the (staggered) grid points."""
    n, dx = 64, 1e-3
    kg = _grid((n, 8), dx)
    L = n * dx
    x = kg.vec(0)
    m = 5
    kx = 2 * np.pi * m / L
    f = np.repeat(np.sin(kx * x)[:, None], 8, axis=1)
    df = ks.spectral_derivative(f, kg, 0, shift)
    xs = x + shift * dx / 2
    exact = np.repeat((kx * np.cos(kx * xs))[:, None], 8, axis=1)
    assert np.max(np.abs(df - exact)) / kx < 1e-12


@pytest.mark.parametrize("absorb", [False, True])
def test_plane_wave_dimension_invariance(absorb):
    """A plane wave along x is the same in 2-D and 3-D when the lateral axes
    carry no PML (TestAcousticSolver.m:49-316)."""
    nax, nlat, dx, c = 96, 8, 1e-4, 1500.0
    dt = 0.25 * dx / c
    prof = np.exp(-((np.arange(nax) - 40.0) ** 2) / (3.0 ** 2))
    med = {"sound_speed": c, "density": 1000.0}
    if absorb:
        med.update(alpha_coeff=10.0, alpha_power=1.9)
    k2 = _grid((nax, nlat), dx)
    k2.setTime(60, dt)
    o2 = ks.kspace_first_order(k2, med, {"p0": np.repeat(prof[:, None], nlat, 1)}, {"record": ["p_final"]},
                               PMLSize=[10, 0], Smooth=False)["p_final"]
    k3 = _grid((nax, nlat, nlat), dx)
    k3.setTime(60, dt)
    o3 = ks.kspace_first_order(k3, med, {"p0": np.broadcast_to(prof[:, None, None], (nax, nlat, nlat)).copy()},
                               {"record": ["p_final"]}, PMLSize=[10, 0, 0], Smooth=False)["p_final"]
    for j in range(nlat):
        assert ks.rel_l2(o2[:, j], o2[:, 0]) < 1e-12
        assert ks.rel_l2(o3[:, j, j], o2[:, 0]) < 1e-10


def test_pml_leaves_interior_untouched():
    """Before the wave reaches the PML, the field with absorbing layers equals
    the field without them (TestSplitFieldPML.m:74-106)."""
    N, dx, c = 64, 1e-4, 1500.0
    kg = _grid((N, N), dx)
    kg.setTime(10, 0.3 * dx / c)
    p0 = np.zeros((N, N))
    p0[30:34, 30:34] = 1.0
    a = ks.kspace_first_order(kg, {"sound_speed": c, "density": 1000.0}, {"p0": p0}, {"record": ["p_final"]},
                              PMLSize=12, PMLAlpha=2.0, Smooth=False)["p_final"]
    b = ks.kspace_first_order(kg, {"sound_speed": c, "density": 1000.0}, {"p0": p0}, {"record": ["p_final"]},
                              PMLSize=12, PMLAlpha=0.0, Smooth=False)["p_final"]
    inner = (slice(20, 44), slice(20, 44))
    assert ks.rel_l2(a[inner], b[inner]) < 1e-6
    assert ks.rel_l2(a, b) > 0        # the layers do act at the edges


def test_auto_time_step():
    """makeTime: dt = CFL dx / c_max, Nt = floor(t_end / dt) + 1 with
    t_end = diagonal / c_min (kWaveGrid.m:612-664)."""
    kg = _grid((128, 128), 1e-4)
    Nt, dt = kg.makeTime(np.array([1500.0, 1800.0]), 0.3)
    assert dt == pytest.approx(0.3 * 1e-4 / 1800.0, rel=1e-15)
    assert Nt == int(np.floor(np.sqrt(2) * 128e-4 / 1500.0 / dt)) + 1


def test_golden_fixtures_reproduce():
    g = np.load(os.path.join(GOLDEN, "cfg1_small.npz"))
    N, dx = int(g["N"]), float(g["dx"])
    kg = _grid((N, N), dx)
    kg.setTime(int(g["Nt"]), float(g["dt"]))
    out = ks.kspace_first_order(kg, {"sound_speed": float(g["c"]), "density": 1000.0}, {"p0": g["p0"]},
                                {"mask": g["sensor_mask"]}, PMLSize=10, CartInterp="nearest")
    assert ks.rel_l2(out, g["p"]) < 1e-12

    g = np.load(os.path.join(GOLDEN, "time_reversal_2d.npz"))
    N, dx = int(g["N"]), float(g["dx"])
    kg = _grid((N, N), dx)
    kg.setTime(int(g["Nt"]), float(g["dt"]))
    p = ks.kspace_first_order(kg, {"sound_speed": float(g["c"]), "density": 1000.0}, {},
                              {"mask": g["sensor_mask"], "time_reversal_boundary_data": g["data"]}, PMLSize=8)
    assert ks.rel_l2(p, g["p_final"]) < 1e-12


def test_golden_absorbing_3d_reproduces():
    g = np.load(os.path.join(GOLDEN, "absorbing_3d.npz"))
    shape = tuple(int(v) for v in g["shape"])
    kg = _grid(shape, float(g["dx"]))
    kg.setTime(int(g["Nt"]), float(g["dt"]))
    med = {"sound_speed": g["c"], "density": g["rho"], "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
    out = ks.kspace_first_order(kg, med, {"p_mask": g["p_mask"], "p": g["sig"]},
                                {"mask": g["sensor_mask"], "record": ["p", "p_max", "p_final"]}, PMLSize=4)
    for k in ("p", "p_max", "p_final"):
        assert ks.rel_l2(out[k], g["out_" + k]) < 1e-12


def test_cart2grid_nearest_and_reorder():
    kg = _grid((32, 32), 1e-3)
    pts = ks.make_cart_circle(10e-3, 12)
    mask, order_index, reorder_index = ks.cart2grid(kg, pts)
    assert mask.sum() == 12
    # reorder_index lists, in find(mask) order, the Cartesian point of each cell
    idx = np.flatnonzero(mask.ravel(order="F"))
    for m, gi in enumerate(idx):
        x, y = np.unravel_index(gi, (32, 32), order="F")
        p = reorder_index[m] - 1
        assert round(pts[0, p] / 1e-3) + 16 == x
        assert round(pts[1, p] / 1e-3) + 16 == y
    # rows in find(mask) order carrying their Cartesian point number come
    # back in Cartesian order
    data = reorder_index[:, None] * np.ones((1, 3))
    back = ks.reorder_binary_sensor_data(data, reorder_index)
    assert np.array_equal(back[:, 0], np.arange(1, 13))


def test_plane_wave_intensity():
    """For a plane wave travelling along x, u = p / (rho c): the intensity
    the oracle forms from p and the unstaggered, dt/2-shifted velocity
    (kspaceFirstOrder_saveIntensity.m) is p^2 / (rho c) at every time step,
    its time average is <p^2> / (rho c), and the transverse intensity is 0."""
    N0, N1, dx, c, rho = 160, 16, 1e-4, 1500.0, 1000.0
    kg = ks.KWaveGrid(N0, dx, N1, dx)
    dt = 0.3 * dx / c
    kg.setTime(500, dt)
    pm = np.zeros((N0, N1))
    pm[30, :] = 1
    t = np.arange(500) * dt
    sig = np.sin(2 * np.pi * 1e6 * t) * np.exp(-((t - 3e-6) / 1e-6) ** 2)
    sm = np.zeros((N0, N1))
    sm[100, :] = 1
    out = ks.kspace_first_order(kg, {"sound_speed": c, "density": rho}, {"p_mask": pm, "p": sig[None, :]},
                                {"mask": sm, "record": ["p", "I", "I_avg"]}, PMLSize=[20, 0])
    p = out["p"]
    assert ks.rel_l2(out["Ix"], p ** 2 / (rho * c)) < 1e-4
    assert np.allclose(out["Ix_avg"], (p ** 2).mean(axis=1) / (rho * c), rtol=1e-5)
    assert np.abs(out["Iy"]).max() <= 1e-6 * np.abs(out["Ix"]).max()
    assert "ux_non_staggered" not in out


def test_gaussian_filter_passes_centre_frequency():
    """gaussianFilter.m keeps a tone at the centre frequency and attenuates
    one at twice the half-power bandwidth away by the Gaussian's value."""
    fs, f0, bw, N = 50e6, 2e6, 50.0, 1000
    t = np.arange(N) / fs
    sig = np.sin(2 * np.pi * f0 * t)[None, :]
    assert ks.rel_l2(ks.gaussian_filter(sig, fs, f0, bw), sig) < 1e-3
    off = f0 + bw / 100 * f0            # two half-widths away: gain exp(-4 ln 2) = 1/16
    sig2 = np.sin(2 * np.pi * off * t)[None, :]
    gain = np.abs(np.fft.rfft(ks.gaussian_filter(sig2, fs, f0, bw)[0])).max() / np.abs(np.fft.rfft(sig2[0])).max()
    assert abs(gain - 1 / 16) < 5e-3

"""Adjoint form: kw_adjoint_gradient against the FP64 discrete adjoint.

The oracle's adjoint (oracle/adjoint.py) is pinned by central finite
differences on the CPU (tests/test_oracle_adjoint.py).  Here the library's
gradient of J = 1/2 sum (p(sensor) - d)^2 with respect to the sound speed and
the density, computed from the FP32 loop with FP64 accumulation and sqrt(Nt)
checkpointing, must match it: relative L2 error <= 1e-3 over the grid (the
loop runs in FP32; the residual is the same array for both).  Every
checkpoint interval must give the same gradient.
"""
import numpy as np
import pytest

from cases import adjoint_problem

TOL = 1e-3


def _rel(a, b):
    return float(np.linalg.norm((np.asarray(a) - b).ravel()) / np.linalg.norm(np.ravel(b)))


def _grid(mod, shape, dx, Nt, dt):
    args = []
    for s in shape:
        args += [s, dx]
    g = (mod.kWaveGrid if hasattr(mod, "kWaveGrid") else mod.KWaveGrid)(*args)
    g.setTime(Nt, dt)
    return g


@pytest.mark.gpu
@pytest.mark.parametrize("shape,Nt", [((32, 28), 60), ((64, 64), 120), ((12, 14, 10), 25), ((32, 64, 48), 40),
                                      ((32, 48, 64), 40)])
def test_gradient_matches_oracle_adjoint(shape, Nt):
    import kwave_b200 as kw
    from oracle import adjoint as adj
    from oracle import kspace as ks
    shape, dx, Nt, dt, c, rho, pm, sig, sm = adjoint_problem(shape, Nt)
    dim = len(shape)
    medium = {"sound_speed": c, "density": rho, "sound_speed_ref": 1700.0}
    sim = kw.Simulation(dim, _grid(kw, shape, dx, Nt, dt), medium, {"p_mask": pm, "p": sig[None, :]},
                        {"mask": sm}, PMLSize=4, Smooth=False)
    y = sim.run()
    ops = adj.setup(_grid(ks, shape, dx, Nt, dt), c, rho, pm, sig, sm, pml_size=4, c_ref=1700.0)
    y64 = adj.forward(ops)
    assert ks.rel_l2(y, y64) < 1e-4
    rng = np.random.default_rng(3)
    d = 0.9 * y64 + 0.01 * np.abs(y64).max() * rng.standard_normal(y64.shape)
    r = y.astype(np.float64) - d
    gc, gr = sim.adjoint_gradient(r)
    rc, rr = adj.gradient(ops, r)
    ec, er = _rel(gc, rc), _rel(gr, rr)
    assert ec <= TOL and er <= TOL, "rel-L2 dJ/dc %.2e dJ/drho %.2e" % (ec, er)
    # checkpoint interval changes memory, not the result
    for K in (1, 7, Nt):
        gc2, gr2 = sim.adjoint_gradient(r, checkpoint_interval=K)
        assert np.array_equal(gc2, gc) and np.array_equal(gr2, gr), K
    # the plan still runs and its outputs are unchanged
    assert np.array_equal(sim.run(), y)
    sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("shape,Nt,K", [((32, 28), 60, 0), ((64, 64), 120, 11), ((12, 14, 10), 25, 4)])
def test_kept_checkpoints_give_the_same_gradient(shape, Nt, K):
    """kw_keep_checkpoints: the misfit's own run keeps the states the
    adjoint would recompute, so the gradient that follows skips its forward
    pass (fewer launches) and is bit-identical; an incomplete run or a reset
    discards them (the gradient then runs its own forward pass)."""
    import kwave_b200 as kw
    shape, dx, Nt, dt, c, rho, pm, sig, sm = adjoint_problem(shape, Nt)
    dim = len(shape)
    medium = {"sound_speed": c, "density": rho, "sound_speed_ref": 1700.0}
    with kw.Simulation(dim, _grid(kw, shape, dx, Nt, dt), medium, {"p_mask": pm, "p": sig[None, :]},
                       {"mask": sm}, PMLSize=4, Smooth=False) as sim:
        y = sim.run()
        r = 0.1 * y.astype(np.float64)
        gc, gr = sim.adjoint_gradient(r, checkpoint_interval=K)
        n0 = sim.launch_count()
        gc_again, _ = sim.adjoint_gradient(r, checkpoint_interval=K)
        plain_launches = sim.launch_count() - n0
        assert np.array_equal(gc_again, gc)
        sim.keep_checkpoints(True, K)
        assert np.array_equal(sim.run(), y)      # recording is unchanged
        n1 = sim.launch_count()
        gc2, gr2 = sim.adjoint_gradient(r, checkpoint_interval=K)
        kept_launches = sim.launch_count() - n1
        assert np.array_equal(gc2, gc) and np.array_equal(gr2, gr)
        assert kept_launches < plain_launches    # the forward pass was skipped
        # a partial run keeps nothing usable: the gradient recomputes, same result
        sim.reset()
        sim.step(Nt // 2)
        gc3, _ = sim.adjoint_gradient(r, checkpoint_interval=K)
        assert np.array_equal(gc3, gc)
        sim.keep_checkpoints(False)
        gc4, _ = sim.adjoint_gradient(r, checkpoint_interval=K)
        assert np.array_equal(gc4, gc)


@pytest.mark.gpu
def test_gradient_rejects_unsupported_media():
    import kwave_b200 as kw
    shape, dx, Nt, dt, c, rho, pm, sig, sm = adjoint_problem((32, 28), 20)
    medium = {"sound_speed": c, "density": rho, "alpha_coeff": 0.5, "alpha_power": 1.5}
    with kw.Simulation(2, _grid(kw, shape, dx, Nt, dt), medium, {"p_mask": pm, "p": sig[None, :]},
                       {"mask": sm}, PMLSize=4) as sim:
        y = sim.run()
        with pytest.raises(kw.KWaveError, match="lossless"):
            sim.adjoint_gradient(np.zeros_like(y))


@pytest.mark.gpu
def test_gradient_agrees_with_time_reversal_image():
    """The reference's own time-reversal run, fed the residual, back-propagates
    it; the classic image sum_t (2/c) dp/dt q of that field with the forward
    field points the same way as the exact adjoint gradient (cosine > 0.95
    inside a 64-element ring around a blob medium)."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import kwave_b200 as kw
    N, dx, Nt = 96, 1e-4, 600
    rng = np.random.default_rng(3)
    ax = np.arange(N) - N / 2
    c_true = np.full((N, N), 1500.0)
    for _ in range(3):
        cx, cy = rng.uniform(-20, 20, 2)
        sg = rng.uniform(4, 8)
        c_true += rng.uniform(-60, 100) * np.exp(-((ax[:, None] - cx) ** 2 + (ax[None, :] - cy) ** 2) / (2 * sg * sg))
    c0 = np.full((N, N), 1500.0)
    rho = np.full((N, N), 1000.0)
    dt = 0.3 * dx / 1800.0
    ring = np.zeros((N, N))
    for a in np.linspace(0, 2 * np.pi, 64, endpoint=False):
        ring[int(round(N / 2 + 38 * np.cos(a))), int(round(N / 2 + 38 * np.sin(a)))] = 1
    cells = np.flatnonzero(ring.ravel(order="F"))
    pm = np.zeros((N, N))
    pm[np.unravel_index(cells[0], (N, N), order="F")] = 1
    sig = 1e3 * bench.ricker(dt, Nt)

    def run(c):
        g = kw.kWaveGrid(N, dx, N, dx)
        g.setTime(Nt, dt)
        return kw.Simulation(2, g, {"sound_speed": c, "density": rho, "sound_speed_ref": 1800.0},
                             {"p_mask": pm, "p": sig[None, :]}, {"mask": ring}, PMLSize=10, Smooth=False)
    with run(c_true) as s:
        d = s.run().astype(np.float64)
    with run(c0) as s:
        r = s.run().astype(np.float64) - d
        g_adj, _ = s.adjoint_gradient(r, density=False)
    inside = (ax[:, None] ** 2 + ax[None, :] ** 2) < 30 ** 2
    cos = bench.tr_gradient_cosine(kw, c0, rho, (N, dx, N, dx), Nt, dt, pm, sig, ring, 1800.0, 10, r, g_adj, inside)
    assert cos > 0.95, cos

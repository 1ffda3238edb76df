"""Pins of the FP64 discrete adjoint (CPU only).

The reference has no adjoint, so the oracle's adjoint (oracle/adjoint.py) is
pinned in two ways: its step-by-step forward must reproduce the oracle's
restatement of kspaceFirstOrder2D/3D exactly, and its gradients of
J = 1/2 sum (p(sensor) - d)^2 with respect to the sound speed and the density
must match central finite differences of J.
"""
import numpy as np
import pytest

from cases import adjoint_problem
from oracle import adjoint as adj
from oracle import kspace as ks


def make_problem(shape, Nt):
    shape, dx, Nt, dt, c, rho, pm, sig, sm = adjoint_problem(shape, Nt)
    args = []
    for s in shape:
        args += [s, dx]
    kg = ks.KWaveGrid(*args)
    kg.setTime(Nt, dt)
    return kg, c, rho, pm, sig, sm


@pytest.mark.parametrize("shape,Nt", [((32, 28), 60), ((12, 14, 10), 25)])
def test_forward_matches_oracle_loop(shape, Nt):
    kg, c, rho, pm, sig, sm = make_problem(shape, Nt)
    ops = adj.setup(kg, c, rho, pm, sig, sm, pml_size=4, c_ref=1700.0)
    ref = ks.kspace_first_order(kg, {"sound_speed": c, "density": rho, "sound_speed_ref": 1700.0},
                                {"p_mask": pm, "p": sig[None, :]}, {"mask": sm}, PMLSize=4, Smooth=False)
    assert ks.rel_l2(adj.forward(ops), ref) < 1e-13


@pytest.mark.parametrize("shape,Nt", [((32, 28), 60), ((12, 14, 10), 25)])
def test_gradient_matches_central_differences(shape, Nt):
    kg, c, rho, pm, sig, sm = make_problem(shape, Nt)
    ops = adj.setup(kg, c, rho, pm, sig, sm, pml_size=4, c_ref=1700.0)
    rng = np.random.default_rng(5)
    y = adj.forward(ops)
    d = 0.9 * y + 0.01 * np.abs(y).max() * rng.standard_normal(y.shape)
    _, r = adj.misfit(ops, d)
    gc, gr = adj.gradient(ops, r)
    cells = np.argsort(np.abs(gc).ravel())[::-1][:2].tolist() + rng.integers(0, gc.size, 2).tolist()
    for k in cells:
        cell = np.unravel_index(k, shape)
        for name, base, g in (("c", c, gc), ("rho0", rho, gr)):
            h = 1e-3 * base[cell]
            plus, minus = base.copy(), base.copy()
            plus[cell] += h
            minus[cell] -= h
            key = "c" if name == "c" else "rho0"
            fd = (adj.misfit(ops, d, **{key: plus})[0] - adj.misfit(ops, d, **{key: minus})[0]) / (2 * h)
            assert abs(g[cell] - fd) <= 2e-4 * abs(fd) + 1e-9 * np.abs(g).max(), (name, cell, g[cell], fd)

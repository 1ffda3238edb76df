"""Generate the golden fixtures of the parity tests.

The reference (MATLAB) cannot run here, so the fixtures are outputs of the
FP64 oracle (oracle/kspace.py) on small seeded cases, which the oracle pins
to closed-form and recipe known answers (tests/test_oracle.py).  Run from the
repo root:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
from oracle import kspace as ks  # noqa: E402


def cfg1_small():
    """Config 1 recipe at 64^2 (disc p0, smoothed; 32-point Cartesian circle,
    nearest-neighbour; lossless homogeneous; t_end = 1.2 x diagonal / c)."""
    N, dx, c = 64, 1e-4, 1500.0
    kg = ks.KWaveGrid(N, dx, N, dx)
    t_end = 1.2 * np.sqrt(2) * N * dx / c
    kg.makeTime(c, 0.3, t_end)
    p0 = ks.make_disc(N, N, N // 2 + 1, N // 2 + 1, 5)
    sensor = {"mask": ks.make_cart_circle(20 * dx, 32)}
    out = ks.kspace_first_order(kg, {"sound_speed": c, "density": 1000.0}, {"p0": p0}, sensor,
                                PMLSize=10, PMLAlpha=2.0, CartInterp="nearest")
    return dict(kind="2d", N=N, dx=dx, c=c, Nt=kg.Nt, dt=kg.dt, p0=p0, sensor_mask=sensor["mask"], p=out)


def absorbing_3d():
    """3-D heterogeneous absorbing nonlinear medium with an additive plane source."""
    rng = np.random.default_rng(20240601)
    shape = (24, 20, 28)
    dx = 2e-4
    c = 1500.0 + 120.0 * rng.random(shape)
    rho = 1000.0 + 0.6 * (c - 1500.0)
    dt = 0.3 * dx / c.max()
    Nt = 40
    pm = np.zeros(shape)
    pm[4, 6:14, 8:20] = 1
    n = 12
    sig = 1e6 * np.sin(2 * np.pi * np.arange(n) / n) * np.hanning(n)
    mask = np.zeros(shape)
    mask[:, :, 14] = 1
    kg = ks.KWaveGrid(shape[0], dx, shape[1], dx, shape[2], dx)
    kg.setTime(Nt, dt)
    med = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
    out = ks.kspace_first_order(kg, med, {"p_mask": pm, "p": sig}, {"mask": mask, "record": ["p", "p_max", "p_final"]},
                                PMLSize=4)
    return dict(kind="3d", shape=np.array(shape), dx=dx, Nt=Nt, dt=dt, c=c, rho=rho, p_mask=pm, sig=sig,
                sensor_mask=mask, **{"out_" + k: v for k, v in out.items()})


def time_reversal_2d():
    """2-D time reversal of boundary data on two sensor lines."""
    N, dx, c = 48, 1e-4, 1500.0
    dt = 0.3 * dx / c
    Nt = 80
    mask = np.zeros((N, N))
    mask[6, :] = 1
    mask[41, :] = 1
    rng = np.random.default_rng(7)
    data = np.cumsum(rng.standard_normal((int(mask.sum()), Nt)), axis=1) * 1e-2
    kg = ks.KWaveGrid(N, dx, N, dx)
    kg.setTime(Nt, dt)
    p = ks.kspace_first_order(kg, {"sound_speed": c, "density": 1000.0}, {}, {"mask": mask,
                              "time_reversal_boundary_data": data}, PMLSize=8)
    return dict(kind="tr", N=N, dx=dx, c=c, Nt=Nt, dt=dt, sensor_mask=mask, data=data, p_final=p)


if __name__ == "__main__":
    for name, fn in (("cfg1_small", cfg1_small), ("absorbing_3d", absorbing_3d), ("time_reversal_2d", time_reversal_2d)):
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **fn())
        print("wrote", name)

"""kWaveGrid: the computational grid object passed to kspaceFirstOrder2D/3D.

Mirrors +kwave/+legacy/kWaveGrid.m (constructor 342-437, setTime 588-604,
makeTime 612-664, makeDim 779-797) for the properties the time loop uses.
Arrays follow MATLAB indexing: ``a[x, y, z]`` is ``a(x, y, z)``.
"""
from __future__ import annotations

import math

import numpy as np


def _make_dim(n: int, d: float) -> np.ndarray:
    """Wavenumbers of one axis in natural order with an exact zero at the DC
    index (kWaveGrid.m:779-797)."""
    if n % 2 == 0:
        frac = np.arange(-(n // 2), n // 2, dtype=np.float64) / n
    else:
        frac = np.arange(-((n - 1) // 2), (n - 1) // 2 + 1, dtype=np.float64) / n
    frac[n // 2] = 0.0
    return (2.0 * math.pi / d) * frac


class kWaveGrid:
    """``kWaveGrid(Nx, dx)``, ``kWaveGrid(Nx, dx, Ny, dy)`` or
    ``kWaveGrid(Nx, dx, Ny, dy, Nz, dz)``."""

    CFL_DEFAULT = 0.3

    def __init__(self, *args):
        if len(args) not in (2, 4, 6):
            raise ValueError("Incorrect number of input arguments.")
        ns = [int(args[i]) for i in range(0, len(args), 2)]
        ds = [float(args[i]) for i in range(1, len(args), 2)]
        if any(n < 1 for n in ns) or any(d <= 0 for d in ds):
            raise ValueError("grid sizes must be positive")
        self.dim = len(ns)
        self._n = ns + [1] * (3 - self.dim)
        self._d = ds + [0.0] * (3 - self.dim)
        self._kvec = [_make_dim(n, d) for n, d in zip(ns, ds)]
        self.Nt = None
        self.dt = None
        self.t_array = "auto"

    # sizes and spacings
    Nx = property(lambda s: s._n[0])
    Ny = property(lambda s: s._n[1])
    Nz = property(lambda s: s._n[2])
    dx = property(lambda s: s._d[0])
    dy = property(lambda s: s._d[1])
    dz = property(lambda s: s._d[2])

    @property
    def shape(self):
        return tuple(self._n[: self.dim])

    @property
    def spacing(self):
        return tuple(self._d[: self.dim])

    @property
    def total_grid_points(self):
        return int(np.prod(self.shape))

    def k_vec(self, axis):
        return self._kvec[axis]

    kx_vec = property(lambda s: s._kvec[0])
    ky_vec = property(lambda s: s._kvec[1] if s.dim > 1 else np.zeros(1))
    kz_vec = property(lambda s: s._kvec[2] if s.dim > 2 else np.zeros(1))

    @property
    def k(self):
        out = np.zeros(self.shape)
        for a in range(self.dim):
            shp = [1] * self.dim
            shp[a] = -1
            out = out + self._kvec[a].reshape(shp) ** 2
        return np.sqrt(out)

    @property
    def k_max(self):
        return min(float(np.max(np.abs(v))) for v in self._kvec)

    def grid_vec(self, axis):
        """x_vec / y_vec / z_vec (kWaveGrid.m:494-505)."""
        n, d = self._n[axis], self._d[axis]
        return n * d * self._kvec[axis] * d / (2.0 * math.pi)

    x_vec = property(lambda s: s.grid_vec(0))
    y_vec = property(lambda s: s.grid_vec(1))
    z_vec = property(lambda s: s.grid_vec(2))

    @property
    def size(self):
        return tuple(n * d for n, d in zip(self.shape, self.spacing))

    def setTime(self, Nt, dt):
        if round(Nt) != Nt or Nt <= 0:
            raise ValueError("Nt must be a positive integer.")
        if dt <= 0:
            raise ValueError("dt must be positive.")
        self.Nt, self.dt = int(Nt), float(dt)
        self.t_array = np.arange(self.Nt) * self.dt

    def makeTime(self, c, cfl=None, t_end=None):
        """dt from the CFL number and the fastest speed; Nt from the time to
        cross the grid diagonal at the slowest speed (kWaveGrid.m:612-664)."""
        cfl = self.CFL_DEFAULT if cfl is None else cfl
        c = np.asarray(c, dtype=np.float64)
        c_max, c_min = float(c.max()), float(c.min())
        if t_end is None:
            t_end = math.sqrt(sum(s * s for s in self.size)) / c_min
        dt = cfl * min(self.spacing) / c_max
        Nt = int(math.floor(t_end / dt)) + 1
        if math.floor(t_end / dt) != math.ceil(t_end / dt) and math.fmod(t_end, dt) == 0:
            Nt += 1
        self.setTime(Nt, dt)
        return self.t_array, self.dt

"""Input-building helpers of the k-Wave API that feed the time loop.

Host-side (NumPy, FP64) restatements of the reference's MATLAB helpers:
getWin.m (1-3-D windows, radial 'Rotation'), smooth.m (window filter in
k-space used for the default p0 smoothing), makeDisc.m / makeBall.m /
makeCircle-style masks via private/makePixelMap.m, makeCartCircle.m,
cart2grid.m (nearest grid point) and reorderBinarySensorData.m.
They run once before the loop, on the host, exactly where the reference runs
them (in MATLAB before the native hand-off).
"""
from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------------------
# getWin.m
# ---------------------------------------------------------------------------

def _cos_sum(n, N, coeffs):
    out = np.full(n.shape, coeffs[0], dtype=np.float64)
    for i, c in enumerate(coeffs[1:], start=1):
        out += (-1.0) ** i * c * np.cos(2.0 * math.pi * i * n / (N - 1))
    return out


def _win1(N, kind, param, symmetric):
    Ne = N if symmetric else N + 1
    n = np.arange(Ne, dtype=np.float64)
    if kind == "Blackman":
        a = 0.16 if param is None else float(param)
        w = _cos_sum(n, Ne, [(1.0 - a) / 2.0, 0.5, a / 2.0])
    elif kind == "Hanning":
        w = 0.5 - 0.5 * np.cos(2.0 * math.pi * n / (Ne - 1))
    elif kind == "Hamming":
        w = 0.54 - 0.46 * np.cos(2.0 * math.pi * n / (Ne - 1))
    elif kind == "Rectangular":
        w = np.ones(Ne)
    else:
        raise ValueError("Unknown window type: " + str(kind))
    return w[:N]


def getWin(N, kind, Rotation=False, Symmetric=True, Param=None):
    """Window of size N (1-3 dims).  ``Rotation`` makes a radially symmetric
    window by linear interpolation of a 1-D window (getWin.m:299-343)."""
    dims = np.atleast_1d(np.asarray(N, dtype=np.int64))
    sym = np.broadcast_to(np.atleast_1d(np.asarray(Symmetric, dtype=bool)), dims.shape)
    if dims.size == 1:
        return _win1(int(dims[0]), kind, Param, bool(sym[0]))
    ext = dims + (~sym).astype(np.int64)
    if Rotation:
        L = int(ext.max())
        lin = _win1(L, kind, Param, True)
        radius = (L - 1) / 2.0
        ll = np.linspace(-radius, radius, L)
        coords = np.meshgrid(*[np.linspace(-radius, radius, int(e)) for e in ext], indexing="ij")
        r = np.sqrt(sum(c * c for c in coords))
        r = np.minimum(r, radius)
        win = np.interp(r, ll, lin)
    else:
        win = _win1(int(ext[0]), kind, Param, True)
        for e in ext[1:]:
            win = np.multiply.outer(win, _win1(int(e), kind, Param, True))
    return win[tuple(slice(0, int(d)) for d in dims)]


def smooth(mat, restore_max=False, window_type="Blackman"):
    """smooth.m:110-137: multiply the spectrum by a radially symmetric window
    (symmetric for odd sizes so the DC gain is 1), optionally restoring the
    maximum magnitude."""
    mat = np.asarray(mat, dtype=np.float64)
    shape = [s for s in mat.shape if s != 1] or [mat.size]
    sym = [bool(s % 2) for s in shape]
    win = np.abs(getWin(shape, window_type, Rotation=True, Symmetric=sym)).reshape(mat.shape)
    out = np.real(np.fft.ifftn(np.fft.fftn(mat) * np.fft.ifftshift(win)))
    if restore_max:
        out *= np.max(np.abs(mat)) / np.max(np.abs(out))
    return out


# ---------------------------------------------------------------------------
# shapes (makeDisc.m, makeBall.m, makeCartCircle.m)
# ---------------------------------------------------------------------------

def _pixel_axis(n, shifted):
    # private/makePixelMap.m createPixelDim with 'single' origin
    if n % 2:
        return np.arange(-(n - 1) // 2, (n - 1) // 2 + 1)
    return np.arange(-n // 2 + 1, n // 2 + 1) if shifted else np.arange(-n // 2, n // 2)


def makeDisc(Nx, Ny, cx, cy, radius):
    """Binary disc of the given radius (grid points) centred at (cx, cy),
    1-based; a zero centre coordinate means the grid centre."""
    cx = int(round(cx)) if cx else Nx // 2 + 1
    cy = int(round(cy)) if cy else Ny // 2 + 1
    if not (1 <= cx <= Nx and 1 <= cy <= Ny):
        raise ValueError("Disc center must be within grid.")
    X, Y = np.meshgrid(_pixel_axis(Nx, True), _pixel_axis(Ny, True), indexing="ij")
    disc = (np.hypot(X, Y) <= radius).astype(np.float64)
    return np.roll(disc, (cx - math.ceil(Nx / 2), cy - math.ceil(Ny / 2)), axis=(0, 1))


def makeBall(Nx, Ny, Nz, cx, cy, cz, radius):
    """Ball of ones (makeBall.m, non-binary form)."""
    c = [int(round(v)) if v else n // 2 + 1 for v, n in ((cx, Nx), (cy, Ny), (cz, Nz))]
    X, Y, Z = np.meshgrid(np.arange(1, Nx + 1) - c[0], np.arange(1, Ny + 1) - c[1],
                          np.arange(1, Nz + 1) - c[2], indexing="ij")
    return (X * X + Y * Y + Z * Z <= radius * radius).astype(np.float64)


def makeCartCircle(radius, num_points, center_pos=(0.0, 0.0)):
    """2 x num_points Cartesian points on a full circle, starting at +pi/2
    and running clockwise in (x, y) (makeCartCircle.m)."""
    ang = math.pi / 2 + np.arange(num_points) * (2.0 * math.pi / num_points)
    pts = np.empty((2, num_points))
    pts[0] = radius * np.cos(ang) + center_pos[0]
    pts[1] = -radius * np.sin(ang) + center_pos[1]
    return pts


# ---------------------------------------------------------------------------
# cart2grid.m (nearest grid point) and the output reorder
# ---------------------------------------------------------------------------

def _round_half_away(v):
    return np.sign(v) * np.floor(np.abs(v) + 0.5)


def cart2grid(kgrid, cart_data):
    """Map Cartesian points to the nearest grid points.  Returns
    ``(mask, order_index, reorder_index)`` as cart2grid.m does (indices 1-based)."""
    cart = np.atleast_2d(np.asarray(cart_data, dtype=np.float64))
    subs = []
    for a in range(kgrid.dim):
        s = _round_half_away(cart[a] / kgrid.spacing[a]) + kgrid.shape[a] // 2 + 1
        if s.min() < 1 or s.max() > kgrid.shape[a]:
            raise ValueError("Cartesian points must lie within the grid defined by kgrid.")
        subs.append(s.astype(np.int64) - 1)
    grid = np.zeros(kgrid.shape)
    # later points overwrite earlier ones on the same cell, as the MATLAB loop does
    grid[tuple(subs)] = 0
    for p in range(cart.shape[1]):
        grid[tuple(s[p] for s in subs)] = p + 1
    flat = grid.ravel(order="F")
    reorder_index = flat[flat != 0].astype(np.int64)
    order_index = np.argsort(reorder_index, kind="stable") + 1
    return (grid != 0).astype(np.float64), order_index, reorder_index


def reorderBinarySensorData(data, reorder_index):
    """Rows sorted by reorder_index (reorderBinarySensorData.m)."""
    return np.asarray(data)[np.argsort(np.asarray(reorder_index), kind="stable")]


def cartLinearWeights(shape, spacing, cart_data):
    """Barycentric interpolation of Cartesian points on a grid of the given
    shape and spacing (grid origin at the centre, as kWaveGrid): returns the
    containing simplex as 0-based column-major grid indices (M x (D+1)) and
    the weights (M x (D+1)).

    The reference triangulates every grid point with delaunayTriangulation and
    locates the points in it (gridDataFast2D.m / gridDataFast3D.m).  On a
    regular grid the Delaunay triangulation is not unique (each cell's
    corners are co-circular), so this uses one documented choice, the Kuhn
    triangulation: inside the cell with lower corner b and fractional offsets
    f, the simplex walks the axes in decreasing order of f (ties: lower axis
    first) and the weights are (1 - f_(1), f_(1) - f_(2), ..., f_(D))."""
    cart = np.atleast_2d(np.asarray(cart_data, dtype=np.float64))
    dim = len(shape)
    M = cart.shape[1]
    frac = np.empty((dim, M))
    base = np.empty((dim, M), dtype=np.int64)
    for a in range(dim):
        n = int(shape[a])
        fi = cart[a] / spacing[a] + n // 2
        if np.any(fi < -1e-9) or np.any(fi > n - 1 + 1e-9):
            raise ValueError("Cartesian points must lie within the k-space grid defined by kgrid.")
        fi = np.clip(fi, 0, n - 1)
        b = np.minimum(np.floor(fi).astype(np.int64), n - 2)
        base[a] = b
        frac[a] = fi - b
    order = np.argsort(-frac, axis=0, kind="stable")
    fs = np.take_along_axis(frac, order, axis=0)
    tri = np.empty((M, dim + 1), dtype=np.int64)
    bc = np.empty((M, dim + 1))
    v = base.copy()
    cols = np.arange(M)
    tri[:, 0] = np.ravel_multi_index(tuple(v), tuple(shape), order="F")
    bc[:, 0] = 1.0 - fs[0]
    for k in range(dim):
        v[order[k], cols] += 1
        tri[:, k + 1] = np.ravel_multi_index(tuple(v), tuple(shape), order="F")
        bc[:, k + 1] = fs[k] - (fs[k + 1] if k + 1 < dim else 0.0)
    return tri, bc


class TransducerSource:
    """The transmit side of a kWaveTransducer used as ``source``: the
    properties the reference's setup reads for the loop's transducer hook
    (kspaceFirstOrder_inputChecking.m:1160-1209, kspaceFirstOrder3D.m:888-904).

    ``active_elements_mask``: grid of the active elements' points;
    ``delay_mask``: per-point beamforming delay in samples (0 = the first
    sample of ``input_signal``); ``input_signal``: the one drive series;
    ``transmit_apodization``: 'Rectangular' or anything else, in which case
    ``transmit_apodization_mask`` holds the per-point weights.  Building the
    masks from element geometry (kWaveTransducer itself) is outside this
    library.
    """

    def __init__(self, active_elements_mask, delay_mask, input_signal, transmit_apodization="Rectangular",
                 transmit_apodization_mask=None):
        self.active_elements_mask = active_elements_mask
        self.delay_mask = delay_mask
        self.input_signal = input_signal
        self.transmit_apodization = transmit_apodization
        self.transmit_apodization_mask = transmit_apodization_mask

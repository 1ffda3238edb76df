"""CPU oracle for the k-space first-order acoustic time loop -- TEST INFRASTRUCTURE ONLY.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference`` legs
of ``bench.py`` may import it.  The shipped library must never route through it.

It is an FP64 NumPy/SciPy restatement of k-Wave's legacy ``kspaceFirstOrder2D``
and ``kspaceFirstOrder3D`` (MATLAB), written from the reference's semantics:

* time loop, update order and p0 initial condition:
  ``+kwave/+legacy/kspaceFirstOrder3D.m:769-1208`` and
  ``+kwave/+legacy/kspaceFirstOrder2D.m:712-1044``;
* staggered density, PML and k-space operators:
  ``kspaceFirstOrder3D.m:585-661`` / ``kspaceFirstOrder2D.m:547-611``;
* input checking and defaults: ``+kwave/+legacy/private/kspaceFirstOrder_inputChecking.m``,
  ``kspaceFirstOrder_setDefaults.m``;
* absorption variables: ``private/kspaceFirstOrder_createAbsorptionVariables.m:29-101``;
* source scaling: ``private/kspaceFirstOrder_scaleSourceTerms.m``;
* sensor extraction: ``private/kspaceFirstOrder_extractSensorData.m:33-569``;
* helpers: ``kWaveGrid.m``, ``getPML.m``, ``getWin.m``, ``smooth.m``, ``makeDisc.m``,
  ``makeBall.m``, ``makeCartCircle.m``, ``cart2grid.m``, ``db2neper.m``,
  ``private/sinc.m``, ``private/makePixelMap.m``, ``expandMatrix.m``,
  ``reorderBinarySensorData.m``.

Parity status.  The reference is MATLAB and cannot run in this environment, and
its tests store no golden vectors.  The oracle is pinned against the
known-answer recipes that the reference's own tests use (analytic wavenumber
formula ``+kwave/+tests/+unit/TestGrid.m:135-194``; analytic spectral
derivatives ``TestFourierCollocation.m:47-300``; plane-wave dimension invariance
``TestAcousticSolver.m:49-316``; PML interior invariance ``TestSplitFieldPML.m:74-106``)
and against the closed-form homogeneous lossless solution the reference's
documentation claims the scheme reproduces (``kspaceFirstOrder3D.m:23-25``).
MATLAB's own ``fftn`` (FFTW inside the closed MATLAB runtime) is not
reproducible here, so bit-level agreement with MATLAB output is *parity
unpinned*; the FFT is ``scipy.fft`` in FP64.

Array convention: NumPy arrays are indexed ``a[x, y, z]`` exactly like MATLAB
``a(x, y, z)``; MATLAB linear indices (``find``) are column-major, i.e.
``np.flatnonzero(mask.ravel(order='F'))`` (0-based here).
"""
from __future__ import annotations

import math
import os
from types import SimpleNamespace

import numpy as np
import scipy.fft as sfft

_WORKERS = max(1, os.cpu_count() or 1)

# wall-clock seconds spent in the time loop by the last kspace_first_order call
LAST_LOOP_SECONDS = 0.0


def fftn(a):
    return sfft.fftn(a, workers=_WORKERS)


def ifftn(a):
    return sfft.ifftn(a, workers=_WORKERS)


# ---------------------------------------------------------------------------
# kWaveGrid (kWaveGrid.m:342-437 ctor, 588-664 setTime/makeTime, 779-797 makeDim)
# ---------------------------------------------------------------------------

def make_dim(n, d):
    """kWaveGrid.makeDim (kWaveGrid.m:779-797): FFT wavenumbers in natural order."""
    if n % 2 == 0:
        nx = np.arange(-n // 2, n // 2, dtype=np.float64) / n
    else:
        nx = np.arange(-(n - 1) // 2, (n - 1) // 2 + 1, dtype=np.float64) / n
    nx[n // 2] = 0.0
    return (2.0 * np.pi / d) * nx


class KWaveGrid:
    """Restatement of ``kWaveGrid`` for 1-3 dimensions (only what the loop uses)."""

    def __init__(self, Nx, dx, Ny=None, dy=None, Nz=None, dz=None):
        self.Nx, self.dx = int(Nx), float(dx)
        self.Ny, self.dy = (int(Ny), float(dy)) if Ny is not None else (1, 0.0)
        self.Nz, self.dz = (int(Nz), float(dz)) if Nz is not None else (1, 0.0)
        self.dim = 1 + (Ny is not None) + (Nz is not None)
        self.kx_vec = make_dim(self.Nx, self.dx)
        self.ky_vec = make_dim(self.Ny, self.dy) if self.dim >= 2 else np.zeros(1)
        self.kz_vec = make_dim(self.Nz, self.dz) if self.dim >= 3 else np.zeros(1)
        self.Nt = None
        self.dt = None

    @property
    def shape(self):
        return tuple([self.Nx, self.Ny, self.Nz][: self.dim])

    @property
    def spacing(self):
        return [self.dx, self.dy, self.dz][: self.dim]

    def k_vecs(self):
        return [self.kx_vec, self.ky_vec, self.kz_vec][: self.dim]

    @property
    def k(self):
        """|k| on the grid in natural (unshifted) order (kWaveGrid.m:399-433)."""
        vecs = self.k_vecs()
        k2 = np.zeros(self.shape)
        for i, v in enumerate(vecs):
            k2 = k2 + _axis(v, i, self.dim) ** 2
        return np.sqrt(k2)

    @property
    def k_max(self):
        return min(np.max(np.abs(v)) for v in self.k_vecs())

    def vec(self, axis):
        """x_vec / y_vec / z_vec (kWaveGrid.m:494-505): Ni*di*ki*di/(2 pi)."""
        n = [self.Nx, self.Ny, self.Nz][axis]
        d = self.spacing[axis]
        return n * d * self.k_vecs()[axis] * d / (2.0 * np.pi)

    @property
    def size(self):
        return [n * d for n, d in zip(self.shape, self.spacing)]

    def setTime(self, Nt, dt):
        if round(Nt) != Nt or Nt <= 0:
            raise ValueError("Nt must be a positive integer.")
        if dt <= 0:
            raise ValueError("dt must be positive.")
        self.Nt, self.dt = int(Nt), float(dt)

    def makeTime(self, c, cfl=0.3, t_end=None):
        c = np.asarray(c, dtype=np.float64)
        c_max, c_min = float(c.max()), float(c.min())
        if t_end is None:
            t_end = math.sqrt(sum(s * s for s in self.size)) / c_min
        self.dt = cfl * min(self.spacing) / c_max
        self.Nt = int(math.floor(t_end / self.dt)) + 1
        if math.floor(t_end / self.dt) != math.ceil(t_end / self.dt) and math.fmod(t_end, self.dt) == 0:
            self.Nt += 1
        return self.Nt, self.dt


def _axis(v, axis, dim):
    shape = [1] * dim
    shape[axis] = -1
    return np.reshape(v, shape)


# ---------------------------------------------------------------------------
# small helpers
# ---------------------------------------------------------------------------

def sinc(x):
    """private/sinc.m: sin(x)/x with sinc(0)=1."""
    x = np.asarray(x, dtype=np.float64)
    z = x == 0
    return np.sin(x + np.pi * z) / (x + z) + z


def db2neper(alpha, y=1.0):
    """db2neper.m:52."""
    return 100.0 * np.asarray(alpha, dtype=np.float64) * (1e-6 / (2 * np.pi)) ** y / (20.0 * np.log10(np.e))


def get_pml(n, d, dt, c, pml_size, pml_alpha, staggered):
    """getPML.m:52-87 (returned as a 1-D vector)."""
    pml = np.ones(n)
    if pml_size == 0:
        return pml
    x = np.arange(1, pml_size + 1, dtype=np.float64)
    xs = x + 0.5 if staggered else x
    left = pml_alpha * (c / d) * ((xs - pml_size - 1) / (0 - pml_size)) ** 4
    right = pml_alpha * (c / d) * (xs / pml_size) ** 4
    pml[:pml_size] = np.exp(-left * dt / 2)
    pml[n - pml_size:] = np.exp(-right * dt / 2)
    return pml


def ifftshift(a):
    return np.fft.ifftshift(a)


def expand_matrix(mat, sizes, edge_val=None):
    """expandMatrix.m: pad by ``sizes`` on both sides; edge replication when
    ``edge_val`` is None, else a constant."""
    pad = [(s, s) for s in sizes]
    if edge_val is None:
        return np.pad(mat, pad, mode="edge")
    return np.pad(mat, pad, mode="constant", constant_values=edge_val)


# ---------------------------------------------------------------------------
# windows and smoothing (getWin.m:104-365, smooth.m:72-137)
# ---------------------------------------------------------------------------

def _cosine_series(n, N, coeffs):
    s = coeffs[0] + 0 * n
    for i in range(1, len(coeffs)):
        s = s + (-1) ** i * coeffs[i] * np.cos(i * 2 * np.pi * n / (N - 1))
    return s


def get_win_1d(N, wtype, param=None, symmetric=True):
    N0 = N
    N = N + (0 if symmetric else 1)
    n = np.arange(N, dtype=np.float64)
    if wtype == "Blackman":
        a = 0.16 if param is None else param
        win = _cosine_series(n, N, [(1 - a) / 2, 0.5, a / 2])
    elif wtype == "Hanning":
        win = 0.5 - 0.5 * np.cos(2 * np.pi * n / (N - 1))
    elif wtype == "Hamming":
        win = 0.54 - 0.46 * np.cos(2 * np.pi * n / (N - 1))
    elif wtype == "Rectangular":
        win = np.ones(N)
    elif wtype == "Tukey":
        a = 0.5 if param is None else param
        win = np.ones(N)
        index = np.arange(0, (N - 1) * a / 2 + 1e-12 * 0 + np.finfo(float).eps * 0, 1.0)
        index = index[index <= (N - 1) * a / 2]
        pa = a * N
        win[: len(index)] = 0.5 * (1 + np.cos(2 * np.pi / pa * (index - pa / 2)))
        win[N - len(index):] = win[: len(index)][::-1]
    else:
        raise ValueError("window type not restated: " + wtype)
    return win[:N0]


def get_win(N, wtype="Blackman", rotation=False, symmetric=True, param=None):
    """getWin.m for 1-3 dimensions ('Rotation' radial windows via interp1)."""
    N = np.atleast_1d(np.asarray(N, dtype=int))
    sym = np.broadcast_to(np.atleast_1d(np.asarray(symmetric, dtype=bool)), N.shape)
    if len(N) == 1:
        return get_win_1d(int(N[0]), wtype, param, bool(sym[0]))
    Ne = N + (~sym).astype(int)
    if rotation:
        L = int(Ne.max())
        win_lin = get_win_1d(L, wtype, param, True)
        radius = (L - 1) / 2
        ll = np.linspace(-radius, radius, L)
        axes = [np.linspace(-radius, radius, int(n)) for n in Ne]
        grids = np.meshgrid(*axes, indexing="ij")
        r = np.sqrt(sum(g ** 2 for g in grids))
        r[r > radius] = radius
        win = np.interp(r, ll, win_lin)
    else:
        wins = [get_win_1d(int(n), wtype, param, True) for n in Ne]
        win = wins[0]
        for w in wins[1:]:
            win = np.multiply.outer(win, w)
    sl = tuple(slice(0, int(n)) for n in N)
    return win[sl]


def smooth(mat, restore_max=False, wtype="Blackman"):
    """smooth.m:110-137: radially symmetric window filter in k-space."""
    mat = np.asarray(mat, dtype=np.float64)
    shape = [s for s in mat.shape if s != 1] if mat.ndim > 1 else list(mat.shape)
    sym = [bool(s % 2) for s in shape]
    win = np.abs(get_win(shape, wtype, rotation=True, symmetric=sym))
    win = np.reshape(win, mat.shape)
    out = np.real(ifftn(fftn(mat) * ifftshift(win)))
    if restore_max:
        out = (np.max(np.abs(mat)) / np.max(np.abs(out))) * out
    return out


# ---------------------------------------------------------------------------
# geometry helpers (makeDisc.m, makeBall.m, makeCartCircle.m, cart2grid.m)
# ---------------------------------------------------------------------------

def _pixel_dim(n, shift):
    if n % 2 == 0:
        return np.arange(-n // 2, n // 2) if shift == 1 else np.arange(-n // 2 + 1, n // 2 + 1)
    return np.arange(-(n - 1) // 2, (n - 1) // 2 + 1)


def make_disc(Nx, Ny, cx, cy, radius):
    """makeDisc.m: binary disc, centre (cx, cy) 1-based (0 -> grid centre)."""
    cx = int(round(cx)) or Nx // 2 + 1
    cy = int(round(cy)) or Ny // 2 + 1
    rx, ry = np.meshgrid(_pixel_dim(Nx, 0), _pixel_dim(Ny, 0), indexing="ij")
    disc = (np.sqrt(rx ** 2 + ry ** 2) <= radius).astype(np.float64)
    return np.roll(disc, (cx - math.ceil(Nx / 2), cy - math.ceil(Ny / 2)), axis=(0, 1))


def make_ball(Nx, Ny, Nz, cx, cy, cz, radius):
    """makeBall.m (non-binary, ball of ones)."""
    cx = int(round(cx)) or Nx // 2 + 1
    cy = int(round(cy)) or Ny // 2 + 1
    cz = int(round(cz)) or Nz // 2 + 1
    X, Y, Z = np.meshgrid(np.arange(1, Nx + 1) - cx, np.arange(1, Ny + 1) - cy,
                          np.arange(1, Nz + 1) - cz, indexing="ij")
    return ((X ** 2 + Y ** 2 + Z ** 2) <= radius ** 2).astype(np.float64)


def make_cart_circle(radius, num_points, center=(0.0, 0.0)):
    """makeCartCircle.m (full circle)."""
    angles = np.arange(num_points + 1) * 2 * np.pi / num_points + np.pi / 2
    angles = angles[:-1]
    c = np.vstack([radius * np.cos(angles), radius * np.sin(-angles)])
    c[0] += center[0]
    c[1] += center[1]
    return c


def _mround(x):
    """MATLAB round (half away from zero)."""
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def cart2grid(kgrid, cart):
    """cart2grid.m:67-194 (nearest grid point).  Returns the binary mask,
    order_index and reorder_index (both 1-based like MATLAB)."""
    cart = np.atleast_2d(np.asarray(cart, dtype=np.float64))
    dim = kgrid.dim
    idx = []
    for a in range(dim):
        v = _mround(cart[a] / kgrid.spacing[a]) + kgrid.shape[a] // 2 + 1
        if v.max() > kgrid.shape[a] or v.min() < 1:
            raise ValueError("Cartesian points must lie within the grid defined by kgrid.")
        idx.append(v.astype(int) - 1)
    grid = np.zeros(kgrid.shape)
    for p in range(cart.shape[1]):
        grid[tuple(i[p] for i in idx)] = p + 1
    flat = grid.ravel(order="F")
    reorder_index = flat[flat != 0].astype(int)
    order_index = np.argsort(reorder_index, kind="stable") + 1
    mask = (grid != 0).astype(np.float64)
    return mask, order_index, reorder_index


def cart_linear(kgrid, cart):
    """Containing simplex (0-based column-major grid indices, M x (D+1)) and
    barycentric weights of Cartesian points in a Delaunay triangulation of
    the grid points, as gridDataFast2D.m / gridDataFast3D.m obtain with
    delaunayTriangulation + pointLocation.  A regular grid is a degenerate
    Delaunay case (each cell's corners are co-circular), so the triangulation
    is not unique and MATLAB's choice of cell diagonals is not documented.
    This restatement uses the Kuhn triangulation: in the cell with lower
    corner b and fractional offsets f, the simplex walks the axes in
    decreasing order of f (ties: lower axis first), with weights
    (1 - f_(1), f_(1) - f_(2), ..., f_(D))."""
    dim = kgrid.dim
    cart = np.atleast_2d(np.asarray(cart, dtype=np.float64))
    M = cart.shape[1]
    f = np.empty((dim, M))
    base = np.empty((dim, M), dtype=np.int64)
    for a in range(dim):
        n = kgrid.shape[a]
        fi = cart[a] / kgrid.spacing[a] + n // 2
        if np.any(fi < -1e-9) or np.any(fi > n - 1 + 1e-9):
            raise ValueError("Cartesian points must lie within the k-space grid defined by kgrid.")
        fi = np.clip(fi, 0, n - 1)
        b = np.minimum(np.floor(fi).astype(np.int64), n - 2)
        base[a] = b
        f[a] = fi - b
    order = np.argsort(-f, axis=0, kind="stable")
    fs = np.take_along_axis(f, order, axis=0)
    tri = np.empty((M, dim + 1), dtype=np.int64)
    bc = np.empty((M, dim + 1))
    v = base.copy()
    cols = np.arange(M)
    tri[:, 0] = np.ravel_multi_index(tuple(v), kgrid.shape, order="F")
    bc[:, 0] = 1.0 - fs[0]
    for k in range(dim):
        v[order[k], cols] += 1
        tri[:, k + 1] = np.ravel_multi_index(tuple(v), kgrid.shape, order="F")
        bc[:, k + 1] = fs[k] - (fs[k + 1] if k + 1 < dim else 0.0)
    return tri, bc


def reorder_binary_sensor_data(data, reorder_index):
    """reorderBinarySensorData.m: sort rows by reorder_index."""
    order = np.argsort(reorder_index, kind="stable")
    return data[order]


def fourier_shift(data, shift):
    """Shift data along its last axis by `shift` samples with the Fourier
    interpolant (fourierShift.m): real(ifft(ifftshift(exp(i k shift)) fft(data)))
    with k = 2 pi (-N/2 .. N/2-1) / N (odd N: -(N-1)/2 .. (N-1)/2), k at
    index floor(N/2) (0-based) set to zero."""
    data = np.asarray(data, dtype=np.float64)
    N = data.shape[-1]
    if N % 2 == 0:
        k = 2 * np.pi * np.arange(-N // 2, N // 2) / N
    else:
        k = 2 * np.pi * np.arange(-(N - 1) // 2, (N - 1) // 2 + 1) / N
    k[N // 2] = 0.0
    return np.real(np.fft.ifft(np.fft.ifftshift(np.exp(1j * k * shift)) * np.fft.fft(data, axis=-1), axis=-1))


def gaussian_filter(signal, fs, freq, bandwidth):
    """gaussianFilter.m: each row of signal filtered in frequency by
    max(G(f - freq), G(f + freq)), G a unit-height Gaussian whose FWHM is
    bandwidth % of freq."""
    signal = np.asarray(signal, dtype=np.float64)
    N = signal.shape[-1]
    if N % 2 == 0:
        f = np.arange(-N // 2, N // 2) * fs / N
    else:
        f = np.arange(-(N - 1) // 2, (N - 1) // 2 + 1) * fs / N
    var = (bandwidth / 100.0 * freq / (2 * np.sqrt(2 * np.log(2)))) ** 2
    g = np.maximum(np.exp(-(f - freq) ** 2 / (2 * var)), np.exp(-(f + freq) ** 2 / (2 * var)))
    spec = np.fft.fftshift(np.fft.fft(signal, axis=-1), axes=-1)
    return np.real(np.fft.ifft(np.fft.ifftshift(g * spec, axes=-1), axis=-1))


def tone_burst_hann(sample_freq, signal_freq, num_cycles):
    """A sine tone burst of ``num_cycles`` cycles sampled at ``sample_freq``,
    windowed by getWin(N, 'Hanning') (toneBurst.m:102-180 time axis)."""
    dt = 1.0 / sample_freq
    tone_length = num_cycles / signal_freq
    t = np.arange(0.0, tone_length + dt * 1e-9, dt)
    t = t[t <= tone_length + 1e-15]
    burst = np.sin(2 * np.pi * signal_freq * t)
    return burst * get_win_1d(len(burst), "Hanning")


# ---------------------------------------------------------------------------
# the solver
# ---------------------------------------------------------------------------


# ---------------------------------------------------------------------------
# Array backends of the time loop.  The set-up always runs in NumPy; the loop
# runs on NumPy (the default) or, as a fast FP64 oracle for full-size checks,
# on torch.float64 tensors (CPU or CUDA, torch.fft).  Both execute the same
# statements in the same order; only the array library differs.  Flat
# indices handed to a backend are C-order (row-major) indices of arrays
# indexed a[x, y, z], converted once from MATLAB's column-major ones.
# ---------------------------------------------------------------------------

class _NumpyBackend:
    """``single``: the loop in FP32 / complex64 (scipy.fft keeps single
    precision), the FP32 variant of the CPU baseline."""
    name = "numpy"

    def __init__(self, single=False):
        self.f = np.float32 if single else np.float64
        self.c = np.complex64 if single else np.complex128

    def put(self, a):
        if isinstance(a, np.ndarray) and a.ndim > 0 and a.dtype.kind in "fc":
            return a.astype(self.c if a.dtype.kind == "c" else self.f, copy=False)
        return a

    def fftn(self, a):
        return fftn(a)

    def ifftn(self, a):
        return ifftn(a)

    def fft(self, a, axis):
        return np.fft.fft(a, axis=axis)

    def ifft(self, a, axis):
        return np.fft.ifft(a, axis=axis)

    real = staticmethod(np.real)
    maximum = staticmethod(np.maximum)
    minimum = staticmethod(np.minimum)
    sqrt = staticmethod(np.sqrt)

    def zeros(self, shape, complex_=False):
        return np.zeros(shape, dtype=self.c if complex_ else self.f)

    def full(self, v, shape):
        return np.array(np.broadcast_to(v, shape), dtype=self.f)

    def copy(self, a):
        return a.copy()

    def take(self, field, idx):
        return np.ascontiguousarray(field).reshape(-1)[idx]

    def scatter_set(self, field, idx, vals):
        f = np.array(field, dtype=self.f, copy=True)
        f.reshape(-1)[idx] = vals
        return f

    def scatter_add(self, field, idx, vals):
        f = np.array(field, dtype=self.f, copy=True)
        f.reshape(-1)[idx] += vals
        return f

    def numpy(self, a):
        return np.asarray(a)


class _TorchBackend:
    """The loop on torch.float64 / complex128 tensors (``device``: "cpu" or "cuda")."""
    name = "torch"

    def __init__(self, device):
        import torch
        self.t = torch
        self.device = torch.device(device)

    def put(self, a):
        if a is None:
            return None
        if isinstance(a, (int, float, complex)):
            return a
        a = np.asarray(a)
        if a.ndim == 0 or a.size == 1 and a.ndim == 0:
            return complex(a) if np.iscomplexobj(a) else float(a)
        if a.dtype.kind in "iu":
            return self.t.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=self.device)
        dt = self.t.complex128 if np.iscomplexobj(a) else self.t.float64
        return self.t.as_tensor(np.ascontiguousarray(a), dtype=dt, device=self.device)

    def fftn(self, a):
        return self.t.fft.fftn(a)

    def ifftn(self, a):
        return self.t.fft.ifftn(a)

    def fft(self, a, axis):
        return self.t.fft.fft(a, dim=axis)

    def ifft(self, a, axis):
        return self.t.fft.ifft(a, dim=axis)

    def real(self, a):
        return a.real

    def maximum(self, a, b):
        return self.t.maximum(a, b)

    def minimum(self, a, b):
        return self.t.minimum(a, b)

    def sqrt(self, a):
        return self.t.sqrt(a)

    def zeros(self, shape, complex_=False):
        return self.t.zeros(shape, dtype=self.t.complex128 if complex_ else self.t.float64, device=self.device)

    def full(self, v, shape):
        if isinstance(v, self.t.Tensor):
            return v.expand(shape).clone()
        return self.t.full(shape, float(v), dtype=self.t.float64, device=self.device)

    def copy(self, a):
        return a.clone()

    def take(self, field, idx):
        return field.reshape(-1)[idx]

    def scatter_set(self, field, idx, vals):
        f = field.clone()
        f.view(-1)[idx] = vals
        return f

    def scatter_add(self, field, idx, vals):
        f = field.clone()
        f.view(-1)[idx] += vals
        return f

    def numpy(self, a):
        if isinstance(a, self.t.Tensor):
            return a.detach().cpu().numpy()
        return np.asarray(a)


def _backend(device, single=False):
    return _NumpyBackend(single) if device is None else _TorchBackend(device)


def _f2c(idx, shape):
    """MATLAB column-major linear indices -> C-order flat indices of a[x, y, z]."""
    idx = np.asarray(idx, dtype=np.int64)
    return np.ravel_multi_index(np.unravel_index(idx, shape, order="F"), shape).astype(np.int64)


RECORD_FLAGS = ("p", "p_max", "p_min", "p_rms", "p_max_all", "p_min_all", "p_final",
                "u", "u_max", "u_min", "u_rms", "u_max_all", "u_min_all", "u_final",
                "u_non_staggered", "I", "I_avg")


def _get(obj, name, default=None):
    if obj is None:
        return default
    if isinstance(obj, dict):
        return obj.get(name, default)
    return getattr(obj, name, default)


def _has(obj, name):
    return _get(obj, name, None) is not None


def kspace_first_order(kgrid, medium, source, sensor, **opts):
    """Restatement of ``kspaceFirstOrder2D`` / ``kspaceFirstOrder3D``.

    ``medium``/``source``/``sensor`` are dicts (or namespaces) with the MATLAB
    field names.  Options use the MATLAB names: PMLSize, PMLAlpha, PMLInside,
    Smooth, UsekSpace, UseSG, CartInterp.  Returns what the MATLAB function
    returns: the ``p`` matrix (M x Nt) when ``sensor.record`` is absent, the
    ``p_final`` array in time-reversal mode, otherwise a dict of outputs.

    ``StepCallback`` (not a reference option) is called as f(t, p) with the
    pressure field after every time step t, for tests that need the field
    history.  ``Device`` (not a reference option) runs the loop on
    torch.float64 tensors on that device ("cpu" or "cuda") instead of NumPy:
    the fast FP64 oracle of the full-size checks.  ``Single`` (not a
    reference option, NumPy only) runs the loop in FP32: the reference's
    ``DataCast = 'single'``, used as the FP32 CPU baseline.
    """
    step_callback = opts.pop("StepCallback", None)
    device = opts.pop("Device", None)
    single = bool(opts.pop("Single", False))
    dim = kgrid.dim
    if dim not in (2, 3):
        raise ValueError("only 2D and 3D are restated")
    # ---- defaults (setDefaults.m:151-170) ----
    pml_default = 20 if dim == 2 else 10
    pml_size = opts.get("PMLSize", pml_default)
    pml_size = [int(v) for v in np.broadcast_to(np.atleast_1d(pml_size), (dim,))]
    pml_alpha = [float(v) for v in np.broadcast_to(np.atleast_1d(opts.get("PMLAlpha", 2.0)), (dim,))]
    pml_inside = bool(opts.get("PMLInside", True))
    smooth_opt = opts.get("Smooth", [True, False, False])
    smooth_opt = list(np.broadcast_to(np.atleast_1d(smooth_opt), (3,)))
    use_kspace = bool(opts.get("UsekSpace", True))
    use_sg = bool(opts.get("UseSG", True))
    cart_interp = opts.get("CartInterp", "linear")

    c = np.asarray(_get(medium, "sound_speed"), dtype=np.float64)
    if _has(medium, "density"):
        rho0 = np.asarray(_get(medium, "density"), dtype=np.float64)
    else:
        rho0 = np.asarray(1.0)

    # ---- equation of state (inputChecking.m:148-281) ----
    alpha_mode = _get(medium, "alpha_mode")
    if _has(medium, "alpha_coeff") or _has(medium, "alpha_power"):
        if alpha_mode == "stokes":
            eos = "stokes"
            alpha_power = 2.0
        else:
            eos = "absorbing"
            alpha_power = float(_get(medium, "alpha_power"))
            if not (0 <= alpha_power < 3):
                raise ValueError("medium.alpha_power must be a real number between 0 and 3.")
            if alpha_power == 1 and alpha_mode != "no_dispersion":
                raise ValueError("alpha_power = 1 needs alpha_mode = 'no_dispersion'")
        alpha_coeff = np.asarray(_get(medium, "alpha_coeff"), dtype=np.float64)
    else:
        eos = "lossless"
    nonlinear = _has(medium, "BonA")
    BonA = np.asarray(_get(medium, "BonA"), dtype=np.float64) if nonlinear else None
    alpha_filter = None
    if eos == "absorbing" and _has(medium, "alpha_filter"):
        alpha_filter = np.asarray(_get(medium, "alpha_filter"), dtype=np.float64)

    # c_ref (setSoundSpeedRef.m:30-49)
    cref_opt = _get(medium, "sound_speed_ref")
    if cref_opt is None or cref_opt == "max":
        c_ref = float(c.max())
    elif cref_opt == "min":
        c_ref = float(c.min())
    elif cref_opt == "mean":
        c_ref = float(c.mean())
    else:
        c_ref = float(cref_opt)

    # ---- sensor (inputChecking.m:288-672) ----
    use_sensor = sensor is not None
    time_rev = use_sensor and _has(sensor, "time_reversal_boundary_data")
    record = set()
    record_given = use_sensor and _has(sensor, "record")
    if record_given:
        for r in _get(sensor, "record"):
            if r not in RECORD_FLAGS:
                raise ValueError("'%s' is not a valid input for sensor.record." % r)
        record = set(_get(sensor, "record"))
    elif use_sensor and not time_rev:
        record = {"p"}
    if time_rev:
        record = set()
    rec_user = set(record)
    if record & {"I", "I_avg"}:
        # intensity needs the pressure and the unstaggered velocity series
        # (createStorageVariables.m:89-148, 309)
        record |= {"p", "u_non_staggered"}
    needs_mask = bool(record & {"p", "p_max", "p_min", "p_rms", "u", "u_non_staggered",
                                "u_max", "u_min", "u_rms", "I", "I_avg"})
    blank_sensor = use_sensor and not needs_mask and not time_rev
    record_start = int(_mround(_get(sensor, "record_start_index", 1))) if use_sensor else 1
    reorder_index = None
    mask = None
    cart_points = None
    cuboids = None
    if use_sensor and not blank_sensor:
        m = np.asarray(_get(sensor, "mask"), dtype=np.float64)
        if m.shape == kgrid.shape:
            mask = m
        elif m.ndim == 2 and m.shape[0] == 2 * dim:
            # cuboid corners [x1, y1, (z1,) x2, y2, (z2)] per column, 1-based
            # (inputChecking.m:517-575)
            if np.any(np.mod(m, 1) != 0):
                raise ValueError("sensor.mask cuboid corner indices must be integers.")
            if np.any(m[dim:] - m[:dim] < 0):
                raise ValueError("sensor.mask cuboid corners must be defined with x2 => x1, etc.")
            if np.any(m < 1) or any(np.any(m[[a, a + dim]] > kgrid.shape[a]) for a in range(dim)):
                raise ValueError("sensor.mask cuboid corners must be within the grid.")
            cuboids = m.astype(np.int64)
        elif m.ndim == 2 and m.shape[0] == dim:
            if cart_interp == "linear" and not time_rev:
                # recorded by barycentric interpolation (createStorageVariables.m:376-400)
                cart_points = m
            else:
                mask, order_index, reorder_index = cart2grid(kgrid, m)
        else:
            raise ValueError("sensor.mask shape not understood")

    # ---- source (inputChecking.m:713-1220) ----
    p0 = _get(source, "p0")
    source_p0 = p0 is not None and np.any(np.asarray(p0) != 0)
    if source_p0:
        p0 = np.asarray(p0, dtype=np.float64)
    source_p = 0
    p_freq_ref = u_freq_ref = None
    if _has(source, "p"):
        sp = np.atleast_2d(np.asarray(_get(source, "p"), dtype=np.float64))
        p_mask = np.asarray(_get(source, "p_mask"))
        p_mode = _get(source, "p_mode", "additive")
        p_freq_ref = _get(source, "p_frequency_ref")
        if p_freq_ref is not None:
            # inputChecking.m:820-836: the k-space correction as a function of w
            p_mode = "additive-no-correction"
        source_p = sp.shape[1]
        if source_p0:
            raise ValueError("source.p0 and source.p can't be defined in the same simulation.")
    u_comps = ["ux", "uy", "uz"][:dim]
    source_u = [0] * dim
    su = [None] * dim
    if any(_has(source, n) for n in u_comps) or _has(source, "u_mask"):
        u_mask = np.asarray(_get(source, "u_mask"))
        u_mode = _get(source, "u_mode", "additive")
        u_freq_ref = _get(source, "u_frequency_ref")
        if u_freq_ref is not None:
            # inputChecking.m:923-939
            u_mode = "additive-no-correction"
        for i, n in enumerate(u_comps):
            if _has(source, n):
                su[i] = np.atleast_2d(np.asarray(_get(source, n), dtype=np.float64))
                source_u[i] = su[i].shape[1]

    # transducer source (inputChecking.m:1160-1209)
    tr_src = None
    if _has(source, "active_elements_mask") and _has(source, "input_signal"):
        ta = _get(source, "transmit_apodization", "Rectangular")
        tr_src = dict(mask=np.asarray(_get(source, "active_elements_mask"), dtype=np.float64),
                      delay=np.asarray(_get(source, "delay_mask"), dtype=np.float64),
                      apod=None if (isinstance(ta, str) and ta == "Rectangular")
                      else np.asarray(_get(source, "transmit_apodization_mask"), dtype=np.float64),
                      sig=np.asarray(_get(source, "input_signal"), dtype=np.float64).ravel())

    # ---- time (inputChecking.m:1227-1268) ----
    if kgrid.Nt is None:
        if time_rev or source_p or any(source_u):
            raise ValueError("kgrid.t_array (Nt and dt) must be defined explicitly")
        kgrid.makeTime(c, 0.3)
    Nt, dt = kgrid.Nt, kgrid.dt

    # ---- smoothing (inputChecking.m:1501-1544, 1574-1604) ----
    if source_p0 and smooth_opt[0]:
        p0 = smooth(p0, True)
    if smooth_opt[1] and c.ndim == dim and c.size > 1:
        c = smooth(c)
    if smooth_opt[2] and rho0.ndim == dim and rho0.size > 1:
        rho0 = smooth(rho0)

    # ---- PMLInside = false (expandGridMatrices.m) ----
    if not pml_inside:
        kg = KWaveGrid(*sum(([kgrid.shape[a] + 2 * pml_size[a], kgrid.spacing[a]] for a in range(dim)), []))
        kg.setTime(Nt, dt)
        kgrid = kg
        if c.size > 1:
            c = expand_matrix(c, pml_size)
        if rho0.size > 1:
            rho0 = expand_matrix(rho0, pml_size)
        if eos != "lossless" and alpha_coeff.size > 1:
            alpha_coeff = expand_matrix(alpha_coeff, pml_size)
        if nonlinear and BonA.size > 1:
            BonA = expand_matrix(BonA, pml_size)
        if alpha_filter is not None:
            alpha_filter = expand_matrix(alpha_filter, pml_size, 0)
        if source_p0:
            p0 = expand_matrix(p0, pml_size, 0)
        if source_p:
            p_mask = expand_matrix(p_mask, pml_size, 0)
        if any(source_u):
            u_mask = expand_matrix(u_mask, pml_size, 0)
        if tr_src is not None:
            for key in ("mask", "delay") + (("apod",) if tr_src["apod"] is not None else ()):
                tr_src[key] = expand_matrix(tr_src[key], pml_size, 0)
        if mask is not None:
            mask = expand_matrix(mask, pml_size, 0)
        if cuboids is not None:
            cuboids = cuboids + np.array(pml_size * 2, dtype=np.int64)[:, None]
        inside = [slice(pml_size[a], kgrid.shape[a] - pml_size[a]) for a in range(dim)]
    else:
        inside = [slice(0, kgrid.shape[a]) for a in range(dim)]
    shape = kgrid.shape

    def find(m):
        return np.flatnonzero(np.asarray(m).ravel(order="F") != 0)

    sensor_interp = cart_linear(kgrid, cart_points) if cart_points is not None else None

    sensor_idx = find(mask) if mask is not None else None
    if cuboids is not None:
        # concatenation of every cuboid's find() (inputChecking.m:1610-1633)
        parts = []
        for ci in range(cuboids.shape[1]):
            tm = np.zeros(shape)
            tm[tuple(slice(cuboids[a, ci] - 1, cuboids[a + dim, ci]) for a in range(dim))] = 1
            parts.append(find(tm))
        sensor_idx = np.concatenate(parts)

    # source indices / labels
    def sig_index(msk, nrows):
        pos = find(msk)
        vals = np.asarray(msk).ravel(order="F")[pos]
        uniq = np.unique(msk)
        if uniq.size <= 2 and uniq.sum() == 1:
            labelled = False
            sig = np.arange(pos.size) if nrows > 1 else np.zeros(pos.size, dtype=int)
        else:
            labelled = True
            sig = vals.astype(int) - 1
        return pos, sig, labelled

    if source_p:
        p_pos, p_sig, _ = sig_index(p_mask, sp.shape[0])
    if any(source_u):
        nrows = max(s.shape[0] for s in su if s is not None)
        u_pos, u_sig, _ = sig_index(u_mask, nrows)

    # ---- absorption (createAbsorptionVariables.m:29-101) ----
    kmag = kgrid.k
    if eos == "absorbing":
        a_np = db2neper(alpha_coeff, alpha_power)
        if alpha_mode != "no_absorption":
            with np.errstate(divide="ignore"):
                nabla1 = kmag ** (alpha_power - 2)
            nabla1[np.isinf(nabla1)] = 0
            nabla1 = ifftshift(nabla1)
            tau = -2 * a_np * c ** (alpha_power - 1)
        else:
            nabla1, tau = 0.0, 0.0
        if alpha_mode != "no_dispersion":
            with np.errstate(divide="ignore"):
                nabla2 = kmag ** (alpha_power - 1)
            nabla2[np.isinf(nabla2)] = 0
            nabla2 = ifftshift(nabla2)
            eta = 2 * a_np * c ** alpha_power * np.tan(np.pi * alpha_power / 2)
        else:
            nabla2, eta = 0.0, 0.0
        if alpha_filter is not None:
            # createAbsorptionVariables.m:56-76: filter in natural order
            nabla1 = np.fft.ifftshift(np.fft.fftshift(np.broadcast_to(nabla1, shape)) * alpha_filter)
            nabla2 = np.fft.ifftshift(np.fft.fftshift(np.broadcast_to(nabla2, shape)) * alpha_filter)
        if _has(medium, "alpha_sign"):
            sgn = np.asarray(_get(medium, "alpha_sign"), dtype=np.float64)
            tau = np.sign(sgn[0]) * tau
            eta = np.sign(sgn[1]) * eta
    elif eos == "stokes":
        a_np = db2neper(alpha_coeff, 2)
        tau = -2 * a_np * c
        if _has(medium, "alpha_sign"):
            tau = np.sign(np.asarray(_get(medium, "alpha_sign"))[0]) * tau

    c0 = c
    # c0 in column-major (find) order, for the per-point source scaling
    c0f = c0.ravel(order="F") if c0.size > 1 else None
    # ---- source scaling (scaleSourceTerms.m) ----
    if source_p:
        sp = sp.copy()
        if p_freq_ref is not None:
            # scaleSourceTerms.m:43-45
            sp = sp * np.cos(2 * np.pi * float(p_freq_ref) * dt / 2)
        if p_mode == "dirichlet":
            if c0.size == 1:
                sp = sp / (dim * c0 ** 2)
            else:
                for r in range(sp.shape[0]):
                    sp[r] = sp[r] / (dim * c0f[p_pos[r]] ** 2)
        else:
            if c0.size == 1:
                sp = sp * (2 * dt / (dim * c0 * kgrid.dx))
            else:
                for r in range(sp.shape[0]):
                    sp[r] = sp[r] * (2 * dt / (dim * c0f[p_pos[r]] * kgrid.dx))
    if any(source_u) and u_freq_ref is not None:
        # scaleSourceTerms.m:272-282
        su = [None if v is None else v * np.cos(2 * np.pi * float(u_freq_ref) * dt / 2) for v in su]
    if any(source_u) and u_mode != "dirichlet":
        for i in range(dim):
            if su[i] is None:
                continue
            su[i] = su[i].copy()
            d = kgrid.spacing[i] if i > 0 else kgrid.dx
            if c0.size == 1:
                su[i] = su[i] * (2 * c0 * dt / d)
            else:
                for r in range(su[i].shape[0]):
                    su[i][r] = su[i][r] * (2 * c0f[u_pos[r]] * dt / d)

    # transducer drive: points, delays and apodization in find() order, the
    # signal scaled by 2 c0 dt / dx with c0 averaged over the points
    # (scaleSourceTerms.m:377-390); active while t <= length - max(delay)
    if tr_src is not None:
        tr_pos = find(tr_src["mask"])
        tr_delay = np.rint(tr_src["delay"].ravel(order="F")[tr_pos]).astype(np.int64)
        tr_apod = np.ones(tr_pos.size) if tr_src["apod"] is None else tr_src["apod"].ravel(order="F")[tr_pos]
        cmean = float(c0) if c0.size == 1 else float(np.mean(c0f[tr_pos]))
        tr_sig = tr_src["sig"] * (2 * cmean * dt / kgrid.dx)
        tr_steps = tr_sig.size - int(tr_delay.max())
    else:
        tr_steps = 0

    # ---- staggered density (kspaceFirstOrder3D.m:585-607) ----
    rho_sg_inv = []
    for a in range(dim):
        if rho0.ndim == dim and rho0.size > 1 and use_sg:
            r = rho0.copy()
            sl_lo = [slice(None)] * dim
            sl_hi = [slice(None)] * dim
            sl_lo[a] = slice(0, shape[a] - 1)
            sl_hi[a] = slice(1, shape[a])
            r[tuple(sl_lo)] = 0.5 * (rho0[tuple(sl_lo)] + rho0[tuple(sl_hi)])
            rho_sg_inv.append(1.0 / r)
        else:
            rho_sg_inv.append(1.0 / rho0)

    # ---- PML and k-space operators (kspaceFirstOrder3D.m:619-661) ----
    pml = []
    pml_sg = []
    for a in range(dim):
        pml.append(_axis(get_pml(shape[a], kgrid.spacing[a], dt, c_ref, pml_size[a], pml_alpha[a], False), a, dim))
        pml_sg.append(_axis(get_pml(shape[a], kgrid.spacing[a], dt, c_ref, pml_size[a], pml_alpha[a], use_sg), a, dim))
    dd_pos, dd_neg = [], []
    for a, kv in enumerate(kgrid.k_vecs()):
        d = kgrid.spacing[a]
        if use_sg:
            pos = ifftshift(1j * kv * np.exp(1j * kv * d / 2))
            neg = ifftshift(1j * kv * np.exp(-1j * kv * d / 2))
        else:
            pos = ifftshift(1j * kv)
            neg = ifftshift(1j * kv)
        dd_pos.append(_axis(pos, a, dim))
        dd_neg.append(_axis(neg, a, dim))
    if use_kspace:
        kappa = ifftshift(sinc(c_ref * kmag * dt / 2))
        source_kappa = ifftshift(np.cos(c_ref * kmag * dt / 2))
    else:
        kappa = 1.0
        source_kappa = 1.0

    # ---- storage (createStorageVariables.m) ----
    xp = _backend(device, single)
    X = xp.put
    num_rec = Nt - record_start + 1
    out = {}
    M = sensor_idx.size if sensor_idx is not None else (cart_points.shape[1] if cart_points is not None else 0)
    if "p" in record:
        out["p"] = xp.zeros((M, num_rec))
    if "p_rms" in record:
        out["p_rms"] = xp.zeros(M)
    if "u" in record:
        for i in range(dim):
            out[u_comps[i]] = xp.zeros((M, num_rec))
    if "u_non_staggered" in record:
        for i in range(dim):
            out[u_comps[i] + "_non_staggered"] = xp.zeros((M, num_rec))
    if "u_rms" in record:
        for i in range(dim):
            out[u_comps[i] + "_rms"] = xp.zeros(M)
    shift_neg = None
    if "u_non_staggered" in record:
        shift_neg = []
        for a, kv in enumerate(kgrid.k_vecs()):
            s = ifftshift(np.exp(-1j * kv * kgrid.spacing[a] / 2)) if use_sg else np.ones(shape[a])
            shift_neg.append(X(_axis(s, a, dim)))

    # ---- time reversal data ----
    if time_rev:
        trd = np.atleast_2d(np.asarray(_get(sensor, "time_reversal_boundary_data"), dtype=np.float64))
        if reorder_index is not None:
            # inputChecking.m:640-648: rows re-sorted into find(mask) order
            trd = trd[np.argsort(order_index, kind="stable")]
        trd = X(np.ascontiguousarray(trd[:, ::-1]))
        index_end = Nt - 1
    else:
        index_end = Nt

    # ---- loop operands on the backend ----
    sidx = X(_f2c(sensor_idx, shape)) if sensor_idx is not None else None
    if sensor_interp is not None:
        tri_c = X(_f2c(sensor_interp[0].ravel(order="C"), shape).reshape(sensor_interp[0].shape))
        bc_x = X(sensor_interp[1])

    def gather_s(field):
        """the recorded value at every sensor point (extractSensorData.m:63-100, 301-352)"""
        if sensor_interp is None:
            return xp.take(field, sidx)
        return (xp.take(field, tri_c) * bc_x).sum(1)

    if source_p:
        p_pos_x, p_sig_x, sp_x = X(_f2c(p_pos, shape)), X(p_sig), X(sp)
    if tr_steps > 0:
        tr_pos_x, tr_delay_x, tr_apod_x, tr_sig_x = X(_f2c(tr_pos, shape)), X(tr_delay), X(tr_apod), X(tr_sig)
    if any(source_u):
        u_pos_x, u_sig_x = X(_f2c(u_pos, shape)), X(u_sig)
        su_x = [X(v) for v in su]
        u_row0 = X(np.zeros_like(u_sig))
    pml, pml_sg = [X(v) for v in pml], [X(v) for v in pml_sg]
    rho_sg_inv = [X(v) for v in rho_sg_inv]
    dd_pos, dd_neg = [X(v) for v in dd_pos], [X(v) for v in dd_neg]
    kappa, source_kappa = X(kappa), X(source_kappa)
    if eos == "absorbing":
        nabla1, nabla2, tau, eta = X(nabla1), X(nabla2), X(tau), X(eta)
    elif eos == "stokes":
        tau = X(tau)
    rho0_x = X(rho0)
    BonA_x = X(BonA) if nonlinear else None
    if source_p0:
        p0_x = X(p0)

    # ---- loop ----
    p = xp.zeros(shape)
    rho = [xp.zeros(shape) for _ in range(dim)]
    u = [xp.zeros(shape) for _ in range(dim)]
    p_k = xp.zeros(shape, complex_=True)
    c2 = X(c0 ** 2)

    import time as _time
    _t0 = _time.perf_counter()
    for t in range(1, index_end + 1):
        if time_rev:
            p = xp.scatter_set(p, sidx, trd[:, t - 1])
            p_k = xp.fftn(p)
            rmod = p / (dim * c2) if dim == 3 else 0.5 * p / c2
            rmod = xp.full(rmod, shape)
            for i in range(dim):
                rho[i] = xp.scatter_set(rho[i], sidx, xp.take(rmod, sidx))

        # momentum (kspaceFirstOrder3D.m:792-803)
        for i in range(dim):
            u[i] = pml_sg[i] * (pml_sg[i] * u[i] - dt * rho_sg_inv[i] * xp.real(xp.ifftn(dd_pos[i] * kappa * p_k)))

        # velocity sources (kspaceFirstOrder3D.m:806-886)
        for i in range(dim):
            if source_u[i] >= t:
                rows = u_sig_x if su[i].shape[0] > 1 else u_row0
                vals = su_x[i][rows, t - 1]
                if u_mode == "dirichlet":
                    u[i] = xp.scatter_set(u[i], u_pos_x, vals)
                elif u_mode == "additive":
                    smat = xp.scatter_set(xp.zeros(shape), u_pos_x, vals)
                    u[i] = u[i] + xp.real(xp.ifftn(source_kappa * xp.fftn(smat)))
                else:
                    u[i] = xp.scatter_add(u[i], u_pos_x, vals)

        # transducer source (kspaceFirstOrder3D.m:888-904)
        if tr_steps >= t:
            u[0] = xp.scatter_add(u[0], tr_pos_x, tr_apod_x * tr_sig_x[tr_delay_x + (t - 1)])

        # divergence (kspaceFirstOrder3D.m:907-909)
        du = [xp.real(xp.ifftn(dd_neg[i] * kappa * xp.fftn(u[i]))) for i in range(dim)]

        # mass conservation (kspaceFirstOrder3D.m:912-927)
        if not nonlinear:
            for i in range(dim):
                rho[i] = pml[i] * (pml[i] * rho[i] - dt * rho0_x * du[i])
        else:
            r0pr = 2 * sum(rho) + rho0_x
            for i in range(dim):
                rho[i] = pml[i] * (pml[i] * rho[i] - dt * r0pr * du[i])

        # pressure sources (kspaceFirstOrder3D.m:930-962)
        if source_p >= t:
            vals = sp_x[p_sig_x, t - 1]
            if p_mode == "dirichlet":
                for i in range(dim):
                    rho[i] = xp.scatter_set(rho[i], p_pos_x, vals)
            elif p_mode == "additive":
                smat = xp.scatter_set(xp.zeros(shape), p_pos_x, vals)
                smat = xp.real(xp.ifftn(source_kappa * xp.fftn(smat)))
                for i in range(dim):
                    rho[i] = rho[i] + smat
            else:
                for i in range(dim):
                    rho[i] = xp.scatter_add(rho[i], p_pos_x, vals)

        # equation of state (kspaceFirstOrder3D.m:965-1019)
        srho = sum(rho)
        sdu = sum(du)
        if eos == "lossless":
            p = c2 * srho
        elif eos == "absorbing":
            p = c2 * (srho + tau * xp.real(xp.ifftn(nabla1 * xp.fftn(rho0_x * sdu)))
                      - eta * xp.real(xp.ifftn(nabla2 * xp.fftn(srho))))
        else:
            p = c2 * (srho + tau * rho0_x * sdu)
        if nonlinear:
            p = p + c2 * BonA_x * srho ** 2 / (2 * rho0_x)
        p = xp.full(p, shape)

        # p0 initial condition (kspaceFirstOrder3D.m:1023-1037)
        if t == 1 and source_p0:
            p = xp.copy(p0_x)
            for i in range(dim):
                rho[i] = xp.full(p0_x / (dim * c2), shape)
            pk0 = xp.fftn(p)
            for i in range(dim):
                u[i] = dt * rho_sg_inv[i] * xp.real(xp.ifftn(dd_pos[i] * kappa * pk0)) / 2
                u[i] = xp.full(u[i], shape)

        p_k = xp.fftn(p)
        if step_callback is not None:
            step_callback(t, p)

        # sensors (extractSensorData.m)
        if use_sensor and not time_rev and t >= record_start:
            fi = t - record_start + 1
            if sensor_idx is not None or sensor_interp is not None:
                ps = gather_s(p)
                if "p" in record:
                    out["p"][:, fi - 1] = ps
                if "p_max" in record:
                    out["p_max"] = xp.copy(ps) if fi == 1 else xp.maximum(out["p_max"], ps)
                if "p_min" in record:
                    out["p_min"] = xp.copy(ps) if fi == 1 else xp.minimum(out["p_min"], ps)
                if "p_rms" in record:
                    out["p_rms"] = xp.sqrt((out["p_rms"] ** 2 * (fi - 1) + ps ** 2) / fi)
                for i in range(dim):
                    us = gather_s(u[i])
                    n = u_comps[i]
                    if "u" in record:
                        out[n][:, fi - 1] = us
                    if "u_max" in record:
                        out[n + "_max"] = xp.copy(us) if fi == 1 else xp.maximum(out[n + "_max"], us)
                    if "u_min" in record:
                        out[n + "_min"] = xp.copy(us) if fi == 1 else xp.minimum(out[n + "_min"], us)
                    if "u_rms" in record:
                        out[n + "_rms"] = xp.sqrt((out[n + "_rms"] ** 2 * (fi - 1) + us ** 2) / fi)
                    if "u_non_staggered" in record:
                        ush = xp.real(xp.ifft(shift_neg[i] * xp.fft(u[i], i), i))
                        out[n + "_non_staggered"][:, fi - 1] = gather_s(ush)
            ins = tuple(inside)
            if "p_max_all" in record:
                out["p_max_all"] = xp.copy(p[ins]) if fi == 1 else xp.maximum(out["p_max_all"], p[ins])
            if "p_min_all" in record:
                out["p_min_all"] = xp.copy(p[ins]) if fi == 1 else xp.minimum(out["p_min_all"], p[ins])
            for i in range(dim):
                n = u_comps[i]
                if "u_max_all" in record:
                    out[n + "_max_all"] = xp.copy(u[i][ins]) if fi == 1 else xp.maximum(out[n + "_max_all"], u[i][ins])
                if "u_min_all" in record:
                    out[n + "_min_all"] = xp.copy(u[i][ins]) if fi == 1 else xp.minimum(out[n + "_min_all"], u[i][ins])

    global LAST_LOOP_SECONDS
    LAST_LOOP_SECONDS = _time.perf_counter() - _t0
    if time_rev:
        p = xp.scatter_set(p, sidx, trd[:, index_end])
        record.add("p_final")
    ins = tuple(inside)
    if "p_final" in record:
        out["p_final"] = xp.copy(p[ins])
    if "u_final" in record:
        for i in range(dim):
            out[u_comps[i] + "_final"] = xp.copy(u[i][ins])
    out = {k: np.array(xp.numpy(v), dtype=np.float64) for k, v in out.items()}

    # intensity (kspaceFirstOrder_saveIntensity.m): u_non_staggered shifted
    # forward in time by dt/2, times p; I_avg is its time average
    if use_sensor and not time_rev and rec_user & {"I", "I_avg"}:
        for i in range(dim):
            n = u_comps[i]
            inten = out["p"] * fourier_shift(out[n + "_non_staggered"], 0.5)
            if "I" in rec_user:
                out["I" + n[1:]] = inten
            if "I_avg" in rec_user:
                out["I" + n[1:] + "_avg"] = inten.mean(axis=-1)
        if "u_non_staggered" not in rec_user:
            for i in range(dim):
                del out[u_comps[i] + "_non_staggered"]
        if "p" not in rec_user:
            del out["p"]

    # Cartesian nearest-neighbour reorder (reorderCartData.m)
    if reorder_index is not None and not time_rev:
        for key in list(out.keys()):
            if key.endswith("_all") or key.endswith("_final"):
                continue
            out[key] = reorder_binary_sensor_data(out[key], reorder_index)

    # sensor frequency response (kspaceFirstOrder3D.m:1345-1348)
    if use_sensor and not time_rev and _has(sensor, "frequency_response") and "p" in out:
        fr = np.asarray(_get(sensor, "frequency_response"), dtype=np.float64).ravel()
        out["p"] = gaussian_filter(out["p"], 1.0 / dt, fr[0], fr[1])

    if cuboids is not None and not time_rev:
        out = _reorder_cuboids(out, cuboids, dim)

    if not use_sensor:
        return None
    if time_rev:
        return out["p_final"]
    if not record_given and cuboids is None:
        return out["p"]
    return out


def _reorder_cuboids(out, cuboids, dim):
    """kspaceFirstOrder_reorderCuboidCorners.m: one dict per cuboid, its
    rows of every sensor output reshaped to [X, Y, (Z,) T] (column-major);
    the _final and _all outputs go to the first cuboid only."""
    res = []
    start = 0
    for ci in range(cuboids.shape[1]):
        size = tuple(int(cuboids[a + dim, ci] - cuboids[a, ci] + 1) for a in range(dim))
        n = int(np.prod(size))
        d = {}
        for k, v in out.items():
            if k.endswith("_all") or k.endswith("_final"):
                if ci == 0:
                    d[k] = v
            elif v.ndim == 2:
                d[k] = v[start:start + n].reshape(size + (v.shape[1],), order="F")
            else:
                d[k] = v[start:start + n].reshape(size, order="F")
        res.append(d)
        start += n
    return res


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


def spectral_derivative(f, kgrid, axis, shift=0):
    """real(ifft(i k exp(shift * i k d / 2) fft(f))) along one axis: the
    staggered derivative operators of kspaceFirstOrder3D.m:629-650
    (shift = +1: ddx_k_shift_pos, -1: ddx_k_shift_neg, 0: unstaggered)."""
    kv = kgrid.k_vecs()[axis]
    d = kgrid.spacing[axis]
    op = ifftshift(1j * kv * np.exp(shift * 1j * kv * d / 2))
    op = _axis(op, axis, f.ndim)
    return np.real(np.fft.ifft(op * np.fft.fft(f, axis=axis), axis=axis))

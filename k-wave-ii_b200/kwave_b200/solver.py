"""kspaceFirstOrder2D / kspaceFirstOrder3D on the B200 library.

The Python side plays the role MATLAB plays in the reference's native
hand-off (+kwave/+legacy/kspaceFirstOrder3DC.m:530-546): it runs the setup of
+kwave/+legacy/private/kspaceFirstOrder_inputChecking.m -- option parsing,
equation-of-state selection, reference sound speed, sensor and source
parsing, p0 smoothing, PML expansion, find(mask) indices, source scaling and
the staggered density interpolation of kspaceFirstOrder3D.m:585-607 -- and
hands the resulting variable set (private/kspaceFirstOrder_saveToDisk.m) to
the C ABI.  The time loop itself runs only on the GPU; if the library is
missing the call raises.

Inputs follow the MATLAB API: ``medium``, ``source`` and ``sensor`` are
structs given as dicts or attribute objects with the MATLAB field names, and
the optional inputs use the MATLAB names (``PMLSize=...``, ``Smooth=...``).
Arrays are indexed ``a[x, y, z]`` like MATLAB ``a(x, y, z)``.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _abi
from .helpers import cart2grid, cartLinearWeights, reorderBinarySensorData, smooth
from .kgrid import kWaveGrid

RECORD_FLAGS = ("p", "p_max", "p_min", "p_rms", "p_max_all", "p_min_all", "p_final",
                "u", "u_max", "u_min", "u_rms", "u_max_all", "u_min_all", "u_final",
                "u_non_staggered", "I", "I_avg")

# optional inputs (private/kspaceFirstOrder_checkOptionalInputs.m:35-481)
_KNOWN_OPTIONS = {
    "CartInterp", "CreateLog", "DataCast", "DataRecast", "DisplayMask", "LogScale", "MeshPlot",
    "MovieArgs", "MovieName", "MovieType", "MovieProfile", "PlotFreq", "PlotLayout", "PlotPML",
    "PlotScale", "PlotSim", "PMLAlpha", "PMLInside", "PMLSize", "RecordMovie", "ScaleSourceTerms",
    "Smooth", "UsekSpace", "UseSG", "StreamToDisk", "SaveToDisk", "SaveToDiskExit",
    "HDFCompressionLevel", "MultiAxialPMLRatio", "PMLRange", "RadialSymmetry", "UseFD", "DeviceNum",
}
# kspaceFirstOrder_setDefaults.m:181, 197
STREAM_TO_DISK_STEPS_DEF = 200
STREAM_TO_DISK_FILENAME = "temp_sensor_data.bin"
_DATA_CASTS = {"off", "double", "single", "gsingle", "gdouble", "GPUsingle", "GPUdouble",
               "gpuArray-single", "gpuArray-double"}


class KWaveInputError(ValueError):
    """Input rejected during setup (the reference raises MATLAB error(...))."""


def _field(obj, name, default=None):
    if obj is None:
        return default
    if isinstance(obj, dict):
        return obj.get(name, default)
    return getattr(obj, name, default)


def _has(obj, name):
    return _field(obj, name) is not None


def _pick(values, dim):
    """x, y, z values chosen as v(1), v(ceil((end+1)/2)), v(end) from a 1..dim
    element input (checkOptionalInputs.m:257-330)."""
    v = list(np.atleast_1d(values))
    if len(v) > dim:
        raise KWaveInputError("Optional input must be a 1 or %d element array." % dim)
    if dim == 2:
        return [v[0], v[-1]]
    return [v[0], v[int(math.ceil((len(v) + 1) / 2)) - 1], v[-1]]


# Full-grid host passes (masks, FP32 conversion, reductions) run over slabs
# of the first axis in a few threads: NumPy releases the GIL inside them.
_POOL = None
_PAR_MIN = 1 << 20


def _pool():
    global _POOL
    if _POOL is None:
        import concurrent.futures
        _POOL = concurrent.futures.ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)))
    return _POOL


def _slabs(a):
    n0 = a.shape[0]
    k = max(1, min(n0, 4 * _pool()._max_workers))
    edges = np.linspace(0, n0, k + 1).astype(int)
    return [slice(int(lo), int(hi)) for lo, hi in zip(edges[:-1], edges[1:]) if hi > lo]


def _par(fn, a, combine):
    """combine([fn(a[s]) for slabs s]) with the slabs in parallel (small arrays inline)."""
    a = np.asarray(a)
    if a.ndim == 0 or a.size < _PAR_MIN:
        return combine([fn(a)])
    return combine(list(_pool().map(lambda s: fn(a[s]), _slabs(a))))


def _any(fn, a):
    return _par(lambda x: bool(np.any(fn(x))), a, any)


def _find(mask):
    """MATLAB find(mask ~= 0): 0-based column-major indices, increasing.

    Found in the array's own memory order and sorted, so no column-major
    copy of the grid is made."""
    m = np.asarray(mask)
    if m.ndim < 2:
        return np.flatnonzero(m)
    if m.size >= _PAR_MIN:
        stride = m.size // m.shape[0]
        nz = np.concatenate(list(_pool().map(lambda s: np.flatnonzero(m[s] != 0) + s.start * stride, _slabs(m))))
    else:
        nz = np.flatnonzero(m)
    f = np.ravel_multi_index(np.unravel_index(nz, m.shape), m.shape, order="F")
    f.sort()
    return f


def _at(a, fidx):
    """Values of grid array a at 0-based column-major linear indices."""
    a = np.asarray(a)
    return a[np.unravel_index(fidx, a.shape, order="F")]


def _grid32(a):
    """A grid-sized array as FP32 in row-major (C) order, the layout the
    library transposes on the device (KW_ROW_MAJOR)."""
    a = np.asarray(a)
    if a.ndim == 0 or a.size < _PAR_MIN or (a.dtype == np.float32 and a.flags.c_contiguous):
        return np.ascontiguousarray(a, dtype=np.float32)
    out = np.empty(a.shape, dtype=np.float32)

    def conv(sl):
        out[sl] = a[sl]
    list(_pool().map(conv, _slabs(a)))
    return out


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"), dtype=np.float32)


class _Prepared:
    """Everything the C ABI needs, plus what the post-processing needs."""


def _prepare(dim, kgrid, medium, source, sensor, options):
    for k in options:
        if k not in _KNOWN_OPTIONS:
            raise KWaveInputError("Unknown optional input %r." % k)
    if kgrid.dim != dim:
        raise KWaveInputError("kgrid must be %dD for kspaceFirstOrder%dD" % (dim, dim))
    P = _Prepared()
    P.dim = dim

    # ---- optional inputs (setDefaults.m:151-170, checkOptionalInputs.m) ----
    for o in ("SaveToDisk", "SaveToDiskExit", "HDFCompressionLevel"):
        if options.get(o) not in (None, False):
            raise KWaveInputError("Optional input %r (the HDF5 input file of the native binaries) is not supported by "
                                  "this solver: no HDF5 library." % o)
    # StreamToDisk (checkOptionalInputs.m:353-374): true -> 200 steps; the
    # series goes through a file named as the reference names it
    stream = options.get("StreamToDisk", False)
    if stream is not False and stream is not None:
        if dim != 3:
            raise KWaveInputError("Optional input 'StreamToDisk' is currently only compatible with 3D fluid simulations.")
        if isinstance(stream, (bool, np.bool_)):
            stream = STREAM_TO_DISK_STEPS_DEF if stream else 0
        elif np.size(stream) != 1 or not np.isfinite(stream) or stream < 0:
            raise KWaveInputError("Optional input 'StreamToDisk' must be a single scalar or Boolean value.")
        stream = int(stream)
    else:
        stream = 0
    for o in ("MultiAxialPMLRatio", "PMLRange", "RadialSymmetry", "UseFD"):
        if o in options:
            raise KWaveInputError("Optional input %r is not valid for kspaceFirstOrder%dD." % (o, dim))
    if options.get("RecordMovie"):
        raise KWaveInputError("'RecordMovie' needs MATLAB figures; this solver runs headless.")
    dc = options.get("DataCast", "off")
    if dc not in _DATA_CASTS:
        raise KWaveInputError("Invalid input for 'DataCast'.")
    pml_size = options.get("PMLSize", 20 if dim == 2 else 10)
    if isinstance(pml_size, str):
        raise KWaveInputError("'PMLSize' set to 'auto' is not supported by this solver.")
    pml_size = [int(_round(v)) for v in _pick(pml_size, dim)]
    pml_alpha = [float(v) for v in _pick(options.get("PMLAlpha", 2.0), dim)]
    pml_inside = bool(options.get("PMLInside", True))
    sm = options.get("Smooth", [True, False, False])
    sm = list(np.atleast_1d(sm))
    if len(sm) > 3 or not all(isinstance(b, (bool, np.bool_)) for b in sm):
        raise KWaveInputError("Optional input 'Smooth' must be a 1, 2 or 3 element Boolean array.")
    smooth_p0, smooth_c0, smooth_rho0 = bool(sm[0]), bool(sm[int(math.ceil((len(sm) + 1) / 2)) - 1]), bool(sm[-1])
    use_kspace = bool(options.get("UsekSpace", True))
    use_sg = bool(options.get("UseSG", True))
    scale_source_terms = bool(options.get("ScaleSourceTerms", True))
    cart_interp = options.get("CartInterp", "linear")
    if cart_interp not in ("linear", "nearest"):
        raise KWaveInputError("Optional input 'CartInterp' must be set to 'linear' or 'nearest'.")

    # ---- medium (inputChecking.m:115-281) ----
    if medium is None or not _has(medium, "sound_speed"):
        raise KWaveInputError("The field medium.sound_speed must be defined.")
    c0 = np.asarray(_field(medium, "sound_speed"), dtype=np.float64)
    if _has(medium, "density"):
        rho0 = np.asarray(_field(medium, "density"), dtype=np.float64)
        user_density = True
    elif c0.size == 1:
        rho0 = np.asarray(1.0)
        user_density = False
    else:
        raise KWaveInputError("The field medium.density must be defined.")
    alpha_mode = _field(medium, "alpha_mode")
    if alpha_mode is not None and alpha_mode not in ("no_absorption", "no_dispersion", "stokes"):
        raise KWaveInputError("medium.alpha_mode must be set to 'no_absorption', 'no_dispersion', or 'stokes'.")
    alpha_coeff = None
    alpha_power = 0.0
    if _has(medium, "alpha_coeff") or _has(medium, "alpha_power"):
        if not _has(medium, "alpha_coeff"):
            raise KWaveInputError("The field medium.alpha_coeff must be defined.")
        alpha_coeff = np.asarray(_field(medium, "alpha_coeff"), dtype=np.float64)
        if alpha_mode == "stokes":
            eos = "stokes"
            alpha_power = 2.0
        else:
            eos = "absorbing"
            if not _has(medium, "alpha_power"):
                raise KWaveInputError("The field medium.alpha_power must be defined.")
            ap = np.asarray(_field(medium, "alpha_power"), dtype=np.float64)
            if ap.size != 1:
                raise KWaveInputError("medium.alpha_power must be scalar.")
            alpha_power = float(ap)
            if alpha_power >= 3 or alpha_power < 0:
                raise KWaveInputError("medium.alpha_power must be a real number between 0 and 3.")
            if alpha_power == 1 and alpha_mode != "no_dispersion":
                raise KWaveInputError("The power law dispersion term in the equation of state is not valid "
                                      "for medium.alpha_power = 1.")
        if _any(lambda x: x < 0, alpha_coeff):
            raise KWaveInputError("medium.alpha_coeff must be non-negative and real.")
    else:
        eos = "lossless"
    # absorption filter in natural wavenumber order (createAbsorptionVariables.m:56-76)
    alpha_filter = None
    if _has(medium, "alpha_filter"):
        if eos == "stokes":
            raise KWaveInputError("Input option medium.alpha_filter is not supported with the axisymmetric code or "
                                  "medium.alpha_mode = 'stokes'.")
        alpha_filter = np.asarray(_field(medium, "alpha_filter"), dtype=np.float64)
        if alpha_filter.shape != kgrid.shape:
            raise KWaveInputError("medium.alpha_filter must be the same size as the computational grid.")
        if eos == "lossless":
            alpha_filter = None     # no absorption operators to filter
    alpha_sign = [1.0, 1.0]
    if _has(medium, "alpha_sign"):
        s = np.asarray(_field(medium, "alpha_sign"), dtype=np.float64).ravel()
        if s.size != 2:
            raise KWaveInputError("medium.alpha_sign must be given as a 2 element numerical array.")
        alpha_sign = [float(s[0]), float(s[1])]
    nonlinear = _has(medium, "BonA")
    BonA = np.asarray(_field(medium, "BonA"), dtype=np.float64) if nonlinear else None
    cref = _field(medium, "sound_speed_ref")
    if cref is None or (isinstance(cref, str) and cref == "max"):
        c_ref = float(_par(np.max, c0, max))
    elif isinstance(cref, str) and cref == "min":
        c_ref = float(_par(np.min, c0, min))
    elif isinstance(cref, str) and cref == "mean":
        c_ref = float(c0.mean())
    elif isinstance(cref, str):
        raise KWaveInputError("Unknown input for medium.sound_speed_ref.")
    else:
        c_ref = float(cref)

    # ---- sensor (inputChecking.m:288-672) ----
    use_sensor = sensor is not None
    time_rev = use_sensor and _has(sensor, "time_reversal_boundary_data")
    record_given = use_sensor and _has(sensor, "record")
    record = set()
    if use_sensor and _has(sensor, "record_mode"):
        raise KWaveInputError("sensor.record_mode input has been deprecated.")
    if record_given:
        rec = _field(sensor, "record")
        if isinstance(rec, str):
            raise KWaveInputError("sensor.record must be given as a cell array, e.g., {'p', 'u'}.")
        for r in rec:
            if r not in RECORD_FLAGS:
                raise KWaveInputError("'%s' is not a valid input for sensor.record." % r)
        record = set(rec)
    elif use_sensor:
        record = {"p"}
    if time_rev:
        record = set()
    P.record_user = set(record)
    if record & {"I", "I_avg"}:
        # intensity is formed after the loop from p and the unstaggered
        # velocity (createStorageVariables.m:89-148, 309; saveIntensity.m)
        record |= {"p", "u_non_staggered"}
    needs_mask = bool(record & {"p", "p_max", "p_min", "p_rms", "u", "u_max", "u_min", "u_rms", "u_non_staggered"})
    blank = use_sensor and not needs_mask and not time_rev
    rsi = _field(sensor, "record_start_index", 1) if use_sensor else 1
    record_start = int(_round(rsi))
    P.frequency_response = None
    if use_sensor and not time_rev and _has(sensor, "frequency_response"):
        fr = np.asarray(_field(sensor, "frequency_response"), dtype=np.float64).ravel()
        if fr.size != 2:
            raise KWaveInputError("sensor.frequency_response must be a 2 element numerical array.")
        P.frequency_response = (float(fr[0]), float(fr[1]))
    P.cuboid_list = None
    P.reorder_index = None
    mask = None
    if use_sensor and not blank:
        if not _has(sensor, "mask"):
            raise KWaveInputError("The field sensor.mask must be defined.")
        m = np.asarray(_field(sensor, "mask"), dtype=np.float64)
        if m.shape == kgrid.shape:
            if _any(lambda x: (x != 0) & (x != 1), m):
                raise KWaveInputError("sensor.mask must be a binary grid (numeric values must be 0 or 1).")
            if not _any(lambda x: x, m):
                raise KWaveInputError("sensor.mask must be a binary grid with at least one element set to 1.")
            mask = m
        elif m.ndim == 2 and m.shape[0] == 2 * dim:
            if np.any(np.mod(m, 1) != 0):
                raise KWaveInputError("sensor.mask cuboid corner indices must be integers.")
            if np.any(m[dim:] - m[:dim] < 0):
                raise KWaveInputError("sensor.mask cuboid corners must be defined as [x1, y1, ... x2, y2, ...] where x2 => x1.")
            if np.any(m < 1) or any(np.any(m[[a, a + dim]] > kgrid.shape[a]) for a in range(dim)):
                raise KWaveInputError("sensor.mask cuboid corners must be within the grid.")
            P.cuboid_list = m.astype(np.int64)
            mask = np.zeros(kgrid.shape)
            for c in range(m.shape[1]):
                sl = tuple(slice(int(m[a, c]) - 1, int(m[a + dim, c])) for a in range(dim))
                mask[sl] = 1
        elif m.ndim == 2 and m.shape[0] == dim:
            if cart_interp == "linear" and not time_rev:
                # recorded by barycentric interpolation on the grid
                # (createStorageVariables.m:376-400, extractSensorData.m:301-352)
                P.cart_points = m
            else:
                mask, order_index, reorder_index = cart2grid(kgrid, m)
                P.reorder_index = None if time_rev else reorder_index
                P.order_index = order_index
        else:
            raise KWaveInputError("Cartesian sensor.mask for a %dD simulation must be given as a %d by N array." % (dim, dim))

    # ---- source (inputChecking.m:713-1220) ----
    p0 = _field(source, "p0")
    source_p0 = p0 is not None and np.size(p0) > 0 and _any(lambda x: x != 0, p0)
    if source_p0:
        p0 = np.asarray(p0, dtype=np.float64)
        if p0.shape != kgrid.shape:
            raise KWaveInputError("source.p0 must be the same size as the computational grid.")
    psrc = None
    if _has(source, "p"):
        if not _has(source, "p_mask"):
            raise KWaveInputError("The field source.p_mask must be defined.")
        pm = np.asarray(_field(source, "p_mask"))
        if pm.shape != kgrid.shape:
            raise KWaveInputError("source.p_mask must be the same size as the computational grid.")
        if not _any(lambda x: x, pm):
            raise KWaveInputError("source.p_mask must be a binary grid with at least one element set to 1.")
        if source_p0:
            raise KWaveInputError("source.p0 and source.p can't be defined in the same simulation.")
        mode = _field(source, "p_mode", "additive")
        if mode not in _abi.SOURCE_MODES:
            raise KWaveInputError("source.p_mode must be set to 'additive', 'additive-no-correction', or 'dirichlet'.")
        sig = np.atleast_2d(np.asarray(_field(source, "p"), dtype=np.float64))
        freq_ref = _frequency_ref(source, "p_frequency_ref", kgrid, c0)
        if freq_ref is not None:
            # the k-space source correction as a function of w instead of k
            # (inputChecking.m:820-836): the source is injected without the
            # spatial correction
            mode = "additive-no-correction"
        psrc = dict(mask=pm, mode=mode, sig=sig, freq_ref=freq_ref)
    usrc = None
    ucomp = ["ux", "uy", "uz"][:dim]
    if any(_has(source, n) for n in ucomp) or _has(source, "u_mask"):
        if not _has(source, "u_mask"):
            raise KWaveInputError("The field source.u_mask must be defined.")
        um = np.asarray(_field(source, "u_mask"))
        if um.shape != kgrid.shape:
            raise KWaveInputError("source.u_mask must be the same size as the computational grid.")
        if not _any(lambda x: x, um):
            raise KWaveInputError("source.u_mask must be a binary grid with at least one element set to 1.")
        mode = _field(source, "u_mode", "additive")
        if mode not in _abi.SOURCE_MODES:
            raise KWaveInputError("source.u_mode must be set to 'additive', 'additive-no-correction', or 'dirichlet'.")
        freq_ref = _frequency_ref(source, "u_frequency_ref", kgrid, c0)
        if freq_ref is not None:
            mode = "additive-no-correction"   # inputChecking.m:923-939
        sigs = [np.atleast_2d(np.asarray(_field(source, n), dtype=np.float64)) if _has(source, n) else None
                for n in ucomp]
        usrc = dict(mask=um, mode=mode, sigs=sigs, freq_ref=freq_ref)
    # a transducer as the source (kspaceFirstOrder_inputChecking.m:1160-1209):
    # any object exposing active_elements_mask, delay_mask, input_signal and
    # transmit_apodization(_mask), as kWaveTransducer does
    tsrc = None
    if _has(source, "active_elements_mask") and _has(source, "input_signal"):
        if dim != 3:
            raise KWaveInputError("Transducer inputs are only compatible with 3D simulations.")
        if psrc is not None or usrc is not None or source_p0:
            raise KWaveInputError("A transducer source cannot be combined with source.p, source.u or source.p0.")
        am = np.asarray(_field(source, "active_elements_mask")) != 0
        dm = np.asarray(_field(source, "delay_mask"))
        if am.shape != kgrid.shape or dm.shape != kgrid.shape:
            raise KWaveInputError("The transducer masks must be the same size as the computational grid.")
        apod = None
        ta = _field(source, "transmit_apodization", "Rectangular")
        if not (isinstance(ta, str) and ta == "Rectangular"):
            apod = np.asarray(_field(source, "transmit_apodization_mask"), dtype=np.float64)
        tsrc = dict(mask=am, delay=dm, apod=apod,
                    sig=np.asarray(_field(source, "input_signal"), dtype=np.float64).ravel())
    if not user_density and (usrc is not None or tsrc is not None or record & {"u", "u_max", "u_rms"}):
        raise KWaveInputError("medium.density must be explicitly defined if velocity inputs or outputs are used, "
                              "even in homogeneous media.")
    if not user_density and nonlinear:
        raise KWaveInputError("medium.density must be explicitly defined if medium.BonA is specified.")

    # ---- time (inputChecking.m:1227-1268) ----
    if kgrid.Nt is None:
        if time_rev:
            raise KWaveInputError("kgrid.t_array (Nt and dt) must be defined explicitly in time reversal mode.")
        if psrc is not None or usrc is not None:
            raise KWaveInputError("kgrid.t_array (Nt and dt) must be defined explicitly when using a time-varying source.")
        kgrid.makeTime(c0, 0.3)
    Nt, dt = int(kgrid.Nt), float(kgrid.dt)
    if use_sensor and (record_start > Nt or record_start < 1):
        raise KWaveInputError("sensor.record_start_index must be between 1 and the number of time steps.")
    if pml_inside and any(2 * pml_size[a] > kgrid.shape[a] for a in range(dim)):
        raise KWaveInputError("The size of the PML must be smaller than the size of the grid.")

    # ---- smoothing (inputChecking.m:1501-1604) ----
    if source_p0 and smooth_p0:
        p0 = smooth(p0, True)
    if smooth_c0 and c0.ndim == dim and c0.size > 1:
        c0 = smooth(c0)
    if smooth_rho0 and rho0.ndim == dim and rho0.size > 1:
        rho0 = smooth(rho0)

    # ---- grid expansion when the PML is outside (expandGridMatrices.m) ----
    shape = kgrid.shape
    spacing = kgrid.spacing
    if not pml_inside:
        def grow(a, edge):
            pad = [(s, s) for s in pml_size]
            return np.pad(a, pad, mode="edge") if edge else np.pad(a, pad)
        shape = tuple(shape[a] + 2 * pml_size[a] for a in range(dim))
        if c0.size > 1:
            c0 = grow(c0, True)
        if rho0.size > 1:
            rho0 = grow(rho0, True)
        if alpha_coeff is not None and alpha_coeff.size > 1:
            alpha_coeff = grow(alpha_coeff, True)
        if alpha_filter is not None:
            alpha_filter = grow(alpha_filter, False)     # expandGridMatrices.m:165-168, zeros
        if nonlinear and BonA.size > 1:
            BonA = grow(BonA, True)
        if source_p0:
            p0 = grow(p0, False)
        if psrc is not None:
            psrc["mask"] = grow(psrc["mask"], False)
        if usrc is not None:
            usrc["mask"] = grow(usrc["mask"], False)
        if tsrc is not None:
            # the delays stay as they are (inputChecking.m:1196-1198)
            tsrc["mask"] = grow(tsrc["mask"], False)
            tsrc["delay"] = grow(tsrc["delay"], False)
            if tsrc["apod"] is not None:
                tsrc["apod"] = grow(tsrc["apod"], False)
        if mask is not None:
            mask = grow(mask, False)
        inside = [(pml_size[a] + 1, shape[a] - pml_size[a]) for a in range(dim)]
    else:
        inside = [(1, shape[a]) for a in range(dim)]
    P.shape = shape
    N = int(np.prod(shape))

    # ---- indices ----
    if P.cuboid_list is not None:
        # sensor_mask_index is the concatenation of each cuboid's find()
        # (inputChecking.m:1612-1633); the library needs increasing indices,
        # so the rows are gathered from the union mask afterwards
        idx_parts = []
        for c in range(P.cuboid_list.shape[1]):
            tm = np.zeros(shape)
            off = [pml_size[a] if not pml_inside else 0 for a in range(dim)]
            sl = tuple(slice(int(P.cuboid_list[a, c]) - 1 + off[a], int(P.cuboid_list[a + dim, c]) + off[a])
                       for a in range(dim))
            tm[sl] = 1
            idx_parts.append(_find(tm))
        P.cuboid_rows = idx_parts
    sensor_idx = _find(mask) if mask is not None else np.zeros(0, dtype=np.int64)
    sensor_w = None
    if getattr(P, "cart_points", None) is not None:
        try:
            tri, sensor_w = cartLinearWeights(shape, spacing, P.cart_points)
        except ValueError as e:
            raise KWaveInputError(str(e))
        sensor_idx = tri

    # ---- source scaling (scaleSourceTerms.m) ----
    hetero_c = c0.size > 1
    src_struct = []
    if psrc is not None:
        pos = _find(psrc["mask"])
        labels = _at(psrc["mask"], pos)
        sig = psrc["sig"].copy()
        rows = _signal_rows(labels, sig.shape[0], pos.size, "source.p", "source.p_mask")
        cpos = _at(c0, pos[:sig.shape[0]]) if hetero_c else None
        if scale_source_terms and psrc["freq_ref"] is not None:
            sig = sig * math.cos(2 * math.pi * psrc["freq_ref"] * dt / 2)   # scaleSourceTerms.m:43-45
        if scale_source_terms:
            if psrc["mode"] == "dirichlet":
                for r in range(sig.shape[0]):
                    cc = c0 if cpos is None else cpos[r]
                    sig[r] = sig[r] / (dim * cc ** 2)
            else:
                for r in range(sig.shape[0]):
                    cc = c0 if cpos is None else cpos[r]
                    sig[r] = sig[r] * (2.0 * dt / (dim * cc * kgrid.dx))
        src_struct.append(("p", psrc["mode"], pos, rows, [sig]))
    if usrc is not None:
        pos = _find(usrc["mask"])
        labels = _at(usrc["mask"], pos)
        sigs = [s.copy() if s is not None else None for s in usrc["sigs"]]
        nrows = max(s.shape[0] for s in sigs if s is not None) if any(s is not None for s in sigs) else 1
        rows = _signal_rows(labels, nrows, pos.size, "source.ux (etc)", "source.u_mask")
        cpos = _at(c0, pos[:nrows]) if hetero_c else None
        if scale_source_terms and usrc["freq_ref"] is not None:
            w = math.cos(2 * math.pi * usrc["freq_ref"] * dt / 2)          # scaleSourceTerms.m:272-282
            sigs = [None if s_ is None else s_ * w for s_ in sigs]
        if scale_source_terms and usrc["mode"] != "dirichlet":
            for i, s in enumerate(sigs):
                if s is None:
                    continue
                d = spacing[i]
                for r in range(s.shape[0]):
                    cc = c0 if cpos is None else cpos[r]
                    s[r] = s[r] * (2.0 * cc * dt / d)
        src_struct.append(("u", usrc["mode"], pos, rows, sigs))

    if tsrc is not None:
        pos = _find(tsrc["mask"])
        tsrc["pos"] = pos
        tsrc["delay_pts"] = np.rint(_at(tsrc["delay"], pos)).astype(np.uint64)
        tsrc["apod_pts"] = None if tsrc["apod"] is None else _at(tsrc["apod"], pos)
        sig = tsrc["sig"]
        if scale_source_terms:
            # scaleSourceTerms.m:377-390: one drive signal, scaled with the
            # mean sound speed over the transducer's points
            cc = float(c0) if c0.size == 1 else float(np.mean(_at(c0, pos)))
            sig = sig * (2.0 * cc * dt / kgrid.dx)
        tsrc["sig_scaled"] = sig

    # ---- staggered density (kspaceFirstOrder3D.m:585-607) ----
    # the midpoint averages are formed on the device from rho0
    derive_rho_sg = rho0.ndim == dim and rho0.size > 1 and use_sg

    # ---- the C problem ----
    keep = []   # arrays referenced by raw pointers must outlive the call

    def arr(a):
        if a is None:
            return _abi.f32p()
        x = _f32(a)
        keep.append(x)
        return _abi.fptr(x)

    def grid_arr(a):
        x = _grid32(a)
        keep.append(x)
        return _abi.fptr(x)

    def idx_arr(i):
        x = np.ascontiguousarray(np.asarray(i, dtype=np.uint64) + 1)
        keep.append(x)
        return _abi.uptr(x)

    pr = _abi.kw_problem()
    pr.abi_version = _abi.KW_ABI_VERSION
    pr.dim = dim
    pr.Nx = shape[0]
    pr.Ny = shape[1]
    pr.Nz = shape[2] if dim == 3 else 1
    pr.Nt = Nt
    pr.dx = spacing[0]
    pr.dy = spacing[1]
    pr.dz = spacing[2] if dim == 3 else 0.0
    pr.dt = dt
    pr.c_ref = c_ref
    pr.array_order = _abi.KW_ROW_MAJOR
    if c0.size > 1:
        pr.c0 = grid_arr(c0)
    else:
        pr.c0_scalar = float(c0)
    if rho0.size > 1:
        pr.rho0 = grid_arr(rho0)
    else:
        pr.rho0_scalar = float(rho0)
    pr.derive_rho0_sg = int(derive_rho_sg)
    pr.pml_x_size, pr.pml_y_size = pml_size[0], pml_size[1]
    pr.pml_z_size = pml_size[2] if dim == 3 else 0
    pr.pml_x_alpha, pr.pml_y_alpha = pml_alpha[0], pml_alpha[1]
    pr.pml_z_alpha = pml_alpha[2] if dim == 3 else 0.0
    pr.use_kspace = int(use_kspace)
    pr.use_sg = int(use_sg)
    pr.nonlinear_flag = int(nonlinear)
    if nonlinear:
        if BonA.size > 1:
            pr.BonA = grid_arr(BonA)
        else:
            pr.BonA_scalar = float(BonA)
    pr.absorbing_flag = {"lossless": 0, "absorbing": 1, "stokes": 2}[eos]
    if alpha_coeff is not None:
        if alpha_coeff.size > 1:
            pr.alpha_coeff = grid_arr(alpha_coeff)
        else:
            pr.alpha_coeff_scalar = float(alpha_coeff)
    pr.alpha_power = alpha_power
    if tsrc is not None:
        ts = pr.transducer_source
        ts.num_points = tsrc["pos"].size
        ts.index = idx_arr(tsrc["pos"])
        d = np.ascontiguousarray(tsrc["delay_pts"], dtype=np.uint64)
        keep.append(d)
        ts.delay = _abi.uptr(d)
        ts.apodization = arr(tsrc["apod_pts"]) if tsrc["apod_pts"] is not None else _abi.f32p()
        ts.signal_length = tsrc["sig_scaled"].size
        ts.input_signal = arr(tsrc["sig_scaled"])
    if alpha_filter is not None:
        pr.alpha_filter = grid_arr(alpha_filter)
    pr.alpha_mode = _abi.ALPHA_MODES.get(alpha_mode if alpha_mode != "stokes" else None, 0)
    pr.alpha_sign[0], pr.alpha_sign[1] = alpha_sign
    for kind, mode, pos, rows, sigs in src_struct:
        targets = [pr.p_source] if kind == "p" else [pr.u_source[i] for i in range(dim)]
        pos_p = idx_arr(pos)
        # a binary mask (one row for every point, or row i for point i) passes
        # no signal index, so a one-row component can sit beside per-point
        # ones (MATLAB's source.ux(':', t) with one row drives every point)
        binary = bool(np.all(rows == 0)) or bool(np.array_equal(rows, np.arange(pos.size)))
        row_p = _abi.u64p() if binary else idx_arr(rows)
        for tgt, s in zip(targets, sigs):
            if s is None:
                continue
            x = np.ascontiguousarray(s.ravel(order="F"), dtype=np.float32)
            keep.append(x)
            tgt.num_time_samples = s.shape[1]
            tgt.mode = _abi.SOURCE_MODES[mode]
            tgt.num_points = pos.size
            tgt.index = pos_p
            tgt.num_signals = s.shape[0]
            tgt.signal_index = row_p
            tgt.input = _abi.fptr(x)
    if source_p0:
        pr.p0_source_input = grid_arr(p0)
    if sensor_w is not None:
        # M points x (D+1) vertices, column-major
        pr.sensor_num = sensor_idx.shape[0]
        pr.sensor_vertices = sensor_idx.shape[1]
        pr.sensor_mask_index = idx_arr(np.asfortranarray(sensor_idx).ravel(order="F"))
        pr.sensor_weights = arr(np.asfortranarray(sensor_w))
    else:
        pr.sensor_num = sensor_idx.size
        if sensor_idx.size:
            pr.sensor_mask_index = idx_arr(sensor_idx)
    pr.record_start_index = record_start
    bits = 0
    for r in record:
        if r in _abi.REC_BITS:
            bits |= 1 << _abi.REC_BITS[r]
    pr.record = bits
    if stream:
        # inputChecking.m:1369-1375
        if not use_sensor or time_rev or mask is None and getattr(P, "cart_points", None) is None:
            raise KWaveInputError("The optional input 'StreamToDisk' is currently only compatible with forward "
                                  "simulations using a non-zero sensor mask.")
        if record_given and set(record) != {"p"}:
            raise KWaveInputError("The optional input 'StreamToDisk' is currently only compatible with sensor.record "
                                  "= {'p'} (the default).")
        pr.stream_to_disk = stream
        fname = STREAM_TO_DISK_FILENAME.encode()
        keep.append(fname)
        pr.stream_to_disk_file = fname
    if time_rev:
        trd = np.atleast_2d(np.asarray(_field(sensor, "time_reversal_boundary_data"), dtype=np.float64))
        if P.reorder_index is None and getattr(P, "order_index", None) is not None:
            # Cartesian rows put into find(mask) order (inputChecking.m:640-648)
            trd = trd[np.argsort(P.order_index, kind="stable")]
        if trd.shape != (sensor_idx.size, Nt):
            raise KWaveInputError("sensor.time_reversal_boundary_data must be [num_sensor_points x Nt].")
        pr.time_reversal_input = arr(trd)
    for a in range(dim):
        pr.inside_lo[a] = inside[a][0]
        pr.inside_hi[a] = inside[a][1]

    pr.device = int(options.get("DeviceNum", 0))
    P.problem = pr
    P.keep = keep
    P.h2d_bytes = int(sum(a.nbytes for a in keep if isinstance(a, np.ndarray)))
    P.record = record
    P.record_given = record_given
    P.time_rev = time_rev
    P.use_sensor = use_sensor
    P.M = int(pr.sensor_num)
    P.dt = dt
    P.Nt = Nt
    P.record_start = record_start
    P.inside = inside
    return P


def _round(v):
    v = float(v)
    return math.copysign(math.floor(abs(v) + 0.5), v)


def _signal_rows(labels, nrows, npts, sname, mname):
    """0-based signal row of each source point (inputChecking.m:853-887);
    labels are the mask's non-zero values in find() order."""
    uniq = np.unique(labels)
    if uniq.size == 1 and uniq[0] == 1:
        if nrows > 1 and nrows != npts:
            raise KWaveInputError("The number of time series in %s must match the number of source elements in %s."
                                  % (sname, mname))
        return np.arange(npts) if nrows > 1 else np.zeros(npts, dtype=np.int64)
    u = uniq[uniq != 0]
    if np.any(np.diff(u) != 1) or u[0] != 1:
        raise KWaveInputError("If using a labelled %s, the source labels must be monotonically increasing and "
                              "start from 1." % mname)
    if nrows != u.size:
        raise KWaveInputError("The number of time series in %s must match the number of labelled source elements "
                              "in %s." % (sname, mname))
    return labels.astype(np.int64) - 1


class Simulation:
    """A prepared kspaceFirstOrder run bound to a device plan.

    ``Simulation(dim, kgrid, medium, source, sensor, **options)`` runs the
    setup and uploads everything; ``run()`` executes the time loop on the GPU
    and returns what kspaceFirstOrder2D/3D returns.  ``run()`` may be called
    again (the loop restarts from the initial state).
    """

    def __init__(self, dim, kgrid, medium, source, sensor, **options):
        self._bind(_prepare(dim, kgrid, medium, source, sensor, options))
        self.prep.keep = None    # the library copied everything it needs

    @classmethod
    def from_prepared(cls, prep):
        """A plan for a problem prepared by ``Server.prepare`` (which stays
        usable for further plans or submissions)."""
        self = cls.__new__(cls)
        self._bind(prep)
        return self

    def _bind(self, prep):
        self._lib = _abi.load_library()
        self.prep = prep
        h = C.c_void_p()
        _abi.check(self._lib.kw_plan_create(C.byref(prep.problem), C.byref(h)))
        self.handle = h
        self.h2d_bytes = prep.h2d_bytes
        d = _abi.kw_output_desc()
        _abi.check(self._lib.kw_plan_outputs(self.handle, C.byref(d)))
        self.desc = d

    def close(self):
        if getattr(self, "handle", None):
            self._lib.kw_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- split API used by benchmarks ---------------------------------------
    def run_device(self):
        _abi.check(self._lib.kw_run_device(self.handle))

    def step(self, n):
        _abi.check(self._lib.kw_step(self.handle, n))

    def reset(self):
        _abi.check(self._lib.kw_reset(self.handle))

    def set_timing(self, classes):
        mask = 0
        for c in classes:
            mask |= 1 << _abi.KCLASS[c]
        _abi.check(self._lib.kw_set_timing(self.handle, mask))

    def timing(self, cls):
        ms = C.c_double()
        n = C.c_uint64()
        _abi.check(self._lib.kw_get_timing(self.handle, _abi.KCLASS[cls], C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def run_timed(self, n):
        ms = C.c_double()
        _abi.check(self._lib.kw_run_timed(self.handle, n, C.byref(ms)))
        return ms.value

    def launch_count(self):
        n = C.c_uint64()
        _abi.check(self._lib.kw_launch_count(self.handle, C.byref(n)))
        return n.value

    def tiles(self):
        """(z, y, x) lines per block of the compile-time transform kernels (0: runtime kernels)."""
        t = (C.c_int32 * 3)()
        _abi.check(self._lib.kw_plan_tiles(self.handle, t))
        return tuple(t)

    def set_tiles(self, tiles):
        t = (C.c_int32 * 3)(*tiles)
        _abi.check(self._lib.kw_set_tiles(self.handle, t))

    def device_bytes(self):
        b = C.c_uint64()
        _abi.check(self._lib.kw_plan_device_bytes(self.handle, C.byref(b)))
        return b.value

    # -- adjoint -----------------------------------------------------------------
    def keep_checkpoints(self, enable=True, checkpoint_interval=0):
        """Let the next complete run keep the adjoint's checkpoints (the
        state after every checkpoint_interval-th step, 0: round(sqrt(Nt))), so
        that an ``adjoint_gradient`` with the same interval after it skips its
        own forward pass (kw_keep_checkpoints).  The gradient is unchanged."""
        _abi.check(self._lib.kw_keep_checkpoints(self.handle, 1 if enable else 0, int(checkpoint_interval)))

    def adjoint_gradient(self, residual, checkpoint_interval=0, density=True):
        """Gradient of a sensor misfit J with respect to the sound speed and
        the density at every grid cell (the library's discrete adjoint of this
        plan's loop; lossless linear media, additive pressure sources).

        ``residual`` is dJ/dp with the shape and row order of the recorded
        ``p`` output (for J = 1/2 sum (p - d)^2, ``p - d``).  Returns
        ``(dJ/dc0, dJ/drho0)`` shaped like the grid (``dJ/drho0`` is None when
        ``density`` is False).  c_ref, dt, the PML and the scaled source
        signal are held fixed."""
        P = self.prep
        T = P.Nt - P.record_start + 1
        r = np.asarray(residual, dtype=np.float64)
        if r.shape != (P.M, T):
            raise ValueError("residual must be %d x %d (sensor points x recorded steps)" % (P.M, T))
        if P.reorder_index is not None:
            # rows came back in Cartesian order: put them back in find(mask) order
            raw = np.empty_like(r)
            raw[np.argsort(np.asarray(P.reorder_index), kind="stable")] = r
            r = raw
        r = np.asfortranarray(r, dtype=np.float32)
        shape = P.shape
        gc = np.zeros(int(np.prod(shape)), dtype=np.float64)
        gr = np.zeros_like(gc) if density else None
        _abi.check(self._lib.kw_adjoint_gradient(self.handle, r.ctypes.data_as(C.c_void_p), int(checkpoint_interval),
                                                 gc.ctypes.data_as(C.c_void_p),
                                                 gr.ctypes.data_as(C.c_void_p) if density else None))
        gc = gc.reshape(shape, order="F")
        return gc, (gr.reshape(shape, order="F") if density else None)

    # -- outputs ---------------------------------------------------------------
    def copy_outputs(self):
        o, host = _alloc_outputs(self.prep)
        _abi.check(self._lib.kw_copy_outputs(self.handle, C.byref(o)))
        return _finish(self.prep, host)

    def run(self):
        o, host = _alloc_outputs(self.prep)
        _abi.check(self._lib.kw_run(self.handle, C.byref(o)))
        return _finish(self.prep, host)


class Server:
    """Continuous batching of independent kspaceFirstOrder runs on one GPU.

    No counterpart in the reference, which runs one simulation per call.
    ``submit`` runs the same setup as kspaceFirstOrder2D/3D and hands the
    problem to the library's serving loop, which admits it against an HBM
    budget, keeps it resident next to the other admitted runs, advances
    every resident run by a slice of time steps per round on its own stream
    and retires it when its loop ends; ``result`` returns exactly what the
    plain call returns for the same inputs.
    """

    def __init__(self, device=0, hbm_budget_bytes=0, max_active=0, steps_per_slice=0, request_timeout_ms=0,
                 fill_cells=0):
        self._lib = _abi.load_library()
        cfg = _abi.kw_server_config(device=device, hbm_budget_bytes=hbm_budget_bytes, max_active=max_active,
                                    steps_per_slice=steps_per_slice, request_timeout_ms=request_timeout_ms,
                                    fill_cells=fill_cells)
        h = C.c_void_p()
        _abi.check(self._lib.kw_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h
        self._preps = {}

    @staticmethod
    def prepare(dim, kgrid, medium, source, sensor, **options):
        """Input checking and setup only (host side), for submitting later."""
        return _prepare(dim, kgrid, medium, source, sensor, options)

    def submit(self, dim, kgrid, medium, source, sensor, **options):
        return self.submit_prepared(self.prepare(dim, kgrid, medium, source, sensor, **options))

    def submit_prepared(self, prep):
        t = C.c_uint64()
        _abi.check(self._lib.kw_server_submit(self.handle, C.byref(prep.problem), C.byref(t)))
        self._preps[t.value] = prep
        return t.value

    def result(self, ticket, with_latency=False, timeout_ms=None):
        """What the plain call returns for this request.  timeout_ms bounds
        the wait (KWaveError with status KW_ERR_TIMEOUT when the request has
        not finished by then; the ticket stays valid)."""
        prep = self._preps[ticket]
        o, host = _alloc_outputs(prep)
        ms = C.c_double()
        if timeout_ms is None:
            st = self._lib.kw_server_wait(self.handle, ticket, C.byref(o), C.byref(ms))
        else:
            st = self._lib.kw_server_wait_for(self.handle, ticket, int(timeout_ms), C.byref(o), C.byref(ms))
        if st != _abi.KW_ERR_TIMEOUT or timeout_ms is None:
            self._preps.pop(ticket)
        _abi.check(st)
        out = _finish(prep, host)
        return (out, ms.value) if with_latency else out

    def stats(self):
        st = _abi.kw_server_stats()
        _abi.check(self._lib.kw_server_get_stats(self.handle, C.byref(st)))
        return {k: getattr(st, k) for k, _ in st._fields_}

    def close(self):
        if getattr(self, "handle", None):
            self._lib.kw_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _inside_shape(prep):
    pr = prep.problem
    return tuple(int(pr.inside_hi[a] - pr.inside_lo[a] + 1) for a in range(prep.dim))


def _alloc_outputs(prep):
    """Host buffers for every recorded output and the kw_outputs naming them."""
    P = prep
    M, T = P.M, P.Nt - P.record_start + 1
    ins = _inside_shape(P)
    host = {}
    o = _abi.kw_outputs()
    rec = P.record

    def buf(key, shape, slot, idx=None):
        a = np.zeros(int(np.prod(shape)), dtype=np.float32)
        host[key] = (a, shape)
        if idx is None:
            setattr(o, slot, _abi.fptr(a))
        else:
            getattr(o, slot)[idx] = _abi.fptr(a)

    if not P.time_rev:
        if "p" in rec:
            buf("p", (M, T), "p")
        for k in ("p_max", "p_min", "p_rms"):
            if k in rec:
                buf(k, (M,), k)
        for k in ("p_max_all", "p_min_all"):
            if k in rec:
                buf(k, ins, k)
        comps = ["ux", "uy", "uz"][:P.dim]
        for i, n in enumerate(comps):
            if "u" in rec:
                buf(n, (M, T), "u", i)
            for k in ("max", "min", "rms"):
                if "u_" + k in rec:
                    buf(n + "_" + k, (M,), "u_" + k, i)
            for k in ("max_all", "min_all"):
                if "u_" + k in rec:
                    buf(n + "_" + k, ins, "u_" + k, i)
            if "u_final" in rec:
                buf(n + "_final", ins, "u_final", i)
            if "u_non_staggered" in rec:
                buf(n + "_non_staggered", (M, T), "u_non_staggered", i)
    if "p_final" in rec or P.time_rev:
        buf("p_final", ins, "p_final")
    return o, host


def _finish(P, host):
    """Shape the raw outputs the way kspaceFirstOrder2D/3D returns them."""
    out = {}
    for k, (a, shape) in host.items():
        out[k] = a.reshape(shape, order="F")
    user = getattr(P, "record_user", P.record)
    if not P.time_rev and user & {"I", "I_avg"}:
        # kspaceFirstOrder_saveIntensity.m: u_non_staggered shifted forward by
        # dt/2 in time (fourierShift.m), times p; I_avg is its time average
        for i in range(P.dim):
            n = ("ux", "uy", "uz")[i]
            inten = out["p"].astype(np.float64) * _fourier_shift(out[n + "_non_staggered"], 0.5)
            if "I" in user:
                out["I" + n[1:]] = inten.astype(np.float32)
            if "I_avg" in user:
                out["I" + n[1:] + "_avg"] = inten.mean(axis=-1).astype(np.float32)
        if "u_non_staggered" not in user:
            for i in range(P.dim):
                del out[("ux", "uy", "uz")[i] + "_non_staggered"]
        if "p" not in user:
            del out["p"]
    # Cartesian nearest-neighbour reorder (reorderCartData.m)
    if P.reorder_index is not None:
        for k in list(out):
            if k.endswith("_all") or k.endswith("_final"):
                continue
            out[k] = reorderBinarySensorData(out[k], P.reorder_index)
    # sensor frequency response (kspaceFirstOrder3D.m:1345-1348)
    if P.frequency_response is not None and "p" in out:
        out["p"] = _gaussian_filter(out["p"], 1.0 / P.dt, *P.frequency_response).astype(np.float32)
    if P.cuboid_list is not None:
        out = _cuboids(P, out)
    if not P.use_sensor:
        return None
    if P.time_rev:
        return out["p_final"]
    if not P.record_given and P.cuboid_list is None:
        return out["p"]
    return out


def _frequency_ref(source, name, kgrid, c0):
    """source.p_frequency_ref / u_frequency_ref checked as
    kspaceFirstOrder_inputChecking.m:820-836 / 923-939 does; None if unset."""
    if not _has(source, name):
        return None
    f = np.asarray(_field(source, name), dtype=np.float64)
    if f.size != 1 or not np.isfinite(f).all() or float(f.ravel()[0]) < 0:
        raise KWaveInputError("Expected input source.%s to be a nonnegative scalar." % name)
    f = float(f.ravel()[0])
    if f > kgrid.k_max * float(np.min(c0)) / (2 * math.pi):
        raise KWaveInputError("source.%s is higher than the maximum frequency supported by the spatial grid." % name)
    return f


def _cuboids(P, out):
    """Per-cuboid outputs shaped [X, Y, (Z,) T] (reorderCuboidCorners.m)."""
    all_idx = _find_union(P.cuboid_rows)
    pos = {v: i for i, v in enumerate(all_idx)}
    res = []
    for c, rows in enumerate(P.cuboid_rows):
        sel = np.array([pos[v] for v in rows], dtype=np.int64)
        lo = P.cuboid_list[:P.dim, c]
        hi = P.cuboid_list[P.dim:, c]
        size = tuple(int(h - l + 1) for l, h in zip(lo, hi))
        d = {}
        for k, v in out.items():
            if k.endswith("_all") or k.endswith("_final"):
                # whole-grid outputs belong to the first cuboid only
                if c == 0:
                    d[k] = v
            elif v.ndim == 2:
                d[k] = v[sel].reshape(size + (v.shape[1],), order="F")
            else:
                d[k] = v[sel].reshape(size, order="F")
        res.append(d)
    return res


def _gaussian_filter(signal, fs, freq, bandwidth):
    """gaussianFilter.m: every row filtered in frequency by
    max(G(f - freq), G(f + freq)), G a unit-height Gaussian of FWHM
    bandwidth % of freq."""
    signal = np.asarray(signal, dtype=np.float64)
    N = signal.shape[-1]
    if N % 2 == 0:
        f = np.arange(-N // 2, N // 2) * fs / N
    else:
        f = np.arange(-(N - 1) // 2, (N - 1) // 2 + 1) * fs / N
    var = (bandwidth / 100.0 * freq / (2 * math.sqrt(2 * math.log(2)))) ** 2
    g = np.maximum(np.exp(-(f - freq) ** 2 / (2 * var)), np.exp(-(f + freq) ** 2 / (2 * var)))
    spec = np.fft.fftshift(np.fft.fft(signal, axis=-1), axes=-1)
    return np.real(np.fft.ifft(np.fft.ifftshift(g * spec, axes=-1), axis=-1))


def _fourier_shift(data, shift):
    """fourierShift.m along the last axis: real(ifft(ifftshift(exp(i k shift)) fft(data)))
    with k = 2 pi (-N/2 .. N/2-1) / N (odd N: -(N-1)/2 .. (N-1)/2) and k at
    index floor(N/2) set to zero."""
    data = np.asarray(data, dtype=np.float64)
    N = data.shape[-1]
    if N % 2 == 0:
        k = 2 * np.pi * np.arange(-N // 2, N // 2) / N
    else:
        k = 2 * np.pi * np.arange(-(N - 1) // 2, (N - 1) // 2 + 1) / N
    k[N // 2] = 0.0
    return np.real(np.fft.ifft(np.fft.ifftshift(np.exp(1j * k * shift)) * np.fft.fft(data, axis=-1), axis=-1))


def _find_union(parts):
    return np.unique(np.concatenate(parts))


def kspaceFirstOrder2D(kgrid, medium, source, sensor, **options):
    """2-D drop-in for kspaceFirstOrder2D (+kwave/+legacy/kspaceFirstOrder2D.m)."""
    with Simulation(2, kgrid, medium, source, sensor, **options) as sim:
        return sim.run()


def kspaceFirstOrder3D(kgrid, medium, source, sensor, **options):
    """3-D drop-in for kspaceFirstOrder3D (+kwave/+legacy/kspaceFirstOrder3D.m)."""
    with Simulation(3, kgrid, medium, source, sensor, **options) as sim:
        return sim.run()

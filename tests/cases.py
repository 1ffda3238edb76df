"""Seeded parity cases shared by the GPU tests (inputs only; no oracle here).

Each case returns (dim, grid args, Nt, dt, medium, source, sensor, options).
"""
import zlib

import numpy as np


def blob_medium(shape, rng, n_blobs=4, c_bg=1500.0):
    c = np.full(shape, c_bg)
    grids = np.meshgrid(*[np.arange(s) for s in shape], indexing="ij")
    for _ in range(n_blobs):
        ctr = [rng.uniform(0.25 * s, 0.75 * s) for s in shape]
        sig = rng.uniform(0.06, 0.15) * min(shape)
        amp = rng.uniform(-100, 200)
        r2 = sum((g - c0) ** 2 for g, c0 in zip(grids, ctr))
        c += amp * np.exp(-r2 / (2 * sig * sig))
    rho = 1000.0 + 0.6 * (c - c_bg)
    return c, rho


def disc_p0(shape, r):
    grids = np.meshgrid(*[np.arange(s) - s // 2 for s in shape], indexing="ij")
    return (np.sqrt(sum(g * g for g in grids)) <= r).astype(float)


def tone(dt, f0, cycles, n_total, amp=1.0):
    n = int(round(cycles / f0 / dt)) + 1
    t = np.arange(n) * dt
    s = amp * np.sin(2 * np.pi * f0 * t) * (0.5 - 0.5 * np.cos(2 * np.pi * np.arange(n) / (n - 1)))
    out = np.zeros(n_total)
    out[: min(n, n_total)] = s[: n_total]
    return out


def make_case(name):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    dx = 1e-4
    if name == "2d_homog_p0":
        shape = (64, 64)
        mask = np.zeros(shape); mask[16, :] = 1; mask[:, 40] = 1
        return 2, shape, dx, 150, 0.3 * dx / 1500, {"sound_speed": 1500.0, "density": 1000.0}, \
            {"p0": disc_p0(shape, 4)}, {"mask": mask, "record": ["p", "p_max", "p_min", "p_rms", "p_final", "u", "u_max", "u_min", "u_rms", "u_final"]}, {"PMLSize": 10}
    if name == "2d_hetero_abs_nl":
        shape = (72, 60)
        c, rho = blob_medium(shape, rng)
        mask = (rng.random(shape) < 0.02).astype(float)
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
        return 2, shape, dx, 200, 0.3 * dx / c.max(), med, {"p0": 1e5 * disc_p0(shape, 5)}, \
            {"mask": mask, "record": ["p", "p_max", "p_rms", "p_max_all", "p_min_all"]}, {"PMLSize": 12}
    if name == "2d_stokes_dirichlet":
        shape = (48, 64)
        pm = np.zeros(shape); pm[10, 20:40] = 1
        dt = 0.3 * dx / 1500
        med = {"sound_speed": 1500.0, "density": 1000.0, "alpha_coeff": 0.5, "alpha_mode": "stokes"}
        src = {"p_mask": pm, "p": tone(dt, 1.5e6, 3, 180) * 1e3, "p_mode": "dirichlet"}
        mask = np.zeros(shape); mask[35, :] = 1
        return 2, shape, dx, 180, dt, med, src, {"mask": mask}, {"PMLSize": 8}
    if name == "2d_nocorr_multi":
        shape = (64, 48)
        pm = np.zeros(shape); pm[20, 10:30] = 1
        dt = 0.3 * dx / 1500
        sig = np.stack([tone(dt, 1e6 + 2e4 * i, 3, 160) for i in range(20)]) * 1e3
        med = {"sound_speed": 1500.0, "density": 1000.0}
        src = {"p_mask": pm, "p": sig, "p_mode": "additive-no-correction"}
        mask = np.zeros(shape); mask[45, :] = 1
        return 2, shape, dx, 160, dt, med, src, {"mask": mask}, {"PMLSize": 8}
    if name == "2d_u_additive":
        shape = (64, 64)
        um = np.zeros(shape); um[12, 24:40] = 1
        dt = 0.3 * dx / 1500
        c, rho = blob_medium(shape, rng)
        med = {"sound_speed": c, "density": rho}
        src = {"u_mask": um, "ux": tone(dt, 1e6, 3, 170), "uy": 0.5 * tone(dt, 1e6, 3, 170)}
        mask = np.zeros(shape); mask[50, :] = 1
        return 2, shape, dx, 170, 0.3 * dx / c.max(), med, src, {"mask": mask, "record": ["p", "u"]}, {"PMLSize": 10}
    if name == "2d_u_dirichlet":
        shape = (60, 50)
        um = np.zeros(shape); um[30, 10:40] = 1
        dt = 0.3 * dx / 1500
        med = {"sound_speed": 1500.0, "density": 1000.0}
        src = {"u_mask": um, "ux": tone(dt, 1e6, 3, 140), "u_mode": "dirichlet"}
        mask = np.zeros(shape); mask[10, :] = 1
        return 2, shape, dx, 140, dt, med, src, {"mask": mask, "record": ["p", "u_max"]}, {"PMLSize": 8}
    if name == "2d_odd_sizes":
        shape = (45, 36)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[5, :] = 1; mask[:, 7] = 1
        return 2, shape, dx, 120, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho}, \
            {"p0": disc_p0(shape, 3)}, {"mask": mask}, {"PMLSize": 6}
    if name == "2d_pml_outside":
        shape = (40, 44)
        mask = np.zeros(shape); mask[8, :] = 1
        return 2, shape, dx, 100, 0.3 * dx / 1500, {"sound_speed": 1500.0, "density": 1000.0}, \
            {"p0": disc_p0(shape, 3)}, {"mask": mask, "record": ["p", "p_final"]}, {"PMLSize": 10, "PMLInside": False}
    if name == "3d_hetero_abs_nl_plane":
        shape = (32, 32, 32)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[6, 8:24, 8:24] = 1
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
        src = {"p_mask": pm, "p": 1e6 * tone(dt, 1e6, 3, 100)}
        mask = np.zeros(shape); mask[:, :, 16] = 1; mask[20, 16, :] = 1
        return 3, shape, dx, 100, dt, med, src, {"mask": mask, "record": ["p", "p_max"]}, {"PMLSize": 6}
    if name == "3d_multi_signal_additive":
        shape = (24, 30, 20)
        dt = 0.3 * dx / 1500
        pm = np.zeros(shape); pm[5, 10:20, 5:15] = 1
        npts = int(pm.sum())
        sig = np.stack([tone(dt, 1e6, 2, 90) * (1 + 0.01 * i) for i in range(npts)]) * 1e3
        med = {"sound_speed": 1500.0, "density": 1000.0, "alpha_coeff": 0.5, "alpha_power": 1.2,
               "alpha_mode": "no_dispersion"}
        src = {"p_mask": pm, "p": sig}
        mask = np.zeros(shape); mask[18, :, :] = 1
        return 3, shape, dx, 90, dt, med, src, {"mask": mask, "record": ["p", "p_rms"]}, {"PMLSize": 4}
    if name == "3d_p0_u":
        shape = (30, 24, 36)
        c, rho = blob_medium(shape, rng)
        mask = (rng.random(shape) < 0.01).astype(float)
        return 3, shape, dx, 80, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho, "BonA": 5.0}, \
            {"p0": disc_p0(shape, 3)}, {"mask": mask, "record": ["p", "u", "u_rms", "p_final", "u_final"]}, {"PMLSize": 5}
    if name == "2d_time_reversal":
        shape = (64, 64)
        mask = np.zeros(shape); mask[10, :] = 1; mask[54, :] = 1
        data = np.stack([tone(0.3 * dx / 1500, 1e6 + 1e4 * i, 2, 100) for i in range(int(mask.sum()))])
        return 2, shape, dx, 100, 0.3 * dx / 1500, {"sound_speed": 1500.0, "density": 1000.0}, \
            {}, {"mask": mask, "time_reversal_boundary_data": data}, {"PMLSize": 8}
    if name == "3d_time_reversal_abs":
        shape = (24, 24, 24)
        mask = np.zeros(shape); mask[4, :, :] = 1
        data = np.stack([tone(0.3 * dx / 1500, 1e6, 2, 60) * (1 + 0.01 * i) for i in range(int(mask.sum()))])
        med = {"sound_speed": 1500.0, "density": 1000.0, "alpha_coeff": 0.75, "alpha_power": 1.5}
        return 3, shape, dx, 60, 0.3 * dx / 1500, med, {}, {"mask": mask, "time_reversal_boundary_data": data}, {"PMLSize": 4}
    if name == "3d_static_mixed_radix":
        # 96 x 160 x 64 takes the compile-time kernels (radix 16/2/3, 16/2/5, 16/4)
        shape = (96, 160, 64)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[8, 60:100, 20:44] = 1
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5, "BonA": 6.0}
        src = {"p_mask": pm, "p": 1e6 * tone(dt, 1e6, 3, 60)}
        mask = np.zeros(shape); mask[:, :, 32] = 1
        return 3, shape, dx, 60, dt, med, src, {"mask": mask, "record": ["p", "p_max", "p_rms"]}, {"PMLSize": 8}
    if name == "3d_static_128":
        shape = (128, 128, 128)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[64, :, :] = 1
        return 3, shape, dx, 30, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho}, \
            {"p0": disc_p0(shape, 6)}, {"mask": mask, "record": ["p", "u_max", "p_final"]}, {"PMLSize": 10}
    if name == "2d_intensity":
        shape = (72, 60)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[12, 20:40] = 1
        mask = (rng.random(shape) < 0.02).astype(float)
        return 2, shape, dx, 160, dt, {"sound_speed": c, "density": rho}, {"p_mask": pm, "p": 1e5 * tone(dt, 1.5e6, 3, 160)}, \
            {"mask": mask, "record": ["p", "u_non_staggered", "I", "I_avg"]}, {"PMLSize": 10}
    if name == "3d_intensity_static":
        # 64^3: every pass on the compile-time (narrow-tile) kernels; p not requested
        shape = (64, 64, 64)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[40, :, 32] = 1; mask[:, 20, 10] = 1
        return 3, shape, dx, 50, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho, "alpha_coeff": 0.5,
                                                      "alpha_power": 1.5}, \
            {"p0": disc_p0(shape, 5)}, {"mask": mask, "record": ["u_non_staggered", "I_avg", "p_max"]}, {"PMLSize": 8}
    if name == "2d_cart_linear":
        # Cartesian circle recorded with the default CartInterp 'linear'
        shape = (64, 64)
        c, rho = blob_medium(shape, rng)
        r = 22 * dx
        ang = np.linspace(0, 2 * np.pi, 40, endpoint=False) + 0.1
        pts = np.stack([r * np.cos(ang), r * np.sin(ang)])
        return 2, shape, dx, 150, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho}, \
            {"p0": disc_p0(shape, 4)}, {"mask": pts, "record": ["p", "p_max", "u", "u_non_staggered"]}, {"PMLSize": 10}
    if name == "3d_cart_linear":
        shape = (32, 28, 30)
        c, rho = blob_medium(shape, rng)
        pts = (rng.random((3, 25)) - 0.5) * np.array([[20], [18], [20]]) * dx
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 0.5, "alpha_power": 1.5}
        return 3, shape, dx, 60, 0.3 * dx / c.max(), med, {"p0": disc_p0(shape, 4)}, \
            {"mask": pts, "record": ["p", "p_rms", "I_avg"], "frequency_response": [1.5e6, 60.0]}, {"PMLSize": 5}
    if name == "2d_full_mask_odd":
        # every cell is a sensor and the cell count (1575) is not a multiple
        # of 4: the index-free gather of the scalar sensor kernel
        shape = (45, 35)
        c, rho = blob_medium(shape, rng)
        return 2, shape, dx, 90, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho, "alpha_coeff": 0.5,
                                                      "alpha_power": 1.5}, \
            {"p0": disc_p0(shape, 4)}, {"mask": np.ones(shape), "record": ["p", "p_max", "p_rms", "u_max"]}, \
            {"PMLSize": 6}
    if name == "3d_layered_full_volume":
        # the large layered recipe at 64^3: rough interfaces, per-cell alpha_coeff
        # and BonA, a focused phased plane source (one signal per point),
        # p_max / p_rms over every cell
        import bench
        w = bench.layered_workload(seed=3, N=64, Nt=60, pml=6, f0=2e6, cycles=3, focus=20, src=16, amp=1e5)
        return 3, w["shape"], w["dx"], w["Nt"], w["dt"], w["medium"], w["source"], w["sensor"], w["options"]
    raise KeyError(name)


CASES = ["2d_homog_p0", "2d_hetero_abs_nl", "2d_stokes_dirichlet", "2d_nocorr_multi", "2d_u_additive",
         "2d_u_dirichlet", "2d_odd_sizes", "2d_pml_outside", "3d_hetero_abs_nl_plane", "3d_multi_signal_additive",
         "3d_p0_u", "2d_time_reversal", "3d_time_reversal_abs", "3d_static_mixed_radix", "3d_static_128",
         "2d_intensity", "3d_intensity_static", "2d_cart_linear", "3d_cart_linear", "3d_layered_full_volume",
         "2d_full_mask_odd"]


def adjoint_problem(shape, Nt, seed=0, dx=1e-4):
    """Heterogeneous lossless medium, one additive point source, a sensor
    plane: (shape, dx, Nt, dt, c, rho, p_mask, signal, sensor_mask)."""
    rng = np.random.default_rng(seed)
    dim = len(shape)
    c = 1500 + 100 * rng.random(shape)
    rho = 1000 + 80 * rng.random(shape)
    dt = 0.3 * dx / c.max()
    pm = np.zeros(shape)
    pm[(shape[0] // 3,) + tuple(s // 2 for s in shape[1:])] = 1
    sig = 1e3 * np.sin(2 * np.pi * 2e6 * np.arange(Nt) * dt) * np.hanning(Nt)
    sm = np.zeros(shape)
    sl = [slice(None)] * dim
    sl[0] = 2 * shape[0] // 3
    sm[tuple(sl)] = 1
    return shape, dx, Nt, dt, c, rho, pm, sig, sm

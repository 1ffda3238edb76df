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
    # ---- grid sizes with prime factors above 7 (direct-sum radix stages) ----
    if name == "2d_prime_22x26":
        shape = (22, 26)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[4, :] = 1; mask[:, 19] = 1
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 0.75, "alpha_power": 1.5}
        return 2, shape, dx, 90, 0.3 * dx / c.max(), med, {"p0": disc_p0(shape, 3)}, \
            {"mask": mask, "record": ["p", "p_max", "u"]}, {"PMLSize": 4}
    if name == "3d_prime_26x22x34":
        shape = (26, 22, 34)
        c, rho = blob_medium(shape, rng)
        med = {"sound_speed": c, "density": rho, "BonA": 6.0}
        mask = np.zeros(shape); mask[:, :, 20] = 1
        return 3, shape, dx, 70, 0.3 * dx / c.max(), med, {"p0": disc_p0(shape, 3)}, \
            {"mask": mask, "record": ["p", "p_rms", "p_final"]}, {"PMLSize": 4}
    if name == "2d_long_axis_1030":
        # a 4-digit axis with a prime factor of 103 (1030 = 2 x 5 x 103)
        shape = (1030, 36)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[40, 10:26] = 1
        mask = np.zeros(shape); mask[900, :] = 1; mask[:, 18] = 1
        return 2, shape, dx, 160, dt, {"sound_speed": c, "density": rho, "alpha_coeff": 0.5, "alpha_power": 1.3}, \
            {"p_mask": pm, "p": 1e4 * tone(dt, 1.5e6, 3, 160)}, {"mask": mask, "record": ["p", "p_max"]}, {"PMLSize": 10}
    if name == "2d_long_y_4096":
        # the real-to-complex axis at its 4096-point limit (2-D y maps to it)
        shape = (24, 4096)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[6:18, 300] = 1
        mask = np.zeros(shape); mask[12, :] = 1; mask[:, 3900] = 1
        return 2, shape, dx, 120, dt, {"sound_speed": c, "density": rho, "alpha_coeff": 0.5, "alpha_power": 1.5,
                                       "BonA": 5.0}, \
            {"p_mask": pm, "p": 1e5 * tone(dt, 2e6, 3, 120)}, {"mask": mask, "record": ["p", "p_max"]}, {"PMLSize": 8}
    if name == "3d_long_z_3000":
        # a 3000-point real-to-complex axis (8 x 3 x 5^3), runtime-radix kernels
        shape = (20, 16, 3000)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[10, 8, :] = 1
        return 3, shape, dx, 60, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho, "alpha_coeff": 0.75,
                                                      "alpha_power": 1.5}, \
            {"p0": disc_p0(shape, 3)}, {"mask": mask, "record": ["p", "p_max", "u"]}, {"PMLSize": 4}
    # ---- operator options (kspaceFirstOrder3D.m:629-661) ----
    if name == "2d_no_sg":
        shape = (60, 52)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[10, 15:35] = 1
        mask = np.zeros(shape); mask[44, :] = 1
        return 2, shape, dx, 140, dt, {"sound_speed": c, "density": rho}, {"p_mask": pm, "p": 1e3 * tone(dt, 1.5e6, 3, 140)}, \
            {"mask": mask, "record": ["p", "u", "u_non_staggered"]}, {"PMLSize": 8, "UseSG": False}
    if name == "3d_no_kspace":
        shape = (28, 24, 30)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[20, :, :] = 1
        return 3, shape, dx, 60, 0.2 * dx / c.max(), {"sound_speed": c, "density": rho, "alpha_coeff": 0.5,
                                                      "alpha_power": 1.5}, \
            {"p0": disc_p0(shape, 3)}, {"mask": mask, "record": ["p", "p_max"]}, {"PMLSize": 4, "UsekSpace": False}
    # ---- absorption variants (createAbsorptionVariables.m:29-101) ----
    if name == "2d_no_absorption_sign":
        shape = (64, 56)
        c, rho = blob_medium(shape, rng)
        mask = (rng.random(shape) < 0.03).astype(float)
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 2.0, "alpha_power": 1.7, "alpha_mode": "no_absorption",
               "alpha_sign": [1, -1]}
        return 2, shape, dx, 150, 0.3 * dx / c.max(), med, {"p0": disc_p0(shape, 4)}, \
            {"mask": mask, "record": ["p", "p_final"]}, {"PMLSize": 8}
    if name == "2d_alpha_sign":
        shape = (48, 64)
        c, rho = blob_medium(shape, rng)
        mask = np.zeros(shape); mask[36, :] = 1
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 1.5, "alpha_power": 1.4, "alpha_sign": [-1, 1]}
        return 2, shape, dx, 120, 0.3 * dx / c.max(), med, {"p0": disc_p0(shape, 4)}, \
            {"mask": mask, "record": ["p", "p_rms"]}, {"PMLSize": 8}
    if name == "2d_stokes_sign":
        shape = (48, 48)
        mask = np.zeros(shape); mask[30, :] = 1
        med = {"sound_speed": 1500.0, "density": 1000.0, "alpha_coeff": 0.8, "alpha_mode": "stokes", "alpha_sign": [-1, 1]}
        return 2, shape, dx, 100, 0.3 * dx / 1500, med, {"p0": disc_p0(shape, 4)}, {"mask": mask}, {"PMLSize": 6}
    # ---- reference sound speed (setSoundSpeedRef.m:30-49) ----
    if name in ("2d_cref_min", "3d_cref_mean", "2d_cref_value"):
        shape = (56, 48) if name.startswith("2d") else (24, 28, 26)
        c, rho = blob_medium(shape, rng)
        cref = {"2d_cref_min": "min", "3d_cref_mean": "mean", "2d_cref_value": 1650.0}[name]
        mask = np.zeros(shape)
        mask[(shape[0] - 8,) + (slice(None),) * (len(shape) - 1)] = 1
        med = {"sound_speed": c, "density": rho, "sound_speed_ref": cref, "alpha_coeff": 0.5, "alpha_power": 1.5}
        return len(shape), shape, dx, 90, 0.25 * dx / c.max(), med, {"p0": disc_p0(shape, 3)}, \
            {"mask": mask, "record": ["p", "p_max"]}, {"PMLSize": 5}
    # ---- smoothing of c and rho (inputChecking.m:1501-1544) ----
    if name == "2d_smooth_all":
        shape = (60, 60)
        c, rho = blob_medium(shape, rng)
        c = c + 40.0 * (rng.random(shape) > 0.7)
        mask = np.zeros(shape); mask[12, :] = 1
        return 2, shape, dx, 120, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho}, {"p0": disc_p0(shape, 5)}, \
            {"mask": mask, "record": ["p", "p_final"]}, {"PMLSize": 8, "Smooth": [True, True, True]}
    # ---- sensor.record_start_index > 1 ----
    if name == "2d_record_start":
        shape = (64, 48)
        c, rho = blob_medium(shape, rng)
        mask = (rng.random(shape) < 0.02).astype(float)
        return 2, shape, dx, 130, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho}, {"p0": disc_p0(shape, 4)}, \
            {"mask": mask, "record": ["p", "p_max", "p_min", "p_rms", "u", "u_rms", "p_max_all", "u_non_staggered"],
             "record_start_index": 47}, {"PMLSize": 8}
    # ---- velocity sources ----
    if name == "2d_u_nocorr":
        shape = (56, 64)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        um = np.zeros(shape); um[14, 20:44] = 1
        src = {"u_mask": um, "ux": tone(dt, 1e6, 3, 150), "uy": 0.3 * tone(dt, 1.2e6, 3, 150),
               "u_mode": "additive-no-correction"}
        mask = np.zeros(shape); mask[44, :] = 1
        return 2, shape, dx, 150, dt, {"sound_speed": c, "density": rho}, src, {"mask": mask, "record": ["p", "u"]}, \
            {"PMLSize": 8}
    if name in ("3d_u_additive", "3d_u_dirichlet"):
        shape = (30, 28, 32)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        um = np.zeros(shape); um[6, 8:20, 10:22] = 1
        n = int(um.sum())
        src = {"u_mask": um, "ux": tone(dt, 1e6, 2, 80), "uy": 0.5 * tone(dt, 1.3e6, 2, 80),
               "uz": np.stack([0.2 * tone(dt, 1e6, 2, 80) * (1 + 0.01 * i) for i in range(n)]),
               "u_mode": "additive" if name == "3d_u_additive" else "dirichlet"}
        mask = np.zeros(shape); mask[22, :, :] = 1
        return 3, shape, dx, 80, dt, {"sound_speed": c, "density": rho, "alpha_coeff": 0.5, "alpha_power": 1.5}, src, \
            {"mask": mask, "record": ["p", "u_max", "u_rms"]}, {"PMLSize": 4}
    # ---- frequency-domain source correction (scaleSourceTerms.m:43-45, 272-282) ----
    if name == "2d_p_freq_ref":
        shape = (60, 48)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        pm = np.zeros(shape); pm[10, 12:36] = 1
        mask = np.zeros(shape); mask[46, :] = 1
        return 2, shape, dx, 140, dt, {"sound_speed": c, "density": rho}, \
            {"p_mask": pm, "p": 1e3 * tone(dt, 1.5e6, 3, 140), "p_frequency_ref": 1.5e6}, \
            {"mask": mask, "record": ["p", "p_max"]}, {"PMLSize": 8}
    if name == "3d_u_freq_ref":
        shape = (28, 26, 30)
        dt = 0.3 * dx / 1500
        um = np.zeros(shape); um[5, 8:18, 8:20] = 1
        src = {"u_mask": um, "ux": tone(dt, 1e6, 2, 70), "uz": 0.4 * tone(dt, 1e6, 2, 70), "u_frequency_ref": 1e6}
        mask = np.zeros(shape); mask[20, :, :] = 1
        return 3, shape, dx, 70, dt, {"sound_speed": 1500.0, "density": 1000.0}, src, \
            {"mask": mask, "record": ["p", "u"]}, {"PMLSize": 4}
    # ---- cuboid-corner sensor masks (inputChecking.m:517-575, reorderCuboidCorners.m) ----
    if name == "3d_cuboids":
        shape = (32, 30, 28)
        c, rho = blob_medium(shape, rng)
        # the third cuboid is a single cell (outside the 4-cell PML)
        corners = np.array([[6, 5, 4, 12, 9, 20], [10, 12, 14, 24, 13, 15], [17, 16, 9, 17, 16, 9]]).T
        return 3, shape, dx, 60, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho, "alpha_coeff": 0.5,
                                                      "alpha_power": 1.5}, \
            {"p0": disc_p0(shape, 4)}, {"mask": corners, "record": ["p", "p_max", "u_rms", "p_final"]}, {"PMLSize": 4}
    if name == "2d_cuboids_pml_outside":
        shape = (40, 36)
        c, rho = blob_medium(shape, rng)
        corners = np.array([[5, 6, 30, 9], [12, 20, 14, 33]]).T
        return 2, shape, dx, 80, 0.3 * dx / c.max(), {"sound_speed": c, "density": rho}, {"p0": disc_p0(shape, 4)}, \
            {"mask": corners, "record": ["p", "p_rms", "p_max_all"]}, {"PMLSize": 6, "PMLInside": False}
    # ---- medium.alpha_filter (createAbsorptionVariables.m:56-76): a low-pass
    # in natural wavenumber order with a slight asymmetry, so the Hermitian
    # projection of the operator matters ----
    if name in ("2d_alpha_filter", "3d_alpha_filter_pml_outside"):
        shape = (60, 52) if name.startswith("2d") else (26, 24, 28)
        c, rho = blob_medium(shape, rng)
        grids = np.meshgrid(*[np.arange(n) - n // 2 for n in shape], indexing="ij")
        filt = np.exp(-sum((g / (0.3 * n)) ** 2 for g, n in zip(grids, shape))) * (1 + 0.2 * grids[0] / shape[0])
        med = {"sound_speed": c, "density": rho, "alpha_coeff": 3.0, "alpha_power": 1.5, "alpha_filter": filt}
        mask = np.zeros(shape)
        mask[(shape[0] - 6,) + (slice(None),) * (len(shape) - 1)] = 1
        opts = {"PMLSize": 6} if name.startswith("2d") else {"PMLSize": 4, "PMLInside": False}
        return len(shape), shape, dx, 100, 0.3 * dx / c.max(), med, {"p0": disc_p0(shape, 3)}, \
            {"mask": mask, "record": ["p", "p_final"]}, opts
    # ---- transducer source (kspaceFirstOrder3D.m:888-904): a 4-element
    # linear array on an x plane, steered by per-element delays, apodised ----
    if name in ("3d_transducer", "3d_transducer_pml_outside"):
        shape = (32, 36, 30)
        c, rho = blob_medium(shape, rng)
        dt = 0.3 * dx / c.max()
        active = np.zeros(shape); delay = np.zeros(shape); apod = np.zeros(shape)
        for e in range(4):
            ys = slice(6 + 6 * e, 10 + 6 * e)
            active[5, ys, 10:20] = 1
            delay[5, ys, 10:20] = 3 * e
            apod[5, ys, 10:20] = 0.5 + 0.5 * np.sin(np.pi * (e + 0.5) / 4)
        sig = tone(dt, 1.5e6, 2, 70)
        src = {"active_elements_mask": active, "delay_mask": delay, "input_signal": sig,
               "transmit_apodization": "Hanning", "transmit_apodization_mask": apod}
        mask = np.zeros(shape); mask[24, :, :] = 1
        opts = {"PMLSize": 4} if name == "3d_transducer" else {"PMLSize": 4, "PMLInside": False}
        return 3, shape, dx, 80, dt, {"sound_speed": c, "density": rho}, src, \
            {"mask": mask, "record": ["p", "u_max"]}, opts
    # ---- TestAcousticSolver.m:320-453 (testAgainstLegacyAbsorption), the
    # legacy 2-D and 3-D runs: 256 axial cells, 16 lateral, dx = 4 mm, PML 20
    # outside the grid along the axial axis only (296 = 8 x 37 cells), power
    # law absorption, Nt + 1 = 151 steps, no smoothing, p_final ----
    if name in ("legacy_abs_2dx", "legacy_abs_2dy", "legacy_abs_3dx"):
        nax, nlat, ldx, c0 = 256, 16, 4e-3, 1500.0
        dt = 0.25 * ldx / c0
        xv = (np.arange(nax) - nax // 2) * ldx
        prof = np.exp(-((xv - 25e-3) ** 2) / (5 * ldx) ** 2)
        if name == "legacy_abs_2dx":
            shape, p0 = (nax, nlat), np.repeat(prof[:, None], nlat, 1)
            med = {"sound_speed": c0, "density": 1000.0, "alpha_coeff": 10.0, "alpha_power": 1.9,
                   "alpha_mode": "no_dispersion"}
            pml = [20, 0]
        elif name == "legacy_abs_2dy":
            shape, p0 = (nlat, nax), np.repeat(prof[None, :], nlat, 0)
            med = {"sound_speed": c0, "density": 1000.0, "alpha_coeff": 10.0, "alpha_power": 1.9,
                   "alpha_mode": "no_absorption"}
            pml = [0, 20]
        else:
            shape, p0 = (nax, nlat, nlat), np.broadcast_to(prof[:, None, None], (nax, nlat, nlat)).copy()
            med = {"sound_speed": c0, "density": 1000.0, "alpha_coeff": 9.0, "alpha_power": 1.2}
            pml = [20, 0, 0]
        return len(shape), shape, ldx, 151, dt, med, {"p0": p0}, {"record": ["p_final"]}, \
            {"PMLSize": pml, "PMLInside": False, "Smooth": False}
    raise KeyError(name)


CASES = ["2d_homog_p0", "2d_hetero_abs_nl", "2d_stokes_dirichlet", "2d_nocorr_multi", "2d_u_additive",
         "2d_u_dirichlet", "2d_odd_sizes", "2d_pml_outside", "3d_hetero_abs_nl_plane", "3d_multi_signal_additive",
         "3d_p0_u", "2d_time_reversal", "3d_time_reversal_abs", "3d_static_mixed_radix", "3d_static_128",
         "2d_intensity", "3d_intensity_static", "2d_cart_linear", "3d_cart_linear", "3d_layered_full_volume",
         "2d_full_mask_odd",
         "2d_prime_22x26", "3d_prime_26x22x34", "2d_long_axis_1030", "2d_long_y_4096", "3d_long_z_3000", "2d_no_sg",
         "3d_no_kspace",
         "2d_no_absorption_sign", "2d_alpha_sign", "2d_stokes_sign", "2d_cref_min", "3d_cref_mean", "2d_cref_value",
         "2d_smooth_all", "2d_record_start", "2d_u_nocorr", "3d_u_additive", "3d_u_dirichlet", "2d_p_freq_ref",
         "3d_u_freq_ref", "3d_cuboids", "2d_cuboids_pml_outside", "legacy_abs_2dx", "legacy_abs_2dy",
         "legacy_abs_3dx", "2d_alpha_filter", "3d_alpha_filter_pml_outside", "3d_transducer",
         "3d_transducer_pml_outside"]


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

"""FP64 discrete adjoint of the k-space first-order loop -- TEST INFRASTRUCTURE ONLY.

The checker for the library's gradient entry point (``kw_adjoint_gradient``);
only ``tests/`` may import it, and the shipped library never routes through it.

The reference has no adjoint (it offers time reversal only), so this module
restates, for the subset the gradient supports -- lossless linear media,
additive pressure sources, a binary sensor mask recording p -- the forward
loop of ``+kwave/+legacy/kspaceFirstOrder3D.m`` step by step:

* momentum ``u_i = pml_sg_i (pml_sg_i u_i - dt rho_sg_i^-1 G_i p)`` (:792-803),
  with ``G_i f = real(ifftn(ddx_k_shift_pos_i kappa fftn(f)))``;
* divergence ``du_i = D_i u_i``, ``D_i`` with ``ddx_k_shift_neg_i`` (:907-909);
* mass ``rho_i = pml_i (pml_i rho_i - dt rho0 du_i)`` (:912-927);
* additive pressure source, filtered by ``source_kappa`` (:930-962);
* equation of state ``p = c0^2 sum_i rho_i`` (:965-1019, lossless);
* sensor ``p(sensor_mask_index)`` (``private/kspaceFirstOrder_extractSensorData.m:63-100``);

and its exact discrete adjoint.  With ``J`` a function of the recorded
pressure and ``r_m(t) = dJ/dp_m(t)``, the backward recursion over
``t = Nt .. 1`` is (``lambda`` at ``Nt + 1`` is zero)::

    mu      = S^T r(t) + dt sum_i D_i(rho_sg_i^-1 pml_sg_i lambda_u_i)
    lambda_rho_i = c0^2 mu + pml_i^2 lambda_rho_i
    lambda_u_i   = pml_sg_i^2 lambda_u_i + dt G_i(rho0 pml_i lambda_rho_i)

using ``G_i^T = -D_i`` (the transpose of a real spectral operator has the
conjugate symbol, and conj(i k e^{i k d/2}) = -i k e^{-i k d/2}).  The
gradients collect ``dJ/dc0 = sum_t mu 2 c0 sum_i rho_i``,
``dJ/drho0 = sum_t sum_i lambda_rho_i (-dt pml_i du_i)`` and, through
``rho_sg_i`` (midpoint average of rho0, kspaceFirstOrder3D.m:585-601),
``dJ/drho_sg_i^-1 = sum_t lambda_u_i (-dt pml_sg_i G_i p(t-1))``.
``c_ref``, ``dt``, the PML profiles and the scaled source signal are held
fixed.  The module is pinned by central finite differences of ``J``.
"""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from oracle.kspace import _axis, fftn, get_pml, ifftn, ifftshift, sinc


def setup(kgrid, c, rho0, p_mask, signal, sensor_mask, pml_size, pml_alpha=2.0, c_ref=None, use_kspace=True):
    """Operators of one problem.  ``signal`` is the pressure source signal
    (one row) before scaleSourceTerms.m; it is scaled here once with the c0
    given (so finite differences hold it fixed)."""
    dim = kgrid.dim
    shape = kgrid.shape
    c = np.asarray(c, dtype=np.float64) * np.ones(shape)
    rho0 = np.asarray(rho0, dtype=np.float64) * np.ones(shape)
    dt = kgrid.dt
    c_ref = float(c.max()) if c_ref is None else float(c_ref)
    ps = [int(pml_size)] * dim if np.isscalar(pml_size) else list(pml_size)
    pa = [float(pml_alpha)] * dim if np.isscalar(pml_alpha) else list(pml_alpha)
    ops = SimpleNamespace(dim=dim, shape=shape, dt=dt, Nt=kgrid.Nt, c_ref=c_ref)
    ops.pml = [_axis(get_pml(shape[a], kgrid.spacing[a], dt, c_ref, ps[a], pa[a], False), a, dim) for a in range(dim)]
    ops.pml_sg = [_axis(get_pml(shape[a], kgrid.spacing[a], dt, c_ref, ps[a], pa[a], True), a, dim)
                  for a in range(dim)]
    kmag = kgrid.k
    kappa = ifftshift(sinc(c_ref * kmag * dt / 2)) if use_kspace else 1.0
    ops.source_kappa = ifftshift(np.cos(c_ref * kmag * dt / 2)) if use_kspace else 1.0
    ops.G, ops.Dn = [], []
    for a, kv in enumerate(kgrid.k_vecs()):
        d = kgrid.spacing[a]
        ops.G.append(_axis(ifftshift(1j * kv * np.exp(1j * kv * d / 2)), a, dim) * kappa)
        ops.Dn.append(_axis(ifftshift(1j * kv * np.exp(-1j * kv * d / 2)), a, dim) * kappa)
    ops.p_pos = np.flatnonzero(np.asarray(p_mask).ravel(order="F") != 0)
    sig = np.atleast_2d(np.asarray(signal, dtype=np.float64))[0]
    # additive source scaling with c0 at the first source point (scaleSourceTerms.m)
    c_src = c.ravel(order="F")[ops.p_pos[0]]
    ops.signal = sig * (2.0 * dt / (dim * c_src * kgrid.dx))
    ops.sensor_idx = np.flatnonzero(np.asarray(sensor_mask).ravel(order="F") != 0)
    ops.c, ops.rho0 = c, rho0
    return ops


def _apply(sym, f):
    return np.real(ifftn(sym * fftn(f)))


def _rho_sg_inv(rho0, dim):
    out = []
    for a in range(dim):
        r = rho0.copy()
        lo = [slice(None)] * dim
        hi = [slice(None)] * dim
        lo[a] = slice(0, rho0.shape[a] - 1)
        hi[a] = slice(1, rho0.shape[a])
        r[tuple(lo)] = 0.5 * (rho0[tuple(lo)] + rho0[tuple(hi)])
        out.append(1.0 / r)
    return out


def _scatter(shape, idx, vals):
    f = np.zeros(int(np.prod(shape)))
    f[idx] = vals
    return f.reshape(shape, order="F")


def forward(ops, c=None, rho0=None, keep_states=False):
    """Recorded pressure y (M x Nt) and, optionally, the states after every step."""
    c = ops.c if c is None else c
    rho0 = ops.rho0 if rho0 is None else rho0
    dim, shape, dt = ops.dim, ops.shape, ops.dt
    rsi = _rho_sg_inv(rho0, dim)
    p = np.zeros(shape)
    u = [np.zeros(shape) for _ in range(dim)]
    rho = [np.zeros(shape) for _ in range(dim)]
    y = np.zeros((ops.sensor_idx.size, ops.Nt))
    states = [(p, u, rho)] if keep_states else None
    for t in range(1, ops.Nt + 1):
        u = [ops.pml_sg[i] * (ops.pml_sg[i] * u[i] - dt * rsi[i] * _apply(ops.G[i], p)) for i in range(dim)]
        du = [_apply(ops.Dn[i], u[i]) for i in range(dim)]
        rho = [ops.pml[i] * (ops.pml[i] * rho[i] - dt * rho0 * du[i]) for i in range(dim)]
        if t <= ops.signal.size:
            src = _apply(ops.source_kappa, _scatter(shape, ops.p_pos, ops.signal[t - 1]))
            rho = [r + src for r in rho]
        p = c ** 2 * sum(rho)
        y[:, t - 1] = p.ravel(order="F")[ops.sensor_idx]
        if keep_states:
            states.append((p, u, rho))
    return (y, states) if keep_states else y


def misfit(ops, d, c=None, rho0=None):
    """J = 1/2 sum (y - d)^2 and its residual dJ/dy."""
    y = forward(ops, c, rho0)
    r = y - d
    return 0.5 * float(np.sum(r * r)), r


def gradient(ops, residual, c=None, rho0=None):
    """(dJ/dc0, dJ/drho0) for dJ/dp_m(t) = residual[m, t-1]."""
    c = ops.c if c is None else c
    rho0 = ops.rho0 if rho0 is None else rho0
    dim, shape, dt = ops.dim, ops.shape, ops.dt
    rsi = _rho_sg_inv(rho0, dim)
    _, states = forward(ops, c, rho0, keep_states=True)
    lu = [np.zeros(shape) for _ in range(dim)]
    lr = [np.zeros(shape) for _ in range(dim)]
    g_c = np.zeros(shape)
    g_r0 = np.zeros(shape)
    g_R = [np.zeros(shape) for _ in range(dim)]
    for t in range(ops.Nt, 0, -1):
        p_t, u_t, rho_t = states[t]
        p_prev = states[t - 1][0]
        mu = _scatter(shape, ops.sensor_idx, residual[:, t - 1])
        mu = mu + dt * sum(_apply(ops.Dn[i], rsi[i] * ops.pml_sg[i] * lu[i]) for i in range(dim))
        lr = [c ** 2 * mu + ops.pml[i] ** 2 * lr[i] for i in range(dim)]
        g_c += mu * 2.0 * c * sum(rho_t)
        g_r0 += sum(lr[i] * (-dt * ops.pml[i] * _apply(ops.Dn[i], u_t[i])) for i in range(dim))
        lu = [ops.pml_sg[i] ** 2 * lu[i] + dt * _apply(ops.G[i], rho0 * ops.pml[i] * lr[i]) for i in range(dim)]
        for i in range(dim):
            g_R[i] += lu[i] * (-dt * ops.pml_sg[i] * _apply(ops.G[i], p_prev))
    # rho_sg_i^-1 = 1 / midpoint(rho0): chain back onto rho0
    g_rho = g_r0.copy()
    for a in range(dim):
        h = g_R[a] * (-(rsi[a] ** 2))        # dJ/drho_sg_a
        lo = [slice(None)] * dim
        hi = [slice(None)] * dim
        last = [slice(None)] * dim
        lo[a] = slice(0, shape[a] - 1)
        hi[a] = slice(1, shape[a])
        last[a] = slice(shape[a] - 1, shape[a])
        g_rho[tuple(lo)] += 0.5 * h[tuple(lo)]
        g_rho[tuple(hi)] += 0.5 * h[tuple(lo)]
        g_rho[tuple(last)] += h[tuple(last)]
    return g_c, g_rho

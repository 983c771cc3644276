"""Seeded initial states for compressible Navier-Stokes HDG problems.

Conserved variables per node are ``[rho, rho*v_1..rho*v_nd, rho*E]`` followed by
the ``nd`` gradient blocks ``q`` (``UDG = [u, q_x, q_y(, q_z)]``, the reference's
``npv x nc`` element layout).  ``q`` starts at zero; the solver makes it
consistent with ``u`` and ``uhat`` (``getQ``) before the first assembly, as
``solvers/dgsolvers.cpp:464-474`` does.

Free stream: rho = 1, |v| = 1, p = 1/(gamma M^2) (``examples/FM/ns/naca0012/
runns.m:14-19``).  ``uhat`` starts as the average of the adjacent elements'
face-node values (``utilities/inituhat.m``).
"""
from __future__ import annotations

import numpy as np

from .master import Master
from .mesh import Mesh


def primitive_to_conserved(rho, vel, p, gamma):
    """rho, vel (nd, ...), p -> conserved (nd+2, ...)."""
    mom = rho[None] * vel
    e = p / (gamma - 1.0) + 0.5 * rho * np.sum(vel * vel, axis=0)
    return np.concatenate([rho[None], mom, e[None]], axis=0)


def isentropic_vortex(x, y, gamma, mach, strength=5.0, centre=(5.0, 5.0)):
    """Isentropic vortex on a uniform x-directed free stream.

    Radial balance dp/dr = rho v_theta^2 / r with p = K rho^gamma gives
    T = p/rho = T_inf - (gamma-1) beta^2 / (8 gamma pi^2) exp(1 - r^2).
    """
    t_inf = 1.0 / (gamma * mach * mach)
    dx, dy = x - centre[0], y - centre[1]
    r2 = dx * dx + dy * dy
    amp = strength / (2.0 * np.pi) * np.exp(0.5 * (1.0 - r2))
    u = 1.0 - amp * dy
    v = amp * dx
    temp = t_inf - (gamma - 1.0) * strength ** 2 / (8.0 * gamma * np.pi ** 2) * np.exp(1.0 - r2)
    rho = (temp / t_inf) ** (1.0 / (gamma - 1.0))
    p = rho * temp
    return rho, np.stack([u, v]), p


def fourier_field(x, gamma, mach, seed, nmodes=8, amplitude=0.05, length=1.0):
    """Uniform x-directed base flow plus seeded Fourier modes on rho, v and p."""
    rng = np.random.default_rng(seed)
    nd = x.shape[0]
    p_inf = 1.0 / (gamma * mach * mach)
    rho = np.ones(x.shape[1:])
    vel = np.zeros(x.shape)
    vel[0] += 1.0
    p = np.full(x.shape[1:], p_inf)
    for _ in range(nmodes):
        k = rng.integers(-2, 3, size=nd)
        while not np.any(k):
            k = rng.integers(-2, 3, size=nd)
        phase = rng.uniform(0.0, 2.0 * np.pi, size=nd + 2)
        coef = rng.uniform(-1.0, 1.0, size=nd + 2)
        arg = 2.0 * np.pi * np.tensordot(k, x, axes=(0, 0)) / length
        rho = rho + amplitude * coef[0] * np.sin(arg + phase[0])
        for d in range(nd):
            vel[d] = vel[d] + amplitude * coef[1 + d] * np.sin(arg + phase[1 + d])
        p = p + amplitude * p_inf * coef[-1] * np.sin(arg + phase[-1])
    return rho, vel, p


def taylor_green(x, gamma, mach):
    """3D Taylor-Green vortex; density follows the pressure at constant temperature."""
    p0 = 1.0 / (gamma * mach * mach)
    xx, yy, zz = x
    u = np.sin(xx) * np.cos(yy) * np.cos(zz)
    v = -np.cos(xx) * np.sin(yy) * np.cos(zz)
    w = np.zeros_like(u)
    p = p0 + (np.cos(2 * xx) + np.cos(2 * yy)) * (np.cos(2 * zz) + 2.0) / 16.0
    rho = p / p0
    return rho, np.stack([u, v, w]), p


def make_udg(master: Master, mesh: Mesh, kind: str, gamma: float, mach: float, seed: int = 0,
             noise: float = 0.0, **kw) -> np.ndarray:
    """UDG (ne, nc, npv) with q = 0."""
    nd = mesh.nd
    ncu = nd + 2
    nc = ncu * (nd + 1)
    x = np.transpose(mesh.dgnodes, (1, 0, 2))            # (nd, ne, npv)
    if kind == "vortex":
        rho, vel, p = isentropic_vortex(x[0], x[1], gamma, mach, **kw)
    elif kind == "fourier":
        rho, vel, p = fourier_field(x, gamma, mach, seed=seed, **kw)
    elif kind == "tgv":
        rho, vel, p = taylor_green(x, gamma, mach)
    elif kind == "uniform":
        rho = np.ones(x.shape[1:])
        vel = np.zeros(x.shape)
        vel[0] += 1.0
        p = np.full(x.shape[1:], 1.0 / (gamma * mach * mach))
    else:
        raise ValueError(kind)
    cons = primitive_to_conserved(rho, vel, p, gamma)      # (ncu, ne, npv)
    if noise > 0.0:
        rng = np.random.default_rng(seed + 7919)
        cons = cons + rng.uniform(-noise, noise, size=cons.shape)
    udg = np.zeros((mesh.ne, nc, mesh.npv))
    udg[:, :ncu, :] = np.transpose(cons, (1, 0, 2))
    return udg


def init_uhat(master: Master, mesh: Mesh, udg: np.ndarray) -> np.ndarray:
    """UH (ndofuh, nch): mean of the element face-node values at each trace node."""
    ncu = mesh.nd + 2
    perm = master.perm.reshape(-1)                             # (nfe*npf,)
    vals = udg[:, :ncu, :][:, :, perm]                         # (ne, ncu, ndf)
    uh = np.zeros((mesh.ndofuh, ncu))
    cnt = np.zeros(mesh.ndofuh)
    idx = mesh.elcon.reshape(-1)
    np.add.at(uh, idx, np.transpose(vals, (0, 2, 1)).reshape(-1, ncu))
    np.add.at(cnt, idx, 1.0)
    return uh / cnt[:, None]

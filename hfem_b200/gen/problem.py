"""HDG Navier-Stokes problem definitions (master + mesh + physics + state).

A :class:`Problem` holds everything the element hot path reads, in the
reference's layouts (element-major numpy arrays = the reference's
column-major ``npv x nc x ne`` etc.).  The named workloads are:

* ``ns2d_vortex``: [0,10]^2 periodic, n x n quads split in 2 triangles,
  isentropic vortex (strength 5 at (5,5)) plus seeded U(-1e-3, 1e-3) noise on
  the conserved variables; gamma 1.4, Re 100, Pr 0.72, Mach 0.5.
* ``ns3d_fourier``: periodic unit cube, n^3 hexes split in 6 tetrahedra,
  uniform flow plus 8 seeded Fourier modes of amplitude 0.05; Re 400, Mach 0.3.
* ``ns3d_tgv``: [0, 2 pi]^3 periodic, Taylor-Green vortex; Re 1600, Mach 0.1.

Physics parameters are ``param = [gamma, eps, Re, Pr, Mach, tau]``
(``application/FM/nsNew/flux_ns2dNEW.c:7-12``, ``runns.m:31``), constant
stabilisation ``tau = 2`` (``convStabMethod = 0``) and constant viscosity
(``viscosityModel = 0``) unless :func:`with_models` selects the Lax-Friedrichs
or Roe stabilisation tensor or Sutherland's law.  Every problem here carries the time term of one
implicit stage: ``s += SH - fc_u * u`` with ``SH = fc_u * UDG_n``
(``elementassembly.cpp:293-304``), which is how both the DIRK driver and a
pseudo-transient Newton step call the assembly.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .master import Master, make_master
from .mesh import Mesh, build_mesh
from .state import init_uhat, make_udg


@dataclass
class Problem:
    name: str
    master: Master
    mesh: Mesh
    param: np.ndarray            # [gamma, eps, Re, Pr, Mach, tau]
    tdep: int
    fc_u: float
    fc_q: float
    time: float
    udg: np.ndarray              # (ne, nc, npv)
    uh: np.ndarray               # (ndofuh, nch)
    sh: np.ndarray               # (ne, nc, npv)
    dt: float = 0.0
    meta: dict = field(default_factory=dict)
    bcm: np.ndarray = None       # boundary condition type per boundary index (app.bcm); None: periodic
    bcs: np.ndarray = None       # (nbnd, nch) boundary states (app.bcs)
    appname: int = 1             # app.appname: 1 compressible Navier-Stokes, 0 Euler (inviscid, no q equation)
    conv_stab: int = 0           # app.convStabMethod: 0 constant tau, 1 Lax-Friedrichs, 2 Roe
    viscosity_model: int = 0     # app.viscosityModel: 0 constant viscosity, 1 Sutherland's law

    @property
    def nd(self):
        return self.master.nd

    @property
    def ncu(self):
        return self.nd + 2

    @property
    def nc(self):
        return self.ncu * (self.nd + 1)

    @property
    def nch(self):
        return self.ncu

    @property
    def n_local(self):           # size of D
        return self.master.npv * self.ncu

    @property
    def n_trace(self):           # size of H
        return self.master.npf * self.master.nfe * self.nch

    @property
    def bsz(self):
        return self.master.npf * self.nch

    def copy_state(self):
        return self.udg.copy(), self.uh.copy()


def _finish(name, master, mesh, udg, gamma, re, pr, mach, tau, dt, meta):
    uh = init_uhat(master, mesh, udg)
    fc_u = 1.0 / dt if dt > 0 else 0.0
    sh = np.zeros_like(udg)
    ncu = master.nd + 2
    sh[:, :ncu, :] = fc_u * udg[:, :ncu, :]
    param = np.array([gamma, 0.0, re, pr, mach, tau], dtype=np.float64)
    return Problem(name=name, master=master, mesh=mesh, param=param, tdep=1 if dt > 0 else 0,
                   fc_u=fc_u, fc_q=1.0, time=0.0, udg=udg, uh=uh, sh=sh, dt=dt, meta=meta)


def ns2d_vortex(n=32, porder=2, seed=0, mach=0.5, re=100.0, dt=0.1, noise=1e-3, length=10.0):
    master = make_master(2, porder)
    mesh = build_mesh(master, n, length)
    gamma = 1.4
    udg = make_udg(master, mesh, "vortex", gamma, mach, seed=seed, noise=noise,
                   centre=(0.5 * length, 0.5 * length))
    meta = dict(kind="ns2d_vortex", n=n, porder=porder, seed=seed, mach=mach, re=re, dt=dt,
                noise=noise, length=length)
    return _finish("ns2d_vortex", master, mesh, udg, gamma, re, 0.72, mach, 2.0, dt, meta)


def ns3d_fourier(n=20, porder=3, seed=0, mach=0.3, re=400.0, dt=0.01):
    master = make_master(3, porder)
    mesh = build_mesh(master, n, 1.0)
    gamma = 1.4
    udg = make_udg(master, mesh, "fourier", gamma, mach, seed=seed)
    meta = dict(kind="ns3d_fourier", n=n, porder=porder, seed=seed, mach=mach, re=re, dt=dt)
    return _finish("ns3d_fourier", master, mesh, udg, gamma, re, 0.72, mach, 2.0, dt, meta)


def ns3d_tgv(n=16, porder=3, mach=0.1, re=1600.0, dt=0.01):
    master = make_master(3, porder)
    mesh = build_mesh(master, n, 2.0 * np.pi)
    gamma = 1.4
    udg = make_udg(master, mesh, "tgv", gamma, mach)
    meta = dict(kind="ns3d_tgv", n=n, porder=porder, mach=mach, re=re, dt=dt)
    return _finish("ns3d_tgv", master, mesh, udg, gamma, re, 0.72, mach, 2.0, dt, meta)


def _freestream(nd, gamma, mach):
    """Conserved free-stream state: rho 1, velocity 1 along x, p = 1/(gamma M^2)."""
    p = 1.0 / (gamma * mach * mach)
    u = np.zeros(nd + 2)
    u[0], u[1] = 1.0, 1.0
    u[nd + 1] = p / (gamma - 1.0) + 0.5
    return u


# boundary condition types of the reference's NS boundary flux (application/FM/fbou.cpp)
BC_NOSLIP_ADIABATIC, BC_DIRICHLET, BC_EXTRAPOLATION, BC_SLIP = 2, 5, 6, 7


def ns2d_channel(n=16, porder=2, seed=0, mach=0.5, re=100.0, dt=0.1, noise=1e-3, length=10.0,
                 bcm=(BC_DIRICHLET, BC_EXTRAPOLATION, BC_SLIP, BC_NOSLIP_ADIABATIC)):
    """[0,L]^2 box (not periodic), isentropic vortex + noise.  Sides ib = 2 axis + end:
    0 x=0 (Dirichlet free stream), 1 x=L (extrapolation), 2 y=0 (slip wall),
    3 y=L (no-slip adiabatic wall)."""
    master = make_master(2, porder)
    mesh = build_mesh(master, n, length, periodic=False)
    gamma = 1.4
    udg = make_udg(master, mesh, "vortex", gamma, mach, seed=seed, noise=noise,
                   centre=(0.5 * length, 0.5 * length))
    meta = dict(kind="ns2d_channel", n=n, porder=porder, seed=seed, mach=mach, re=re, dt=dt, noise=noise,
                length=length, bcm=list(bcm))
    p = _finish("ns2d_channel", master, mesh, udg, gamma, re, 0.72, mach, 2.0, dt, meta)
    p.bcm = np.array(bcm, dtype=np.int64)
    p.bcs = np.tile(_freestream(2, gamma, mach), (len(bcm), 1))
    return p


def ns3d_box(n=4, porder=2, seed=0, mach=0.3, re=400.0, dt=0.01,
             bcm=(BC_DIRICHLET, BC_EXTRAPOLATION, BC_SLIP, BC_NOSLIP_ADIABATIC, BC_SLIP, BC_EXTRAPOLATION)):
    """Unit cube (not periodic), uniform flow + Fourier modes; one condition per side
    (ib = 2 axis + end)."""
    master = make_master(3, porder)
    mesh = build_mesh(master, n, 1.0, periodic=False)
    gamma = 1.4
    udg = make_udg(master, mesh, "fourier", gamma, mach, seed=seed)
    meta = dict(kind="ns3d_box", n=n, porder=porder, seed=seed, mach=mach, re=re, dt=dt, bcm=list(bcm))
    p = _finish("ns3d_box", master, mesh, udg, gamma, re, 0.72, mach, 2.0, dt, meta)
    p.bcm = np.array(bcm, dtype=np.int64)
    p.bcs = np.tile(_freestream(3, gamma, mach), (len(bcm), 1))
    return p


def as_euler(prob: Problem) -> Problem:
    """The same mesh, state and boundary conditions with the Euler equations
    (app.appname 0, flag_q 0).  The state keeps the NS layout with q slots: the
    inviscid flux does not depend on q, so every q coupling of the element
    matrices vanishes and they equal those of the q-free formulation."""
    from dataclasses import replace
    udg = prob.udg.copy()
    udg[:, prob.ncu:, :] = 0.0
    sh = prob.sh.copy()
    sh[:, prob.ncu:, :] = 0.0
    meta = dict(prob.meta, physics="euler")
    return replace(prob, name=prob.name + "_euler", udg=udg, sh=sh, appname=0, meta=meta)


def with_models(prob: Problem, conv_stab: int = 0, viscosity_model: int = 0) -> Problem:
    """The same problem with another convective stabilisation tensor
    (app.convStabMethod: 0 constant tau = param[5], 1 Lax-Friedrichs, 2 Roe;
    application/FM/stabilizationTensor.cpp) and viscosity model
    (app.viscosityModel: 0 constant, 1 Sutherland's law; application/FM/getViscosity.c)."""
    from dataclasses import replace
    tag = {0: "", 1: "_lf", 2: "_roe"}[conv_stab] + {0: "", 1: "_suth"}[viscosity_model]
    meta = dict(prob.meta, conv_stab=conv_stab, viscosity_model=viscosity_model)
    return replace(prob, name=prob.name + tag, conv_stab=int(conv_stab), viscosity_model=int(viscosity_model),
                   meta=meta)


def make_problem(kind: str, **kw) -> Problem:
    return {"ns2d_vortex": ns2d_vortex, "ns3d_fourier": ns3d_fourier, "ns3d_tgv": ns3d_tgv,
            "ns2d_channel": ns2d_channel, "ns3d_box": ns3d_box}[kind](**kw)

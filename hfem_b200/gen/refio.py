"""Reader/writer for the reference's float64 input files.

Writes ``<prefix>app.bin``, ``master.bin``, ``mesh.bin`` and ``sol.bin`` in the
layout ``preprocessing/readbinaryfiles.cpp`` reads (serial branch): every
integer is stored as a double, arrays are column-major, and each file starts
with a fixed-length ``ndims`` header (app 40 at ``readbinaryfiles.cpp:16-46``,
master 20 at ``:112-175``, mesh 30 at ``:413-464``, sol 10 at ``:640-652``).
The field order mirrors the MATLAB writers (``preprocessing/digasopre.m:266-300``
and ``mkapp``).
"""
from __future__ import annotations

import numpy as np

from .problem import Problem

# indices into app.flag (initializestructs.cpp:91-107, 186-204)
FLAG_LEN = 28
PROBLEM_LEN = 14


def app_arrays(prob: Problem, preconditioner=0, newton_tol=1e-10, gmres_tol=1e-10, newton_maxiter=1,
               dirk_stage=1, dirk_order=1, dt_list=None):
    flag = np.zeros(FLAG_LEN)
    flag[0] = prob.tdep
    flag[5] = 1 if prob.appname == 1 else 0   # flag_q: q eliminated by the local solve (NS only)
    flag[9] = 1                      # overlapping level
    flag[16] = preconditioner        # serial reference accepts -1 or 0
    flag[17] = 0                     # left preconditioning
    flag[18] = 1                     # quasi-Newton storage precision (unused)
    flag[19] = 0                     # MGS
    flag[24] = 1                     # preconditioner precision: double
    flag[25] = 1                     # matvec precision: double
    flag[26] = 1                     # orthogonalisation precision: double
    factor = np.array([prob.fc_u, prob.fc_q, 0.0, prob.time, 0.0, 0.0])
    problem = np.zeros(PROBLEM_LEN)
    problem[0] = 0                   # HDG
    problem[1] = prob.appname        # app.appname: 1 compressible Navier-Stokes, 0 Euler
    problem[3] = dirk_order
    problem[4] = dirk_stage
    problem[5] = getattr(prob, "conv_stab", 0)           # app.convStabMethod: 0 constant tau, 1 LF, 2 Roe
    problem[8] = getattr(prob, "viscosity_model", 0)     # app.viscosityModel: 0 constant, 1 Sutherland
    problem[12] = 1                  # GMRES
    problem[13] = newton_maxiter
    dt = np.array(dt_list if dt_list is not None else [prob.dt if prob.dt > 0 else 1.0])
    return flag, factor, problem, dt, np.array([newton_tol, gmres_tol])


def _w(f, arr):
    """Natural (row, col) arrays and 1-D tables: column-major flattening."""
    np.asarray(arr, dtype=np.float64).ravel(order="F").tofile(f)


def _we(f, arr):
    """Element-major arrays (ne first): C order is the reference's column-major."""
    np.asarray(arr, dtype=np.float64).ravel(order="C").tofile(f)


def write_app(path, prob: Problem, **kw):
    m = prob.master
    flag, factor, problem, dt, solversparam = app_arrays(prob, **kw)
    arrays = [
        np.array([0.0, 1.0]),                 # meshsize (unused serially)
        np.array([0.0, 1.0]),                 # solsize
        np.array([m.porder]),                 # porder
        np.array([0.0]),                      # elemtype
        np.array([0.0]),                      # nodetype
        np.array([m.pgauss]),                 # pgauss
        np.array([m.pgauss]),                 # pgaussR
        np.array([0.0]),                      # quadtype
        np.zeros(0) if prob.bcm is None else np.asarray(prob.bcm, dtype=np.float64),          # bcm
        np.zeros(0) if prob.bcs is None else np.ascontiguousarray(prob.bcs, dtype=np.float64).ravel(),  # bcs[ib*nch + c]
        np.zeros(0), np.zeros(0),             # bcd bcv
        dt, flag, factor, problem, prob.param, solversparam,
    ]
    ndims = np.zeros(40)
    for i, a in enumerate(arrays):
        ndims[i] = a.size
    ndims[18] = 1                             # nproc
    ndims[19] = 1                             # nfile
    ndims[20] = prob.nd
    ndims[21] = prob.nd                       # ncd
    euler = prob.appname == 0
    ndims[22] = prob.ncu if euler else prob.nc  # nc (Euler: no gradient unknowns)
    ndims[23] = prob.ncu
    ndims[24] = prob.nch
    ndims[25] = 0 if euler else prob.ncu * prob.nd   # ncq
    ndims[26] = 0                             # ncp
    ndims[27] = 0                             # nco
    with open(path, "wb") as f:
        _w(f, ndims)
        for a in arrays:
            _w(f, a)


def write_master(path, prob: Problem):
    m = prob.master
    nd = m.nd
    nve = nd + 1
    nle = 3 if nd == 2 else 6
    nplmax = m.porder + 1
    ndims = np.zeros(20)
    ndims[:11] = [nd, 0, 0, m.npv, m.npv, m.ngv, m.ngv, m.nfe, nve, nle, nplmax]
    shapvt = m.fortran("shapvt")
    shapvg = m.fortran("shapvg")
    svsv = m.fortran("shapvgdotshapvl")
    with open(path, "wb") as f:
        _w(f, ndims)
        _w(f, np.full(m.nfe, m.npf))          # npf
        _w(f, np.full(m.nfe, m.npf))          # nmf
        _w(f, np.full(m.nfe, m.ngf))          # ngf
        _w(f, np.full(m.nfe, m.ngf))          # ngfR
        _w(f, np.full(m.nfe, nd))             # nvf
        _w(f, np.full(nle, nplmax))           # npl
        _w(f, np.asfortranarray(m.plocvl))
        _w(f, np.asfortranarray(m.gpvl))
        _w(f, m.gwvl)
        _w(f, shapvt)
        _w(f, shapvg)
        _w(f, shapvt)                         # shapmv (geometry order = solution order)
        _w(f, svsv)
        _w(f, np.asfortranarray(m.gpvl))      # residual rule = Jacobian rule
        _w(f, m.gwvl)
        _w(f, shapvt)
        _w(f, shapvg)
        _w(f, shapvt)
        _w(f, np.zeros(nve))                  # permnode (unused by the hot path)
        _w(f, np.zeros(nle * nplmax))         # permedge (unused by the hot path)
        shapft = m.fortran("shapft")
        shapfg = m.fortran("shapfg")
        sfsf = m.fortran("shapfgdotshapfc")
        for a in range(m.nfe):
            _w(f, np.asfortranarray(m.plocfc))
            _w(f, np.asfortranarray(m.gpfc))
            _w(f, m.gwfc)
            _w(f, shapft)
            _w(f, shapfg)
            _w(f, shapft)                     # shapmf
            _w(f, sfsf)
            _w(f, np.asfortranarray(m.gpfc))
            _w(f, m.gwfc)
            _w(f, shapft)
            _w(f, shapfg)
            _w(f, shapft)
            _w(f, m.perm[a])                  # perm (0-based element nodes)
            _w(f, m.perm[a])                  # permgeom
            _w(f, np.array(m.faces[a]))       # face vertices


def write_mesh(path, prob: Problem):
    me = prob.mesh
    nd = me.nd
    ndims = np.zeros(30)
    ndims[:17] = [nd, nd, me.nfe, nd + 1, nd, me.ne, me.nf, me.nv, me.ndofuh, me.npv, me.npf,
                  prob.nc, prob.ncu, prob.ncu * nd, 0, prob.nch, me.nf]
    ndims[28] = 0                             # HDG
    ndims[29] = 1                             # nproc
    fmat = np.zeros((me.nf, nd + 3))
    fmat[:, 0] = nd
    fmat[:, 1:nd + 1] = me.face_verts
    fmat[:, nd + 1:] = me.face_elems
    with open(path, "wb") as f:
        _w(f, ndims)
        _w(f, np.zeros(me.ne))                # elementtype
        _we(f, me.t)                           # (ne, nve) C order == (nve, ne) column-major
        _we(f, me.dgnodes)
        _we(f, me.elcon)
        _we(f, me.bf)
        _we(f, me.t2f)
        _we(f, me.t2t)
        _we(f, fmat)
        _w(f, np.zeros(me.nf))                # isEDGface


def write_sol(path, prob: Problem, udg=None, uh=None):
    udg = prob.udg if udg is None else udg
    uh = prob.uh if uh is None else uh
    if prob.appname == 0:
        udg = udg[:, :prob.ncu, :]          # the Euler state has no q
    ndims = np.zeros(10)
    ndims[0] = udg.size
    ndims[1] = uh.size
    with open(path, "wb") as f:
        _w(f, ndims)
        _we(f, np.ascontiguousarray(udg))
        _we(f, np.ascontiguousarray(uh))


def write_inputs(prefix: str, prob: Problem, **kw):
    write_app(prefix + "app.bin", prob, **kw)
    write_master(prefix + "master.bin", prob)
    write_mesh(prefix + "mesh.bin", prob)
    write_sol(prefix + "sol.bin", prob)


# ------------------------------------------------------------------ readers
def _rd(f, n):
    a = np.fromfile(f, dtype=np.float64, count=n)
    if a.size != n:
        raise ValueError("file shorter than its header says")
    return a


def read_sol(path, ne=None, npv=None, nc=None):
    """sol.bin (readbinaryfiles.cpp readsolstruct, serial branch): UDG, UH, PDG as flat arrays."""
    with open(path, "rb") as f:
        nd = _rd(f, 10).astype(np.int64)
        udg, uh, pdg = _rd(f, int(nd[0])), _rd(f, int(nd[1])), _rd(f, int(nd[2]))
    if ne is not None:
        udg = udg.reshape(ne, nc, npv)
    return udg, uh, pdg


def read_mesh(path):
    """mesh.bin (readmeshstruct, serial branch) as a dict of element-major arrays."""
    with open(path, "rb") as f:
        nd = _rd(f, 30).astype(np.int64)
        dim, ncd, nfe, nve, nvf, ne, nf = (int(v) for v in nd[:7])
        npe, npf = int(nd[9]), int(nd[10])
        out = dict(ndims=nd)
        out["elementtype"] = _rd(f, ne).astype(np.int64)
        out["t"] = _rd(f, nve * ne).reshape(ne, nve).astype(np.int64)
        out["dgnodes"] = _rd(f, npe * ncd * ne).reshape(ne, ncd, npe)
        out["elcon"] = _rd(f, npf * nfe * ne).reshape(ne, npf * nfe).astype(np.int64)
        out["bf"] = _rd(f, nfe * ne).reshape(ne, nfe).astype(np.int64)
        out["t2f"] = _rd(f, nfe * ne).reshape(ne, nfe).astype(np.int64)
        out["t2t"] = _rd(f, nfe * ne).reshape(ne, nfe).astype(np.int64)
        out["f"] = _rd(f, (nvf + 3) * nf).reshape(nf, nvf + 3).astype(np.int64)
        out["isEDGface"] = _rd(f, nf).astype(np.int64)
    return out


def write_checkpoint(path, udg, uh, ncu=None, with_q=True):
    """Solution file of solstruct::writeSol2File (preprocessing/ioutilities.cpp:256-300):
    [n_udg, n_uh, UDG (u only when with_q is False), UH], float64."""
    udg = np.ascontiguousarray(udg)
    if not with_q:
        udg = np.ascontiguousarray(udg[:, :ncu, :])
    with open(path, "wb") as f:
        np.array([udg.size, np.size(uh)], dtype=np.float64).tofile(f)
        udg.astype(np.float64).tofile(f)
        np.ascontiguousarray(uh, dtype=np.float64).tofile(f)


def read_checkpoint(path):
    with open(path, "rb") as f:
        n = _rd(f, 2).astype(np.int64)
        return _rd(f, int(n[0])), _rd(f, int(n[1]))


def problem_from_files(prefix, prob_template):
    """State of a problem read back from the reference's input files: UDG/UH from
    sol.bin and dgnodes/elcon/t2f checked against the template's mesh."""
    udg, uh, _ = read_sol(prefix + "sol.bin")
    me = read_mesh(prefix + "mesh.bin")
    p = prob_template
    if not (np.array_equal(me["elcon"], p.mesh.elcon) and np.array_equal(me["t2f"], p.mesh.t2f)):
        raise ValueError("mesh file does not match the problem's connectivity")
    p.udg = udg.reshape(p.udg.shape)
    p.uh = uh.reshape(p.uh.shape)
    return p

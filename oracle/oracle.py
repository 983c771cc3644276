"""ctypes front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/liboracle.so`` (the project's restatement, hfem_oracle.cpp) and
runs ``oracle/_ref/hfem_ref`` (the reference's own C++ built from its sources)
on the reference's binary input files.  Only tests, ``__graft_entry__.smoke``
and the CPU-baseline leg of ``bench.py`` use this module, as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_BIN = os.path.join(HERE, "_ref", "hfem_ref")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


class OracleProblem(C.Structure):
    _fields_ = [
        ("nd", C.c_int), ("npv", C.c_int), ("npf", C.c_int), ("nfe", C.c_int),
        ("ngv", C.c_int), ("ngf", C.c_int), ("ne", C.c_int), ("nf", C.c_int),
        ("shapvt", _dp), ("shapvg", _dp), ("shapvgdotshapvl", _dp),
        ("shapft", _dp), ("shapfg", _dp), ("shapfgdotshapfc", _dp),
        ("perm", _ip), ("dgnodes", _dp), ("elcon", _ip), ("t2f", _ip),
        ("rowstart", _ip), ("colidx", _ip),
        ("param", C.c_double * 6), ("tdep", C.c_int),
        ("fc_u", C.c_double), ("fc_q", C.c_double), ("time", C.c_double),
        ("bf", _ip), ("bcm", _ip), ("bcs", _dp), ("appname", C.c_int),
        ("conv_stab", C.c_int), ("visc_model", C.c_int),
    ]

# boundary condition types restated in hfem_oracle.cpp (fbou_point)
BC_TYPES = (1, 2, 5, 6, 7)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        for name in ("oracle_element", "oracle_getq", "oracle_assemble", "oracle_residual",
                     "oracle_update", "oracle_bj_inverse", "oracle_gmres", "oracle_mdf_ordering",
                     "oracle_bilu0_factor", "oracle_gmres_bilu0"):
            getattr(_lib, name).restype = C.c_int
    return _lib


def build(with_reference: bool = False):
    args = ["make", "-C", HERE, "liboracle.so"]
    if with_reference:
        args[-1] = "all"
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class Oracle:
    """Oracle bound to one problem (keeps the converted arrays alive)."""

    def __init__(self, prob):
        m, me = prob.master, prob.mesh
        self.prob = prob
        self._keep = dict(
            shapvt=m.fortran("shapvt"), shapvg=m.fortran("shapvg"), svsv=m.fortran("shapvgdotshapvl"),
            shapft=m.fortran("shapft"), shapfg=m.fortran("shapfg"), sfsf=m.fortran("shapfgdotshapfc"),
            perm=np.ascontiguousarray(m.perm, dtype=np.int32),
            dgnodes=np.ascontiguousarray(me.dgnodes, dtype=np.float64),
            elcon=np.ascontiguousarray(me.elcon, dtype=np.int32),
            t2f=np.ascontiguousarray(me.t2f, dtype=np.int32),
            rowstart=np.ascontiguousarray(me.rowstart, dtype=np.int32),
            colidx=np.ascontiguousarray(me.colidx, dtype=np.int32),
        )
        k = self._keep
        p = OracleProblem()
        p.nd, p.npv, p.npf, p.nfe = m.nd, m.npv, m.npf, m.nfe
        p.ngv, p.ngf, p.ne, p.nf = m.ngv, m.ngf, me.ne, me.nf
        p.shapvt, p.shapvg, p.shapvgdotshapvl = _d(k["shapvt"]), _d(k["shapvg"]), _d(k["svsv"])
        p.shapft, p.shapfg, p.shapfgdotshapfc = _d(k["shapft"]), _d(k["shapfg"]), _d(k["sfsf"])
        p.perm, p.dgnodes, p.elcon, p.t2f = _i(k["perm"]), _d(k["dgnodes"]), _i(k["elcon"]), _i(k["t2f"])
        p.rowstart, p.colidx = _i(k["rowstart"]), _i(k["colidx"])
        for i in range(6):
            p.param[i] = float(prob.param[i])
        p.tdep, p.fc_u, p.fc_q, p.time = prob.tdep, prob.fc_u, prob.fc_q, prob.time
        p.appname = int(getattr(prob, "appname", 1))
        p.conv_stab = int(getattr(prob, "conv_stab", 0))
        p.visc_model = int(getattr(prob, "viscosity_model", 0))
        if getattr(prob, "bcm", None) is not None:
            if any(int(b) not in BC_TYPES for b in prob.bcm):
                raise ValueError(f"boundary condition types {list(prob.bcm)} not all in {BC_TYPES}")
            k["bf"] = np.ascontiguousarray(me.bf, dtype=np.int32)
            k["bcm"] = np.ascontiguousarray(prob.bcm, dtype=np.int32)
            k["bcs"] = np.ascontiguousarray(prob.bcs, dtype=np.float64)
            p.bf, p.bcm, p.bcs = _i(k["bf"]), _i(k["bcm"]), _d(k["bcs"])
        self.p = p
        self.n = prob.n_local
        self.nb = prob.n_trace
        self.bsz = prob.bsz
        self.nblk = int(me.rowstart[-1])

    def getq(self, udg, uh, sh=None):
        udg = np.ascontiguousarray(udg, dtype=np.float64).copy()
        sh = self.prob.sh if sh is None else sh
        lib().oracle_getq(C.byref(self.p), _d(udg), _d(np.ascontiguousarray(uh)), _d(np.ascontiguousarray(sh)))
        return udg

    def element(self, udg, uh, ie, sh=None):
        n, nb = self.n, self.nb
        sh = self.prob.sh if sh is None else sh
        out = dict(D=np.zeros(n * n), F=np.zeros(n * nb), K=np.zeros(nb * n), H=np.zeros(nb * nb),
                   Ru=np.zeros(n), Rh=np.zeros(nb))
        lib().oracle_element(C.byref(self.p), _d(np.ascontiguousarray(udg)), _d(np.ascontiguousarray(uh)),
                             _d(np.ascontiguousarray(sh)), ie, _d(out["D"]), _d(out["F"]), _d(out["K"]),
                             _d(out["H"]), _d(out["Ru"]), _d(out["Rh"]))
        return out

    def assemble(self, udg, uh, sh=None, want_dinv=True, e0=0, e1=-1, elem_blocks=False):
        me = self.prob.mesh
        sh = self.prob.sh if sh is None else sh
        ne = me.ne
        Hg = np.zeros(self.nblk * self.bsz * self.bsz)
        Rg = np.zeros(me.nf * self.bsz)
        Rr = np.zeros(me.nf * self.bsz)
        DinvRu = np.zeros(ne * self.n) if want_dinv else None
        DinvF = np.zeros(ne * self.n * self.nb) if want_dinv else None
        rn = C.c_double(0.0)
        e1v = ne if e1 < 0 else e1
        eH = np.zeros((e1v - e0) * self.nb * self.nb) if elem_blocks else None
        eRh = np.zeros((e1v - e0) * self.nb) if elem_blocks else None
        null = _dp()
        rc = lib().oracle_assemble(C.byref(self.p), _d(np.ascontiguousarray(udg)), _d(np.ascontiguousarray(uh)),
                                   _d(np.ascontiguousarray(sh)), _d(Hg), _d(Rg), _d(Rr),
                                   _d(DinvRu) if want_dinv else null, _d(DinvF) if want_dinv else null,
                                   C.byref(rn), _d(eH) if elem_blocks else null,
                                   _d(eRh) if elem_blocks else null, e0, e1)
        if rc != 0:
            raise RuntimeError(f"oracle_assemble failed ({rc})")
        return dict(Hg=Hg, Rg=Rg, Rr=Rr, DinvRu=DinvRu, DinvF=DinvF, rnorm=rn.value, eH=eH, eRh=eRh)

    def residual(self, udg, uh, sh=None):
        sh = self.prob.sh if sh is None else sh
        rn = C.c_double(0.0)
        lib().oracle_residual(C.byref(self.p), _d(np.ascontiguousarray(udg)), _d(np.ascontiguousarray(uh)),
                              _d(np.ascontiguousarray(sh)), C.byref(rn))
        return rn.value

    def update(self, udg, uh, duh, DinvRu, DinvF, alpha, sh=None):
        sh = self.prob.sh if sh is None else sh
        udg = np.ascontiguousarray(udg).copy()
        uh = np.ascontiguousarray(uh).copy()
        lib().oracle_update(C.byref(self.p), _d(udg), _d(uh), _d(np.ascontiguousarray(sh)), _d(DinvRu),
                            _d(DinvF), _d(np.ascontiguousarray(duh)), C.c_double(alpha))
        return udg, uh

    def bj_inverse(self, Hg):
        me = self.prob.mesh
        Minv = np.zeros(me.nf * self.bsz * self.bsz)
        rc = lib().oracle_bj_inverse(me.nf, self.bsz, self._keep["rowstart"].ctypes.data_as(_ip), _d(Hg), _d(Minv))
        if rc:
            raise RuntimeError("singular diagonal block")
        return Minv

    def gmres(self, Hg, b, Minv=None, restart=50, tol=1e-10, maxit=1000, x0=None):
        me = self.prob.mesh
        x = np.zeros_like(b) if x0 is None else x0.copy()
        it = C.c_int(0)
        hist = np.zeros(maxit + 1)
        flag = lib().oracle_gmres(me.nf, self.bsz, _i(self._keep["rowstart"]), _i(self._keep["colidx"]), _d(Hg),
                                  _d(Minv) if Minv is not None else _dp(), _d(np.ascontiguousarray(b)), _d(x),
                                  restart, C.c_double(tol), maxit, C.byref(it), _d(hist), maxit + 1)
        return x, flag, hist[:it.value]

    # -- BILU0 with the MDF ordering (computeMDFordering.m, computeBILU0.m, applyBILU0.m)
    def _rc(self):
        return _i(self._keep["rowstart"]), _i(self._keep["colidx"])

    def mdf_ordering(self, Hg):
        nf = self.prob.mesh.nf
        o2u = np.zeros(nf, dtype=np.int32)
        u2o = np.zeros(nf, dtype=np.int32)
        if lib().oracle_mdf_ordering(nf, self.bsz, *self._rc(), _d(Hg), _i(o2u), _i(u2o)):
            raise RuntimeError("singular diagonal block")
        return o2u, u2o

    def bilu0_factor(self, Hg, o2u, u2o):
        Mg = np.zeros_like(Hg)
        lib().oracle_bilu0_factor(self.prob.mesh.nf, self.bsz, *self._rc(), _d(Hg), _i(o2u), _i(u2o), _d(Mg))
        return Mg

    def bilu0_apply(self, Mg, o2u, u2o, x):
        v = np.zeros_like(x)
        lib().oracle_bilu0_apply(self.prob.mesh.nf, self.bsz, *self._rc(), _d(Mg), _i(o2u), _i(u2o),
                                 _d(np.ascontiguousarray(x)), _d(v))
        return v

    def gmres_bilu0(self, Hg, Mg, o2u, u2o, b, restart=50, tol=1e-10, maxit=1000):
        x = np.zeros_like(b)
        it = C.c_int(0)
        hist = np.zeros(maxit + 1)
        flag = lib().oracle_gmres_bilu0(self.prob.mesh.nf, self.bsz, *self._rc(), _d(Hg), _d(Mg), _i(o2u), _i(u2o),
                                        _d(np.ascontiguousarray(b)), _d(x), restart, C.c_double(tol), maxit,
                                        C.byref(it), _d(hist), maxit + 1)
        return x, flag, hist[:it.value]


def dirk_table(stages, order):
    """(d = A^-1, t) of the DIRK(s, q) tableaus solvers/DIRKcoeff.cpp lists."""
    if (stages, order) == (1, 1):
        A, t = np.array([[1.0]]), [1.0]
    elif (stages, order) == (2, 2):
        g = 1 - 1 / np.sqrt(2)
        A, t = np.array([[g, 0], [1 - g, g]]), [g, 1.0]
    elif (stages, order) == (3, 3):
        g = 0.4358665
        for _ in range(50):
            g -= (g ** 3 - 3 * g * g + 1.5 * g - 1 / 6) / (3 * g * g - 6 * g + 1.5)
        t2 = (1 + g) / 2
        b1, b2 = -(6 * g * g - 16 * g + 1) / 4, (6 * g * g - 20 * g + 5) / 4
        A, t = np.array([[g, 0, 0], [t2 - g, g, 0], [b1, b2, g]]), [g, t2, 1.0]
    else:
        raise ValueError((stages, order))
    return np.linalg.inv(A), t


def newton_solve(o, udg, uh, sh, tol, maxiter, restart=50, gmres_tol=1e-10):
    """solveNonlinearProblem (solvers/dgsolvers.cpp:106-205) on the oracle."""
    rnorm, it, robust = tol + 1.0, 0, 0
    hist = []
    while rnorm > tol and it < maxiter:
        it += 1
        a = o.assemble(udg, uh, sh=sh)
        old = a["rnorm"]
        hist.append(old)
        x, flag, _ = o.gmres(a["Hg"], a["Rg"], Minv=o.bj_inverse(a["Hg"]), restart=restart, tol=gmres_tol)
        if flag == -1:
            break
        if it == 1 and old < tol:
            rnorm = old
            break
        alpha = 1.0
        while True:
            udg, uh = o.update(udg, uh, x, a["DinvRu"], a["DinvF"], alpha, sh=sh)
            rnorm = o.residual(udg, uh, sh=sh)
            if not np.isfinite(rnorm) or (rnorm > old and rnorm > tol):
                alpha = -abs(alpha / 2)
                if abs(alpha) < 1e-4:
                    if robust == 0:
                        robust = 1
                        alpha = -2 * abs(alpha)
                        udg, uh = o.update(udg, uh, x, a["DinvRu"], a["DinvF"], alpha, sh=sh)
                    break
            else:
                break
    hist.append(rnorm)
    return udg, uh, rnorm < tol, hist


def dirk_step(prob, udg, uh, sh, dt, stages=3, order=3, tol=1e-10, maxiter=10):
    """One step of solveUnsteadyProblem (solvers/dgsolvers.cpp:280-420) on the oracle."""
    d, t = dirk_table(stages, order)
    ncu = prob.ncu
    udgi = udg.copy()
    for s in range(stages):
        if s == 0:
            sh = (d[0, 0] / dt) * udgi
        elif s == 1:
            sh = ((d[1, 0] + d[1, 1]) / dt) * udgi - udg * d[1, 0] / dt
        else:
            sh = (((d[2, 0] + d[2, 1] + d[2, 2]) / dt) * udgi
                  - (d[2, 0] / d[1, 0]) * ((d[1, 0] + d[1, 1]) * udgi / dt - sh) - udg * d[2, 1] / dt)
        sh = sh.copy()
        sh[:, ncu:, :] = 0.0
        prob.fc_u = d[s, s] / dt
        prob.fc_q = 1.0
        prob.tdep = 1
        o = Oracle(prob)
        udg, uh, conv, _ = newton_solve(o, udg, uh, sh, tol, maxiter)
        if not conv:
            raise RuntimeError(f"DIRK stage {s + 1} did not converge")
    return udg, uh, sh


def run_reference(prob, mode="assemble", ndump=0, newton=None, workdir=None):
    """Run the compiled reference on ``prob`` and load its dumps."""
    from hfem_b200.gen.refio import write_inputs

    if not os.path.exists(REF_BIN):
        raise FileNotFoundError("reference oracle not built (make -C oracle with the reference tree)")
    tmp = workdir or tempfile.mkdtemp(prefix="hfemref_")
    inp = os.path.join(tmp, "in_")
    out = os.path.join(tmp, "out_")
    kw = {}
    if newton is not None:
        kw = dict(newton_maxiter=newton["maxiter"], gmres_tol=newton["tol"])
    if mode == "dirk":
        kw.update(dirk_stage=newton["stages"], dirk_order=newton["order"], dt_list=[newton["dt"]],
                  newton_tol=newton["newton_tol"])
    write_inputs(inp, prob, **kw)
    if mode == "assemble":
        cmd = [REF_BIN, "assemble", inp, out, str(ndump)]
    elif mode == "dirk":
        cmd = [REF_BIN, "dirk", inp, out, str(newton["nsteps"]), str(newton["precond"]), str(newton["restart"]),
               repr(newton["tol"])]
    else:
        cmd = [REF_BIN, "newton", inp, out, str(newton["maxiter"]), str(newton["precond"]),
               str(newton["restart"]), repr(newton["tol"])]
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL, env=env)

    def ld(name):
        return np.fromfile(out + name + ".bin", dtype=np.float64)

    if mode == "assemble":
        res = {k: ld(k) for k in ("udg", "Hg", "Rg", "Rr", "DinvRu", "DinvF")}
        res["rnorm"] = float(ld("rnorm")[0])
        if ndump:
            for k in ("eD", "eF", "eK", "eH", "eRu", "eRh"):
                res[k] = ld(k)
        return res
    if mode == "dirk":
        return {"udg_steps": ld("udg_steps").reshape(newton["nsteps"] + 1, *prob.udg.shape)}
    return {k: ld(k) for k in ("udg", "uh", "rnorm_hist", "gmres_iters", "gmres_hist")}

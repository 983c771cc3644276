"""Many independent HDG problems in one GPU context.

Problems of the same element shape are packed into a disjoint-union mesh:
elements, faces and face-block rows are concatenated with offsets, so one
assembly launch covers every problem's elements and the owner-gather scatter
keeps each problem's blocks apart (the union system is block diagonal).  Each
problem keeps its own physics (``hfem_set_problem_map``), residual norm and
line-search step.  The reference runs one problem per process; this packing
is what lets element work of many requests share the GPU.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import replace

import numpy as np

from .core import HDGSolver, load_library
from .gen.mesh import Mesh
from .gen.problem import Problem

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def union_problem(probs: list) -> tuple:
    """Disjoint union of problems sharing one master element.

    Returns (union Problem, eprob, fprob, params (nprob x 8), element offsets,
    trace-dof offsets)."""
    m = probs[0].master
    for p in probs:
        if (p.master.nd, p.master.porder, p.master.ngv) != (m.nd, m.porder, m.ngv):
            raise ValueError("all problems in a union must share the master element")
        if getattr(p, "appname", 1) != getattr(probs[0], "appname", 1):
            raise ValueError("all problems in a union must solve the same equations")
        if (getattr(p, "conv_stab", 0), getattr(p, "viscosity_model", 0)) != \
                (getattr(probs[0], "conv_stab", 0), getattr(probs[0], "viscosity_model", 0)):
            raise ValueError("all problems in a union must share the stabilization tensor and viscosity model")
    npf = m.npf
    eoff = np.cumsum([0] + [p.mesh.ne for p in probs])
    foff = np.cumsum([0] + [p.mesh.nf for p in probs])
    boff = np.cumsum([0] + [int(p.mesh.rowstart[-1]) for p in probs])
    dg = np.concatenate([p.mesh.dgnodes for p in probs])
    elcon = np.concatenate([p.mesh.elcon + foff[i] * npf for i, p in enumerate(probs)])
    t2f = np.concatenate([p.mesh.t2f + foff[i] for i, p in enumerate(probs)])
    t2t = np.concatenate([p.mesh.t2t + eoff[i] for i, p in enumerate(probs)])
    rs = np.concatenate([[0]] + [p.mesh.rowstart[1:] + boff[i] for i, p in enumerate(probs)])
    ci = np.concatenate([p.mesh.colidx + foff[i] for i, p in enumerate(probs)])
    fe = np.concatenate([p.mesh.face_elems + eoff[i] for i, p in enumerate(probs)])
    fv = np.concatenate([p.mesh.face_verts for p in probs])
    tt = np.concatenate([p.mesh.t for p in probs])
    # boundary flags: each problem's boundary indices shifted past the earlier problems'
    bfl, bcm, bcs, nbnd = [], [], [], 0
    for i, p in enumerate(probs):
        pb = getattr(p, "bcm", None)
        bfi = np.where(p.mesh.bf < 0, p.mesh.bf - nbnd, p.mesh.bf + eoff[i])
        bfl.append(bfi)
        if pb is not None:
            bcm.extend(int(x) for x in pb)
            bcs.append(np.asarray(p.bcs, dtype=np.float64))
            nbnd += len(pb)
    bf = np.concatenate(bfl)
    mesh = Mesh(nd=m.nd, ne=int(eoff[-1]), nf=int(foff[-1]), nv=0, npv=m.npv, npf=npf, nfe=m.nfe, dgnodes=dg,
                t=tt, t2f=t2f, t2t=t2t, bf=bf, elcon=elcon, face_verts=fv, face_elems=fe, rowstart=rs,
                colidx=ci)
    eprob = np.repeat(np.arange(len(probs)), [p.mesh.ne for p in probs]).astype(np.int32)
    fprob = np.repeat(np.arange(len(probs)), [p.mesh.nf for p in probs]).astype(np.int32)
    params = np.array([[*p.param, float(p.tdep), p.fc_u] for p in probs], dtype=np.float64)
    u = replace(probs[0], name="union", mesh=mesh, udg=np.concatenate([p.udg for p in probs]),
                uh=np.concatenate([p.uh for p in probs]), sh=np.concatenate([p.sh for p in probs]),
                bcm=np.array(bcm, dtype=np.int64) if bcm else None,
                bcs=np.concatenate(bcs) if bcs else None)
    return u, eprob, fprob, params, eoff, foff * npf


class BatchSolver:
    """Newton iterations for a set of problems packed into one context."""

    def __init__(self, probs: list, device: int = 0, stream: int | None = None):
        self.probs = probs
        t0 = time.perf_counter()
        self.union, self.eprob, self.fprob, self.params, self.eoff, self.hoff = union_problem(probs)
        t1 = time.perf_counter()
        self.s = HDGSolver(self.union, device=device)
        self.build_times = {"repack_union": t1 - t0, "repack_context": time.perf_counter() - t1}
        if stream is not None:
            self.s.set_stream(stream)
        lib = load_library()
        lib.hfem_set_problem_map.argtypes = [C.c_void_p, C.c_int, _ip, _ip, _dp]
        lib.hfem_problem_rnorms.argtypes = [C.c_void_p, _dp]
        lib.hfem_update_problems.argtypes = [C.c_void_p, _dp]
        lib.hfem_gmres_problems.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, _ip, _ip]
        self.lib = lib
        rc = lib.hfem_set_problem_map(self.s.h, len(probs), self.eprob.ctypes.data_as(_ip),
                                      self.fprob.ctypes.data_as(_ip), self.params.ctypes.data_as(_dp))
        self.s._chk(rc, "set_problem_map")
        self.n = len(probs)
        self.phases = {"assemble": 0.0, "gmres": 0.0, "gmres_iterations": 0, "line_search": 0.0}

    def close(self):
        self.s.close()

    def rnorms(self):
        out = np.zeros(self.n)
        self.s._chk(self.lib.hfem_problem_rnorms(self.s.h, out.ctypes.data_as(_dp)), "problem_rnorms")
        return out

    def update(self, alpha):
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        self.s._chk(self.lib.hfem_update_problems(self.s.h, a.ctypes.data_as(_dp)), "update_problems")

    def gmres(self, precond=2, restart=50, tol=1e-10, maxit=1000):
        """Per-problem GMRES (hfem_gmres_problems); returns (conv, iters) arrays."""
        conv = np.zeros(self.n, dtype=np.int32)
        its = np.zeros(self.n, dtype=np.int32)
        self.s._chk(self.lib.hfem_gmres_problems(self.s.h, precond, restart, tol, maxit, conv.ctypes.data_as(_ip),
                                                 its.ctypes.data_as(_ip)), "gmres_problems")
        return conv, its

    def newton_iteration(self, tol, active, gmres_tol=1e-12, restart=50, alpha_min=1e-4):
        """One iteration of solveNonlinearProblem (dgsolvers.cpp:106-205) for every
        problem with active[p]; returns (old norms, new norms)."""
        t0 = time.perf_counter()
        self.s.assembleLinearSystem()
        old = self.rnorms()
        t1 = time.perf_counter()
        conv, its = self.gmres(precond=2, restart=restart, tol=gmres_tol)
        t2 = time.perf_counter()
        self.phases["assemble"] += t1 - t0
        self.phases["gmres"] += t2 - t1
        self.phases["gmres_iterations"] += int(its.max())
        step = np.where(active & (old >= tol), 1.0, 0.0)       # the line search's incremental steps
        alpha = step.copy()
        new = old.copy()
        todo = step > 0
        while np.any(todo):
            self.update(np.where(todo, alpha, 0.0))
            self.s.computeResidualNorm()
            r = self.rnorms()
            new = np.where(todo, r, new)
            bad = todo & (~np.isfinite(r) | ((r > old) & (r > tol)))
            a = np.abs(alpha) / 2
            alpha = np.where(bad, -a, 0.0)
            todo = bad & (a >= alpha_min)
        self.phases["line_search"] += time.perf_counter() - t2
        return old, new

    def state(self, i):
        udg, uh = self.s.get_solution()
        e0, e1 = self.eoff[i], self.eoff[i + 1]
        h0, h1 = self.hoff[i], self.hoff[i + 1]
        return udg[e0:e1], uh[h0:h1]

"""Domain decomposition of one HDG problem over several GPUs (one rank per GPU).

The reference's MPI path (digasopar) partitions the elements, assembles each
part's element blocks locally, exchanges the face blocks of the faces on part
interfaces (assembly/globalassembly.cpp:946-979, 1045-1057), solves with a
GMRES whose dot products are all-reduced (solvers/pDLAK.cpp:322-357) and keeps
the trace increments of interface faces consistent in the update
(solvers/solutionupdate.cpp:113-178).  This module restates that scheme on top
of the single-GPU path:

* :func:`partition` cuts the mesh into slabs of elements along one axis.
  Each part is a complete local problem (its elements, every face they touch,
  the face-block CSR over those faces), so the local GPU assembly is the
  unchanged single-GPU kernel sequence.  A face on a part interface appears
  in both parts; each part's row holds only its own elements' contributions
  (the system is "subassembled": the global row is the sum of the parts').
  The lower rank owns an interface face: only the owner counts it in dot
  products and norms.
* :class:`DDSolver` runs the solver chain with a :class:`Exchange` (sums of
  interface-face values between neighbours and all-reduces of scalars through
  ``torch.distributed``: NCCL over NVLink on GPUs, gloo on CPU).  After the
  local assembly it sums the interface rows of the right-hand side, the
  residual vector and the diagonal blocks (block Jacobi); every GMRES matvec is
  the local block matvec followed by the interface sum; dot products are local
  over owned faces, then all-reduced.  Every rank therefore holds the same
  values on a shared face and takes the same GMRES and Newton decisions.

The local work goes through a backend (``assemble``, ``matvec``, ``update``,
``residual`` and the assembled arrays): :class:`GPUBackend` is the C ABI on
the rank's GPU; tests supply a CPU backend.  Interface traffic per matvec is
one block row segment per interface face; no TMA or multicast is involved.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np
import torch

from .gen.mesh import Mesh
from .gen.problem import Problem


@dataclass
class Part:
    rank: int
    nparts: int
    prob: Problem                # the local problem: local elements, the faces they touch
    elems: np.ndarray            # local element -> global element
    faces: np.ndarray            # local face -> global face (increasing)
    owned: np.ndarray            # per local face: this rank counts it in dot products and norms
    shared: dict                 # neighbour rank -> local faces shared with it (increasing global id)


def element_parts(prob: Problem, nparts: int, axis: int = 0) -> np.ndarray:
    """Part of every element: slabs of equal element counts ordered by the
    element centroid along ``axis`` (ties broken by element id)."""
    cen = prob.mesh.dgnodes[:, axis, :].mean(axis=1)
    order = np.lexsort((np.arange(prob.mesh.ne), cen))
    part = np.empty(prob.mesh.ne, dtype=np.int64)
    for r, chunk in enumerate(np.array_split(order, nparts)):
        part[chunk] = r
    return part


def partition(prob: Problem, nparts: int, rank: int, axis: int = 0) -> Part:
    """The local problem of ``rank`` among ``nparts`` slabs (see the module doc)."""
    me, m = prob.mesh, prob.master
    npf, nfe = m.npf, m.nfe
    part = element_parts(prob, nparts, axis)
    elems = np.nonzero(part == rank)[0]
    faces = np.unique(me.t2f[elems])
    g2l = np.full(me.nf, -1, dtype=np.int64)
    g2l[faces] = np.arange(faces.size)
    # the parts every face touches (a face has one or two elements)
    fparts = [set() for _ in range(me.nf)]
    for e in range(me.ne):
        for f in me.t2f[e]:
            fparts[f].add(int(part[e]))
    owner = np.array([min(s) for s in fparts], dtype=np.int64)
    owned = owner[faces] == rank
    shared = {}
    for lf, gf in enumerate(faces):
        for s in fparts[gf]:
            if s != rank:
                shared.setdefault(s, []).append(lf)
    shared = {s: np.array(v, dtype=np.int64) for s, v in sorted(shared.items())}

    t2f = g2l[me.t2f[elems]]
    elcon = g2l[me.elcon[elems] // npf] * npf + me.elcon[elems] % npf
    e2l = np.full(me.ne, -1, dtype=np.int64)
    e2l[elems] = np.arange(elems.size)
    t2t = np.where(me.t2t[elems] >= 0, e2l[np.maximum(me.t2t[elems], 0)], me.t2t[elems])
    bf = np.where(me.bf[elems] < 0, me.bf[elems], np.maximum(t2t, 0))
    fe = me.face_elems[faces]
    face_elems = np.where(fe >= 0, e2l[np.maximum(fe, 0)], -1)
    face_elems = np.sort(np.where(face_elems < 0, np.iinfo(np.int64).max, face_elems), axis=1)
    face_elems = np.where(face_elems == np.iinfo(np.int64).max, -1, face_elems)
    # face-block CSR over the local faces: diagonal first, then ascending
    rows = [set() for _ in range(faces.size)]
    for fs in t2f:
        for a in fs:
            rows[a].update(int(b) for b in fs)
    rowstart = np.zeros(faces.size + 1, dtype=np.int64)
    cols = []
    for i in range(faces.size):
        cols.append(i)
        cols.extend(sorted(rows[i] - {i}))
        rowstart[i + 1] = len(cols)
    mesh = Mesh(nd=me.nd, ne=elems.size, nf=faces.size, nv=me.nv, npv=me.npv, npf=npf, nfe=nfe,
                dgnodes=np.ascontiguousarray(me.dgnodes[elems]), t=me.t[elems], t2f=t2f, t2t=t2t, bf=bf,
                elcon=elcon, face_verts=me.face_verts[faces], face_elems=face_elems, rowstart=rowstart,
                colidx=np.array(cols, dtype=np.int64))
    uh = prob.uh.reshape(me.nf, npf, -1)[faces].reshape(faces.size * npf, -1)
    local = replace(prob, mesh=mesh, udg=np.ascontiguousarray(prob.udg[elems]), uh=np.ascontiguousarray(uh),
                    sh=np.ascontiguousarray(prob.sh[elems]), meta=dict(prob.meta, part=rank, nparts=nparts))
    return Part(rank=rank, nparts=nparts, prob=local, elems=elems, faces=faces, owned=owned, shared=shared)


class Exchange:
    """Interface sums and scalar all-reduces among the ranks of a process group."""

    def __init__(self, part: Part, bsz: int, device, group=None):
        self.part, self.bsz, self.group, self.device = part, bsz, group, device
        self.idx = {s: torch.as_tensor(v, device=device) for s, v in part.shared.items()}
        self.owned = torch.as_tensor(np.repeat(part.owned, bsz), device=device)

    def interface_sum(self, v: torch.Tensor, width: int = None) -> torch.Tensor:
        """v (faces x width, flattened) += the neighbours' values on shared faces."""
        import torch.distributed as dist
        w = width or self.bsz
        v2 = v.view(-1, w)
        if not self.idx:
            return v
        sends = {s: v2.index_select(0, i).contiguous() for s, i in self.idx.items()}
        recvs = {s: torch.empty_like(t) for s, t in sends.items()}
        ops = []
        for s in sorted(self.idx):
            ops.append(dist.P2POp(dist.isend, sends[s], s, group=self.group))
            ops.append(dist.P2POp(dist.irecv, recvs[s], s, group=self.group))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for s in sorted(self.idx):
            v2.index_add_(0, self.idx[s], recvs[s])
        return v

    def allreduce(self, x: torch.Tensor) -> torch.Tensor:
        import torch.distributed as dist
        dist.all_reduce(x, op=dist.ReduceOp.SUM, group=self.group)
        return x

    def dot(self, a: torch.Tensor, b: torch.Tensor) -> float:
        s = torch.sum(torch.where(self.owned, a * b, torch.zeros((), dtype=a.dtype, device=a.device))).reshape(1)
        return float(self.allreduce(s).item())


class DDSolver:
    """The solver chain of one rank over its part (see the module doc).  The
    backend holds the rank's local problem."""

    def __init__(self, part: Part, backend, exchange: Exchange):
        self.part, self.be, self.ex = part, backend, exchange
        self.bsz = part.prob.bsz

    # -- assembly: local pass, then interface sums
    def assemble(self) -> float:
        self.be.assemble()
        self.rg = self.ex.interface_sum(self.be.Rg().clone())
        self.minv = self._block_jacobi()
        return self._rnorm()

    def residual(self) -> float:
        self.be.residual()
        return self._rnorm()

    def _rnorm(self) -> float:
        rr = self.ex.interface_sum(self.be.Rr().clone())
        s = torch.sum(torch.where(self.ex.owned, rr * rr, torch.zeros((), dtype=rr.dtype, device=rr.device)))
        s = s + torch.sum(self.be.ru2())
        return float(np.sqrt(self.ex.allreduce(s.reshape(1)).item()))

    def _block_jacobi(self) -> torch.Tensor:
        """Inverses of the summed diagonal blocks (kernel/mkBlockJacobi.m)."""
        b = self.bsz
        diag = self.be.diag_blocks().reshape(-1, b * b).clone()     # (nf, b*b), column-major blocks
        diag = self.ex.interface_sum(diag.reshape(-1), width=b * b).view(-1, b, b)
        return torch.linalg.inv(diag.transpose(1, 2)).transpose(1, 2).contiguous()

    def _prec(self, v: torch.Tensor) -> torch.Tensor:
        b = self.bsz
        vb = v.view(-1, b, 1)
        # column-major blocks: y_i = M_i v_i with M_i[r + b c] at [i, c, r]
        return torch.bmm(self.minv.transpose(1, 2), vb).reshape(-1)

    def _op(self, v: torch.Tensor) -> torch.Tensor:
        """M^-1 A v with A the summed (global) system restricted to this part."""
        return self._prec(self.ex.interface_sum(self.be.matvec(v)))

    # -- restarted left-preconditioned GMRES with modified Gram-Schmidt
    # (kernel/gmres_bilu0.m:17-105 with block Jacobi), dots over owned faces
    def gmres(self, restart=50, tol=1e-10, maxit=1000):
        b = self._prec(self.rg)
        x = torch.zeros_like(b)
        nrmb = np.sqrt(self.ex.dot(b, b)) or 1.0
        hist, it, flag = [], 0, -2
        while flag == -2:
            r = b - self._op(x)
            beta = np.sqrt(self.ex.dot(r, r))
            if beta / nrmb <= tol:
                flag = 0
                break
            V = [r / beta]
            H = np.zeros((restart + 1, restart))
            cs, sn = np.zeros(restart), np.zeros(restart)
            g = np.zeros(restart + 1)
            g[0] = beta
            j = 0
            while j < restart:
                w = self._op(V[j])
                for i in range(j + 1):
                    H[i, j] = self.ex.dot(w, V[i])
                    w = w - H[i, j] * V[i]
                H[j + 1, j] = np.sqrt(self.ex.dot(w, w))
                nn = H[j + 1, j]
                for i in range(j):
                    a, c = H[i, j], H[i + 1, j]
                    H[i, j], H[i + 1, j] = cs[i] * a + sn[i] * c, -sn[i] * a + cs[i] * c
                rr = np.sqrt(H[j, j] * H[j, j] + H[j + 1, j] * H[j + 1, j])
                cs[j], sn[j] = H[j, j] / rr, H[j + 1, j] / rr
                H[j, j], H[j + 1, j] = rr, 0.0
                g[j + 1], g[j] = -sn[j] * g[j], cs[j] * g[j]
                it += 1
                hist.append(abs(g[j + 1]) / nrmb)
                j += 1
                if hist[-1] <= tol:
                    flag = 0
                    break
                if it >= maxit:
                    flag = 1
                    break
                if nn == 0.0:
                    flag = -1
                    break
                V.append(w / nn)
            y = np.zeros(j)
            for i in range(j - 1, -1, -1):
                y[i] = (g[i] - H[i, i + 1:j] @ y[i + 1:j]) / H[i, i]
            for i in range(j):
                x = x + float(y[i]) * V[i]
        self.x = x
        return (1 if flag == 0 else (0 if flag == 1 else -1)), np.array(hist)

    def update(self, alpha: float):
        self.be.update(self.x, alpha)

    # -- damped Newton with the reference's line search (dgsolvers.cpp:106-205)
    def newton(self, tol=1e-10, maxiter=10, restart=50, gmres_tol=1e-10):
        rnorm, it, robust, hist = tol + 1.0, 0, 0, []
        while rnorm > tol and it < maxiter:
            it += 1
            old = self.assemble()
            hist.append(old)
            conv, _ = self.gmres(restart=restart, tol=gmres_tol)
            if conv == -1:
                break
            if it == 1 and old < tol:
                rnorm = old
                break
            alpha = 1.0
            while True:
                self.update(alpha)
                rnorm = self.residual()
                if not np.isfinite(rnorm) or (rnorm > old and rnorm > tol):
                    alpha = -abs(alpha / 2)
                    if abs(alpha) < 1e-4:
                        if robust == 0:
                            robust = 1
                            alpha = -2 * abs(alpha)
                            self.update(alpha)
                        break
                else:
                    break
        hist.append(rnorm)
        return rnorm < tol, hist


class GPUBackend:
    """The rank's local problem on its GPU through the C ABI (one context)."""

    def __init__(self, prob: Problem, device: int):
        from .core import HDGSolver
        torch.cuda.set_device(device)
        self.s = HDGSolver(prob, device=device)
        self.s.getQ()
        self.nb = int(prob.mesh.rowstart[-1])
        self.bsz = prob.bsz
        self.rowstart = torch.as_tensor(prob.mesh.rowstart[:-1], device=f"cuda:{device}")

    def assemble(self):
        self.s.assembleLinearSystem()

    def residual(self):
        self.s.computeResidualNorm()

    def Rg(self):
        return self.s.device_tensor("Rg")

    def Rr(self):
        return self.s.device_tensor("Rr")

    def ru2(self):
        return self.s.device_tensor("ru2")

    def diag_blocks(self):
        b2 = self.bsz * self.bsz
        return self.s.device_tensor("Hg").view(-1, b2).index_select(0, self.rowstart)

    def matvec(self, v):
        return self.s.matvec(v)

    def update(self, x, alpha):
        self.s.set_step(x)
        self.s.updateSol(alpha)

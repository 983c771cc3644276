"""Simplex meshes of a box with HDG trace numbering, periodic or bounded.

Builds what the reference's front end builds for a periodic HDG mesh
(``preprocessing/digasopre.m:39-88``): ``t2f`` (``mkt2fmatlab.m``), the HDG
trace numbering ``elcon`` (``mkelconmatlab.m`` hdgelcon: the dofs of face
``i`` are ``i*npf + k`` with ``k`` the face node in the orientation of the
face's first element, and every other element's local face node maps to the
matching node), the periodic matching (``periodicmatlab.m``), and the
face-to-face block sparsity ``ent2ent`` (the reference's closed ``dmdserial``;
rows list the diagonal block first, as ``kernel/computeBILU0.m:15-17`` and
``kernel/mkBlockJacobi.m:10`` require).

Periodicity is handled topologically: vertex ids wrap modulo the grid size,
so faces on opposite sides of the box are the same face; coordinates in
``dgnodes`` stay unwrapped.  Grids need ``n >= 3`` cells per direction so
that distinct faces never share their wrapped vertex set.

Bounded meshes (``periodic=False``) keep the boundary faces with one element;
``bf`` of such an element face is ``-(ib + 1)`` with the side index
``ib = 2 * axis + end`` (``end`` 0 at coordinate 0, 1 at ``length``), the
reference's convention for ``mesh.bf`` (``elementassembly.cpp:1078-1103``:
``ib = -bf - 1``, boundary condition ``app.bcm[ib]``).

All arrays are 0-based and element-major (numpy C order), which is the
reference's column-major layout: ``dgnodes[e, d, n]`` is
``mesh.dgnodes[n + npv*(d + ncd*e)]``.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np

from .master import Master


@dataclass
class Mesh:
    nd: int
    ne: int
    nf: int
    nv: int
    npv: int
    npf: int
    nfe: int
    dgnodes: np.ndarray     # (ne, nd, npv) float64
    t: np.ndarray           # (ne, nd+1) wrapped vertex ids
    t2f: np.ndarray         # (ne, nfe)
    t2t: np.ndarray         # (ne, nfe)
    bf: np.ndarray          # (ne, nfe): >= 0 interior/periodic, < 0 boundary
    elcon: np.ndarray       # (ne, nfe*npf) global trace node ids
    face_verts: np.ndarray  # (nf, nd) canonical vertex order of each face
    face_elems: np.ndarray  # (nf, 2) first and second element of each face
    rowstart: np.ndarray    # (nf+1,) ent2entStart
    colidx: np.ndarray      # (nnz,)  ent2ent, diagonal first in each row

    @property
    def ndofuh(self):
        return self.nf * self.npf


def _square_tris(n: int, length: float, periodic: bool = True):
    h = length / n
    m = n if periodic else n + 1
    verts, wrapped = [], []
    for j in range(n):
        for i in range(n):
            v00, v10, v11, v01 = (i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1)
            for tri in ((v00, v10, v11), (v00, v11, v01)):
                verts.append([[h * a, h * b] for a, b in tri])
                wrapped.append([(a % m) + m * (b % m) for a, b in tri])
    return np.array(verts), np.array(wrapped, dtype=np.int64), m * m


def _cube_tets(n: int, length: float, periodic: bool = True):
    h = length / n
    m = n if periodic else n + 1
    base = []
    for perm in itertools.permutations(range(3)):
        p = [np.zeros(3, dtype=np.int64)]
        for ax in perm:
            q = p[-1].copy()
            q[ax] += 1
            p.append(q)
        x = np.array(p, dtype=np.float64)
        det = np.linalg.det(np.stack([x[1] - x[0], x[2] - x[0], x[3] - x[0]]))
        if det < 0:
            p[1], p[2] = p[2], p[1]
        base.append(p)
    verts, wrapped = [], []
    for k in range(n):
        for j in range(n):
            for i in range(n):
                off = np.array([i, j, k])
                for tet in base:
                    pts = [off + q for q in tet]
                    verts.append([[h * c for c in q] for q in pts])
                    wrapped.append([(q[0] % m) + m * ((q[1] % m) + m * (q[2] % m)) for q in pts])
    return np.array(verts), np.array(wrapped, dtype=np.int64), m ** 3


def _face_node_bary(master: Master):
    """Barycentric coordinates of the face master nodes over the face vertices."""
    s = master.plocfc
    lam = np.concatenate([1.0 - s.sum(axis=1, keepdims=True), s], axis=1)
    return lam                                   # (npf, nvf)


def build_mesh(master: Master, n: int, length: float, periodic: bool = True) -> Mesh:
    nd = master.nd
    if n < 3 and periodic:
        raise ValueError("periodic grids need at least 3 cells per direction")
    if n < 1:
        raise ValueError("need at least one cell per direction")
    if nd == 2:
        vcoord, t, nv = _square_tris(n, length, periodic)
    else:
        vcoord, t, nv = _cube_tets(n, length, periodic)
    ne = t.shape[0]
    nfe, npf, npv = master.nfe, master.npf, master.npv
    nvf = nd

    # dgnodes: affine map of the master nodes
    lam = np.concatenate([1.0 - master.plocvl.sum(axis=1, keepdims=True), master.plocvl], axis=1)
    dg = np.einsum("nv,evd->edn", lam, vcoord)           # (ne, nd, npv)

    # faces by wrapped vertex set, numbered by first appearance
    faces = np.array(master.faces)                       # (nfe, nvf)
    lv = t[:, faces].reshape(ne * nfe, nvf)              # local vertex ids per element face
    key = np.sort(lv, axis=1)
    _, first, inverse = np.unique(key, axis=0, return_index=True, return_inverse=True)
    inverse = inverse.ravel()
    order = np.argsort(first)
    rank = np.empty_like(order)
    rank[order] = np.arange(order.size)
    fid = rank[inverse]                                  # face id per element face
    nf = order.size
    if periodic and nf * 2 != ne * nfe:
        raise RuntimeError("periodic mesh is not closed (every face needs two elements)")
    face_first = first[order]                            # element-face index of the first owner
    canon = lv[face_first]                               # (nf, nvf)

    # node map for every vertex permutation sigma: local face node m -> canonical node k
    blam = _face_node_bary(master)                       # (npf, nvf)
    nodemap = {}
    for sigma in itertools.permutations(range(nvf)):
        lam_c = np.zeros_like(blam)
        lam_c[:, list(sigma)] = blam                     # local vertex i is canonical sigma[i]
        d = np.abs(lam_c[:, None, :] - blam[None, :, :]).sum(axis=2)
        k = np.argmin(d, axis=1)
        if np.max(d[np.arange(npf), k]) > 1e-12:
            raise RuntimeError("face node matching failed")
        nodemap[sigma] = k
    can_of = canon[fid]                                  # (ne*nfe, nvf)
    sig = np.argmax(lv[:, :, None] == can_of[:, None, :], axis=2)   # position of local vertex i in canonical
    elcon = np.empty((ne * nfe, npf), dtype=np.int64)
    for sigma, k in nodemap.items():
        mask = np.all(sig == np.array(sigma)[None, :], axis=1)
        elcon[mask] = fid[mask, None] * npf + k[None, :]
    if np.any(np.sort(sig, axis=1) != np.arange(nvf)[None, :]):
        raise RuntimeError("face vertex permutation invalid")

    t2f = fid.reshape(ne, nfe)
    elem_of = np.repeat(np.arange(ne), nfe)
    face_elems = np.full((nf, 2), -1, dtype=np.int64)
    face_elems[:, 0] = elem_of[face_first]
    second = np.ones(ne * nfe, dtype=bool)
    second[face_first] = False
    face_elems[fid[second], 1] = elem_of[second]
    t2t = np.where(face_elems[t2f, 0] == np.arange(ne)[:, None], face_elems[t2f, 1], face_elems[t2f, 0])
    if np.any(face_elems[t2f, 0] == face_elems[t2f, 1]):
        raise RuntimeError("an element meets itself across a face")
    bf = t2t.copy()
    if not periodic:
        # boundary element faces: side index from the face centroid
        cen = vcoord[:, faces, :].mean(axis=2)           # (ne, nfe, nd)
        for e, a in zip(*np.nonzero(t2t < 0)):
            c = cen[e, a]
            side = -1
            for ax in range(nd):
                if abs(c[ax]) < 1e-9 * length:
                    side = 2 * ax
                elif abs(c[ax] - length) < 1e-9 * length:
                    side = 2 * ax + 1
            if side < 0:
                raise RuntimeError("boundary face off the box")
            bf[e, a] = -(side + 1)

    # ent2ent: faces sharing an element with face i; diagonal first, rest ascending
    rows = [[] for _ in range(nf)]
    for e in range(ne):
        fs = t2f[e]
        for a in fs:
            rows[a].extend(int(b) for b in fs)
    rowstart = np.zeros(nf + 1, dtype=np.int64)
    cols = []
    for i in range(nf):
        others = sorted(set(rows[i]) - {i})
        cols.append(i)
        cols.extend(others)
        rowstart[i + 1] = len(cols)
    colidx = np.array(cols, dtype=np.int64)

    return Mesh(nd=nd, ne=ne, nf=nf, nv=nv, npv=npv, npf=npf, nfe=nfe, dgnodes=np.ascontiguousarray(dg),
                t=t, t2f=t2f, t2t=t2t, bf=bf, elcon=elcon.reshape(ne, nfe * npf),
                face_verts=canon, face_elems=face_elems, rowstart=rowstart, colidx=colidx)

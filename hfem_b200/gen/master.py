"""Master (reference) element tables for triangles and tetrahedra.

Follows ``preprocessing/mkmasterelement.m:1-144`` for what each table means:

* ``shapvl[i, g, d]``: Lagrange basis ``i`` at volume point ``g``; ``d = 0`` is
  the value, ``d = 1..nd`` the derivative w.r.t. reference coordinate ``d-1``.
* ``shapvt = shapvl^T`` (ngv, npv, nd+1), ``shapvg = shapvl * diag(w)``.
* ``shapvgdotshapvl[(jj + npv*ii), g, d] = shapvg[jj, g, d] * shapvl[ii, g, 0]``
  (``mkmasterelement.m:75-79``).
* face tables ``shapft/shapfg/shapfgdotshapfc`` likewise on the face master
  element with ``nd-1`` reference coordinates (``mkmasterelement.m:101-120``).
* ``perm[a][m]``: element node sitting at face node ``m`` of local face ``a``.

Node layouts: triangle nodes follow the reference's uniform layout
(``mkmasternodes.m`` trinodes2d: rows of constant ``eta``, ``xi`` fastest).
Local faces use the reference's vertex lists (triangle faces [2 3],[3 1],[1 2];
tetrahedron faces [2 3 4],[1 4 3],[1 2 4],[1 3 2], ``mkmasternodes.m``), whose
ordering makes ``facegeom`` normals point outward for positively oriented
elements.  Face node ``m`` with face reference coordinates ``s`` sits at
``v0 + sum_k s_k (v_{k+1} - v0)`` over the face's vertices.  The tetrahedron
node layout (layers of constant ``zeta``) is this project's own; the kernels
only rely on ``perm``.

Basis functions are built from a monomial Vandermonde matrix in coordinates
centred on the element centroid (adequate for p <= 4).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .quadrature import line_rule, simplex_rule

TRI_FACES = [(1, 2), (2, 0), (0, 1)]
TET_FACES = [(1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)]
TRI_VERTS = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
TET_VERTS = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])


def simplex_nodes(dim: int, p: int) -> np.ndarray:
    """Uniform Lagrange nodes on the reference simplex."""
    if dim == 1:
        return (np.arange(p + 1) / p).reshape(-1, 1)
    if dim == 2:
        pts = [(i / p, j / p) for j in range(p + 1) for i in range(p + 1 - j)]
        return np.array(pts, dtype=np.float64)
    pts = [(i / p, j / p, k / p)
           for k in range(p + 1) for j in range(p + 1 - k) for i in range(p + 1 - j - k)]
    return np.array(pts, dtype=np.float64)


def _exponents(dim, p):
    if dim == 1:
        return [(a,) for a in range(p + 1)]
    if dim == 2:
        return [(a, b) for t in range(p + 1) for a in range(t + 1) for b in [t - a]]
    return [(a, b, t - a - b) for t in range(p + 1) for a in range(t + 1) for b in range(t - a + 1)]


def lagrange_tables(dim: int, p: int, nodes: np.ndarray, pts: np.ndarray) -> np.ndarray:
    """Values and first derivatives of the nodal basis: (npe, npts, dim+1)."""
    exps = np.array(_exponents(dim, p), dtype=np.int64)
    centre = np.full(dim, 1.0 / (dim + 1))

    def mono(x, deriv):
        x = x - centre
        out = np.ones((x.shape[0], len(exps)))
        for k, e in enumerate(exps):
            for d in range(dim):
                ed = e[d]
                if deriv == d + 1:
                    if ed == 0:
                        out[:, k] = 0.0
                        break
                    out[:, k] *= ed * x[:, d] ** (ed - 1)
                else:
                    out[:, k] *= x[:, d] ** ed
        return out

    vand = mono(nodes, 0)                       # (npe, nmono)
    inv = np.linalg.inv(vand)                   # coefficients of each basis function
    tab = np.empty((nodes.shape[0], pts.shape[0], dim + 1))
    for d in range(dim + 1):
        tab[:, :, d] = (mono(pts, d) @ inv).T
    return tab


@dataclass
class Master:
    """Master element of one simplex type and order (masterstruct subset)."""

    nd: int
    porder: int
    pgauss: int
    npv: int
    npf: int
    nfe: int
    ngv: int
    ngf: int
    plocvl: np.ndarray
    plocfc: np.ndarray
    gpvl: np.ndarray
    gwvl: np.ndarray
    gpfc: np.ndarray
    gwfc: np.ndarray
    shapvl: np.ndarray          # (npv, ngv, nd+1)
    shapfc: np.ndarray          # (npf, ngf, nd)
    perm: np.ndarray            # (nfe, npf) int
    faces: list = field(default_factory=list)

    # --- tables in the reference's memory layouts (column-major flattening)
    @property
    def shapvt(self):           # ngv x npv x (nd+1)
        return np.transpose(self.shapvl, (1, 0, 2))

    @property
    def shapvg(self):           # npv x ngv x (nd+1)
        return self.shapvl * self.gwvl[None, :, None]

    @property
    def shapvgdotshapvl(self):  # (npv*npv) x ngv x (nd+1), row = jj + npv*ii
        g = self.shapvg                                  # [jj, q, d]
        v = self.shapvl[:, :, 0]                         # [ii, q]
        t = g[None, :, :, :] * v[:, None, :, None]       # [ii, jj, q, d]
        return t.reshape(self.npv * self.npv, self.ngv, self.nd + 1)

    @property
    def shapft(self):           # ngf x npf x nd
        return np.transpose(self.shapfc, (1, 0, 2))

    @property
    def shapfg(self):           # npf x ngf x nd
        return self.shapfc * self.gwfc[None, :, None]

    @property
    def shapfgdotshapfc(self):  # (npf*npf) x ngf x nd, row = jj + npf*ii
        g = self.shapfg
        v = self.shapfc[:, :, 0]
        t = g[None, :, :, :] * v[:, None, :, None]
        return t.reshape(self.npf * self.npf, self.ngf, self.nd)

    def fortran(self, name: str) -> np.ndarray:
        """Table flattened in column-major order, as the reference stores it."""
        return np.asfortranarray(getattr(self, name)).ravel(order="F")


def make_master(nd: int, porder: int, pgauss: int | None = None) -> Master:
    if pgauss is None:
        pgauss = max(2 * porder, 1)
    plocvl = simplex_nodes(nd, porder)
    plocfc = simplex_nodes(nd - 1, porder)
    gpvl, gwvl = simplex_rule(nd, pgauss)
    if nd == 2:
        gpfc, gwfc = line_rule(pgauss)
        faces, verts = TRI_FACES, TRI_VERTS
    else:
        gpfc, gwfc = simplex_rule(2, pgauss)
        faces, verts = TET_FACES, TET_VERTS
    shapvl = lagrange_tables(nd, porder, plocvl, gpvl)
    shapfc = lagrange_tables(nd - 1, porder, plocfc, gpfc)
    perm = np.empty((len(faces), plocfc.shape[0]), dtype=np.int64)
    for a, fv in enumerate(faces):
        v0 = verts[fv[0]]
        for m, s in enumerate(plocfc):
            x = v0.copy()
            for k in range(nd - 1):
                x = x + s[k] * (verts[fv[k + 1]] - v0)
            d = np.linalg.norm(plocvl - x[None, :], axis=1)
            idx = int(np.argmin(d))
            if d[idx] > 1e-12:
                raise RuntimeError("face node not found among element nodes")
            perm[a, m] = idx
    return Master(nd=nd, porder=porder, pgauss=pgauss, npv=plocvl.shape[0], npf=plocfc.shape[0],
                  nfe=len(faces), ngv=gpvl.shape[0], ngf=gpfc.shape[0], plocvl=plocvl,
                  plocfc=plocfc, gpvl=gpvl, gwvl=gwvl, gpfc=gpfc, gwfc=gwfc, shapvl=shapvl,
                  shapfc=shapfc, perm=perm, faces=[list(f) for f in faces])

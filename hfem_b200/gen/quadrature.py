"""Quadrature rules on the reference line, triangle and tetrahedron.

The reference picks its rules in ``master/gaussquad.m``:

* line ``[0,1]`` (``master/gaussquad1d.m:23-33``): Gauss-Legendre with
  ``ceil((pgauss-1)/2) + 1`` points (Golub-Welsch on the Legendre Jacobi
  matrix).  Note the count: the reference builds an ``(n+1) x (n+1)`` Jacobi
  matrix, so a degree-4 request gives 3 points.
* triangle (``master/gaussquad2d.m``): fully symmetric rules, 3/6/12/16 points
  for degrees 2/4/6/8 (weights sum to the reference area 1/2).
* tetrahedron (``master/gaussquad3d.m``): fully symmetric rules, 4 points for
  degree 2 and 24 points for degree 6 (weights sum to 1/6).

The symmetric simplex rules are not copied from any table: each is defined by
its orbit structure (the published Dunavant / Keast families) and its free
parameters are solved here from the moment equations (exact integration of
every monomial up to the rule's degree) by Gauss-Newton, starting from rough
literature estimates.  ``check_rule`` verifies exactness to 1e-14.
"""
from __future__ import annotations

import itertools
import math
from functools import lru_cache

import numpy as np


def gauss_legendre_01(npts: int):
    """Gauss-Legendre rule with ``npts`` points on [0, 1]."""
    x, w = np.polynomial.legendre.leggauss(npts)
    return 0.5 * (x + 1.0), 0.5 * w


def line_rule(pgauss: int):
    """Line rule used on the faces of 2D elements (gaussquad1d.m:23-33)."""
    n = int(math.ceil((pgauss - 1) / 2.0))
    x, w = gauss_legendre_01(n + 1)
    return x.reshape(-1, 1), w


# ---------------------------------------------------------------- simplex ---

def _orbit_points(kind: str, params, dim: int):
    """Barycentric points of one symmetry orbit."""
    if dim == 2:
        if kind == "S3":
            bary = [(1 / 3, 1 / 3, 1 / 3)]
        elif kind == "S21":
            a, = params
            base = (a, a, 1 - 2 * a)
            bary = sorted(set(itertools.permutations(base)))
        elif kind == "S111":
            a, b = params
            base = (a, b, 1 - a - b)
            bary = sorted(set(itertools.permutations(base)))
        else:
            raise ValueError(kind)
    else:
        if kind == "S4":
            bary = [(0.25, 0.25, 0.25, 0.25)]
        elif kind == "S31":
            a, = params
            base = (a, a, a, 1 - 3 * a)
            bary = sorted(set(itertools.permutations(base)))
        elif kind == "S22":
            a, = params
            base = (a, a, 0.5 - a, 0.5 - a)
            bary = sorted(set(itertools.permutations(base)))
        elif kind == "S211":
            a, b = params
            base = (a, a, b, 1 - 2 * a - b)
            bary = sorted(set(itertools.permutations(base)))
        else:
            raise ValueError(kind)
    return [tuple(p) for p in bary]


_NPARAM = {"S3": 0, "S21": 1, "S111": 2, "S4": 0, "S31": 1, "S22": 1, "S211": 2}
_NPTS = {"S3": 1, "S21": 3, "S111": 6, "S4": 1, "S31": 4, "S22": 6, "S211": 12}


def _assemble(structure, theta, dim):
    pts, wts = [], []
    k = 0
    for kind in structure:
        npar = _NPARAM[kind]
        params = theta[k:k + npar]
        k += npar
        w = theta[k]
        k += 1
        orb = _orbit_points(kind, params, dim)
        # sorted(set(...)) may merge points when parameters coincide; keep the
        # orbit size fixed by regenerating without set() in that case.
        if len(orb) != _NPTS[kind]:
            raise ValueError("degenerate orbit")
        for b in orb:
            pts.append(b[1:])          # reference coordinates = last dim barycentrics
            wts.append(w)
    return np.array(pts, dtype=np.float64), np.array(wts, dtype=np.float64)


def _monomials(dim, degree):
    out = []
    for tot in range(degree + 1):
        if dim == 2:
            for i in range(tot + 1):
                out.append((i, tot - i))
        else:
            for i in range(tot + 1):
                for j in range(tot - i + 1):
                    out.append((i, j, tot - i - j))
    return out


def _exact(mono):
    num = 1.0
    for e in mono:
        num *= math.factorial(e)
    return num / math.factorial(sum(mono) + len(mono))


def _moment_residual(structure, theta, dim, degree):
    pts, wts = _assemble(structure, theta, dim)
    res = []
    for mono in _monomials(dim, degree):
        val = np.sum(wts * np.prod(pts ** np.array(mono, dtype=np.float64), axis=1))
        res.append(val - _exact(mono))
    return np.array(res)


def _solve(structure, guess, dim, degree):
    theta = np.array(guess, dtype=np.float64)
    for _ in range(60):
        r = _moment_residual(structure, theta, dim, degree)
        if np.max(np.abs(r)) < 1e-16:
            break
        jac = np.empty((r.size, theta.size))
        for j in range(theta.size):
            h = 1e-7 * max(1.0, abs(theta[j]))
            tp = theta.copy()
            tp[j] += h
            tm = theta.copy()
            tm[j] -= h
            jac[:, j] = (_moment_residual(structure, tp, dim, degree)
                         - _moment_residual(structure, tm, dim, degree)) / (2 * h)
        step, *_ = np.linalg.lstsq(jac, -r, rcond=None)
        theta = theta + step
    return theta


# Orbit structures of the published symmetric families with rough starting
# parameters (barycentric orbit parameters, then the weight for unit measure
# scaled to the reference simplex measure below).
_TRI = {
    2: (["S21"], [1 / 6, 1 / 3]),
    4: (["S21", "S21"], [0.44, 0.22, 0.09, 0.11]),
    6: (["S21", "S21", "S111"], [0.25, 0.117, 0.063, 0.051, 0.053, 0.31, 0.083]),
    8: (["S3", "S21", "S21", "S21", "S111"],
        [0.144, 0.459, 0.095, 0.171, 0.103, 0.0505, 0.0325, 0.0084, 0.263, 0.0272]),
}
_TET = {
    2: (["S31"], [0.138, 0.25]),
    4: (["S31", "S31", "S22"], [0.0927, 0.0735, 0.311, 0.1127, 0.4545, 0.0425]),
    6: (["S31", "S31", "S31", "S211"],
        [0.2146, 0.0399, 0.0407, 0.0101, 0.3223, 0.0554, 0.0637, 0.2697, 0.0482]),
}


def _scale_weights(structure, guess, measure):
    g = list(guess)
    k = 0
    for kind in structure:
        k += _NPARAM[kind]
        g[k] *= measure
        k += 1
    return g


@lru_cache(maxsize=None)
def simplex_rule(dim: int, pgauss: int):
    """Symmetric rule exact to degree ``pgauss`` on the reference simplex."""
    table = _TRI if dim == 2 else _TET
    degree = max(pgauss, 1)
    cands = sorted(d for d in table if d >= degree)
    if not cands:
        raise ValueError(f"no {dim}D simplex rule for degree {pgauss}")
    d = cands[0]
    structure, guess = table[d]
    measure = 0.5 if dim == 2 else 1.0 / 6.0
    theta = _solve(structure, _scale_weights(structure, guess, measure), dim, d)
    pts, wts = _assemble(structure, theta, dim)
    err = np.max(np.abs(_moment_residual(structure, theta, dim, d)))
    if err > 1e-14:
        raise RuntimeError(f"{dim}D rule of degree {d} did not converge ({err:.2e})")
    if np.any(wts <= 0) or np.any(pts < -1e-14) or np.any(pts.sum(axis=1) > 1 + 1e-14):
        raise RuntimeError(f"{dim}D rule of degree {d} has points outside or negative weights")
    return pts, wts


def check_rule(pts, wts, dim, degree):
    """Max error over all monomials up to ``degree`` (0 for an exact rule)."""
    err = 0.0
    for mono in _monomials(dim, degree):
        val = np.sum(wts * np.prod(pts ** np.array(mono, dtype=np.float64), axis=1))
        err = max(err, abs(val - _exact(mono)))
    return err

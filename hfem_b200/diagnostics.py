"""Solution diagnostics shared by the GPU path and its checks.

``kinetic_energy`` integrates 1/2 rho |v|^2 over the mesh with the volume
quadrature of the master element (the Taylor-Green history of the DIRK
workload).  The reference has no kinetic-energy routine; both the GPU run and
its CPU check use this function on their own UDG.
"""
from __future__ import annotations

import numpy as np


def kinetic_energy(prob, udg: np.ndarray) -> float:
    m, me = prob.master, prob.mesh
    nd = m.nd
    phi = m.shapvl[:, :, 0]                          # (npv, ngv)
    dphi = m.shapvl[:, :, 1:]                        # (npv, ngv, nd)
    x = me.dgnodes                                   # (ne, nd, npv)
    J = np.einsum("edn,ngr->egdr", x, dphi)          # (ne, ngv, nd, nd)
    detJ = np.abs(np.linalg.det(J))                  # (ne, ngv)
    u = np.einsum("ecn,ng->egc", udg[:, :nd + 2, :], phi)
    rho = u[:, :, 0]
    mom = u[:, :, 1:nd + 1]
    ke = 0.5 * np.sum(mom * mom, axis=2) / rho
    return float(np.sum(ke * detJ * m.gwvl[None, :]))

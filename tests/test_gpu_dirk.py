"""GPU: DIRK(3,3) time stepping (solveUnsteadyProblem) against the oracle.

Small Taylor-Green problem (periodic [0, 2 pi]^3, 3^3 x 6 tetrahedra, p = 2,
Re 1600, Mach 0.1), two steps of dt = 0.01.  The kinetic-energy history
(diagnostics.kinetic_energy on each side's own UDG) must agree to 1e-9
relative, the final state to 1e-8 relative (Newton converged to 1e-10 on
both sides, so the states differ by the solver tolerance, not by rounding).
"""
import numpy as np
import pytest

from hfem_b200.core import HDGSolver
from hfem_b200.diagnostics import kinetic_energy
from hfem_b200.gen.problem import ns3d_tgv
from oracle import Oracle, dirk_step

pytestmark = pytest.mark.gpu


def test_dirk33_tgv_matches_oracle():
    dt, nsteps = 0.01, 2
    prob = ns3d_tgv(n=3, porder=2, dt=dt)
    o = Oracle(prob)
    udg = o.getq(prob.udg, prob.uh)
    uh = prob.uh.copy()
    sh = np.zeros_like(udg)
    ke_ref = [kinetic_energy(prob, udg)]
    for _ in range(nsteps):
        udg, uh, sh = dirk_step(prob, udg, uh, sh, dt, tol=1e-10)
        ke_ref.append(kinetic_energy(prob, udg))

    prob2 = ns3d_tgv(n=3, porder=2, dt=dt)
    s = HDGSolver(prob2)
    try:
        s.getQ()
        u0, _ = s.get_solution()
        ke = [kinetic_energy(prob2, u0)]
        for _ in range(nsteps):
            s.solveUnsteadyStep(dt, stages=3, order=3, newton_tol=1e-10)
            u, h = s.get_solution()
            ke.append(kinetic_energy(prob2, u))
    finally:
        s.close()
    ke, ke_ref = np.array(ke), np.array(ke_ref)
    assert np.max(np.abs(ke - ke_ref) / ke_ref) < 1e-9, (ke, ke_ref)
    assert np.max(np.abs(u - udg)) / np.max(np.abs(udg)) < 1e-8
    assert ke[-1] < ke[0]            # viscous decay

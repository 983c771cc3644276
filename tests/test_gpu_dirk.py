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


@pytest.mark.parametrize("precision", [0, 1, 2, 3], ids=["fp64", "mixed", "fp32_preconditioner", "split_tf32"])
def test_dirk33_tgv_p3_20_steps_match_reference_driver(precision):
    """The Taylor-Green DIRK workload at the size the reference finishes in
    minutes: 4^3 x 6 tetrahedra, p = 3, DIRK(3,3), 20 steps of dt = 0.01, each
    stage solved by Newton to 1e-10.  The fixture holds the kinetic-energy
    history of the reference's own driver (solveUnsteadyProblem, made by
    tests/golden/make_golden.py).  Mixed precision: FP32 block-Jacobi inverses
    with the 3xTF32 element contractions and the TF32 condensation GEMMs (mode
    1), the FP32 inverses alone with the FP64 Jacobian (mode 2, the precision of
    the Taylor-Green workload), or the FP32 inverses with the 3xTF32 element
    contractions (mode 3), with FP64 residuals, Arnoldi and Newton updates in all.  Bar: kinetic energy within 1e-9 relative at every step;
    final state within 1e-8 of the reference's (both converged to 1e-10)."""
    import os
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "tgv_p3_n4_dirk20.npz")))
    dt, nsteps = float(g["dt"][0]), int(g["nsteps"][0])
    prob = ns3d_tgv(n=int(g["n"][0]), porder=int(g["porder"][0]), dt=dt)
    s = HDGSolver(prob)
    try:
        s.set_precision(precision)
        s.getQ()
        u, _ = s.get_solution()
        ke, iters = [kinetic_energy(prob, u)], 0
        for _ in range(nsteps):
            iters += s.solveUnsteadyStep(dt, stages=3, order=3, newton_tol=1e-10)
            u, _ = s.get_solution()
            ke.append(kinetic_energy(prob, u))
    finally:
        s.close()
    ke = np.array(ke)
    err = float(np.max(np.abs(ke - g["ke"]) / g["ke"]))
    print(f"TGV 4^3x6 p3, {nsteps} DIRK(3,3) steps, precision {precision}: {iters} Newton iterations, "
          f"kinetic-energy rel err {err:.2e}")
    assert err < 1e-9, (ke, g["ke"])
    p = np.random.default_rng(20261203).standard_normal((8, u.size))
    d = float(np.max(np.abs(p @ u.ravel() - g["udg_final_proj"])))
    assert d <= 1e-8 * g["udg_final_absmax"][0] * np.sqrt(u.size), d

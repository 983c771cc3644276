"""Euler equations (app.appname 0) on the GPU against the oracle, whose Euler
form is pinned to the reference's own q-free Euler discretisation by the golden
fixture euler2d_channel_p2_n3.

* Element blocks, Hg, DinvF within 1e-12 relative, residual vectors within
  1e-12 of their scale, periodic and bounded, 2D and 3D.
* Newton on a bounded Euler problem converges to 1e-10.
"""
import numpy as np
import pytest

from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import as_euler, ns2d_channel, ns2d_vortex, ns3d_box, ns3d_fourier
from oracle import Oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("2d_p2_periodic", lambda: as_euler(ns2d_vortex(n=4, porder=2))),
    ("2d_p3_channel", lambda: as_euler(ns2d_channel(n=3, porder=3, bcm=(1, 6, 7, 2)))),
    ("3d_p1_periodic", lambda: as_euler(ns3d_fourier(n=3, porder=1))),
    ("3d_p2_box", lambda: as_euler(ns3d_box(n=2, porder=2, bcm=(1, 1, 7, 7, 2, 6)))),
]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_euler_assembly_matches_oracle(name, make):
    p = make()
    o = Oracle(p)
    uq = o.getq(p.udg, p.uh)
    ref = o.assemble(uq, p.uh, elem_blocks=True)
    s = HDGSolver(p)
    s.set_solution(uq, p.uh, p.sh)
    rn = s.assembleLinearSystem()
    assert abs(rn - ref["rnorm"]) <= 1e-12 * ref["rnorm"]
    assert rel(s.download("H"), ref["eH"]) < 1e-12
    assert rel(s.download("Hg"), ref["Hg"]) < 1e-12
    assert rel(s.download("DinvF"), ref["DinvF"]) < 1e-12
    assert np.max(np.abs(s.download("Rg") - ref["Rg"])) <= 1e-12 * max(np.max(np.abs(ref["Rg"])), 1.0)
    s.close()


def test_euler_newton_converges():
    p = as_euler(ns2d_channel(n=6, porder=2, bcm=(1, 1, 7, 7)))
    s = HDGSolver(p)
    s.getQ()
    conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, gmres_tol=1e-12)
    s.close()
    assert conv == 1 and hist[-1] < 1e-10, hist

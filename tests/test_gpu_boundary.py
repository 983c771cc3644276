"""Bounded meshes on the GPU against the oracle (whose boundary rows are pinned
to the reference's fbou.cpp by the golden fixtures).

* Element blocks, Hg, Rg, Rr, DinvF within 1e-12 relative, rnorm 1e-12, for
  2D p1-p3 and 3D p1-p2 with free-stream far field, Dirichlet, extrapolation,
  slip and no-slip adiabatic walls.
* Newton on a bounded channel converges to 1e-10; packed with a periodic
  problem, a bounded problem assembles as it does alone.
"""
import numpy as np
import pytest

from hfem_b200.batch import BatchSolver
from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_channel, ns2d_vortex, ns3d_box
from oracle import Oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("2d_p1", lambda: ns2d_channel(n=4, porder=1)),
    ("2d_p2", lambda: ns2d_channel(n=4, porder=2, bcm=(2, 2, 5, 6))),
    ("2d_p3", lambda: ns2d_channel(n=3, porder=3)),
    ("3d_p1", lambda: ns3d_box(n=2, porder=1)),
    ("3d_p2", lambda: ns3d_box(n=2, porder=2)),
    ("2d_p2_farfield", lambda: ns2d_channel(n=4, porder=2, bcm=(1, 1, 1, 1))),
    ("3d_p1_farfield", lambda: ns3d_box(n=2, porder=1, bcm=(1, 1, 2, 7, 1, 5))),
]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_bounded_assembly_matches_oracle(name, make):
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
    scale = max(np.max(np.abs(ref["Rg"])), 1.0)
    assert np.max(np.abs(s.download("Rg") - ref["Rg"])) <= 1e-12 * scale
    assert np.max(np.abs(s.download("Rr") - ref["Rr"])) <= 1e-12 * max(np.max(np.abs(ref["Rr"])), 1.0)
    s.close()


def test_bounded_newton_converges():
    p = ns2d_channel(n=6, porder=2)
    s = HDGSolver(p)
    s.getQ()
    conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, gmres_tol=1e-12)
    s.close()
    assert conv == 1 and hist[-1] < 1e-10, hist


def test_bounded_problem_packed_with_periodic():
    probs = [ns2d_channel(n=4, porder=2, seed=3), ns2d_vortex(n=4, porder=2, seed=4),
             ns2d_channel(n=3, porder=2, seed=5, bcm=(6, 5, 2, 7))]
    b = BatchSolver(probs)
    b.s.getQ()
    b.s.assembleLinearSystem()
    rn = b.rnorms()
    for i, p in enumerate(probs):
        s = HDGSolver(p)
        s.getQ()
        r = s.assembleLinearSystem()
        assert abs(rn[i] - r) <= 1e-12 * r, (i, rn[i], r)
        s.close()
    b.close()

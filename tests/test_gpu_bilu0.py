"""BILU0 with the MDF ordering on the GPU against the oracle's restatement.

* The ordering (an integer permutation) is bit-exact.
* GMRES(50) with BILU0 to 1e-10: same iteration count (+-1) and solution
  within 1e-8 relative; the first residual estimates agree to 1e-9.
* Newton with BILU0 converges to the FP64 residual tolerance.

Block sizes up to 32 with short levels (the MDF order's) run the one-CTA
factorisation and solves; block size 50 the per-level launches.
"""
import numpy as np
import pytest

from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_channel, ns2d_vortex, ns3d_box, ns3d_fourier, with_models
from oracle import Oracle

pytestmark = pytest.mark.gpu

CASES = [("2d_p2", lambda: ns2d_vortex(n=5, porder=2, seed=4)),
         ("2d_p3", lambda: ns2d_vortex(n=4, porder=3, seed=5)),
         ("3d_p1", lambda: ns3d_fourier(n=3, porder=1, seed=6)),
         # bounded meshes (face blocks of boundary faces have fewer neighbours)
         ("2d_p2_channel", lambda: ns2d_channel(n=4, porder=2, seed=7)),
         ("2d_p2_channel_roe_sutherland", lambda: with_models(ns2d_channel(n=4, porder=2, seed=9), 2, 1)),
         ("3d_p1_box", lambda: ns3d_box(n=2, porder=1)),
         # block size 50: the per-level launches (the one-CTA forms take blocks up to 32)
         ("3d_p3_box", lambda: ns3d_box(n=2, porder=3))]


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_bilu0_matches_oracle(name, make):
    p = make()
    o = Oracle(p)
    uq = o.getq(p.udg, p.uh)
    ref = o.assemble(uq, p.uh)
    o2u, u2o = o.mdf_ordering(ref["Hg"])
    Mg = o.bilu0_factor(ref["Hg"], o2u, u2o)
    x_ref, flag, hist_ref = o.gmres_bilu0(ref["Hg"], Mg, o2u, u2o, ref["Rg"], restart=50, tol=1e-10)
    s = HDGSolver(p)
    s.set_solution(uq, p.uh, p.sh)
    s.assembleLinearSystem()
    conv, hist = s.gmres(precond=0, restart=50, tol=1e-10)
    assert np.array_equal(s.ordering(), o2u)
    x = s.download("x")
    s.close()
    assert conv == 1 and flag == 0
    assert abs(len(hist) - len(hist_ref)) <= 1
    k = min(5, len(hist), len(hist_ref))
    assert np.allclose(hist[:k], hist_ref[:k], rtol=1e-9, atol=0)
    assert np.max(np.abs(x - x_ref)) <= 1e-8 * np.max(np.abs(x_ref))


def test_bilu0_newton_converges():
    p = ns2d_vortex(n=6, porder=2, seed=8)
    s = HDGSolver(p)
    s.getQ()
    conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=10, precond=0, gmres_tol=1e-10)
    s.close()
    assert conv == 1 and hist[-1] < 1e-10

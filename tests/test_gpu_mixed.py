"""Mixed-precision assembly (TF32 tensor-core Schur GEMMs) against the FP64 path.

* The residual norm is computed from FP64 residuals in both modes and agrees
  to 1e-13 relative.
* The condensed blocks Hg and DinvF carry TF32 rounding (unit roundoff 2^-11
  on the operands, FP32 accumulation): max |mixed - FP64| <= 1e-2 max |FP64|.
* Newton with the mixed Jacobian still converges to the FP64 residual
  tolerance 1e-10 (the FP64 residual drives the iteration).
"""
import numpy as np
import pytest

from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_vortex, ns3d_fourier

pytestmark = pytest.mark.gpu

CASES = [
    ("2d_p1", lambda: ns2d_vortex(n=4, porder=1)),
    ("2d_p2", lambda: ns2d_vortex(n=4, porder=2)),
    ("2d_p3", lambda: ns2d_vortex(n=3, porder=3)),
    ("2d_p4", lambda: ns2d_vortex(n=3, porder=4)),
    ("3d_p1", lambda: ns3d_fourier(n=3, porder=1)),
    ("3d_p2", lambda: ns3d_fourier(n=3, porder=2)),
    ("3d_p3", lambda: ns3d_fourier(n=3, porder=3)),
]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_mixed_blocks_close_to_fp64(name, make):
    prob = make()
    s = HDGSolver(prob)
    s.getQ()
    r64 = s.assembleLinearSystem()
    Hg64, DF64 = s.download("Hg"), s.download("DinvF")
    s.set_precision(1)
    r32 = s.assembleLinearSystem()
    Hg32, DF32 = s.download("Hg"), s.download("DinvF")
    s.close()
    assert abs(r32 - r64) <= 1e-13 * r64
    assert rel(Hg32, Hg64) < 1e-2, rel(Hg32, Hg64)
    assert rel(DF32, DF64) < 1e-2, rel(DF32, DF64)
    assert rel(Hg32, Hg64) > 0.0          # the tensor-core path really ran


@pytest.mark.parametrize("name,make", [CASES[1], CASES[6]], ids=["2d_p2", "3d_p3"])
def test_mixed_newton_reaches_fp64_tolerance(name, make):
    prob = make()
    s = HDGSolver(prob)
    s.set_precision(1)
    s.getQ()
    conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, gmres_tol=1e-10)
    s.close()
    assert conv == 1 and hist[-1] < 1e-10, hist


def test_mixed_gmres_reaches_tolerance_with_fp32_preconditioner():
    prob = ns3d_fourier(n=3, porder=2)
    s = HDGSolver(prob)
    s.getQ()
    s.assembleLinearSystem()
    c64, h64 = s.gmres(precond=2, restart=50, tol=1e-10)
    x64 = s.download("x")
    s.set_precision(1)
    s.assembleLinearSystem()
    c32, h32 = s.gmres(precond=2, restart=50, tol=1e-10)
    x32 = s.download("x")
    s.close()
    assert c64 == 1 and c32 == 1
    # the mixed system differs from the FP64 one by TF32 rounding, not by the preconditioner
    assert rel(x32, x64) < 1e-2


def test_mixed_newton_with_fp32_bilu0_factors():
    """BILU0 (MDF order) with FP32 factors in mixed mode: Newton still reaches the
    FP64 residual tolerance, and the GMRES iteration count stays within a few
    of the FP64-factor run (the preconditioner changes the Krylov path only)."""
    prob = ns2d_vortex(n=4, porder=2)
    runs = {}
    for mode in (0, 1):
        s = HDGSolver(make_copy(prob))
        s.set_precision(mode)
        s.getQ()
        s.assembleLinearSystem()
        conv, hist = s.gmres(precond=0, restart=50, tol=1e-10)
        runs[mode] = (conv, len(hist))
        conv_n, nh = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, precond=0, gmres_tol=1e-10)
        s.close()
        assert conv_n == 1 and nh[-1] < 1e-10, nh
    assert runs[0][0] == 1 and runs[1][0] == 1
    assert abs(runs[1][1] - runs[0][1]) <= 3, runs


def make_copy(prob):
    import copy
    return copy.deepcopy(prob)

"""3xTF32 element contractions (precision mode 3) against the FP64 path.

Mode 3 runs the volume (D = Y'Phi, F = Y'Psi) and face (K, H rows)
contractions of the element kernel as split-precision TF32 products on the
tensor cores (hi/lo operands, three MMAs, FP32 accumulation); the element LU,
the Schur GEMMs and the residuals stay FP64.
* The residual norm comes from FP64 residuals: within 1e-13 relative.
* The trace rows K (the contraction output itself) and the condensed blocks
  DinvF and Hg: max |mode 3 - FP64| <= 2e-5 max |FP64| (operands carry about
  21 bits, FP32 sums of up to 96 terms), and nonzero (the split path ran).
* Newton in mode 3 reaches the FP64 residual tolerance 1e-10 in the FP64
  iteration count (+1 at most), and its final state matches the FP64 run's
  to 1e-9 relative (both are converged solutions of the same FP64 residual).
"""
import copy

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
def test_split_contractions_close_to_fp64(name, make):
    prob = make()
    s = HDGSolver(prob)
    s.getQ()
    r64 = s.assembleLinearSystem()
    ref = {k: s.download(k) for k in ("K", "DinvF", "Hg")}
    s.set_precision(3)
    r3 = s.assembleLinearSystem()
    cur = {k: s.download(k) for k in ref}
    s.close()
    assert abs(r3 - r64) <= 1e-13 * r64
    for k in ref:
        e = rel(cur[k], ref[k])
        assert 0.0 < e < 2e-5, (k, e)


@pytest.mark.parametrize("name,make", [CASES[1], CASES[6]], ids=["2d_p2", "3d_p3"])
def test_split_newton_keeps_fp64_iterations(name, make):
    prob = make()
    out = {}
    for mode in (0, 3):
        s = HDGSolver(copy.deepcopy(prob))
        s.set_precision(mode)
        s.getQ()
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, gmres_tol=1e-10)
        u, uh = s.get_solution()
        out[mode] = (conv, hist, u, uh)
        s.close()
    for mode in (0, 3):
        assert out[mode][0] == 1 and out[mode][1][-1] < 1e-10, (mode, out[mode][1])
    assert len(out[3][1]) <= len(out[0][1]) + 1, (out[0][1], out[3][1])
    assert rel(out[3][2], out[0][2]) < 1e-9
    assert rel(out[3][3], out[0][3]) < 1e-9

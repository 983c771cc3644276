"""Stabilization tensors and viscosity models on the GPU against the oracle.

The oracle's Lax-Friedrichs and Roe tensors (app.convStabMethod 1, 2;
application/FM/stabilizationTensor.cpp) and Sutherland's law
(app.viscosityModel 1; application/FM/getViscosity.c) are pinned to the
reference's own assembly by the golden fixtures (tests/test_oracle_golden.py).
* Element blocks H, the system Hg, Rg, Rr, DinvF within 1e-12 relative and
  rnorm within 1e-12, on periodic 2D / 3D meshes and on a walled channel (the
  no-slip wall's energy row takes the tensor through its fhat), Euler included.
* Newton with the Roe tensor and Sutherland's law on a channel reaches 1e-10.
* The C ABI rejects unsupported models.
"""
import numpy as np
import pytest

from hfem_b200.core import HDGSolver, HfemError
from hfem_b200.gen.problem import as_euler, ns2d_channel, ns2d_vortex, ns3d_box, ns3d_fourier, with_models
from oracle import Oracle

pytestmark = pytest.mark.gpu

CASES = [
    ("2d_p2_lf", lambda: with_models(ns2d_vortex(n=4, porder=2), 1, 0)),
    ("2d_p3_roe", lambda: with_models(ns2d_vortex(n=3, porder=3), 2, 0)),
    ("2d_p2_sutherland", lambda: with_models(ns2d_vortex(n=4, porder=2), 0, 1)),
    ("2d_p2_roe_sutherland", lambda: with_models(ns2d_vortex(n=4, porder=2), 2, 1)),
    ("3d_p2_lf", lambda: with_models(ns3d_fourier(n=3, porder=2), 1, 0)),
    ("3d_p3_roe", lambda: with_models(ns3d_fourier(n=3, porder=3), 2, 0)),
    ("3d_p1_lf_sutherland", lambda: with_models(ns3d_fourier(n=3, porder=1), 1, 1)),
    ("3d_p2_sutherland", lambda: with_models(ns3d_fourier(n=3, porder=2), 0, 1)),
    ("2d_channel_roe_sutherland", lambda: with_models(ns2d_channel(n=4, porder=2, bcm=(2, 2, 5, 6)), 2, 1)),
    ("3d_box_lf", lambda: with_models(ns3d_box(n=2, porder=2), 1, 0)),
    ("euler2d_channel_lf", lambda: with_models(as_euler(ns2d_channel(n=3, porder=2, bcm=(1, 6, 7, 2))), 1, 0)),
    ("euler2d_channel_roe", lambda: with_models(as_euler(ns2d_channel(n=3, porder=2, bcm=(1, 6, 7, 2))), 2, 0)),
]


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_models_assembly_matches_oracle(name, make):
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
    assert np.max(np.abs(s.download("Rr") - ref["Rr"])) <= 1e-12 * max(np.max(np.abs(ref["Rr"])), 1.0)
    s.close()


def test_models_newton_converges():
    p = with_models(ns2d_channel(n=6, porder=2), 2, 1)
    s = HDGSolver(p)
    s.getQ()
    conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, gmres_tol=1e-12)
    s.close()
    assert conv == 1 and hist[-1] < 1e-10, hist


def test_unsupported_models_rejected():
    s = HDGSolver(ns2d_vortex(n=3, porder=1))
    for cs, vm in ((3, 0), (-1, 0), (0, 2)):
        with pytest.raises(HfemError):
            s._chk(s.lib.hfem_set_models(s.h, cs, vm), "set_models")
    s.close()


def test_newton_line_search_matches_reference():
    """Newton on a walled channel with the Roe tensor and Sutherland's law: the
    full step raises the residual, so the line search of solveNonlinearProblem
    (dgsolvers.cpp:106-205) halves the step with residual-only passes between
    the updates; history and state against the reference driver's (fixture from
    oracle/_ref/hfem_ref newton) within 1e-12."""
    import os
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                  "ns2d_channel_roe_suth_p2_n4_newton.npz")))
    p = with_models(ns2d_channel(n=4, porder=2), 2, 1)
    s = HDGSolver(p)
    s.getQ()
    conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=2, gmres_tol=1e-10)
    udg, uh = s.get_solution()
    s.close()
    r0 = g["rnorm_hist"][0]
    assert len(hist) == len(g["rnorm_hist"]), (hist, g["rnorm_hist"])
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * r0, (hist, g["rnorm_hist"])
    assert rel(udg.ravel(), g["udg"].ravel()) < 1e-12 and rel(uh.ravel(), g["uh"].ravel()) < 1e-12


def test_batch_line_search_equals_alone():
    """Two packed problems whose full Newton steps are rejected: the batch's
    per-problem line search (residual-only passes between per-problem updates)
    reproduces each problem's own Newton history (per-problem GMRES to 1e-10,
    so histories within 1e-8 of r0)."""
    from hfem_b200.batch import BatchSolver
    probs = [with_models(ns2d_channel(n=4, porder=2, seed=s), 2, 1) for s in (0, 3)]
    alone = []
    for p in probs:
        s = HDGSolver(p)
        s.getQ()
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=2, gmres_tol=1e-10)
        s.close()
        alone.append(hist)
    b = BatchSolver(probs)
    b.s.getQ()
    active = np.ones(len(probs), dtype=bool)
    hb = [[] for _ in probs]
    for it in range(2):
        old, new = b.newton_iteration(1e-10, active, gmres_tol=1e-10)
        for i in range(len(probs)):
            if it == 0:
                hb[i].append(old[i])
            hb[i].append(new[i])
    b.close()
    for i in range(len(probs)):
        h = np.array(hb[i])
        assert h.shape == alone[i].shape, (h, alone[i])
        assert np.max(np.abs(h - alone[i])) <= 1e-8 * alone[i][0], (h, alone[i])
        assert alone[i][1] < alone[i][0]       # the line search took a partial step


@pytest.mark.parametrize("mode", [1, 3], ids=["mixed", "split_tf32"])
def test_mixed_newton_with_line_search_reaches_fp64_tolerance(mode):
    """Mixed precision on the problem whose full steps the line search rejects:
    Newton still ends at the FP64 residual tolerance, at the FP64 run's state."""
    p = with_models(ns2d_channel(n=4, porder=2), 2, 1)
    out = {}
    for m in (0, mode):
        s = HDGSolver(p)
        s.set_precision(m)
        s.getQ()
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=30, gmres_tol=1e-10)
        out[m] = (conv, hist, s.get_solution())
        s.close()
    for m in out:
        assert out[m][0] == 1 and out[m][1][-1] < 1e-10, (m, out[m][1])
    (u0, h0), (u1, h1) = out[0][2], out[mode][2]
    assert rel(u1, u0) < 1e-8 and rel(h1, h0) < 1e-8


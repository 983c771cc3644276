"""GPU: the solver chain and the full-size workloads against the reference.

Pins, through the C ABI, what single assemblies do not:

* updateSol + block-Jacobi GMRES + the Newton driver on the 4 x 4 x 2 vortex
  (2D, p = 2): two Newton iterations against the reference driver's own run
  (``tests/golden/ns2d_p2_n4_newton.npz``, made by oracle/_ref/hfem_ref):
  residual history within 1e-12 of the first residual, GMRES iteration counts
  equal, final udg / uh within 1e-12 relative.
* block-Jacobi GMRES against the oracle's restated GMRES on the same system:
  relative-residual histories within 1e-12 (absolute, in units of |M^-1 b|),
  the same iteration count, solutions within 1e-10 relative.
* the full-size 2D workload (32 x 32 x 2 = 2,048 triangles, p = 2): q from
  getQ within 1e-11 of max |udg| (a discrete gradient, see the test), every
  assembled array against the oracle at 1e-12 on the same state, and one Newton
  step against the reference driver (``ns2d_p2_n32_newton1.npz``) at 1e-12 of
  the first residual.
* the full-size 3D workload (20^3 x 6 = 48,000 tetrahedra, p = 3): 64 seeded
  elements' blocks (K and Rh before condensation, D^-1, the condensed H, Rh,
  D^-1 F and D^-1 Ru) against the oracle's element routine, condensed with
  numpy, at 1e-12 relative to each array's largest entry (D^-1 Ru, a residual:
  1e-12 of max(|D^-1 Ru|, 1), as the other residual checks).
* the mixed-precision Newton (TF32 Schur GEMMs, FP32 block-Jacobi inverses,
  FP64 residuals, Arnoldi and update): its converged state against the FP64
  oracle's converged state (both to a residual of 1e-10).  Two states that each
  satisfy the residual tolerance differ by about the tolerance times the
  conditioning, so the bar is 1e-8 relative; the measured error is printed.
"""
import os

import numpy as np
import pytest

from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_vortex, ns3d_fourier
from oracle import Oracle, newton_solve

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def rel(a, b):
    return float(np.max(np.abs(np.ravel(a) - np.ravel(b))) / max(np.max(np.abs(b)), 1e-300))


def projections(a):
    p = np.random.default_rng(20261203).standard_normal((8, np.size(a)))
    return p @ np.ravel(a)


def test_update_gmres_newton_steps_match_reference_driver():
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_p2_n4_newton.npz")))
    prob = ns2d_vortex(n=4, porder=2)
    s = HDGSolver(prob)
    try:
        s.getQ()
        hist, iters = [], []
        for _ in range(2):
            hist.append(s.assembleLinearSystem())
            conv, gh = s.gmres(precond=2, restart=50, tol=1e-10)
            assert conv == 1
            iters.append(len(gh))
            s.updateSol(1.0)
        hist.append(s.computeResidualNorm())
        udg, uh = s.get_solution()
    finally:
        s.close()
    r0 = g["rnorm_hist"][0]
    assert np.max(np.abs(np.array(hist) - g["rnorm_hist"])) <= 1e-12 * r0, (hist, g["rnorm_hist"])
    assert iters == [int(v) for v in g["gmres_iters"]], (iters, g["gmres_iters"])
    assert rel(udg, g["udg"]) < 1e-12, rel(udg, g["udg"])
    assert rel(uh, g["uh"]) < 1e-12, rel(uh, g["uh"])


def test_newton_driver_history_matches_reference_driver():
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_p2_n4_newton.npz")))
    prob = ns2d_vortex(n=4, porder=2)
    s = HDGSolver(prob)
    try:
        s.getQ()
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-14, maxiter=2, precond=2, restart=50, gmres_tol=1e-10)
        udg, uh = s.get_solution()
    finally:
        s.close()
    r0 = g["rnorm_hist"][0]
    assert len(hist) == 3
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * r0, (hist, g["rnorm_hist"])
    assert rel(udg, g["udg"]) < 1e-12 and rel(uh, g["uh"]) < 1e-12


@pytest.mark.parametrize("n", [4, 32], ids=["4x4x2", "32x32x2"])
def test_block_jacobi_gmres_matches_oracle(n):
    prob = ns2d_vortex(n=n, porder=2)
    o = Oracle(prob)
    s = HDGSolver(prob)
    try:
        s.getQ()
        s.assembleLinearSystem()
        Hg, Rg = s.download("Hg"), s.download("Rg")
        conv, gh = s.gmres(precond=2, restart=50, tol=1e-10)
        x = s.download("x")
    finally:
        s.close()
    xr, flag, hr = o.gmres(Hg, Rg, Minv=o.bj_inverse(Hg), restart=50, tol=1e-10)
    assert conv == 1 and flag == 0
    assert len(gh) == len(hr), (len(gh), len(hr))
    dh = float(np.max(np.abs(gh - hr)))
    print(f"BJ-GMRES n={n}: {len(gh)} iterations, history diff {dh:.2e}, x rel {rel(x, xr):.2e}")
    assert dh <= 1e-12, dh
    assert rel(x, xr) < 1e-10, rel(x, xr)


@pytest.fixture(scope="module")
def config1():
    prob = ns2d_vortex(n=32, porder=2)
    o = Oracle(prob)
    udg_q = o.getq(prob.udg, prob.uh)
    ref = o.assemble(udg_q, prob.uh)
    return prob, udg_q, ref


def test_full_size_2d_assembly_matches_oracle(config1):
    prob, udg_q, ref = config1
    s = HDGSolver(prob)
    try:
        s.getQ()
        udg, _ = s.get_solution()
        # q is the discrete gradient of u (sums of O(1) terms that cancel to the
        # gradient of a 1e-3 perturbation), so its rounding is ~1e3 times that of
        # u: 1e-11 of max |udg| here (1.3e-12 measured on B200)
        assert np.array_equal(udg[:, :prob.ncu], prob.udg[:, :prob.ncu])
        assert rel(udg, udg_q) < 1e-11
        s.set_solution(udg_q, prob.uh, prob.sh)
        rn = s.assembleLinearSystem()
        got = {k: s.download(k) for k in ("Hg", "Rg", "Rr", "DinvF", "DinvRu")}
    finally:
        s.close()
    assert rel(got["Hg"], ref["Hg"]) < 1e-12
    assert np.array_equal(got["Hg"] == 0.0, ref["Hg"] == 0.0)
    assert rel(got["DinvF"], ref["DinvF"]) < 1e-12
    scale = max(np.max(np.abs(ref["Rr"])), np.max(np.abs(ref["Rg"])))
    for k in ("Rg", "Rr"):
        assert np.max(np.abs(got[k] - ref[k])) <= 1e-12 * scale, k
    assert np.max(np.abs(got["DinvRu"] - ref["DinvRu"])) <= 1e-12 * max(np.max(np.abs(ref["DinvRu"])), 1.0)
    assert abs(rn - ref["rnorm"]) <= 1e-12 * ref["rnorm"]


def test_full_size_2d_newton_step_matches_reference_driver():
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_p2_n32_newton1.npz")))
    prob = ns2d_vortex(n=32, porder=2)
    s = HDGSolver(prob)
    try:
        s.getQ()
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-14, maxiter=1, precond=2, restart=50, gmres_tol=1e-10)
        udg, uh = s.get_solution()
    finally:
        s.close()
    r0 = g["rnorm_hist"][0]
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * r0, (hist, g["rnorm_hist"])
    for k, v in (("udg", udg), ("uh", uh)):
        d = np.max(np.abs(projections(v) - g[k + "_proj"]))
        assert d <= 1e-12 * g[k + "_absmax"][0] * np.sqrt(v.size), (k, d)


def test_full_size_3d_sampled_elements_match_oracle():
    prob = ns3d_fourier(n=20, porder=3)
    n, nb, ne = prob.n_local, prob.n_trace, prob.mesh.ne
    assert ne == 48000
    elems = np.sort(np.random.default_rng(2026).choice(ne, size=64, replace=False))
    s = HDGSolver(prob)
    try:
        s.getQ()
        s.assembleLinearSystem()
        udg, uh = s.get_solution()
        got = {k: s.download_elements(k, elems) for k in ("K", "Ro", "Dinv", "H", "Rh", "DinvF", "DinvRu")}
    finally:
        s.close()
    o = Oracle(prob)
    ref = {k: [] for k in got}
    for ie in elems:
        e = o.element(udg, uh, int(ie))
        D = e["D"].reshape(n, n, order="F")
        F = e["F"].reshape(n, nb, order="F")
        K = e["K"].reshape(nb, n, order="F")
        H = e["H"].reshape(nb, nb, order="F")
        Dinv = np.linalg.inv(D)
        DinvF, DinvRu = Dinv @ F, Dinv @ e["Ru"]
        ref["K"].append(e["K"])
        ref["Ro"].append(e["Rh"])
        ref["Dinv"].append(Dinv.ravel(order="F"))
        ref["DinvF"].append(DinvF.ravel(order="F"))
        ref["DinvRu"].append(DinvRu)
        ref["H"].append((H - K @ DinvF).ravel(order="F"))
        ref["Rh"].append(e["Rh"] - K @ DinvRu)
    for k in got:
        r = np.array(ref[k])
        err = rel(got[k], r)
        if k == "DinvRu":
            # a residual: relative to the scale of the terms that cancel in it
            # (the convention of the other residual checks), not to its own size
            err = float(np.max(np.abs(got[k] - r)) / max(np.max(np.abs(r)), 1.0))
        print(f"48k-element workload, {len(elems)} sampled elements: {k} err {err:.2e}")
        assert err < 1e-12, (k, err)


@pytest.mark.parametrize("make", [lambda: ns2d_vortex(n=4, porder=2), lambda: ns3d_fourier(n=3, porder=3)],
                         ids=["2d_p2", "3d_p3"])
def test_mixed_newton_state_matches_fp64_oracle(make):
    prob = make()
    o = Oracle(prob)
    udg0 = o.getq(prob.udg, prob.uh)
    udg_ref, uh_ref, ok, hist_ref = newton_solve(o, udg0, prob.uh.copy(), prob.sh, 1e-10, 12)
    assert ok
    s = HDGSolver(prob)
    try:
        s.set_precision(1)
        s.getQ()
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=12, gmres_tol=1e-10)
        udg, uh = s.get_solution()
    finally:
        s.close()
    assert conv == 1 and hist[-1] < 1e-10
    eu, eh = rel(udg, udg_ref), rel(uh, uh_ref)
    print(f"mixed Newton vs FP64 oracle: {len(hist) - 1} vs {len(hist_ref) - 1} iterations, "
          f"udg rel err {eu:.2e}, uh rel err {eh:.2e}")
    assert eu < 1e-8 and eh < 1e-8, (eu, eh)

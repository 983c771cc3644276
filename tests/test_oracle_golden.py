"""CPU: the oracle restatement against fixtures made by the reference's own C++.

The fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py with
oracle/_ref/hfem_ref) hold seeded inputs and the reference's outputs.  These
tests pin (1) the input generator: regenerated inputs equal the stored ones, and
(2) the oracle: on the stored inputs it reproduces the reference's q, element
blocks, Hg, Rg, Rr, D^-1 Ru, D^-1 F and rNorm within 1e-12 relative (residual
vectors: 1e-12 of the scale of the terms that cancel in them).
"""
import os

import numpy as np
import pytest

from hfem_b200.gen.problem import as_euler, ns2d_channel, ns2d_vortex, ns3d_box, ns3d_fourier, with_models
from oracle import Oracle, newton_solve

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {
    "ns2d_p1_n3": lambda: ns2d_vortex(n=3, porder=1),
    "ns2d_p2_n3": lambda: ns2d_vortex(n=3, porder=2),
    "ns2d_p3_n3": lambda: ns2d_vortex(n=3, porder=3),
    "ns3d_p1_n3": lambda: ns3d_fourier(n=3, porder=1),
    "ns3d_p3_n3": lambda: ns3d_fourier(n=3, porder=3),
    "ns2d_channel_p2_n3": lambda: ns2d_channel(n=3, porder=2),
    "ns3d_box_p1_n2": lambda: ns3d_box(n=2, porder=1),
    "ns2d_farfield_p2_n3": lambda: ns2d_channel(n=3, porder=2, bcm=(1, 1, 1, 1)),
    # Euler (app.appname 0, flag_q 0): the reference stores no q
    "euler2d_channel_p2_n3": lambda: as_euler(ns2d_channel(n=3, porder=2, bcm=(1, 6, 7, 2))),
    # stabilization tensors (app.convStabMethod 1 Lax-Friedrichs, 2 Roe) and
    # Sutherland's law (app.viscosityModel 1)
    "ns2d_lf_p2_n3": lambda: with_models(ns2d_vortex(n=3, porder=2), 1, 0),
    "ns2d_roe_p2_n3": lambda: with_models(ns2d_vortex(n=3, porder=2), 2, 0),
    "ns2d_suth_p2_n3": lambda: with_models(ns2d_vortex(n=3, porder=2), 0, 1),
    "ns3d_lf_p2_n3": lambda: with_models(ns3d_fourier(n=3, porder=2), 1, 0),
    "ns3d_roe_p2_n3": lambda: with_models(ns3d_fourier(n=3, porder=2), 2, 0),
    "ns3d_suth_p2_n3": lambda: with_models(ns3d_fourier(n=3, porder=2), 0, 1),
    "ns2d_channel_roe_suth_p2_n3": lambda: with_models(ns2d_channel(n=3, porder=2), 2, 1),
    "euler2d_channel_lf_p2_n3": lambda: with_models(as_euler(ns2d_channel(n=3, porder=2, bcm=(1, 6, 7, 2))), 1, 0),
}


def rel(a, b):
    return float(np.max(np.abs(np.ravel(a) - np.ravel(b))) / max(np.max(np.abs(b)), 1e-300))


def compare(name, got, g, tol=1e-12, scale=None):
    if name in g:
        ref = g[name]
        if scale is None:
            assert rel(got, ref) < tol, (name, rel(got, ref))
        else:
            assert np.max(np.abs(np.ravel(got) - ref)) <= tol * scale, name
    else:
        p = np.random.default_rng(20261203).standard_normal((8, np.size(got)))
        proj = p @ np.ravel(got)
        assert np.max(np.abs(proj - g[name + "_proj"])) <= tol * g[name + "_absmax"][0] * np.sqrt(np.size(got)) * 8, name


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    g = dict(np.load(os.path.join(HERE, request.param + ".npz")))
    prob = CASES[request.param]()
    return request.param, prob, g


def test_generator_reproduces_inputs(case):
    name, prob, g = case
    assert rel(prob.udg, g["udg_in"]) < 1e-13
    assert rel(prob.uh, g["uh_in"]) < 1e-13
    assert rel(prob.mesh.dgnodes, g["dgnodes"]) < 1e-13
    assert np.array_equal(prob.mesh.elcon, g["elcon"])


def test_oracle_matches_reference(case):
    name, prob, g = case
    o = Oracle(prob)
    udg_q = o.getq(g["udg_in"], g["uh_in"])
    if prob.appname == 0:
        # the reference's Euler state holds u only; q stays unused in the NS layout
        ncu = prob.ncu
        assert rel(udg_q[:, :ncu, :], g["udg"].reshape(prob.mesh.ne, ncu, -1)) < 1e-12
        ref_udg = udg_q
    else:
        assert rel(udg_q, g["udg"]) < 1e-12
        ref_udg = g["udg"].reshape(udg_q.shape)
    for ie in range(2):
        e = o.element(ref_udg, g["uh_in"], ie)
        for k in ("D", "F", "K", "H", "Rh"):
            blk = g["e" + k].reshape(2, -1)[ie]
            assert rel(e[k], blk) < 1e-12, (k, ie)
        ru = g["eRu"].reshape(2, -1)[ie]
        assert np.max(np.abs(e["Ru"] - ru)) <= 1e-12 * max(np.max(np.abs(e["Rh"])), np.max(np.abs(ru)))
    a = o.assemble(ref_udg, g["uh_in"])
    compare("Hg", a["Hg"], g)
    compare("DinvF", a["DinvF"], g)
    scale = max(np.max(np.abs(g["Rr"])), np.max(np.abs(g["Rg"])))
    compare("Rg", a["Rg"], g, scale=scale)
    compare("Rr", a["Rr"], g, scale=scale)
    compare("DinvRu", a["DinvRu"], g, scale=max(np.max(np.abs(g["DinvRu"])), 1.0))
    assert abs(a["rnorm"] - g["rnorm"][0]) <= 1e-12 * g["rnorm"][0]


def test_newton_history_matches_reference():
    g = dict(np.load(os.path.join(HERE, "ns2d_p2_n4_newton.npz")))
    prob = ns2d_vortex(n=4, porder=2)
    o = Oracle(prob)
    udg = o.getq(prob.udg, prob.uh)
    uh = prob.uh.copy()
    hist, iters = [], []
    for _ in range(2):
        a = o.assemble(udg, uh)
        hist.append(a["rnorm"])
        x, flag, gh = o.gmres(a["Hg"], a["Rg"], Minv=o.bj_inverse(a["Hg"]), restart=50, tol=1e-10)
        assert flag == 0
        iters.append(len(gh))
        udg, uh = o.update(udg, uh, x, a["DinvRu"], a["DinvF"], 1.0)
    hist.append(o.residual(udg, uh))
    r0 = g["rnorm_hist"][0]
    assert np.max(np.abs(np.array(hist) - g["rnorm_hist"])) <= 1e-12 * r0
    assert iters == [int(v) for v in g["gmres_iters"]]
    assert rel(udg.ravel(), g["udg"]) < 1e-12
    assert rel(uh.ravel(), g["uh"]) < 1e-12


def projections(name, a):
    """The fixed random projections make_golden.py stores for large arrays."""
    p = np.random.default_rng(20261203).standard_normal((8, a.size))
    return p @ np.ravel(a)


def test_newton_step_full_size_2d_matches_reference():
    """One Newton step of the reference driver on the full-size 2D workload
    (32 x 32 x 2 triangles, p = 2, block-Jacobi GMRES(50) to 1e-10)."""
    g = dict(np.load(os.path.join(HERE, "ns2d_p2_n32_newton1.npz")))
    prob = ns2d_vortex(n=32, porder=2)
    o = Oracle(prob)
    udg = o.getq(prob.udg, prob.uh)
    a = o.assemble(udg, prob.uh)
    x, flag, gh = o.gmres(a["Hg"], a["Rg"], Minv=o.bj_inverse(a["Hg"]), restart=50, tol=1e-10)
    assert flag == 0 and len(gh) == int(g["gmres_iters"][0])
    udg, uh = o.update(udg, prob.uh, x, a["DinvRu"], a["DinvF"], 1.0)
    hist = np.array([a["rnorm"], o.residual(udg, uh)])
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * g["rnorm_hist"][0]
    for k, v in (("udg", udg), ("uh", uh)):
        assert np.max(np.abs(projections(k, v) - g[k + "_proj"])) <= 1e-12 * g[k + "_absmax"][0] * np.sqrt(v.size)


def test_newton_with_roe_and_sutherland_matches_reference():
    """The reference's Newton driver with the Roe tensor and Sutherland's law on
    a walled channel (two iterations, line search as solveNonlinearProblem)."""
    g = dict(np.load(os.path.join(HERE, "ns2d_channel_roe_suth_p2_n4_newton.npz")))
    prob = with_models(ns2d_channel(n=4, porder=2), 2, 1)
    o = Oracle(prob)
    udg = o.getq(prob.udg, prob.uh)
    udg, uh, _, hist = newton_solve(o, udg, prob.uh.copy(), prob.sh, 1e-10, 2)
    r0 = g["rnorm_hist"][0]
    assert len(hist) == len(g["rnorm_hist"])
    assert np.max(np.abs(np.array(hist) - g["rnorm_hist"])) <= 1e-12 * r0
    assert rel(udg.ravel(), g["udg"].ravel()) < 1e-12 and rel(uh.ravel(), g["uh"].ravel()) < 1e-12

"""Generates the golden fixtures in this folder from the reference's own C++.

Runs oracle/_ref/hfem_ref (the reference's serial hot path compiled from its
sources by oracle/Makefile; needs the reference tree) on small seeded problems
and stores its outputs next to the generated inputs:

    python tests/golden/make_golden.py [fixture names]

Each fixture holds the inputs (so the CPU tests also pin the generator) and
the reference outputs: q from getQ, Hg / Rg / Rr, D^-1 Ru, D^-1 F, rNorm and the
pre-condensation blocks of the first elements; large 3D arrays are stored as
fixed random projections instead of in full.  The Newton fixture holds the
reference driver's residual history and GMRES iteration counts; the full-size
2D workload (32 x 32 x 2 triangles, p = 2) gets one Newton step of the same
driver, and the Taylor-Green fixture the kinetic-energy history of 20 steps of
the reference's DIRK(3,3) driver (solveUnsteadyProblem).

    python tests/golden/make_golden.py newton          # the Newton fixtures only
    python tests/golden/make_golden.py dirk            # the DIRK fixture only
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from hfem_b200.diagnostics import kinetic_energy  # noqa: E402
from hfem_b200.gen.problem import (as_euler, ns2d_channel, ns2d_vortex, ns3d_box, ns3d_fourier,  # noqa: E402
                                   ns3d_tgv, with_models)
from oracle import run_reference  # noqa: E402

CASES = {
    "ns2d_p1_n3": lambda: ns2d_vortex(n=3, porder=1),
    "ns2d_p2_n3": lambda: ns2d_vortex(n=3, porder=2),
    "ns2d_p3_n3": lambda: ns2d_vortex(n=3, porder=3),
    "ns3d_p1_n3": lambda: ns3d_fourier(n=3, porder=1),
    "ns3d_p3_n3": lambda: ns3d_fourier(n=3, porder=3),
    # bounded meshes: Dirichlet, extrapolation, slip and no-slip adiabatic walls
    "ns2d_channel_p2_n3": lambda: ns2d_channel(n=3, porder=2),
    "ns3d_box_p1_n2": lambda: ns3d_box(n=2, porder=1),
    "ns2d_farfield_p2_n3": lambda: ns2d_channel(n=3, porder=2, bcm=(1, 1, 1, 1)),
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
FULL_LIMIT = 400_000          # store arrays up to this many entries in full



def squeeze(name, a, limit=FULL_LIMIT):
    a = np.asarray(a)
    if a.size <= limit:
        return {name: a}
    p = np.random.default_rng(20261203).standard_normal((8, a.size))
    return {name + "_proj": p @ a.ravel(), name + "_absmax": np.array([np.max(np.abs(a))])}


def newton_fixtures():
    if not os.path.exists(os.path.join(HERE, "ns2d_p2_n4_newton.npz")):
        prob = ns2d_vortex(n=4, porder=2)
        ref = run_reference(prob, mode="newton", newton=dict(maxiter=2, precond=2, restart=50, tol=1e-10))
        np.savez_compressed(os.path.join(HERE, "ns2d_p2_n4_newton.npz"), rnorm_hist=ref["rnorm_hist"],
                            gmres_iters=ref["gmres_iters"], udg=ref["udg"], uh=ref["uh"])
        print("newton", ref["rnorm_hist"], ref["gmres_iters"])
    # the Roe tensor and Sutherland's law on a walled channel, two Newton iterations
    prob = with_models(ns2d_channel(n=4, porder=2), 2, 1)
    ref = run_reference(prob, mode="newton", newton=dict(maxiter=2, precond=2, restart=50, tol=1e-10))
    np.savez_compressed(os.path.join(HERE, "ns2d_channel_roe_suth_p2_n4_newton.npz"), rnorm_hist=ref["rnorm_hist"],
                        gmres_iters=ref["gmres_iters"], udg=ref["udg"], uh=ref["uh"])
    print("newton roe+sutherland channel", ref["rnorm_hist"], ref["gmres_iters"])
    # the full-size 2D workload: 2,048 elements, one Newton step
    prob = ns2d_vortex(n=32, porder=2)
    ref = run_reference(prob, mode="newton", newton=dict(maxiter=1, precond=2, restart=50, tol=1e-10))
    out = dict(rnorm_hist=ref["rnorm_hist"], gmres_iters=ref["gmres_iters"])
    out.update(squeeze("udg", ref["udg"], limit=0))
    out.update(squeeze("uh", ref["uh"], limit=0))
    np.savez_compressed(os.path.join(HERE, "ns2d_p2_n32_newton1.npz"), **out)
    print("newton n32", ref["rnorm_hist"], ref["gmres_iters"])


DIRK_CASE = dict(n=4, porder=3, dt=0.01, nsteps=20)


def dirk_fixture():
    """Taylor-Green vortex, 4^3 x 6 tetrahedra, p = 3, DIRK(3,3), 20 steps of
    dt = 0.01, each stage solved by Newton to 1e-10 with block-Jacobi GMRES(50)."""
    c = DIRK_CASE
    prob = ns3d_tgv(n=c["n"], porder=c["porder"], dt=c["dt"])
    ref = run_reference(prob, mode="dirk", newton=dict(maxiter=10, precond=2, restart=50, tol=1e-10, stages=3,
                                                       order=3, dt=c["dt"], newton_tol=1e-10, nsteps=c["nsteps"]))
    steps = ref["udg_steps"]
    ke = np.array([kinetic_energy(prob, u) for u in steps])
    out = dict(ke=ke, **{k: np.array([v]) for k, v in c.items()})
    out.update(squeeze("udg_final", steps[-1], limit=0))
    np.savez_compressed(os.path.join(HERE, "tgv_p3_n4_dirk20.npz"), **out)
    print("dirk", ke)


def main(only=None):
    if only and "newton" in only:
        return newton_fixtures()
    if only and "dirk" in only:
        return dirk_fixture()
    for key, make in CASES.items():
        if only and key not in only:
            continue
        prob = make()
        ref = run_reference(prob, ndump=2)
        out = dict(udg_in=prob.udg, uh_in=prob.uh, dgnodes=prob.mesh.dgnodes, elcon=prob.mesh.elcon,
                   rnorm=np.array([ref["rnorm"]]))
        for k in ("udg", "Hg", "Rg", "Rr", "DinvRu", "DinvF", "eD", "eF", "eK", "eH", "eRu", "eRh"):
            out.update(squeeze(k, ref[k]))
        np.savez_compressed(os.path.join(HERE, key + ".npz"), **out)
        print(key, {k: v.shape for k, v in out.items()})
    if only:
        return
    newton_fixtures()
    dirk_fixture()


if __name__ == "__main__":
    main(sys.argv[1:] or None)      # optional: names of the fixtures to (re)make

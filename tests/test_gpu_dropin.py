"""GPU: the reference's own Newton driver on the B200 path (the drop-in check).

oracle/_ref/digasoser_b200 is the reference's serial solver chain compiled from
its sources with solvers/dgsolvers.cpp unchanged and its assembly, solution
update and closed solver routines replaced by hfem_b200/shim/reference_shim.cpp
on libhfem_b200.so (built by oracle/Makefile where the reference tree is
present; the binary travels with the repository).  Its Newton residual history
and final state must match the reference's own run (oracle/_ref/hfem_ref,
stored in tests/golden) within 1e-12 of the first residual / 1e-12 relative:
  * the 4 x 4 x 2 vortex (2D, p = 2), two Newton iterations;
  * the full-size 2D workload (32 x 32 x 2 = 2,048 triangles, p = 2), one step;
  * a walled channel with the Roe stabilization tensor and Sutherland's law
    (app.convStabMethod 2, app.viscosityModel 1, read by the reference's own
    set-up and handed to the library by the shim), two iterations.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from hfem_b200.gen.problem import ns2d_channel, ns2d_vortex, with_models
from hfem_b200.gen.refio import write_inputs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "digasoser_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def run_driver(prob, maxiter):
    if not os.path.exists(DRIVER):
        pytest.skip("oracle/_ref/digasoser_b200 not built (make -C oracle REF=<reference tree> all)")
    tmp = tempfile.mkdtemp(prefix="hfem_dropin_")
    inp, out = os.path.join(tmp, "in_"), os.path.join(tmp, "out_")
    write_inputs(inp, prob, newton_maxiter=maxiter, gmres_tol=1e-10)
    r = subprocess.run([DRIVER, "newton", inp, out, str(maxiter), "2", "50", "1e-10"], capture_output=True,
                       text=True, env=dict(os.environ, OPENBLAS_NUM_THREADS="1"))
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
    ld = lambda k: np.fromfile(out + k + ".bin", dtype=np.float64)  # noqa: E731
    return ld("rnorm_hist"), ld("udg"), ld("uh")


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def test_reference_newton_driver_on_gpu_two_steps():
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_p2_n4_newton.npz")))
    hist, udg, uh = run_driver(ns2d_vortex(n=4, porder=2), 2)
    r0 = g["rnorm_hist"][0]
    print("drop-in driver, 4x4x2 p2:", hist, "reference:", g["rnorm_hist"])
    assert hist.shape == g["rnorm_hist"].shape
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * r0
    assert rel(udg, g["udg"].ravel()) < 1e-12 and rel(uh, g["uh"].ravel()) < 1e-12


def test_reference_newton_driver_on_gpu_full_size_2d():
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_p2_n32_newton1.npz")))
    hist, udg, uh = run_driver(ns2d_vortex(n=32, porder=2), 1)
    r0 = g["rnorm_hist"][0]
    print("drop-in driver, 32x32x2 p2:", hist, "reference:", g["rnorm_hist"])
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * r0
    for k, v in (("udg", udg), ("uh", uh)):
        p = np.random.default_rng(20261203).standard_normal((8, v.size))
        d = np.max(np.abs(p @ v - g[k + "_proj"]))
        assert d <= 1e-12 * g[k + "_absmax"][0] * np.sqrt(v.size), (k, d)


def test_reference_newton_driver_on_gpu_roe_sutherland_channel():
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_channel_roe_suth_p2_n4_newton.npz")))
    hist, udg, uh = run_driver(with_models(ns2d_channel(n=4, porder=2), 2, 1), 2)
    r0 = g["rnorm_hist"][0]
    print("drop-in driver, Roe + Sutherland channel:", hist, "reference:", g["rnorm_hist"])
    assert hist.shape == g["rnorm_hist"].shape
    assert np.max(np.abs(hist - g["rnorm_hist"])) <= 1e-12 * r0
    assert rel(udg, g["udg"].ravel()) < 1e-12 and rel(uh, g["uh"].ravel()) < 1e-12

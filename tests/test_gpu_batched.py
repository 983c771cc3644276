"""Mixed-order batched assembly in one CUDA graph (GPU).

* Every mesh's residual norm from the graph equals its norm from a plain
  per-mesh assembly to 1e-13 relative (same kernels, same element data).
* The face-block system of each packed shape equals the per-mesh systems
  (1e-13 relative), whichever batched-GEMM tiling the autotuner picked.
* Replaying the graph gives the same result twice (it is a pure function of
  the resident state).
"""
import numpy as np
import pytest

from hfem_b200.batched import MixedOrderAssembly, autotune
from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_vortex, ns3d_fourier

pytestmark = pytest.mark.gpu


def _probs():
    return [ns2d_vortex(n=4, porder=1, seed=1, mach=0.3), ns2d_vortex(n=5, porder=2, seed=2, mach=0.7),
            ns2d_vortex(n=3, porder=3, seed=3, mach=0.5), ns2d_vortex(n=4, porder=4, seed=4, mach=0.25),
            ns2d_vortex(n=6, porder=2, seed=5, mach=0.45), ns2d_vortex(n=3, porder=1, seed=6, mach=0.8),
            ns3d_fourier(n=3, porder=2, seed=7)]


def test_graph_assembly_equals_per_mesh(tmp_path, monkeypatch):
    monkeypatch.setenv("HFEM_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    probs = _probs()
    m = MixedOrderAssembly(probs, precision=0, tune=True)
    m.launch()
    rn = m.finish()
    m.launch()
    rn2 = m.finish()
    assert np.array_equal(rn, rn2)
    for i, p in enumerate(probs):
        s = HDGSolver(p)
        s.getQ()
        r = s.assembleLinearSystem()
        assert abs(rn[i] - r) <= 1e-13 * r, (i, rn[i], r)
        s.close()
    # the packed face-block system of the p=2 group equals the per-mesh ones
    k = m.keys.index((2, 2))
    b = m.solvers[k]
    Hg = b.s.download("Hg")
    bsz2 = b.probs[0].bsz ** 2
    rs = b.union.mesh.rowstart
    foff = np.cumsum([0] + [q.mesh.nf for q in b.probs])
    for j, q in enumerate(b.probs):
        s = HDGSolver(q)
        s.getQ()
        s.assembleLinearSystem()
        ref = s.download("Hg")
        got = Hg[rs[foff[j]] * bsz2:rs[foff[j + 1]] * bsz2]
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
        s.close()
    m.close()


def test_autotune_picks_valid_tilings(tmp_path):
    p = ns3d_fourier(n=3, porder=3)
    s = HDGSolver(p)
    s.getQ()
    ref = s.assembleLinearSystem()
    Hg0 = s.download("Hg")
    g1, g2, ms = autotune(s, "3d_p3", cache=str(tmp_path / "t.json"))
    assert ms is not None and np.all(ms > 0)
    if (g1, g2) != (-1, -1):         # (-1, -1): the fused kernel beat the best pair
        assert ms[0, g1] == ms[0].min() and ms[1, g2] == ms[1].min()
    r = s.assembleLinearSystem()
    assert abs(r - ref) <= 1e-13 * ref
    assert np.max(np.abs(s.download("Hg") - Hg0)) <= 1e-13 * np.max(np.abs(Hg0))
    # cached choice is reused
    g1b, g2b, ms2 = autotune(s, "3d_p3", cache=str(tmp_path / "t.json"))
    assert (g1b, g2b) == (g1, g2) and ms2 is None
    s.close()


def test_mixed_graph_residuals_match_fp64():
    probs = _probs()[:4]
    a = MixedOrderAssembly(probs, precision=0, tune=False)
    a.launch()
    r64 = a.finish()
    a.close()
    b = MixedOrderAssembly(probs, precision=1, tune=False)
    b.launch()
    r32 = b.finish()
    b.close()
    assert np.allclose(r32, r64, rtol=1e-13, atol=0)

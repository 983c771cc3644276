"""Multi-problem contexts and the serving loop on the GPU.

* A problem packed with others assembles exactly what it assembles alone:
  its element blocks, its face-block rows of Hg and its residual norm agree
  to 1e-13 relative (the same kernels run on the same element data; only the
  element and face offsets differ).
* Every request served in the mix ends at the state that a plain FP64 solve
  of it alone reaches: both are solved to a Newton residual below 1e-10, and
  the states agree to 1e-8 relative to the state's magnitude (the distance
  between two iterates that both satisfy the residual tolerance).
"""
import numpy as np
import pytest

from hfem_b200.batch import BatchSolver
from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_vortex
from hfem_b200.serve import Request, sequential, serve

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def test_packed_assembly_equals_alone():
    probs = [ns2d_vortex(n=4, porder=2, seed=1, re=80.0, mach=0.3),
             ns2d_vortex(n=3, porder=2, seed=2, re=300.0, mach=0.6),
             ns2d_vortex(n=5, porder=2, seed=3, re=150.0, mach=0.45)]
    b = BatchSolver(probs)
    b.s.getQ()
    b.s.assembleLinearSystem()
    rn = b.rnorms()
    Hg_u, H_u = b.s.download("Hg"), b.s.download("H")
    bsz2, nb2 = probs[0].bsz ** 2, probs[0].n_trace ** 2
    blk = b.union.mesh.rowstart
    foff = np.cumsum([0] + [p.mesh.nf for p in probs])
    for i, p in enumerate(probs):
        s = HDGSolver(p)
        s.getQ()
        r_alone = s.assembleLinearSystem()
        assert abs(rn[i] - r_alone) <= 1e-13 * r_alone
        H = s.download("H")
        assert _rel(H_u[b.eoff[i] * nb2:b.eoff[i + 1] * nb2], H) < 1e-13
        Hg = s.download("Hg")
        assert _rel(Hg_u[blk[foff[i]] * bsz2:blk[foff[i + 1]] * bsz2], Hg) < 1e-13
        s.close()
    b.close()


def test_per_problem_gmres_equals_alone():
    probs = [ns2d_vortex(n=4, porder=3, seed=4, re=70.0, mach=0.25),
             ns2d_vortex(n=6, porder=3, seed=5, re=450.0, mach=0.65),
             ns2d_vortex(n=3, porder=3, seed=6, re=200.0, mach=0.4)]
    b = BatchSolver(probs)
    b.s.getQ()
    b.s.assembleLinearSystem()
    conv, its = b.gmres(precond=2, restart=20, tol=1e-10)
    x_u = b.s.download("x")
    foff = np.cumsum([0] + [p.mesh.nf for p in probs]) * probs[0].bsz
    for i, p in enumerate(probs):
        s = HDGSolver(p)
        s.getQ()
        s.assembleLinearSystem()
        c1, hist = s.gmres(precond=2, restart=20, tol=1e-10)
        x = s.download("x")
        assert conv[i] == c1 == 1
        assert abs(int(its[i]) - len(hist)) <= 1, (its, len(hist))
        assert _rel(x_u[foff[i]:foff[i + 1]], x) < 1e-8
        s.close()
    b.close()


class _StepClock:
    """A clock that advances a fixed amount per reading, so arrivals land
    between iteration boundaries deterministically."""

    def __init__(self, dt):
        self.t, self.dt = 0.0, dt

    def __call__(self):
        self.t += self.dt
        return self.t


def _requests():
    spec = [(4, 2, 90.0, 0.3, 0.0), (3, 1, 400.0, 0.6, 0.0), (5, 3, 200.0, 0.5, 0.1),
            (6, 2, 60.0, 0.45, 0.2), (3, 3, 480.0, 0.25, 0.3), (4, 1, 120.0, 0.7, 0.4)]
    return [Request(rid=i, arrival=t, n=n, porder=p, re=re, mach=m, seed=100 + i)
            for i, (n, p, re, m, t) in enumerate(spec)]


def test_served_result_equals_alone():
    mix = _requests()
    # immediate admission, so later arrivals join groups in flight
    st = serve(mix, tol=1e-10, keep_states=True, clock=_StepClock(0.05), hbm_budget=1 << 34, join_fraction=0.0,
               max_wait=0)
    assert st.completed == len(mix)
    alone = _requests()
    sequential(alone, tol=1e-10, keep_states=True, clock=_StepClock(100.0))
    for a, m in zip(alone, mix):
        assert a.rnorm < 1e-10 and m.rnorm < 1e-10, (a.rid, a.rnorm, m.rnorm)
        assert _rel(m.udg, a.udg) < 1e-8, a.rid
        assert _rel(m.uh, a.uh) < 1e-8, a.rid
    # later arrivals joined groups already in flight
    assert st.mean_batch > 1.0


def test_admission_waits_for_memory():
    mix = _requests()
    # a budget that holds about one request at a time still completes every request
    from hfem_b200.serve import footprint_bytes, build_problem
    budget = max(footprint_bytes(build_problem(r)) for r in mix)
    st = serve(mix, tol=1e-10, clock=_StepClock(0.05), hbm_budget=budget)
    assert st.completed == len(mix) and st.max_rnorm < 1e-10
    assert st.peak_bytes <= budget


def test_served_result_equals_alone_batched_admission():
    # the default policy: admissions batched, groups driven by concurrent host threads
    mix = _requests()
    st = serve(mix, tol=1e-10, keep_states=True, clock=_StepClock(0.05), hbm_budget=1 << 34)
    assert st.completed == len(mix)
    alone = _requests()
    sequential(alone, tol=1e-10, keep_states=True, clock=_StepClock(100.0))
    for a, m in zip(alone, mix):
        assert a.rnorm < 1e-10 and m.rnorm < 1e-10, (a.rid, a.rnorm, m.rnorm)
        assert _rel(m.udg, a.udg) < 1e-8, a.rid
        assert _rel(m.uh, a.uh) < 1e-8, a.rid

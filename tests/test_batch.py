"""Host logic of multi-problem packing and the request stream (no GPU)."""
import numpy as np

from hfem_b200.batch import union_problem
from hfem_b200.gen.problem import ns2d_vortex
from hfem_b200.serve import footprint_bytes, make_requests


def _probs():
    return [ns2d_vortex(n=4, porder=2, seed=1, re=80.0, mach=0.3),
            ns2d_vortex(n=3, porder=2, seed=2, re=300.0, mach=0.6),
            ns2d_vortex(n=5, porder=2, seed=3, re=150.0, mach=0.45)]


def test_union_offsets_and_block_diagonal():
    probs = _probs()
    u, eprob, fprob, params, eoff, hoff = union_problem(probs)
    m = u.mesh
    assert m.ne == sum(p.mesh.ne for p in probs) and m.nf == sum(p.mesh.nf for p in probs)
    assert list(eoff) == list(np.cumsum([0] + [p.mesh.ne for p in probs]))
    assert hoff[-1] == m.nf * m.npf == u.uh.shape[0]
    assert np.all(np.diff(m.rowstart) > 0) and m.rowstart[-1] == m.colidx.size
    foff = np.cumsum([0] + [p.mesh.nf for p in probs])
    for i, p in enumerate(probs):
        e0, e1 = eoff[i], eoff[i + 1]
        assert np.all(eprob[e0:e1] == i)
        assert np.all(fprob[foff[i]:foff[i + 1]] == i)
        # every face, block column and trace dof of problem i stays inside problem i
        assert np.array_equal(m.t2f[e0:e1] - foff[i], p.mesh.t2f)
        assert np.array_equal(m.elcon[e0:e1] - hoff[i], p.mesh.elcon)
        rows = slice(m.rowstart[foff[i]], m.rowstart[foff[i + 1]])
        assert np.array_equal(m.colidx[rows] - foff[i], p.mesh.colidx)
        assert np.array_equal(u.udg[e0:e1], p.udg) and np.array_equal(u.uh[hoff[i]:hoff[i + 1]], p.uh)
        assert np.allclose(params[i], [*p.param, p.tdep, p.fc_u])


def test_union_rejects_mixed_orders():
    import pytest
    with pytest.raises(ValueError):
        union_problem([ns2d_vortex(n=3, porder=1), ns2d_vortex(n=3, porder=2)])


def test_request_stream_is_seeded():
    a = make_requests(200, rate=50.0, seed=7)
    b = make_requests(200, rate=50.0, seed=7)
    assert [(r.arrival, r.n, r.porder, r.re, r.mach) for r in a] == [(r.arrival, r.n, r.porder, r.re, r.mach) for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0)
    assert abs(len(a) / arr[-1] - 50.0) < 15.0                  # Poisson rate
    ne = np.array([r.elements for r in a])
    assert ne.min() >= 200 and ne.max() <= 17000
    assert {r.porder for r in a} == {1, 2, 3}
    assert all(50 <= r.re <= 500 and 0.2 <= r.mach <= 0.7 for r in a)


def test_footprint_grows_with_order_and_size():
    f1 = footprint_bytes(ns2d_vortex(n=4, porder=1))
    f2 = footprint_bytes(ns2d_vortex(n=4, porder=3))
    f3 = footprint_bytes(ns2d_vortex(n=8, porder=3))
    assert 0 < f1 < f2 < f3

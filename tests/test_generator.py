"""CPU: quadrature, master element and mesh invariants of the input generator."""
import numpy as np
import pytest

from hfem_b200.gen.master import make_master
from hfem_b200.gen.mesh import build_mesh
from hfem_b200.gen.quadrature import check_rule, line_rule, simplex_rule


@pytest.mark.parametrize("dim,deg,npts", [(2, 2, 3), (2, 4, 6), (2, 6, 12), (2, 8, 16), (3, 2, 4), (3, 4, 14),
                                          (3, 6, 24)])
def test_simplex_rules_exact(dim, deg, npts):
    p, w = simplex_rule(dim, deg)
    assert len(w) == npts
    assert check_rule(p, w, dim, deg) < 1e-14
    assert np.all(w > 0)


@pytest.mark.parametrize("pgauss,npts", [(2, 2), (4, 3), (6, 4), (8, 5)])
def test_line_rule_counts(pgauss, npts):
    x, w = line_rule(pgauss)
    assert len(w) == npts and abs(w.sum() - 1.0) < 1e-15


@pytest.mark.parametrize("nd,p", [(2, 1), (2, 2), (2, 3), (2, 4), (3, 1), (3, 2), (3, 3)])
def test_master_partition_of_unity(nd, p):
    m = make_master(nd, p)
    assert np.allclose(m.shapvl[:, :, 0].sum(axis=0), 1.0, atol=1e-13)
    assert np.allclose(m.shapvl[:, :, 1:].sum(axis=0), 0.0, atol=1e-11)
    assert np.allclose(m.shapfc[:, :, 0].sum(axis=0), 1.0, atol=1e-13)
    # every face node is an element node on that face
    assert m.perm.shape == (nd + 1, m.npf) and np.all(m.perm < m.npv)


@pytest.mark.parametrize("nd,p,n", [(2, 2, 4), (2, 1, 3), (3, 3, 3), (3, 1, 3)])
def test_mesh_trace_numbering(nd, p, n):
    m = make_master(nd, p)
    L = 1.0
    me = build_mesh(m, n, L)
    # every trace node is shared by exactly two elements at the same (periodic) position
    pos = {}
    cnt = np.zeros(me.ndofuh, dtype=int)
    for e in range(me.ne):
        for a in range(me.nfe):
            i = me.t2f[e, a]
            for k in range(me.npf):
                g = me.elcon[e, a * me.npf + k]
                assert i * me.npf <= g < (i + 1) * me.npf
                x = me.dgnodes[e, :, m.perm[a, k]] % L
                if g in pos:
                    d = np.abs(pos[g] - x)
                    assert np.max(np.minimum(d, L - d)) < 1e-9
                else:
                    pos[g] = x
                cnt[g] += 1
    assert np.all(cnt == 2)
    # face-block CSR: diagonal first, 2 nfe - 1 blocks per row
    rs, ci = me.rowstart, me.colidx
    for i in range(me.nf):
        assert ci[rs[i]] == i
        assert rs[i + 1] - rs[i] == 2 * me.nfe - 1
    # positively oriented elements (outward facegeom normals rely on it)
    ref_verts = np.vstack([np.zeros(nd), np.eye(nd)])
    vid = [int(np.argmin(np.linalg.norm(m.plocvl - v, axis=1))) for v in ref_verts]
    for e in range(0, me.ne, max(1, me.ne // 17)):
        v = me.dgnodes[e][:, vid]
        assert np.linalg.det(v[:, 1:] - v[:, :1]) > 0


def test_small_periodic_grid_rejected():
    with pytest.raises(ValueError):
        build_mesh(make_master(2, 1), 2, 1.0)

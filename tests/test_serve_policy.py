"""CPU: the server's admission policy (which iteration boundary packs the
requests that arrived into their order's group)."""
from types import SimpleNamespace

from hfem_b200.serve import _Group


def _req(ne, live=True):
    return SimpleNamespace(prob=SimpleNamespace(mesh=SimpleNamespace(ne=ne)), live=live)


def test_joiners_pack_at_once_into_an_idle_group():
    g = _Group()
    g.joining = [_req(100)]
    assert g.join_due(0.5, 3)


def test_small_joiners_wait_for_share_or_iterations():
    g = _Group()
    g.members = [_req(1000), _req(1000)]
    g.joining = [_req(300)]
    assert not g.join_due(0.5, 3)           # 300 < 0.5 * 2000 live elements
    g.joining.append(_req(800))
    assert g.join_due(0.5, 3)               # 1100 >= 1000
    g.joining = [_req(10)]
    g.waited = 3
    assert g.join_due(0.5, 3)               # waited long enough


def test_immediate_admission_and_retired_members():
    g = _Group()
    g.members = [_req(1000), _req(500, live=False)]
    g.joining = [_req(1)]
    assert g.join_due(0.0, 0)
    assert not g.join_due(0.5, 3)           # live elements are 1000, not 1500
    g.joining = []
    assert not g.join_due(0.0, 0)

"""CPU: the domain decomposition of hfem_b200/dd.py (several GPUs) on its host logic.

The local assembly of each part is the oracle here (a CPU backend); the
partition, the interface sums, the all-reduced dot products and the
distributed GMRES / Newton are the module's own code, run as world_size 2
``gloo`` ranks.  Checks:
  * the parts' subassembled face-block rows sum to the single-domain Hg and Rg
    (1e-12 relative), each element in exactly one part;
  * the two-rank block-Jacobi GMRES reproduces the single-domain GMRES
    (restated oracle): same iteration count, relative-residual history within
    1e-12, solution within 1e-12 relative;
  * two damped-Newton iterations over two ranks reproduce the single-domain
    Newton residual history within 1e-12 of the first residual;
  * on a walled channel with the Roe tensor and Sutherland's law, where the
    full steps are rejected and the line search halves them, two ranks
    reproduce the reference driver's history (tests/golden fixture) to 1e-12.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest
import torch

from hfem_b200.dd import DDSolver, Exchange, partition
from hfem_b200.gen.problem import ns2d_channel, ns2d_vortex, with_models
from oracle import Oracle, newton_solve


def problem():
    prob = ns2d_vortex(n=4, porder=2)
    prob.udg = Oracle(prob).getq(prob.udg, prob.uh)
    return prob


class OracleBackend:
    """Local work of one part on the CPU oracle (test backend)."""

    def __init__(self, prob):
        self.prob, self.o = prob, Oracle(prob)
        self.udg, self.uh = prob.udg.copy(), prob.uh.copy()
        self.b = prob.bsz
        self.rs, self.ci = prob.mesh.rowstart, prob.mesh.colidx

    def _pass(self, want):
        a = self.o.assemble(self.udg, self.uh, want_dinv=want)
        self._Rr = torch.from_numpy(a["Rr"])
        # sum of ||Ru_e||^2 over the part's elements (the interface rows of Rr are
        # partial sums, so it is not rnorm^2 - ||Rr||^2 of the local pass)
        ru2 = sum(float(np.sum(self.o.element(self.udg, self.uh, e)["Ru"] ** 2)) for e in range(self.prob.mesh.ne))
        self._ru2 = torch.tensor([ru2], dtype=torch.float64)
        return a

    def assemble(self):
        a = self._pass(True)
        self.Hg, self.DinvRu, self.DinvF = a["Hg"], a["DinvRu"], a["DinvF"]
        self._Rg = torch.from_numpy(a["Rg"])

    def residual(self):
        self._pass(False)

    def Rg(self):
        return self._Rg

    def Rr(self):
        return self._Rr

    def ru2(self):
        return self._ru2

    def diag_blocks(self):
        b2 = self.b * self.b
        return torch.from_numpy(self.Hg.reshape(-1, b2)[self.rs[:-1]].copy())

    def matvec(self, v):
        b, x = self.b, v.numpy().reshape(-1, self.b)
        blocks = self.Hg.reshape(-1, b, b)                  # [k, c, r] = block k (r, c)
        y = np.zeros_like(x)
        for i in range(self.rs.size - 1):
            for k in range(self.rs[i], self.rs[i + 1]):
                y[i] += blocks[k].T @ x[self.ci[k]]
        return torch.from_numpy(y.reshape(-1))

    def update(self, x, alpha):
        self.udg, self.uh = self.o.update(self.udg, self.uh, x.numpy(), self.DinvRu, self.DinvF, alpha)


def test_parts_subassemble_the_global_system():
    prob = problem()
    ref = Oracle(prob).assemble(prob.udg, prob.uh)
    b = prob.bsz
    rs, ci = prob.mesh.rowstart, prob.mesh.colidx
    blk = {(i, int(ci[k])): k for i in range(prob.mesh.nf) for k in range(rs[i], rs[i + 1])}
    Hg, Rg = np.zeros_like(ref["Hg"]).reshape(-1, b * b), np.zeros_like(ref["Rg"]).reshape(-1, b)
    seen = np.zeros(prob.mesh.ne, dtype=int)
    for r in range(2):
        p = partition(prob, 2, r)
        seen[p.elems] += 1
        a = Oracle(p.prob).assemble(p.prob.udg, p.prob.uh)
        lrs, lci = p.prob.mesh.rowstart, p.prob.mesh.colidx
        for i in range(p.faces.size):
            Rg[p.faces[i]] += a["Rg"].reshape(-1, b)[i]
            for k in range(lrs[i], lrs[i + 1]):
                Hg[blk[(int(p.faces[i]), int(p.faces[lci[k]]))]] += a["Hg"].reshape(-1, b * b)[k]
        # interface faces are shared with the other rank and owned by exactly one
        assert set(p.shared) <= {1 - r}
    assert np.all(seen == 1)
    assert np.max(np.abs(Hg.ravel() - ref["Hg"])) <= 1e-12 * np.max(np.abs(ref["Hg"]))
    assert np.max(np.abs(Rg.ravel() - ref["Rg"])) <= 1e-12 * np.max(np.abs(ref["Rg"]))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        prob = problem()
        part = partition(prob, world, rank)
        dd = DDSolver(part, OracleBackend(part.prob), Exchange(part, prob.bsz, "cpu"))
        r0 = dd.assemble()
        conv, hist = dd.gmres(restart=50, tol=1e-10)
        x = dd.x.numpy().reshape(-1, prob.bsz)
        dd2 = DDSolver(part, OracleBackend(part.prob), Exchange(part, prob.bsz, "cpu"))
        ok, nhist = dd2.newton(tol=1e-14, maxiter=2)
        torch.save(dict(r0=r0, conv=conv, hist=hist, faces=part.faces[part.owned], x=x[part.owned],
                        nhist=np.array(nhist)), os.path.join(out, f"rank{rank}.pt"))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.fixture(scope="module")
def two_ranks(tmp_path_factory):
    import torch.multiprocessing as mp
    out = str(tmp_path_factory.mktemp("dd"))
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    return [torch.load(os.path.join(out, f"rank{r}.pt"), weights_only=False) for r in range(2)]


def test_two_rank_gmres_matches_single_domain(two_ranks):
    prob = problem()
    o = Oracle(prob)
    a = o.assemble(prob.udg, prob.uh)
    xr, flag, hr = o.gmres(a["Hg"], a["Rg"], Minv=o.bj_inverse(a["Hg"]), restart=50, tol=1e-10)
    assert flag == 0
    x = np.zeros((prob.mesh.nf, prob.bsz))
    for res in two_ranks:
        assert res["conv"] == 1
        assert abs(res["r0"] - a["rnorm"]) <= 1e-12 * a["rnorm"]
        assert len(res["hist"]) == len(hr)
        assert np.max(np.abs(res["hist"] - hr)) <= 1e-12
        x[res["faces"]] = res["x"]
    assert np.max(np.abs(x.ravel() - xr)) <= 1e-12 * np.max(np.abs(xr))


def test_two_rank_newton_matches_single_domain(two_ranks):
    prob = problem()
    _, _, _, href = newton_solve(Oracle(prob), prob.udg, prob.uh.copy(), prob.sh, 1e-14, 2)
    for res in two_ranks:
        assert len(res["nhist"]) == len(href)
        assert np.max(np.abs(res["nhist"] - np.array(href))) <= 1e-12 * href[0]


def _channel_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        prob = with_models(ns2d_channel(n=4, porder=2), 2, 1)
        prob.udg = Oracle(prob).getq(prob.udg, prob.uh)
        part = partition(prob, world, rank)
        dd = DDSolver(part, OracleBackend(part.prob), Exchange(part, prob.bsz, "cpu"))
        ok, nhist = dd.newton(tol=1e-10, maxiter=2)
        torch.save(dict(nhist=np.array(nhist)), os.path.join(out, f"chan{rank}.pt"))
    finally:
        dist.destroy_process_group()


def test_two_rank_line_search_on_bounded_mesh_matches_reference(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path)
    mp.start_processes(_channel_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    g = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                  "ns2d_channel_roe_suth_p2_n4_newton.npz")))
    for r in range(2):
        h = torch.load(os.path.join(out, f"chan{r}.pt"), weights_only=False)["nhist"]
        assert len(h) == len(g["rnorm_hist"])
        assert np.max(np.abs(h - g["rnorm_hist"])) <= 1e-12 * g["rnorm_hist"][0], (h, g["rnorm_hist"])

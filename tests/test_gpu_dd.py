"""GPU: the domain-decomposition driver (hfem_b200/dd.py) on its GPU backend.

A run here has one GPU, so the decomposition runs as one rank (one part, no
interface); the multi-rank host logic is covered by tests/test_dd.py on CPU
(gloo, two ranks).  This checks the GPU plumbing the ranks use -- the
assembled arrays as device tensors, hfem_matvec, hfem_set_step + updateSol,
the all-reduces over CUDA tensors -- against the single-GPU solver chain:
  * the driver's block-Jacobi GMRES history equals hfem_gmres's within 1e-12
    and its solution within 1e-12 relative;
  * two Newton iterations match the reference driver's history
    (tests/golden/ns2d_p2_n4_newton.npz) within 1e-12 of the first residual;
  * so do two iterations on a walled channel with the Roe tensor and
    Sutherland's law, where the line search rejects the full steps.
"""
import os
import socket
from datetime import timedelta

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def group():
    import torch.distributed as dist
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60))
    yield
    dist.destroy_process_group()


def test_dd_driver_on_gpu_backend(group):
    from hfem_b200.core import HDGSolver
    from hfem_b200.dd import DDSolver, Exchange, GPUBackend, partition
    from hfem_b200.gen.problem import ns2d_vortex
    prob = ns2d_vortex(n=4, porder=2)
    s = HDGSolver(prob)
    try:
        s.getQ()
        s.assembleLinearSystem()
        conv, href = s.gmres(precond=2, restart=50, tol=1e-10)
        xref = s.download("x")
    finally:
        s.close()
    part = partition(prob, 1, 0)
    be = GPUBackend(part.prob, 0)
    dd = DDSolver(part, be, Exchange(part, prob.bsz, "cuda:0"))
    dd.assemble()
    c, hist = dd.gmres(restart=50, tol=1e-10)
    x = dd.x.cpu().numpy()
    assert c == 1 and conv == 1 and len(hist) == len(href)
    assert np.max(np.abs(hist - href)) <= 1e-12
    assert np.max(np.abs(x - xref)) <= 1e-12 * np.max(np.abs(xref))
    be.s.close()

    g = dict(np.load(os.path.join(GOLDEN, "ns2d_p2_n4_newton.npz")))
    be = GPUBackend(partition(prob, 1, 0).prob, 0)
    dd = DDSolver(part, be, Exchange(part, prob.bsz, "cuda:0"))
    ok, nhist = dd.newton(tol=1e-14, maxiter=2)
    be.s.close()
    assert np.max(np.abs(np.array(nhist) - g["rnorm_hist"])) <= 1e-12 * g["rnorm_hist"][0], nhist



def test_dd_line_search_on_gpu_backend(group):
    from hfem_b200.dd import DDSolver, Exchange, GPUBackend, partition
    from hfem_b200.gen.problem import ns2d_channel, with_models
    g = dict(np.load(os.path.join(GOLDEN, "ns2d_channel_roe_suth_p2_n4_newton.npz")))
    prob = with_models(ns2d_channel(n=4, porder=2), 2, 1)
    part = partition(prob, 1, 0)
    be = GPUBackend(part.prob, 0)
    dd = DDSolver(part, be, Exchange(part, prob.bsz, "cuda:0"))
    ok, nhist = dd.newton(tol=1e-10, maxiter=2)
    be.s.close()
    assert np.max(np.abs(np.array(nhist) - g["rnorm_hist"])) <= 1e-12 * g["rnorm_hist"][0], nhist

"""GPU: hfem_assemble_host (state copied from host in pieces, each piece's
element kernel started as soon as it has arrived) equals hfem_set_solution
followed by hfem_assemble, bit for bit."""
import numpy as np
import pytest

from hfem_b200.core import HDGSolver
from hfem_b200.gen.problem import ns2d_channel, ns3d_fourier, with_models

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("make,chunks", [(lambda: ns3d_fourier(n=3, porder=2), 4),
                                         (lambda: ns2d_channel(n=4, porder=3), 3),
                                         (lambda: ns3d_fourier(n=3, porder=1), 1000),
                                         (lambda: with_models(ns2d_channel(n=4, porder=2), 2, 1), 3)])
def test_assemble_host_equals_set_and_assemble(make, chunks):
    import torch
    prob = make()
    s = HDGSolver(prob)
    s.getQ()
    udg, uh = s.get_solution()
    h_udg = torch.from_numpy(np.ascontiguousarray(udg)).pin_memory()
    h_uh = torch.from_numpy(np.ascontiguousarray(uh)).pin_memory()
    h_sh = torch.from_numpy(np.ascontiguousarray(prob.sh)).pin_memory()
    r_ref = s.assembleLinearSystem()
    Hg, Rg, DinvF = s.download("Hg"), s.download("Rg"), s.download("DinvF")
    for _ in range(2):
        r = s.assemble_from_host(h_udg.data_ptr(), h_uh.data_ptr(), h_sh.data_ptr(), chunks=chunks)
        assert r == r_ref
        assert np.array_equal(s.download("Hg"), Hg)
        assert np.array_equal(s.download("Rg"), Rg)
        assert np.array_equal(s.download("DinvF"), DinvF)
    s.close()

"""GPU test of hfem_condense_noalloc, the entry point that allocates nothing.

Callers that cannot call cudaMalloc (programs drawing device memory from their
own caching pool, serving loops that reserve HBM once) pass every input and
output buffer themselves; the element workspace comes from a fixed 32 MiB
device array inside the library.  This test allocates its buffers with torch
(as such a caller would), calls the entry point twice in a row through the C
ABI, and checks every output of both calls -- D^-1, D^-1 F, K, the condensed H
and Rh, D^-1 Ru, Rh before condensation, ||Ru||^2 and the pivot flags --
against the context-based hfem_assemble with the tolerance of the other parity
tests (1e-12 relative), on periodic and bounded meshes and on Euler.
"""
import ctypes as C

import numpy as np
import pytest

from hfem_b200.core import HDGSolver, load_library
from hfem_b200.gen.problem import as_euler, ns2d_channel, ns2d_vortex, ns3d_fourier

pytestmark = pytest.mark.gpu

_dp = C.POINTER(C.c_double)


def _ptr(t):
    return C.c_void_p(t.data_ptr() if t is not None else 0)


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


CASES = [("2d_p2", lambda: ns2d_vortex(n=4, porder=2)),
         ("3d_p3", lambda: ns3d_fourier(n=3, porder=3)),
         ("2d_p2_channel", lambda: ns2d_channel(n=3, porder=2)),
         ("euler_2d_p2_channel", lambda: as_euler(ns2d_channel(n=3, porder=2, bcm=(1, 6, 7, 2))))]
OUTPUTS = ("Dinv", "DinvF", "K", "H", "DinvRu", "Rh", "Ro", "ru2")


@pytest.mark.parametrize("make", [c[1] for c in CASES], ids=[c[0] for c in CASES])
def test_condense_noalloc_matches_assemble(make):
    import torch

    prob = make()
    s = HDGSolver(prob, device=0)
    try:
        s.getQ()
        s.assembleLinearSystem()
        ref = {k: s.download_elements(k, np.arange(prob.mesh.ne)).ravel() for k in OUTPUTS}
        udg_q, uh = s.get_solution()
        dims = s.dims
    finally:
        s.close()

    lib = load_library()
    vp = C.c_void_p
    lib.hfem_condense_noalloc.argtypes = [vp] + [vp] * 12 + [_dp, C.c_int, C.c_double, C.c_double] + \
        [vp, vp, vp, C.c_int] + [vp] * 9 + [vp]
    lib.hfem_condense_noalloc.restype = C.c_int

    dev = torch.device("cuda:0")
    m, me = prob.master, prob.mesh

    def dput(a, dtype=torch.float64):
        return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device=dev)

    tabs = [dput(m.fortran(k)) for k in ("shapvt", "shapvg", "shapvgdotshapvl", "shapft", "shapfg",
                                          "shapfgdotshapfc")]
    perm = dput(m.perm.astype(np.int32), torch.int32)
    dg = dput(me.dgnodes)
    elcon = dput(me.elcon.astype(np.int32), torch.int32)
    d_udg, d_uh, d_sh = dput(udg_q), dput(uh), dput(prob.sh)
    bounded = getattr(prob, "bcm", None) is not None
    bf = dput(me.bf.astype(np.int32), torch.int32) if bounded else None
    bcm = dput(np.asarray(prob.bcm, dtype=np.int32), torch.int32) if bounded else None
    bcs = dput(np.asarray(prob.bcs, dtype=np.float64)) if bounded else None
    ne, n, nb = me.ne, prob.n_local, prob.n_trace
    f64 = dict(dtype=torch.float64, device=dev)
    out = dict(Dinv=torch.empty(ne * n * n, **f64), DinvF=torch.empty(ne * n * nb, **f64),
               K=torch.empty(ne * nb * n, **f64), H=torch.empty(ne * nb * nb, **f64),
               DinvRu=torch.empty(ne * n, **f64), Rh=torch.empty(ne * nb, **f64),
               Ro=torch.empty(ne * nb, **f64), ru2=torch.empty(ne, **f64),
               info=torch.empty(ne, dtype=torch.int32, device=dev))
    param = np.ascontiguousarray(prob.param, dtype=np.float64)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for t in out.values():
            t.fill_(-7)                      # stale contents must not leak into the result
        torch.cuda.synchronize()
        rc = lib.hfem_condense_noalloc(C.byref(dims), *[_ptr(t) for t in tabs], _ptr(perm), _ptr(dg), _ptr(elcon),
                                       _ptr(d_udg), _ptr(d_uh), _ptr(d_sh), param.ctypes.data_as(_dp),
                                       int(prob.tdep), float(prob.fc_u), float(prob.fc_q),
                                       _ptr(bf), _ptr(bcm), _ptr(bcs), int(getattr(prob, "appname", 1)),
                                       *[_ptr(out[k]) for k in OUTPUTS], _ptr(out["info"]), C.c_void_p(stream))
        assert rc == 0, f"call {call}: rc {rc}"
        torch.cuda.synchronize()
        assert int(out["info"].abs().max()) == 0
        for key in OUTPUTS:
            got = out[key].cpu().numpy()
            assert rel(got, ref[key]) < 1e-12, (call, key, rel(got, ref[key]))


def test_condense_noalloc_rejects_unsupported_shape():
    lib = load_library()
    from hfem_b200.core import Dims
    lib.hfem_condense_noalloc.restype = C.c_int
    dims = Dims(2, 7, 3, 3, 6, 3, 10, 15, 75)        # npv = 7: no compiled kernel
    z = C.c_void_p(1)
    param = np.ones(6)
    lib.hfem_condense_noalloc.argtypes = None
    rc = lib.hfem_condense_noalloc(C.byref(dims), *([z] * 12), param.ctypes.data_as(_dp), C.c_int(0),
                                   C.c_double(0.0), C.c_double(1.0), C.c_void_p(0), C.c_void_p(0), C.c_void_p(0),
                                   C.c_int(1), *([z] * 9), C.c_void_p(0))
    assert rc == -2

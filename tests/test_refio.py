"""CPU: the reference's binary formats round-trip (readbinaryfiles.cpp, writeSol2File)."""
import os

import numpy as np

from hfem_b200.gen.problem import ns2d_vortex
from hfem_b200.gen.refio import read_checkpoint, read_mesh, read_sol, write_checkpoint, write_inputs


def test_inputs_round_trip(tmp_path):
    prob = ns2d_vortex(n=3, porder=2)
    prefix = str(tmp_path / "in_")
    write_inputs(prefix, prob)
    udg, uh, pdg = read_sol(prefix + "sol.bin", prob.mesh.ne, prob.master.npv, prob.nc)
    assert np.array_equal(udg, prob.udg) and np.array_equal(uh, prob.uh.ravel()) and pdg.size == 0
    me = read_mesh(prefix + "mesh.bin")
    assert np.array_equal(me["elcon"], prob.mesh.elcon)
    assert np.array_equal(me["t2f"], prob.mesh.t2f)
    assert np.array_equal(me["dgnodes"], prob.mesh.dgnodes)
    # app.bin: 40-entry header then the arrays it sizes
    a = np.fromfile(prefix + "app.bin")
    assert a.size == 40 + int(a[:18].sum())
    assert int(a[20]) == 2 and int(a[22]) == prob.nc


def test_checkpoint_round_trip(tmp_path):
    prob = ns2d_vortex(n=3, porder=1)
    path = str(tmp_path / "solout.bin")
    write_checkpoint(path, prob.udg, prob.uh)
    u, h = read_checkpoint(path)
    assert np.array_equal(u, prob.udg.ravel()) and np.array_equal(h, prob.uh.ravel())
    write_checkpoint(path, prob.udg, prob.uh, ncu=prob.ncu, with_q=False)
    u, h = read_checkpoint(path)
    assert u.size == prob.mesh.ne * prob.master.npv * prob.ncu

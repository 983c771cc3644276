"""Batched assembly of many meshes of mixed polynomial order in one CUDA graph.

Meshes that share an element shape (dimension and order) are packed into one
context (``batch.union_problem``); the assembly kernels of every context are
captured once into a single CUDA graph (``hfem_graph_capture``) with one
branch per shape, so a whole assembly pass over all meshes is one graph
launch.  Each shape's batched-GEMM tilings are picked by ``autotune``: every
tiling compiled into the library is timed on that shape's own operands and
the fastest is kept, cached per device and shape in a JSON file.
"""
from __future__ import annotations

import ctypes as C
import json
import os

import numpy as np

from .batch import BatchSolver
from .core import HfemError, load_library

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

CACHE = os.environ.get("HFEM_AUTOTUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "hfem_b200",
                                                           "autotune.json"))


def _lib():
    lib = load_library()
    if not getattr(lib, "_batched_types", False):
        lib.hfem_autotune.argtypes = [C.c_void_p, C.c_int, _ip, _dp]
        lib.hfem_set_gemm_tiles.argtypes = [C.c_void_p, C.c_int, C.c_int]
        lib.hfem_gemm_candidates.argtypes = []
        lib.hfem_assemble_async.argtypes = [C.c_void_p]
        lib.hfem_assemble_finish.argtypes = [C.c_void_p, _dp]
        lib.hfem_graph_capture.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]
        lib.hfem_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
        lib.hfem_graph_destroy.argtypes = [C.c_void_p]
        lib._batched_types = True
    return lib


def _device_key(device):
    import torch
    return torch.cuda.get_device_name(device).replace(" ", "_")


def autotune(solver, key, device=0, reps=3, cache=CACHE, refresh=False):
    """Pick the batched-GEMM tilings for one context; returns (g1, g2, timings)."""
    lib = _lib()
    table = {}
    if os.path.exists(cache):
        try:
            table = json.load(open(cache))
        except (OSError, ValueError):
            table = {}
    dk = _device_key(device)
    hit = table.get(dk, {}).get(key)
    if hit is not None and not refresh:
        solver._chk(lib.hfem_set_gemm_tiles(solver.h, int(hit[0]), int(hit[1])), "set_gemm_tiles")
        return int(hit[0]), int(hit[1]), None
    nc = lib.hfem_gemm_candidates()
    best = np.zeros(2, dtype=np.int32)
    ms = np.zeros(2 * nc)
    solver._chk(lib.hfem_autotune(solver.h, reps, best.ctypes.data_as(_ip), ms.ctypes.data_as(_dp)), "autotune")
    table.setdefault(dk, {})[key] = [int(best[0]), int(best[1])]
    try:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        json.dump(table, open(cache, "w"), indent=1)
    except OSError:
        pass
    return int(best[0]), int(best[1]), ms.reshape(2, nc)


class MixedOrderAssembly:
    """All meshes' assembly as one graph launch (one context per element shape).

    precision 1 with tune: the TF32 condensation on the shapes where it is
    faster than the tuned FP64 kernels (the others stay FP64, `fp64_shapes`)."""

    def __init__(self, probs, device=0, precision=0, tune=True, stream=None):
        import torch
        self.device = device
        self.stream = stream or torch.cuda.Stream(device=device)
        self.groups = {}
        for i, p in enumerate(probs):
            self.groups.setdefault((p.master.nd, p.master.porder), []).append(i)
        self.keys = sorted(self.groups)
        self.solvers = []
        self.tiles = {}
        self.fp64_shapes = []      # shapes left in FP64 by a mixed-precision build
        for k in self.keys:
            b = BatchSolver([probs[i] for i in self.groups[k]], device=device, stream=self.stream.cuda_stream)
            b.s.getQ()
            if tune:
                self.tiles[k] = autotune(b.s, f"{k[0]}d_p{k[1]}", device=device)[:2]
            b.s.set_precision(precision)
            if tune and precision == 1 and not self._tf32_pays(b):
                b.s.set_precision(0)         # this shape's tuned FP64 condensation is faster
                self.fp64_shapes.append(k)
            self.solvers.append(b)
        self.ne = sum(p.mesh.ne for p in probs)
        lib = _lib()
        arr = (C.c_void_p * len(self.solvers))(*[b.s.h.value for b in self.solvers])
        g = C.c_void_p()
        rc = lib.hfem_graph_capture(arr, len(self.solvers), C.c_void_p(self.stream.cuda_stream), C.byref(g))
        if rc != 0:
            msg = lib.hfem_last_error(self.solvers[0].s.h).decode()
            raise HfemError(f"graph capture failed ({rc}): {msg}")
        self.graph = g

    @staticmethod
    def _tf32_pays(b, reps=2):
        """Time the condensation of one shape both ways (the TF32 tensor-core
        kernel against the tuned FP64 kernels); True when TF32 is faster."""
        def cond_ms(prec):
            b.s.set_precision(prec)
            b.s.assembleLinearSystem()
            b.s.set_timing(True)
            for _ in range(reps):
                b.s.assembleLinearSystem()
            kt = b.s.kernel_times()
            b.s.set_timing(False)
            return sum(v[0] for k, v in kt.items() if k in ("schur_tc", "schur_fused", "gemm_DinvF", "gemm_schur"))
        t_fp64, t_tf32 = cond_ms(0), cond_ms(1)
        return t_tf32 < t_fp64

    def launch(self):
        """Enqueue one assembly pass over every mesh (one graph launch)."""
        rc = _lib().hfem_graph_launch(self.graph, C.c_void_p(self.stream.cuda_stream))
        if rc != 0:
            raise HfemError(f"graph launch failed ({rc})")

    def finish(self):
        """Wait, check every element LU, and return the residual norm per mesh (input order)."""
        lib = _lib()
        out = {}
        for k, b in zip(self.keys, self.solvers):
            rn = C.c_double()
            b.s._chk(lib.hfem_assemble_finish(b.s.h, C.byref(rn)), "assemble_finish")
            for i, r in zip(self.groups[k], b.rnorms()):
                out[i] = float(r)
        return np.array([out[i] for i in range(len(out))])

    def close(self):
        if self.graph:
            _lib().hfem_graph_destroy(self.graph)
            self.graph = None
        for b in self.solvers:
            b.close()
        self.solvers = []

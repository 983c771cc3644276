"""Host-side binding of the sm_100a HDG hot path (``libhfem_b200.so``).

``HDGSolver`` mirrors the reference's solver surface for this path
(``solvers/dgsolvers.cpp``, ``assembly/globalassembly.cpp``): ``getQ``,
``assembleLinearSystem``, ``computeResidualNorm``, ``gmres``, ``updateSol``
and ``solveNonlinearProblem``, all running on the GPU through the C ABI in
``include/hfem_b200.h``.  There is no CPU fallback: without the compiled
library or a CUDA device, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)

ERRORS = {-1: "invalid argument", -2: "unsupported element", -3: "CUDA error", -4: "bad call order",
          -5: "inconsistent mesh", -6: "singular matrix", -7: "out of device memory"}

DOWNLOAD = {"Hg": 0, "Rg": 1, "Rr": 2, "DinvRu": 3, "DinvF": 4, "H": 5, "Rh": 6, "x": 7, "udg": 8, "uh": 9,
            "K": 10, "Ro": 12, "Dinv": 13, "ru2": 14}


class HfemError(RuntimeError):
    pass


class Dims(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("nd", "npv", "npf", "nfe", "ngv", "ngf", "ne", "nf", "nblocks")]


_lib = None


def load_library(path: str = LIB):
    """Load the compiled library; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise HfemError(f"{path} not built; run hfem_b200.build.build() (nvcc, sm_100a)")
    lib = C.CDLL(path)
    lib.hfem_create.argtypes = [C.POINTER(Dims), C.c_int, C.POINTER(C.c_void_p)]
    lib.hfem_destroy.argtypes = [C.c_void_p]
    lib.hfem_last_error.argtypes = [C.c_void_p]
    lib.hfem_last_error.restype = C.c_char_p
    lib.hfem_set_stream.argtypes = [C.c_void_p, C.c_void_p]
    lib.hfem_set_master.argtypes = [C.c_void_p] + [_dp] * 6 + [_ip]
    lib.hfem_set_mesh.argtypes = [C.c_void_p, _dp, _ip, _ip, _ip, _ip]
    lib.hfem_set_boundary.argtypes = [C.c_void_p, _ip, C.c_int, _ip, _dp]
    lib.hfem_set_app.argtypes = [C.c_void_p, C.c_int]
    lib.hfem_set_models.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.hfem_set_physics.argtypes = [C.c_void_p, _dp, C.c_int, C.c_double, C.c_double, C.c_double]
    lib.hfem_set_solution.argtypes = [C.c_void_p, _dp, _dp, _dp]
    lib.hfem_set_solution_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.hfem_assemble_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_double)]
    lib.hfem_get_solution.argtypes = [C.c_void_p, _dp, _dp]
    lib.hfem_getq.argtypes = [C.c_void_p]
    lib.hfem_assemble.argtypes = [C.c_void_p, _dp]
    lib.hfem_residual.argtypes = [C.c_void_p, _dp]
    lib.hfem_gmres.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, _ip, _ip, _dp, C.c_int]
    lib.hfem_update.argtypes = [C.c_void_p, C.c_double]
    lib.hfem_newton.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, _dp,
                                C.c_int, _ip, _ip]
    lib.hfem_download.argtypes = [C.c_void_p, C.c_int, _dp, C.c_size_t]
    lib.hfem_dirk_step.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                   C.c_double, C.c_int, _ip]
    lib.hfem_set_timing.argtypes = [C.c_void_p, C.c_int]
    lib.hfem_set_precision.argtypes = [C.c_void_p, C.c_int]
    lib.hfem_get_ordering.argtypes = [C.c_void_p, _ip]
    lib.hfem_reset_ordering.argtypes = [C.c_void_p]
    lib.hfem_device_buffer.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)]
    lib.hfem_kernel_times.argtypes = [C.c_void_p, C.c_char_p, C.c_size_t, _dp, _ip, C.c_int]
    lib.hfem_matvec.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.hfem_set_step.argtypes = [C.c_void_p, C.c_void_p]
    _lib = lib
    return lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class HDGSolver:
    """GPU state of one HDG problem (one C-ABI context)."""

    def __init__(self, prob, device: int = 0):
        self.lib = load_library()
        self.prob = prob
        m, me = prob.master, prob.mesh
        self.dims = Dims(m.nd, m.npv, m.npf, m.nfe, m.ngv, m.ngf, me.ne, me.nf, int(me.rowstart[-1]))
        h = C.c_void_p()
        rc = self.lib.hfem_create(C.byref(self.dims), device, C.byref(h))
        if rc != 0:
            raise HfemError(f"hfem_create failed: {ERRORS.get(rc, rc)}")
        self.h = h
        self.n = prob.n_local
        self.nb = prob.n_trace
        self.bsz = prob.bsz
        keep = [m.fortran(k) for k in ("shapvt", "shapvg", "shapvgdotshapvl", "shapft", "shapfg", "shapfgdotshapfc")]
        perm = np.ascontiguousarray(m.perm, dtype=np.int32)
        self._chk(self.lib.hfem_set_master(self.h, *[_d(k) for k in keep], _i(perm)), "set_master")
        self.set_mesh(me)
        self._chk(self.lib.hfem_set_app(self.h, int(getattr(prob, "appname", 1))), "set_app")
        self._chk(self.lib.hfem_set_models(self.h, int(getattr(prob, "conv_stab", 0)),
                                           int(getattr(prob, "viscosity_model", 0))), "set_models")
        if getattr(prob, "bcm", None) is not None:
            self.set_boundary(me.bf, prob.bcm, prob.bcs)
        self.set_physics(prob.param, prob.tdep, prob.fc_u, prob.fc_q, prob.time)
        self.set_solution(prob.udg, prob.uh, prob.sh)

    # -- plumbing -------------------------------------------------------
    def _chk(self, rc, what):
        if rc < 0:
            msg = self.lib.hfem_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise HfemError(f"{what}: {ERRORS.get(rc, rc)}: {msg}")
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.lib.hfem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int):
        self._chk(self.lib.hfem_set_stream(self.h, C.c_void_p(stream_ptr)), "set_stream")

    def set_mesh(self, me):
        self._mesh = dict(dg=np.ascontiguousarray(me.dgnodes, dtype=np.float64),
                          elcon=np.ascontiguousarray(me.elcon, dtype=np.int32),
                          t2f=np.ascontiguousarray(me.t2f, dtype=np.int32),
                          rs=np.ascontiguousarray(me.rowstart, dtype=np.int32),
                          ci=np.ascontiguousarray(me.colidx, dtype=np.int32))
        k = self._mesh
        self._chk(self.lib.hfem_set_mesh(self.h, _d(k["dg"]), _i(k["elcon"]), _i(k["t2f"]), _i(k["rs"]), _i(k["ci"])),
                  "set_mesh")

    def set_boundary(self, bf, bcm, bcs):
        self._bnd = (np.ascontiguousarray(bf, dtype=np.int32), np.ascontiguousarray(bcm, dtype=np.int32),
                     np.ascontiguousarray(bcs, dtype=np.float64))
        b = self._bnd
        self._chk(self.lib.hfem_set_boundary(self.h, _i(b[0]), int(b[1].size), _i(b[1]), _d(b[2])), "set_boundary")

    def set_physics(self, param, tdep, fc_u, fc_q, time=0.0):
        p = np.ascontiguousarray(param, dtype=np.float64)
        self._chk(self.lib.hfem_set_physics(self.h, _d(p), int(tdep), float(fc_u), float(fc_q), float(time)),
                  "set_physics")

    def set_solution(self, udg, uh, sh=None):
        udg = np.ascontiguousarray(udg, dtype=np.float64)
        uh = np.ascontiguousarray(uh, dtype=np.float64)
        shp = _d(np.ascontiguousarray(sh, dtype=np.float64)) if sh is not None else _dp()
        self._chk(self.lib.hfem_set_solution(self.h, _d(udg), _d(uh), shp), "set_solution")

    def set_solution_device(self, udg_ptr, uh_ptr, sh_ptr=None):
        self._chk(self.lib.hfem_set_solution_device(self.h, C.c_void_p(udg_ptr), C.c_void_p(uh_ptr),
                                                    C.c_void_p(sh_ptr) if sh_ptr else None), "set_solution_device")

    def get_solution(self):
        udg = np.empty_like(self.prob.udg)
        uh = np.empty_like(self.prob.uh)
        self._chk(self.lib.hfem_get_solution(self.h, _d(udg), _d(uh)), "get_solution")
        return udg, uh

    def download(self, what):
        me, ne = self.prob.mesh, self.prob.mesh.ne
        sizes = {"Hg": int(me.rowstart[-1]) * self.bsz ** 2, "Rg": me.nf * self.bsz, "Rr": me.nf * self.bsz,
                 "DinvRu": ne * self.n, "DinvF": ne * self.n * self.nb, "H": ne * self.nb ** 2,
                 "Rh": ne * self.nb, "x": me.nf * self.bsz, "K": ne * self.nb * self.n,
                 "Ro": ne * self.nb, "Dinv": ne * self.n * self.n, "ru2": ne}
        out = np.empty(sizes[what])
        self._chk(self.lib.hfem_download(self.h, DOWNLOAD[what], _d(out), out.size), f"download {what}")
        return out

    def device_tensor(self, what):
        """A torch view (float64, cuda) of one of the context's device buffers (no copy)."""
        import torch
        ptr, cnt = C.c_void_p(), C.c_size_t()
        self._chk(self.lib.hfem_device_buffer(self.h, DOWNLOAD[what], C.byref(ptr), C.byref(cnt)), f"buffer {what}")

        class _View:
            __cuda_array_interface__ = {"shape": (cnt.value,), "typestr": "<f8", "data": (ptr.value, False),
                                        "version": 3, "strides": None}
        return torch.as_tensor(_View(), device=f"cuda:{torch.cuda.current_device()}")

    def download_elements(self, what, elems):
        """The per-element blocks of the listed elements of an element-major
        buffer (H, Rh, DinvF, DinvRu, K, Ro, Dinv, ru2), gathered on the device,
        as an (len(elems), block size) array."""
        import torch
        t = self.device_tensor(what)
        per = t.numel() // self.prob.mesh.ne
        idx = torch.as_tensor(np.asarray(elems, dtype=np.int64), device=t.device)
        return t.view(-1, per).index_select(0, idx).cpu().numpy()

    def matvec(self, x):
        """y = Hg x for a float64 CUDA tensor x on the context's device (after an assembly)."""
        import torch
        x = x.contiguous()
        y = torch.empty_like(x)
        self._chk(self.lib.hfem_matvec(self.h, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr())), "matvec")
        return y

    def set_step(self, duh):
        """Make duh (float64 CUDA tensor, nf*bsz) the step updateSol applies."""
        duh = duh.contiguous()
        self._chk(self.lib.hfem_set_step(self.h, C.c_void_p(duh.data_ptr())), "set_step")

    # -- reference surface ---------------------------------------------
    def getQ(self):
        self._chk(self.lib.hfem_getq(self.h), "getQ")

    def assembleLinearSystem(self):
        rn = C.c_double()
        self._chk(self.lib.hfem_assemble(self.h, C.byref(rn)), "assembleLinearSystem")
        return rn.value

    def assemble_from_host(self, udg_ptr, uh_ptr, sh_ptr=None, chunks=4):
        """set_solution + assembleLinearSystem with the host-to-device copies of
        the element-wise state overlapped with the element kernel (pointers to
        host memory, pinned for the overlap; e.g. torch pinned tensors' data_ptr)."""
        rn = C.c_double()
        self._chk(self.lib.hfem_assemble_host(self.h, C.c_void_p(udg_ptr), C.c_void_p(uh_ptr),
                                              C.c_void_p(sh_ptr) if sh_ptr else None, int(chunks), C.byref(rn)),
                  "assemble_host")
        return rn.value

    def computeResidualNorm(self):
        rn = C.c_double()
        self._chk(self.lib.hfem_residual(self.h, C.byref(rn)), "computeResidualNorm")
        return rn.value

    def gmres(self, precond=2, restart=50, tol=1e-10, maxit=1000):
        conv, its = C.c_int(), C.c_int()
        hist = np.zeros(maxit + 1)
        self._chk(self.lib.hfem_gmres(self.h, precond, restart, tol, maxit, C.byref(conv), C.byref(its), _d(hist),
                                      hist.size), "gmres")
        return conv.value, hist[:its.value]

    def updateSol(self, alpha=1.0):
        self._chk(self.lib.hfem_update(self.h, float(alpha)), "updateSol")

    def solveNonlinearProblem(self, newton_tol=1e-10, maxiter=10, precond=2, restart=50, gmres_tol=1e-10,
                              gmres_maxit=1000):
        hist = np.zeros(maxiter + 2)
        nit, conv = C.c_int(), C.c_int()
        self._chk(self.lib.hfem_newton(self.h, newton_tol, maxiter, precond, restart, gmres_tol, gmres_maxit, _d(hist),
                                       hist.size, C.byref(nit), C.byref(conv)), "solveNonlinearProblem")
        return conv.value, hist[:nit.value + 1]

    def solveUnsteadyStep(self, dt, stages=3, order=3, newton_tol=1e-10, newton_maxiter=10, precond=2, restart=50,
                          gmres_tol=1e-10, gmres_maxit=1000):
        """One DIRK time step (solveUnsteadyProblem's step loop body); returns Newton iterations."""
        it = C.c_int(0)
        self._chk(self.lib.hfem_dirk_step(self.h, float(dt), stages, order, newton_tol, newton_maxiter, precond,
                                          restart, gmres_tol, gmres_maxit, C.byref(it)), "solveUnsteadyStep")
        return it.value

    def ordering(self):
        """ordered2unordered of the BILU0 ordering in use."""
        o2u = np.zeros(self.prob.mesh.nf, dtype=np.int32)
        self._chk(self.lib.hfem_get_ordering(self.h, _i(o2u)), "get_ordering")
        return o2u

    def set_precision(self, mode):
        """0: FP64 throughout; 1: 3xTF32 element contractions, TF32 tensor-core Schur GEMMs and FP32
        preconditioner; 2: FP32 preconditioner only; 3: 3xTF32 element contractions and FP32
        preconditioner with FP64 Schur (FP64 LU, residuals and Arnoldi in every mode)."""
        self._chk(self.lib.hfem_set_precision(self.h, int(mode)), "set_precision")

    def set_timing(self, on=True):
        self._chk(self.lib.hfem_set_timing(self.h, 1 if on else 0), "set_timing")

    def kernel_times(self):
        names = C.create_string_buffer(4096)
        ms = np.zeros(64)
        cnt = np.zeros(64, dtype=np.int32)
        k = self._chk(self.lib.hfem_kernel_times(self.h, names, 4096, _d(ms), _i(cnt), 64), "kernel_times")
        keys = names.value.decode().split(";") if k > 0 else []
        return {key: (float(ms[i]), int(cnt[i])) for i, key in enumerate(keys)}

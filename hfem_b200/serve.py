"""Continuous-batching server for independent HDG solve requests.

Each request is a 2D Navier-Stokes HDG solve: a periodic square triangle mesh
of 256 to 16,384 elements (log-uniform), order p in {1, 2, 3}, Re in
[50, 500], Mach in [0.2, 0.7] and an isentropic-vortex state from its own
seed, solved to a Newton residual of 1e-10.  The nonlinear system of a
request is the implicit (backward-Euler, dt = 0.1) step of the reference's
driver (``solvers/dgsolvers.cpp:106-205`` with the time term of
``elementassembly.cpp:293-304``), which is well posed for every draw of the
physics; a steady state of a decaying viscous vortex on a periodic box does
not exist.

The server keeps the state of admitted requests on the device.  At every
iteration boundary it admits the requests that have arrived, in arrival
order, while their device footprint fits the HBM budget.  Requests of one
order are packed into one context (``BatchSolver``), so their element
assembly, condensation, scatter and Krylov solve run as single launches,
while each request keeps its own physics, residual and line search.  A
request retires (its state is read back and its latency recorded) at the
first iteration boundary where its residual is below tolerance.  A group is
repacked when requests join it or when retired requests make up more than
half of its elements; until then a retired request rides along with step 0.
``sequential`` serves the same stream one request at a time with plain FP64
solves (``HDGSolver.solveNonlinearProblem``) for comparison.
"""
from __future__ import annotations

import math
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field, replace

import numpy as np

from .batch import BatchSolver
from .core import HDGSolver, load_library
from .gen.problem import ns2d_vortex


@dataclass(eq=False)
class Request:
    rid: int
    arrival: float
    n: int
    porder: int
    re: float
    mach: float
    seed: int
    prob: object = None
    start: float = math.nan
    finish: float = math.nan
    iters: int = 0
    rnorm: float = math.nan
    live: bool = True
    cur: object = None           # the problem with the request's in-flight state
    udg: np.ndarray = None
    uh: np.ndarray = None

    @property
    def elements(self):
        return 2 * self.n * self.n


def make_requests(count, rate, seed=0, min_el=256, max_el=16384, orders=(1, 2, 3)):
    """`count` requests with Poisson arrivals at `rate` req/s; element counts
    log-uniform in [min_el, max_el] (meshes are n x n squares split in 2)."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=count))
    out = []
    for i in range(count):
        ne = math.exp(rng.uniform(math.log(min_el), math.log(max_el)))
        n = max(3, int(round(math.sqrt(ne / 2))))
        out.append(Request(rid=i, arrival=float(t[i]), n=n, porder=int(rng.choice(orders)),
                           re=float(rng.uniform(50, 500)), mach=float(rng.uniform(0.2, 0.7)),
                           seed=seed * 100003 + i))
    return out


def build_problem(r: Request):
    if r.prob is None:
        r.prob = ns2d_vortex(n=r.n, porder=r.porder, seed=r.seed, mach=r.mach, re=r.re)
    return r.prob


def footprint_bytes(prob) -> int:
    """Device bytes one problem holds inside a context (the per-element
    D, F, D^-1 F, K, H blocks dominate; Krylov basis of restart 50 per face),
    with 1/8 added for the allocator's size classes and per-context buffers."""
    n, nb, ne, nf, bsz = prob.n_local, prob.n_trace, prob.mesh.ne, prob.mesh.nf, prob.bsz
    per_elem = 9 * (n * n + 3 * n * nb + nb * nb + 2 * n + 3 * nb + 3 * prob.master.npv * prob.nc)
    per_face = 9 * (8 * bsz * bsz + 60 * bsz)
    return ne * per_elem + nf * per_face


@dataclass
class ServeStats:
    completed: int
    makespan: float
    solves_per_s: float
    p50: float
    p99: float
    mean_batch: float
    iterations: int
    max_rnorm: float
    peak_bytes: int = 0
    phases: dict = field(default_factory=dict)
    latencies: list = field(default_factory=list)

    def as_dict(self):
        d = dict(self.__dict__)
        d.pop("latencies")
        return d


def _stats(reqs, t_end, batches, iterations, peak=0, phases=None):
    lat = np.array([r.finish - r.arrival for r in reqs])
    return ServeStats(phases=phases or {}, completed=len(reqs), makespan=t_end, solves_per_s=len(reqs) / max(t_end, 1e-12),
                      p50=float(np.percentile(lat, 50)), p99=float(np.percentile(lat, 99)),
                      mean_batch=float(np.mean(batches)) if batches else 0.0, iterations=iterations,
                      max_rnorm=float(max(r.rnorm for r in reqs)), peak_bytes=int(peak), latencies=lat.tolist())


def _merge(acc, ph):
    for k, v in ph.items():
        acc[k] = acc.get(k, 0) + v


class _Group:
    """Requests of one order packed into one context."""

    def __init__(self):
        self.members = []        # requests in the current context, in pack order
        self.joining = []        # admitted, not yet packed
        self.solver = None
        self.waited = 0          # group iterations the joining requests have waited

    def live(self):
        return [r for r in self.members if r.live]

    def join_due(self, join_fraction, max_wait):
        """Pack the joining requests now?  Always when nothing is live; else once
        they hold join_fraction of the live elements or have waited max_wait
        iterations (a repack costs about half an iteration, so admissions are
        batched instead of repacking at every iteration boundary)."""
        if not self.joining:
            return False
        live = sum(r.prob.mesh.ne for r in self.live())
        if live == 0:
            return True
        return (sum(r.prob.mesh.ne for r in self.joining) >= join_fraction * live or self.waited >= max_wait)

    def retired_fraction(self):
        tot = sum(r.prob.mesh.ne for r in self.members)
        dead = sum(r.prob.mesh.ne for r in self.members if not r.live)
        return dead / tot if tot else 0.0

    def repack(self, device, stream, phases=None, on_device=True):
        """Rebuild the context from the live members plus the joining
        requests; returns the device bytes of the retired members it drops."""
        keep = self.live()
        freed = sum(footprint_bytes(r.prob) for r in self.members if not r.live)
        t0 = time.perf_counter()
        old = self.solver
        old_pos = {id(r): i for i, r in enumerate(self.members)}
        if old is not None and keep and not on_device:
            udg, uh = old.s.get_solution()
            for r in keep:
                i = old_pos[id(r)]
                r.cur = replace(r.cur, udg=udg[old.eoff[i]:old.eoff[i + 1]].copy(),
                                uh=uh[old.hoff[i]:old.hoff[i + 1]].copy())
        t1 = time.perf_counter()
        # in-flight states (u and uhat only, a small share of a context) are set
        # aside on the device and the old context is closed before the new one is
        # built, so a repack never holds two contexts' element blocks at once
        saved = []
        if old is not None and keep and on_device:
            import torch
            src_u, src_h = old.s.device_tensor("udg"), old.s.device_tensor("uh")
            su = src_u.numel() // old.eoff[-1]
            sh = src_h.numel() // old.hoff[-1]
            for r in keep:
                i = old_pos[id(r)]
                saved.append((src_u[old.eoff[i] * su:old.eoff[i + 1] * su].clone(),
                              src_h[old.hoff[i] * sh:old.hoff[i + 1] * sh].clone()))
            torch.cuda.synchronize(device)
        if old is not None:
            old.close()
        self.members = keep + self.joining
        self.joining = []
        self.waited = 0
        self.solver = None
        if self.members:
            # in-flight requests start from their packed state on the host side
            # and get their current state by device-to-device copies below
            self.solver = BatchSolver([r.cur for r in self.members], device=device, stream=stream)
            if saved:
                import torch
                dst_u, dst_h = self.solver.s.device_tensor("udg"), self.solver.s.device_tensor("uh")
                for j, (u, h) in enumerate(saved):
                    n0, m0 = self.solver.eoff[j], self.solver.hoff[j]
                    dst_u[n0 * su:n0 * su + u.numel()].copy_(u)
                    dst_h[m0 * sh:m0 * sh + h.numel()].copy_(h)
                torch.cuda.synchronize(device)
                del saved
            # q of joining requests from their (u, uhat); in-flight ones already
            # satisfy q = getQ(u, uhat), so recomputing them is a no-op up to rounding
            self.solver.s.getQ()
        if phases is not None:
            phases["repack_readback"] = phases.get("repack_readback", 0.0) + (t1 - t0)
            phases["repack_build"] = phases.get("repack_build", 0.0) + (time.perf_counter() - t1)
            if self.solver is not None:
                for k, v in self.solver.build_times.items():
                    phases[k] = phases.get(k, 0.0) + v
        return freed


def serve(requests, tol=1e-10, hbm_budget=None, max_newton=20, device=0, clock=time.perf_counter,
          keep_states=False, stream=None, repack_fraction=0.5, gmres_tol=1e-10, restart=50, repack_on_device=True,
          join_fraction=0.5, max_wait=3, workers=3):
    """Continuous batching over `requests` (sorted by arrival); returns ServeStats.

    Admitted requests join their order's context at an iteration boundary: at
    once (join_fraction 0, max_wait 0) or batched (the defaults) -- see
    _Group.join_due.  `workers` host threads drive the orders' groups
    concurrently (0: one after another)."""
    if hbm_budget is None:
        import ctypes
        import torch
        free, _ = torch.cuda.mem_get_info(device)
        lib = load_library()
        lib.hfem_pool_cached_bytes.restype = ctypes.c_longlong
        lib.hfem_pool_cached_bytes.argtypes = []
        # blocks idle in the library's pool are reclaimable: they count as free
        hbm_budget = int(0.8 * (free + lib.hfem_pool_cached_bytes()))
    for r in requests:
        build_problem(r)
        r.live, r.iters, r.cur = True, 0, r.prob
    pending = deque(sorted(requests, key=lambda r: r.arrival))
    pool = ThreadPoolExecutor(max_workers=workers) if workers and workers > 1 else None
    try:
        return _serve_loop(requests, pending, pool, tol, hbm_budget, max_newton, device, clock, keep_states, stream,
                           repack_fraction, gmres_tol, restart, repack_on_device, join_fraction, max_wait)
    finally:
        if pool is not None:
            pool.shutdown(wait=True)


def _serve_loop(requests, pending, pool, tol, hbm_budget, max_newton, device, clock, keep_states, stream,
                repack_fraction, gmres_tol, restart, repack_on_device, join_fraction, max_wait):
    groups = {}
    phases = {"repack": 0.0, "retire": 0.0, "assemble": 0.0, "gmres": 0.0, "gmres_iterations": 0, "line_search": 0.0}
    used = peak = 0
    done, batch_sizes, iterations = [], [], 0
    t0 = clock()
    while pending or any(g.members or g.joining for g in groups.values()):
        now = clock() - t0
        while pending and pending[0].arrival <= now:
            r = pending[0]
            need = footprint_bytes(r.prob)
            if used + need > hbm_budget and used > 0:
                break                                    # wait for HBM to free up
            pending.popleft()
            used += need
            peak = max(peak, used)
            r.start = now
            groups.setdefault(r.porder, _Group()).joining.append(r)
        busy = [g for g in groups.values() if g.live() or g.joining]
        if not busy:
            if pending:
                time.sleep(max(0.0, min(0.005, pending[0].arrival - now)))
            continue
        for g in busy:
            if g.join_due(join_fraction, max_wait) or g.retired_fraction() > repack_fraction:
                tr = time.perf_counter()
                if g.solver is not None:
                    _merge(phases, g.solver.phases)
                used -= g.repack(device, stream, phases, repack_on_device)
                phases["repack"] += time.perf_counter() - tr
        # one Newton iteration of every busy group; each group's context has its
        # own stream, and with `workers` each group is driven by its own host
        # thread (the library calls release the interpreter lock), so the groups'
        # launches and host round trips overlap
        runs = []
        for g in busy:
            if g.joining:
                g.waited += 1
            active = np.array([r.live for r in g.members])
            batch_sizes.append(int(active.sum()))
            runs.append((g, active))
        if pool is not None and len(runs) > 1:
            futs = [pool.submit(g.solver.newton_iteration, tol, a, gmres_tol=gmres_tol, restart=restart)
                    for g, a in runs]
            results = [f.result() for f in futs]
        else:
            results = [g.solver.newton_iteration(tol, a, gmres_tol=gmres_tol, restart=restart) for g, a in runs]
        for (g, active), (old, new) in zip(runs, results):
            b = g.solver
            iterations += 1
            finished = []
            for i, r in enumerate(g.members):
                if not r.live:
                    continue
                r.iters += 1
                r.rnorm = float(new[i])
                if new[i] < tol or r.iters >= max_newton or not np.isfinite(new[i]):
                    finished.append(i)
            if finished:
                tr = time.perf_counter()
                # each finished request's result goes back to the host (its slice only)
                du, dh = b.s.device_tensor("udg"), b.s.device_tensor("uh")
                su, sh = du.numel() // b.eoff[-1], dh.numel() // b.hoff[-1]
                for i in finished:
                    r = g.members[i]
                    u = du[b.eoff[i] * su:b.eoff[i + 1] * su].cpu().numpy()
                    h = dh[b.hoff[i] * sh:b.hoff[i + 1] * sh].cpu().numpy()
                    r.udg = u.reshape(r.prob.udg.shape) if keep_states else None
                    r.uh = h.reshape(r.prob.uh.shape) if keep_states else None
                tnow = clock() - t0
                for i in finished:
                    r = g.members[i]
                    r.live = False
                    r.finish = tnow
                    done.append(r)
                if not g.live():
                    used -= sum(footprint_bytes(r.prob) for r in g.members)
                    _merge(phases, b.phases)
                    b.close()
                    g.solver, g.members = None, []
                phases["retire"] += time.perf_counter() - tr
    for g in groups.values():
        if g.solver is not None:
            _merge(phases, g.solver.phases)
            g.solver.close()
    return _stats(done, clock() - t0, batch_sizes, iterations, peak, phases)


def sequential(requests, tol=1e-10, max_newton=20, device=0, clock=time.perf_counter, keep_states=False,
               gmres_tol=1e-10, restart=50):
    """Plain FP64 solves, one request at a time in arrival order."""
    for r in requests:
        build_problem(r)
    t0 = clock()
    for r in sorted(requests, key=lambda r: r.arrival):
        now = clock() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        r.start = clock() - t0
        s = HDGSolver(r.prob, device=device)
        try:
            s.getQ()
            conv, hist = s.solveNonlinearProblem(newton_tol=tol, maxiter=max_newton, gmres_tol=gmres_tol,
                                                 restart=restart)
            r.iters = len(hist) - 1
            r.rnorm = float(hist[-1])
            udg, uh = s.get_solution()
            if keep_states:
                r.udg, r.uh = udg, uh
        finally:
            s.close()
        r.finish = clock() - t0
    return _stats(requests, clock() - t0, [1] * len(requests), sum(r.iters for r in requests))

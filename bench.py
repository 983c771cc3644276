#!/usr/bin/env python
"""Benchmark of the HDG element hot path on B200 (one JSON line on rank 0).

Workload (default): 3D compressible Navier-Stokes HDG, periodic unit cube,
20^3 hexes split into 6 tetrahedra = 48,000 elements, p = 3 (20 nodes, 5
conserved variables + gradients), FP64.  One step = one full pass of element
assembly + static condensation + scatter into the face-block system
(assembleLinearSystem), with the solution resident on the device.

  metric  assembly+Schur elements/s (FP64), whole job (sum over GPUs)
  e2e     the same step through the C ABI (hfem_assemble_host) with the state
          copied from pinned host memory every step, the copies overlapped with
          the element kernel piece by piece, and the residual norm read back
  roofline of the dominant kernel against the measured FP64 roof
  cpu_baseline  the reference's own C++ (oracle/_ref/hfem_ref, built from the
          reference sources) on the host cores, as a reported baseline

``--impl reference`` times only the reference CPU path (all host cores).
Multi-GPU runs are independent replicas (the path has no data exchange in
this single-GPU design): one process per GPU, weak scaling, max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "ns3d_p3_48k": dict(kind="ns3d_fourier", n=20, porder=3,
                        label="3D NS HDG, periodic unit cube 20^3x6 tets = 48000 elements, p=3, Re 400, Mach 0.3"),
    "ns3d_p3_6k": dict(kind="ns3d_fourier", n=10, porder=3,
                       label="3D NS HDG, periodic unit cube 10^3x6 tets = 6000 elements, p=3 (profiling size)"),
    "ns3d_p3_3k": dict(kind="ns3d_fourier", n=8, porder=3,
                       label="3D NS HDG, periodic unit cube 8^3x6 tets = 3072 elements, p=3 (ncu capture size)"),
    "ns2d_p2_2k": dict(kind="ns2d_vortex", n=32, porder=2,
                       label="2D NS HDG, periodic [0,10]^2 32x32x2 tris = 2048 elements, p=2, Re 100, Mach 0.5"),
}
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "hfem_ref")


def flops_per_element(prob):
    """Algorithmic FLOPs of assembly + Schur per element (GEMM and LU structure of the reference)."""
    m = prob.master
    nd, npv, npf, nfe, ngv, ngf = m.nd, m.npv, m.npf, m.nfe, m.ngv, m.ngf
    ncu = nch = nd + 2
    ndf = npf * nfe
    n, nb = npv * ncu, nch * ndf
    vol = (2 * npv * ncu * ngv * (nd + 1) + 2 * npv * (ncu * npv * ncu) * ngv * (nd + 1)
           + 2 * npv * (ncu * ncu * ndf) * ngv * (nd + 1))
    face = (2 * npf * npf * (nfe * nch * ncu) * ngf + 2 * npf * npf * (nfe * nch * nch) * ngf
            + 2 * npf * (nfe * ncu * npv * ncu) * ngf + 2 * npf * (nfe * ncu * ncu * ndf) * ngf)
    schur = (2.0 / 3.0) * n ** 3 + 2 * n * n * nb + 2 * nb * nb * n + 2 * n * n + 2 * nb * n
    return dict(element=float(vol + face), schur=float(schur))


def bytes_per_element(prob):
    """Algorithmic HBM bytes per element: inputs read, condensed outputs written (FP64)."""
    m = prob.master
    nd, npv, npf, nfe = m.nd, m.npv, m.npf, m.nfe
    ncu = nch = nd + 2
    nc = ncu * (nd + 1)
    n, nb = npv * ncu, nch * npf * nfe
    return 8.0 * (npv * nc + npv * nd + npf * nfe * nch) + 8.0 * (nb * nb + nb + n * nb + n)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # the timed region starts once the sampler has written its first line
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.05)
        self.skip = 1 if os.path.getsize(self.path) > 0 else 0

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        # the line written before the timed region is not one of its samples
        for line in open(self.path).readlines()[getattr(self, "skip", 0):]:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- CPU legs
def _write_ref_inputs(tmpdir, kind, porder, n):
    from hfem_b200.gen.problem import make_problem
    from hfem_b200.gen.refio import write_inputs
    prob = make_problem(kind, n=n, porder=porder)
    prefix = os.path.join(tmpdir, "in_")
    write_inputs(prefix, prob)
    return prefix, prob.mesh.ne


def _run_ref_timing(prefix, nelem, reps):
    env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
    out = subprocess.run([REF_BIN, "timing", prefix, str(nelem), str(reps)], check=True, capture_output=True,
                         text=True, env=env).stdout
    return json.loads(out.strip().splitlines()[-1])


# Reference runs time a 4^3 x 6 = 384-element mesh of the workload's element
# type per process: large enough that its assembled system (107 MB for p = 3)
# and element arrays leave the host caches, as the full workload's would.
REF_SAMPLE_N = 4


def reference_cpu(workload, seconds_per_proc=10.0, procs=None, reps=None):
    """Reference C++ assembleLinearSystem on the host cores: P independent processes
    (the reference's MPI driver cannot be built here; its OpenMP is disabled)."""
    if not os.path.exists(REF_BIN):
        return None
    w = WORKLOADS[workload]
    sample_n = REF_SAMPLE_N
    procs = procs or max(1, os.cpu_count() or 1)
    with tempfile.TemporaryDirectory() as tmp:
        prefix, ne = _write_ref_inputs(tmp, w["kind"], w["porder"], sample_n)
        calib = _run_ref_timing(prefix, ne, 1)
        if reps is None:
            reps = max(1, int(seconds_per_proc / max(calib["seconds"], 1e-3)))
        results = [None] * procs

        def worker(i):
            results[i] = _run_ref_timing(prefix, ne, reps)

        th = [threading.Thread(target=worker, args=(i,)) for i in range(procs)]
        t0 = time.time()
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.time() - t0
    total = sum(r["elems_per_s"] for r in results)
    return {"value": total, "unit": "elements/s", "cores": procs, "kind": "reference",
            "single_core_elems_per_s": calib["elems_per_s"],
            "sample": f"{w['kind']} p={w['porder']} on a {sample_n}^3x6={ne}-element periodic mesh, "
                      f"{reps} assembleLinearSystem passes in each of {procs} processes ({wall:.1f} s wall)"}


# ---------------------------------------------------------------- GPU leg
def run_gpu(args, rank, world, local_rank):
    import torch
    from hfem_b200.core import HDGSolver
    from hfem_b200.gen.problem import make_problem
    from hfem_b200.hwpeak import fp64_peak_tflops

    torch.cuda.set_device(local_rank)
    dev = local_rank
    w = WORKLOADS[args.workload]
    prob = make_problem(w["kind"], n=w["n"], porder=w["porder"], **({"seed": rank} if w["kind"] != "ns3d_tgv" else {}))
    ne = prob.mesh.ne
    solver = HDGSolver(prob, device=dev)
    stream = torch.cuda.current_stream()
    solver.set_stream(stream.cuda_stream)
    solver.getQ()
    udg_q, uh0 = solver.get_solution()

    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        dist = dist_mod

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        solver.assembleLinearSystem()
    torch.cuda.synchronize()

    sampler = ClockSampler(dev) if rank == 0 else None
    if sampler:
        sampler.start()
    solver.set_timing(True)
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        rnorm = solver.assembleLinearSystem()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    ktimes = solver.kernel_times()
    solver.set_timing(False)
    clocks = sampler.stop() if sampler else None

    # e2e: state from pinned host memory every step, residual norm back
    h_udg = torch.from_numpy(np.ascontiguousarray(udg_q)).pin_memory()
    h_uh = torch.from_numpy(np.ascontiguousarray(uh0)).pin_memory()
    h_sh = torch.from_numpy(np.ascontiguousarray(prob.sh)).pin_memory()
    def e2e_step():
        # hfem_assemble_host: the state's copies overlap the element kernel piece by piece
        return solver.assemble_from_host(h_udg.data_ptr(), h_uh.data_ptr(), h_sh.data_ptr(), chunks=args.e2e_chunks)

    for _ in range(max(1, args.warmup // 2)):
        e2e_step()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e0.elapsed_time(e1)

    # mixed precision legs: the same step in precision mode 1 (3xTF32 element
    # contractions, TF32 tcgen05 Schur GEMMs) and mode 3 (3xTF32 element
    # contractions, FP64 Schur); errors against this run's FP64 blocks
    def mixed_leg(mode):
        solver.set_precision(0)
        solver.set_solution(udg_q, uh0, prob.sh)
        r64 = solver.assembleLinearSystem()
        ref = {k: solver.device_tensor(k).clone() for k in ("K", "Hg", "DinvF")}
        solver.set_precision(mode)
        for _ in range(max(3, args.warmup)):
            solver.assembleLinearSystem()
        solver.set_timing(True)
        barrier()
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(args.steps):
            r32 = solver.assembleLinearSystem()
        m1.record(stream)
        torch.cuda.synchronize()
        barrier()
        leg_ms = m0.elapsed_time(m1)
        leg_k = solver.kernel_times()
        solver.set_timing(False)
        err = {}
        for k, v in ref.items():
            cur = solver.device_tensor(k)
            err[k] = float((cur - v).abs().max() / v.abs().max())
        err["rnorm"] = abs(r32 - r64) / r64
        del ref
        solver.set_precision(0)
        return leg_ms, leg_k, err

    mixed_ms, mixed_k, mixed_err = 0.0, {}, {}
    split_ms, split_k, split_err = 0.0, {}, {}
    if not args.no_mixed:
        mixed_ms, mixed_k, mixed_err = mixed_leg(1)
        split_ms, split_k, split_err = mixed_leg(3)

    if dist is not None:
        t = torch.tensor([ms, e2e_ms, mixed_ms, split_ms], dtype=torch.float64, device=f"cuda:{dev}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms, mixed_ms, split_ms = float(t[0]), float(t[1]), float(t[2]), float(t[3])
    solver.close()
    if rank != 0:
        return None

    fl = flops_per_element(prob)
    peak = fp64_peak_tflops(dev)
    dom = max(("element", "schur"), key=lambda k: ktimes.get(k, (0.0, 1))[0])
    kms, kcnt = ktimes[dom]
    avg_launch_s = kms / kcnt * 1e-3
    achieved = fl[dom] * ne / avg_launch_s / 1e12
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        tr = json.load(open(tfile)).get(args.workload, {}).get(dom)
        if tr:
            traffic = tr["bytes_per_element"] * ne
    launches = sum(v[1] for v in ktimes.values()) + args.steps   # + the rnorm reduction per step
    value = world * ne * args.steps / (ms * 1e-3)
    e2e_value = world * ne * args.steps / (e2e_ms * 1e-3)
    bpe = bytes_per_element(prob)
    line = {
        "metric": "assembly+Schur elements/s (FP64)",
        "value": value,
        "unit": "elements/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Fourier-mode flow on a generated periodic tetrahedral mesh)",
        "config": {"workload": w["label"], "elements_per_gpu": ne, "porder": prob.master.porder,
                   "local_dofs_D": prob.n_local, "trace_dofs_H": prob.n_trace,
                   "flops_per_element": fl["element"] + fl["schur"],
                   "l2": "inputs larger than L2 (UDG 154 MB, 48 GB of per-pass outputs); no flush needed",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "fp64", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": "measured in this run: FP64 FMA burst kernel (hfem_fp64_peak)",
                     "flops_per_launch": fl[dom] * ne, "avg_launch_ms": avg_launch_s * 1e3,
                     "hbm_view": {"algorithmic_bytes_per_step": bpe * ne,
                                  "achieved_gbs": bpe * ne / (ms * 1e-3 / args.steps) / 1e9}},
        "kernel_ms_per_step": {k: v[0] / args.steps for k, v in ktimes.items()},
        "e2e": {"value": e2e_value, "unit": "elements/s", "ms_per_step": e2e_ms / args.steps,
                "h2d_bytes_per_step": int(h_udg.numel() * 8 + h_uh.numel() * 8 + h_sh.numel() * 8),
                "d2h_bytes_per_step": 8 + 4 * ne},
        "clocks": clocks,
        "gpu_launches": launches,
        "rnorm": rnorm,
    }
    if not args.no_mixed:
        tc_ms = mixed_k.get("schur_tc", (0.0, 1))
        line["mixed"] = {
            "metric": "assembly+Schur elements/s (precision mode 1: 3xTF32 element contractions, TF32 tensor-core "
                      "Schur GEMMs, FP64 LU/residual)",
            "value": world * ne * args.steps / (mixed_ms * 1e-3), "unit": "elements/s",
            "ms_per_step": mixed_ms / args.steps, "speedup_vs_fp64": ms / mixed_ms,
            "error_vs_fp64": mixed_err,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in mixed_k.items()},
            "schur_tc_tflops": (2.0 * prob.n_local * prob.n_trace * (prob.n_local + prob.n_trace)) * ne
                               / (tc_ms[0] / tc_ms[1] * 1e-3) / 1e12 if tc_ms[0] > 0 else None}
        line["mixed_split"] = {
            "metric": "assembly+Schur elements/s (precision mode 3: 3xTF32 element contractions, FP64 LU, Schur "
                      "and residual)",
            "value": world * ne * args.steps / (split_ms * 1e-3), "unit": "elements/s",
            "ms_per_step": split_ms / args.steps, "speedup_vs_fp64": ms / split_ms,
            "error_vs_fp64": split_err,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in split_k.items()}}
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_cpu(args.workload, seconds_per_proc=args.cpu_seconds)
    return line


def run_reference(args, rank):
    if rank != 0:
        return None
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "oracle/_ref/hfem_ref not built (needs the reference sources)"}
    w = WORKLOADS[args.workload]
    procs = max(1, os.cpu_count() or 1)
    with tempfile.TemporaryDirectory() as tmp:
        prefix, ne = _write_ref_inputs(tmp, w["kind"], w["porder"], REF_SAMPLE_N)
        for _ in range(args.warmup):
            _run_ref_timing(prefix, ne, 1)
        results = [None] * procs

        def worker(i):
            results[i] = _run_ref_timing(prefix, ne, args.steps)

        th = [threading.Thread(target=worker, args=(i,)) for i in range(procs)]
        t0 = time.time()
        for t in th:
            t.start()
        for t in th:
            t.join()
        wall = time.time() - t0
    value = sum(r["elems_per_s"] for r in results)
    sample = (f"{w['kind']} p={w['porder']} on a {REF_SAMPLE_N}^3x6={ne}-element periodic mesh, {args.steps} "
              f"assembleLinearSystem passes per process, {procs} processes")
    return {"metric": "assembly+Schur elements/s (FP64)", "value": value, "unit": "elements/s", "impl": "reference",
            "n_gpus": 0, "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": w["label"], "sample": sample},
            "cpu_baseline": {"value": value, "unit": "elements/s", "cores": procs, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ------------------------------------------------------------- other tasks
def run_newton_task(args):
    """Config 1: one Newton step (assembly, BJ-GMRES(50) to 1e-10, update, residual) on
    the 2D p=2 vortex, repeated to the converged state; GPU vs the reference driver."""
    import torch
    from hfem_b200.core import HDGSolver
    from hfem_b200.gen.problem import ns2d_vortex
    prob = ns2d_vortex(n=32, porder=2)
    s = HDGSolver(prob)
    st = torch.cuda.current_stream()
    s.set_stream(st.cuda_stream)
    s.getQ()
    u0, h0 = s.get_solution()
    for _ in range(args.warmup):
        s.set_solution(u0, h0, prob.sh)
        s.solveNonlinearProblem(newton_tol=1e-10, maxiter=1, precond=args.precond)
    times, hist = [], None
    for _ in range(args.steps):
        s.set_solution(u0, h0, prob.sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        conv, hist = s.solveNonlinearProblem(newton_tol=1e-10, maxiter=1, precond=args.precond)
        e1.record(st)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    s.set_timing(True)
    _, gh = s.gmres(precond=args.precond, restart=50, tol=1e-10)
    kt = s.kernel_times()
    s.close()
    ms = float(np.median(times))
    pname = {2: "BJ", 0: "BILU0", -1: "unpreconditioned"}[args.precond]
    line = {"metric": f"Newton steps/s (2D NS p=2, 2048 elements, {pname}-GMRES(50) tol 1e-10)", "value": 1e3 / ms,
            "gmres_kernel_ms": {k: v[0] for k, v in kt.items()},
            "unit": "steps/s", "impl": "hfem", "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup,
            "dtype": "f64", "rnorm_history": [float(v) for v in hist], "gmres_iterations": int(len(gh)),
            "higher_is_better": True}
    if os.path.exists(REF_BIN):
        from hfem_b200.gen.refio import write_inputs
        with tempfile.TemporaryDirectory() as tmp:
            prefix = os.path.join(tmp, "in_")
            write_inputs(prefix, prob, newton_maxiter=1, gmres_tol=1e-10)
            env = dict(os.environ, OPENBLAS_NUM_THREADS="1")
            t0 = time.time()
            subprocess.run([REF_BIN, "newton", prefix, os.path.join(tmp, "out_"), "1", str(args.precond), "50",
                            "1e-10", "1"],
                           check=True, capture_output=True, env=env)
            wall = time.time() - t0
            rh = np.fromfile(os.path.join(tmp, "out_rnorm_hist.bin"))
        line["cpu_baseline"] = {"value": 1.0 / wall, "unit": "steps/s", "cores": 1, "kind": "reference",
                                "sample": "the same Newton step by oracle/_ref/hfem_ref (reference driver, one "
                                          "process, includes its set-up)",
                                "rnorm_history": [float(v) for v in rh]}
    return line


def run_dirk_task(args):
    """Config 4: Taylor-Green 16^3 x 6 tets, p = 3, Re 1600, Mach 0.1, DIRK(3,3),
    dt = 0.01, 20 steps, with the FP32 preconditioner and FP64 Jacobian, Newton
    residual, Arnoldi and update (precision mode 2) by default.
    The same steps in FP64 give the mixed run's kinetic-energy error against
    FP64; the 4^3 x 6 Taylor-Green case, 20 steps in the same precision, is
    checked against the reference driver's kinetic-energy history
    (tests/golden/tgv_p3_n4_dirk20.npz)."""
    import torch
    from hfem_b200.core import HDGSolver
    from hfem_b200.diagnostics import kinetic_energy
    from hfem_b200.gen.problem import ns3d_tgv

    def run(n, precision, steps, timed):
        prob = ns3d_tgv(n=n, porder=3, dt=0.01)
        s = HDGSolver(prob)
        st = torch.cuda.current_stream()
        s.set_stream(st.cuda_stream)
        s.set_precision(precision)
        s.getQ()
        u, _ = s.get_solution()
        ke = [kinetic_energy(prob, u)]
        iters, times = [], []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            iters.append(s.solveUnsteadyStep(0.01, stages=3, order=3, newton_tol=args.dirk_tol))
            e1.record(st)
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
            u, _ = s.get_solution()
            ke.append(kinetic_energy(prob, u))
        s.close()
        return prob, np.array(ke), iters, times

    prob, ke, iters, times = run(args.tgv_n, args.dirk_precision, args.dirk_steps, True)
    out = {"metric": f"DIRK(3,3) time steps/s (3D TGV {args.tgv_n}^3x6 tets = {prob.mesh.ne} elements, p=3)",
           "value": 1e3 / float(np.mean(times)), "unit": "steps/s", "impl": "hfem",
           "dtype": {0: "f64",
                     1: "mixed: f32 preconditioner, 3xtf32 element contractions, tf32 condensation GEMMs, "
                        "f64 Newton/Arnoldi",
                     2: "mixed: f32 preconditioner, f64 Jacobian, Newton and Arnoldi",
                     3: "mixed: f32 preconditioner, 3xtf32 element contractions, f64 condensation, Newton and "
                        "Arnoldi"}[args.dirk_precision],
           "ms_per_step": float(np.mean(times)), "steps": args.dirk_steps, "newton_iterations": iters,
           "newton_tol": args.dirk_tol, "kinetic_energy": ke.tolist(), "higher_is_better": True}
    if args.dirk_precision != 0:
        _, ke64, it64, t64 = run(args.tgv_n, 0, args.dirk_steps, True)
        out["fp64"] = {"ms_per_step": float(np.mean(t64)), "newton_iterations": it64,
                       "kinetic_energy_rel_diff": float(np.max(np.abs(ke - ke64) / ke64))}
    gfile = os.path.join(ROOT, "tests", "golden", "tgv_p3_n4_dirk20.npz")
    if os.path.exists(gfile):
        g = dict(np.load(gfile))
        _, ke4, _, _ = run(int(g["n"][0]), args.dirk_precision, int(g["nsteps"][0]), False)
        out["reference_check"] = {"case": "TGV 4^3x6 tets, p=3, 20 DIRK(3,3) steps of dt 0.01",
                                  "kinetic_energy_rel_err_vs_reference_driver": float(np.max(np.abs(ke4 - g["ke"])
                                                                                              / g["ke"]))}
    return out


def run_serve_task(args):
    """Config 5: a stream of independent 2D NS solve requests (Poisson arrivals,
    256-16,384 elements log-uniform, p in {1,2,3}, Re in [50,500], Mach in
    [0.2,0.7], Newton residual 1e-10), served with continuous batching and, on
    the same stream, by sequential plain FP64 solves."""
    import torch
    from hfem_b200.serve import build_problem, make_requests, sequential, serve
    torch.cuda.init()
    out = {"metric": "HDG solves/s with p50/p99 latency (2D NS request stream)", "unit": "solves/s",
           "impl": "hfem", "dtype": "f64", "higher_is_better": True, "data": "synthetic", "rates": []}
    for rate in args.serve_rates:
        reqs = make_requests(args.serve_requests, rate, seed=args.serve_seed)
        for r in reqs:
            build_problem(r)
        # warm the kernels, contexts and the device pool once with the same stream
        # (untimed), as the other tasks take warm-up steps
        serve([r for r in make_requests(6, 1e6, seed=999, max_el=512)], hbm_budget=None)
        warm = make_requests(args.serve_requests, rate, seed=args.serve_seed)[:args.serve_warm_requests]
        for a, b in zip(warm, reqs):
            a.prob = b.prob
        serve(warm, tol=1e-10, gmres_tol=args.serve_gmres_tol, repack_on_device=not args.serve_host_repack)
        st = serve(reqs, tol=1e-10, gmres_tol=args.serve_gmres_tol, repack_on_device=not args.serve_host_repack)
        seq_reqs = make_requests(args.serve_requests, rate, seed=args.serve_seed)[:args.serve_seq_requests]
        for a, b in zip(seq_reqs, reqs):
            a.prob = b.prob
        sq = sequential(seq_reqs, tol=1e-10, gmres_tol=args.serve_gmres_tol) if args.serve_seq_requests > 0 else None
        out["rates"].append({"rate": rate, "requests": len(reqs), "served": st.as_dict(),
                             "sequential": dict(sq.as_dict(), requests=len(seq_reqs)) if sq else None})
    best = out["rates"][-1]
    out["value"] = best["served"]["solves_per_s"]
    out["sequential_value"] = best["sequential"]["solves_per_s"] if best["sequential"] else None
    return out


def run_batched_task(args):
    """Config 3: 64 periodic 2D NS meshes, 512-32,768 elements (log-uniform), p in
    {1,2,3,4}, Mach U[0.2,0.8], vortex + noise.  One assembly pass over all of
    them as (a) plain per-mesh FP64 calls, (b) one graph launch in FP64 with
    autotuned tilings, (c) one graph launch with the TF32 tensor-core Schur GEMMs."""
    import math
    import torch
    from hfem_b200.batched import MixedOrderAssembly
    from hfem_b200.core import HDGSolver
    from hfem_b200.gen.problem import ns2d_vortex
    rng = np.random.default_rng(args.batched_seed)
    probs = []
    for i in range(args.batched_meshes):
        ne = math.exp(rng.uniform(math.log(512), math.log(32768)))
        n = max(4, int(round(math.sqrt(ne / 2))))
        probs.append(ns2d_vortex(n=n, porder=int(rng.integers(1, 5)), seed=1000 + i,
                                 mach=float(rng.uniform(0.2, 0.8))))
    ne = sum(p.mesh.ne for p in probs)
    # (a) plain FP64: one context and one assembleLinearSystem call per mesh
    plain = [HDGSolver(p) for p in probs]
    for s in plain:
        s.getQ()
        s.assembleLinearSystem()
    torch.cuda.synchronize()
    t_plain = []
    for _ in range(args.steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r_plain = [s.assembleLinearSystem() for s in plain]
        e1.record()
        torch.cuda.synchronize()
        t_plain.append(e0.elapsed_time(e1))
    for s in plain:
        s.close()
    out = {"metric": "batched mixed-order assembly+Schur elements/s (64 2D NS meshes, p 1-4)",
           "unit": "elements/s", "impl": "hfem", "higher_is_better": True, "data": "synthetic",
           "elements": ne, "meshes": len(probs), "steps": args.steps,
           "orders": {str(p): int(sum(q.mesh.ne for q in probs if q.master.porder == p)) for p in (1, 2, 3, 4)},
           "plain_fp64": {"value": ne / (np.median(t_plain) * 1e-3), "ms": float(np.median(t_plain))}}
    for name, prec in (("graph_fp64", 0), ("graph_mixed", 1)):
        m = MixedOrderAssembly(probs, precision=prec, tune=True)
        for _ in range(max(3, args.warmup)):
            m.launch()
        m.finish()
        ts = []
        for _ in range(args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(m.stream)
            m.launch()
            e1.record(m.stream)
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        rn = m.finish()
        out[name] = {"value": ne / (np.median(ts) * 1e-3), "ms": float(np.median(ts)),
                     "max_rnorm_rel_diff_vs_plain": float(np.max(np.abs(rn - np.array(r_plain)) / np.array(r_plain))),
                     "tiles": {f"{k[0]}d_p{k[1]}": v for k, v in m.tiles.items()}}
        if prec == 1:
            out[name]["dtype"] = "3xtf32 element contractions, tf32 Schur GEMMs where the autotuner picks them, f64 element LU / residual"
            out[name]["fp64_shapes"] = [f"{k[0]}d_p{k[1]}" for k in m.fp64_shapes]
        m.close()
    out["value"] = out["graph_mixed"]["value"]
    out["speedup_graph_mixed_vs_plain_fp64"] = out["graph_mixed"]["value"] / out["plain_fp64"]["value"]
    out["speedup_graph_fp64_vs_plain_fp64"] = out["graph_fp64"]["value"] / out["plain_fp64"]["value"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hfem", choices=["hfem", "reference"])
    ap.add_argument("--workload", default="ns3d_p3_48k", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision legs (precision modes 1 and 3)")
    ap.add_argument("--e2e-chunks", type=int, default=8, help="pieces of the element-wise state copied ahead of the element kernel in the e2e leg")
    ap.add_argument("--task", default="assembly", choices=["assembly", "newton", "dirk", "serve", "batched"])
    ap.add_argument("--batched-meshes", type=int, default=64)
    ap.add_argument("--precond", type=int, default=2, choices=[-1, 0, 2],
                    help="GMRES preconditioner of the newton task: 2 block Jacobi, 0 BILU0 (MDF order), -1 none")
    ap.add_argument("--batched-seed", type=int, default=0)
    ap.add_argument("--tgv-n", type=int, default=16)
    ap.add_argument("--dirk-steps", type=int, default=20)
    ap.add_argument("--dirk-tol", type=float, default=1e-10)
    ap.add_argument("--dirk-precision", type=int, default=2, choices=[0, 1, 2, 3],
                    help="0 FP64; 1 3xTF32 element + TF32 Schur + FP32 preconditioner; 2 FP32 preconditioner "
                         "(config 4); 3 3xTF32 element + FP32 preconditioner")
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[20.0, 50.0, 100.0])
    ap.add_argument("--serve-requests", type=int, default=2000)
    ap.add_argument("--serve-seq-requests", type=int, default=2000)
    ap.add_argument("--serve-warm-requests", type=int, default=300,
                    help="requests of the same stream served once, untimed, before the timed pass")
    ap.add_argument("--serve-seed", type=int, default=0)
    ap.add_argument("--serve-gmres-tol", type=float, default=1e-10)
    ap.add_argument("--serve-host-repack", action="store_true",
                    help="carry in-flight states through host memory when a group is repacked")
    args = ap.parse_args()
    if args.task != "assembly":
        line = {"newton": run_newton_task, "dirk": run_dirk_task, "serve": run_serve_task,
                "batched": run_batched_task}[args.task](args)
        print(json.dumps(line), flush=True)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "hfem" else args.warmup

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        line = run_reference(args, rank)
    else:
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(local_rank)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        line = run_gpu(args, rank, world, local_rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark: continuous Q4 Laplace vmult (GDoF/s) on the deformed unit cube.

Workload (one step = one operator application dst = A src over the whole mesh): 128^3
hexahedra of [0,1]^3 mapped by x' = x + 0.1 sin(pi x) sin(pi y) sin(pi z) (per component,
Q4 isoparametric, non-affine Jacobians at 5^3 Gauss points), FE_Q(4), 135,005,697 DoFs, src
uniform[-1,1] from seed 1234, FP64.  Inputs (12.6 GB of geometry) are far larger than L2,
so no L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--cells 128]

--impl b200 (default): the CUDA library through its C ABI.  `value` is device-timed with
the inputs resident in HBM; `e2e` repeats the measurement through the same C-ABI call with
the input in pinned host memory, the host->device copy of src and the device->host copy of
dst inside the timed region.  Under torchrun (N > 1) every rank runs an independent replica
(the operator is not partitioned across GPUs); value sums the ranks' DoFs over the slowest
rank's time.
--impl reference: the CPU restatement of the reference's operator (oracle/pmg_oracle.c;
the reference itself needs deal.II + Kokkos + MPI + p4est, none of which exist here) on all
host cores, on a bounded sample of the same workload (the same deformed-cube mesh family
at 32^3 cells).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "portable-multigrid_b200"))
sys.path.insert(0, ROOT)

METRIC = "Q4 vmult GDoF/s"
WORKLOAD = "Q4 Laplace vmult, deformed unit cube x'=x+0.1 sin(pi x)sin(pi y)sin(pi z)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cells", type=int, default=128, help="cells per direction (power of 2)")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--skip-cpu", action="store_true", help="omit the cpu_baseline leg")
    ap.add_argument("--skip-solve", action="store_true",
                    help="omit the time-to-solution leg (Q6 variable-kappa ph-multigrid CG)")
    ap.add_argument("--case", choices=sorted(PROFILE_CASES), default=None,
                    help="profiling mode: run one representative launch set of a solver path "
                         "inside the NVTX range 'prof' and exit (no bench line)")
    ap.add_argument("--refine", type=int, default=None, help="refinements of the --case mesh")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def slowest_rank_ms(times_ms, device):
    """Each of the local device times (ms) as the maximum over all ranks of the default process
    group (the job is as slow as its slowest replica); unchanged without a process group."""
    import torch
    t = torch.tensor([float(v) for v in times_ms], dtype=torch.float64, device=device)
    dist = torch.distributed
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def replica_rate(n_dofs, world, steps, ms):
    """Whole-job GDoF/s of `world` replicas that each applied the operator `steps` times to
    n_dofs DoFs in `ms` milliseconds (the slowest rank's time)."""
    return n_dofs * world * steps / (ms * 1e-3) / 1e9


def box_for(cells):
    refine = int(round(np.log2(cells)))
    assert 1 << refine == cells, "--cells must be a power of two"
    return refine


# ----------------------------------------------------------------------------------------
# CPU leg: the oracle's OpenMP vmult on a bounded sample (same mesh family, 32^3 cells)
# ----------------------------------------------------------------------------------------
def cpu_vmult_rate(steps=None, seconds=12.0, sample_cells=32):
    from oracle import oracle as O
    refine = box_for(sample_cells)
    box = O.Box.make(refine=refine, deform=1, amp=0.1)
    plain, cons, idx = O.dofs(box, 4)
    G = O.geometry_G(box, 4)
    color = O.colors(box)
    src = np.random.default_rng(1234).uniform(-1.0, 1.0, cons.shape[0])
    O.vmult(4, idx, G, cons, src, color=color)  # warm
    n = 0
    t0 = time.perf_counter()
    while True:
        O.vmult(4, idx, G, cons, src, color=color)
        n += 1
        el = time.perf_counter() - t0
        if (steps is not None and n >= steps) or (steps is None and el >= seconds):
            break
    rate = cons.shape[0] * n / el / 1e9
    return rate, {"n_dofs": int(cons.shape[0]), "vmults": n, "seconds": el,
                  "cores": O.num_threads()}


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    # each step is one vmult of the 32^3 sample
    rate_w, info_w = cpu_vmult_rate(steps=max(1, args.warmup))
    rate, info = cpu_vmult_rate(steps=max(1, args.steps))
    sample = (f"oracle CPU restatement, OpenMP over {info['cores']} threads, {info['vmults']} "
              f"vmults of the 32^3-cell deformed cube (Q4, {info['n_dofs']} DoFs)")
    line = {
        "metric": METRIC, "value": rate, "unit": "GDoF/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": info["seconds"] / info["vmults"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": WORKLOAD + " (32^3-cell sample on the host CPU)",
                   "cells": 32 ** 3, "n_dofs": info["n_dofs"], "degree": 4},
        "cpu_baseline": {"value": rate, "unit": "GDoF/s", "cores": info["cores"], "kind": "port",
                         "sample": sample},
        "e2e": {"value": rate, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------
# GPU arm
# ----------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=10)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(key):
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(key)


def time_vmults(op, dst, src, steps, torch, stream):
    import pmg
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    pmg.profile_reset()
    pmg.profile_enable(True)
    start.record(stream)
    for _ in range(steps):
        op.vmult(dst, src)
    stop.record(stream)
    stop.synchronize()
    pmg.profile_enable(False)
    total_ms = start.elapsed_time(stop)
    cell_ms, cell_n = pmg.profile_query("vmult_cell")
    cons_ms, cons_n = pmg.profile_query("vmult_init")
    return total_ms, cell_ms, cell_n, cons_n


def e2e_vmults(op, src_host, steps, torch, dev, barrier):
    """End-to-end vmults from and to pinned host memory: every step copies its input host ->
    device, applies the operator through the C ABI and copies the result device -> host.
    Returns (pipelined ms, serial ms) for `steps` steps.  Pipelined: step i's H2D, vmult and
    D2H run on three streams, step i+1's H2D overlapping step i's vmult and step i-1's D2H
    (two device buffer pairs, event dependencies); serial: all on one stream."""
    device = f"cuda:{dev}"
    src_pinned = src_host.pin_memory()
    dst_pinned = [torch.empty_like(src_pinned).pin_memory() for _ in range(2)]
    srcs = [torch.empty(src_host.shape, dtype=src_host.dtype, device=device) for _ in range(2)]
    dsts = [torch.empty_like(srcs[0]) for _ in range(2)]
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()

    def pipelined(n):
        h2d = [torch.cuda.Event() for _ in range(n)]
        comp = [torch.cuda.Event() for _ in range(n)]
        d2h = [torch.cuda.Event() for _ in range(n)]
        for i in range(n):
            b = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(comp[i - 2])   # srcs[b] read by step i-2
                srcs[b].copy_(src_pinned, non_blocking=True)
                h2d[i].record(s_in)
            with torch.cuda.stream(s_comp):
                s_comp.wait_event(h2d[i])
                if i >= 2:
                    s_comp.wait_event(d2h[i - 2])  # dsts[b] read back by step i-2
                op.vmult(dsts[b], srcs[b])
                comp[i].record(s_comp)
            with torch.cuda.stream(s_out):
                s_out.wait_event(comp[i])
                dst_pinned[b].copy_(dsts[b], non_blocking=True)
                d2h[i].record(s_out)
        return d2h[-1]

    pipelined(2)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(s_in)
    s_comp.wait_event(ev0)
    s_out.wait_event(ev0)
    last = pipelined(steps)
    s_out.wait_event(last)
    ev1.record(s_out)
    ev1.synchronize()
    t_pipe = ev0.elapsed_time(ev1)
    torch.cuda.synchronize()
    barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        srcs[0].copy_(src_pinned, non_blocking=True)
        op.vmult(dsts[0], srcs[0])
        dst_pinned[0].copy_(dsts[0], non_blocking=True)
    e1.record(stream)
    e1.synchronize()
    t_serial = e0.elapsed_time(e1)
    del srcs, dsts, src_pinned, dst_pinned
    torch.cuda.synchronize()
    return t_pipe, t_serial


def vmult_sweep(torch, pmg, dev, peak, steps=100, warmup=10, sizes=(16, 32, 64)):
    """The deformed-cube Q4 vmult at the smaller sizes of the refinement sweep, FP64 and FP32:
    GDoF/s over `steps` event-timed vmults after `warmup`, and the cell kernel's algorithmic
    bytes over its average event-timed duration as a fraction of the HBM peak.  At 16^3 and
    32^3 the inputs fit in L2 (31 MB / 248 MB FP64), so those rates are L2-resident, not HBM
    rates."""
    out = {}
    stream = torch.cuda.current_stream()
    for cells in sizes:
        mesh = pmg.Mesh(pmg.Box.make(refine=box_for(cells), deform=1, amp=0.1))
        for name, dt, tdt in (("f64", pmg.F64, torch.float64), ("f32", pmg.F32, torch.float32)):
            op = pmg.LaplaceOperator(mesh, 4, dt, pmg.GEOMETRY_FULL, device=dev)
            n = op.m()
            src = torch.from_numpy(np.random.default_rng(1234).uniform(-1.0, 1.0, n)).to(tdt).to(f"cuda:{dev}")
            dst = torch.empty_like(src)
            for _ in range(warmup):
                op.vmult(dst, src)
            torch.cuda.synchronize()
            total_ms, cell_ms, cell_n, _ = time_vmults(op, dst, src, steps, torch, stream)
            bw = op.bytes_per_vmult() / (cell_ms / max(cell_n, 1) * 1e-3) / 1e9
            out[f"{cells}^3_{name}"] = {"n_dofs": n, "gdofs": n * steps / (total_ms * 1e-3) / 1e9,
                                        "cell_kernel_gbs": bw, "frac_of_hbm": bw / peak}
            del op, src, dst
        del mesh
    torch.cuda.empty_cache()
    return out


def plain_method(torch, pmg, dev, repeats=3):
    """The plain method: -lap u = 3 pi^2 sin(pi x) sin(pi y) sin(pi z) on [0,1]^3, FE_Q(2) on 16^3
    cells (35,937 DoFs), geometric multigrid at degree 2 on every level 16^3 .. 2^3,
    Chebyshev(3), FP64 CG to a relative residual of 1e-10; FP64 and FP32 V-cycles, median of
    `repeats` solves after one warm-up, with the L2 error against the exact solution."""
    box = pmg.Box.make(coarse=(2, 2, 2), refine=3)
    res = {}
    for name, dt in (("fp64_mg", pmg.F64), ("fp32_mg", pmg.F32)):
        h = pmg.Hierarchy(box, [2], mg_dtype=dt, cheb_degree=3, h_degree=2, device=dev)
        b = h.fine64.assemble_rhs(1, 4)
        h.estimate()
        h.solve(b, reduce=1e-10)
        times, info, x = [], None, None
        for _ in range(repeats):
            x = h.fine64.initialize_dof_vector()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            x, info = h.solve(b, x=x, reduce=1e-10)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        res[name] = {"seconds": float(np.median(times)), "iterations": info["iterations"],
                     "reduction_per_step": info["reduction_per_step"], "l2_error": h.fine64.l2_error(x, 1)}
        n = h.fine64.m()
        del h, b, x
    res["n_dofs"] = n
    res["config"] = "Q2, 16^3 cells, h-multigrid at degree 2 to 2^3, Chebyshev(3), FP64 CG to 1e-10"
    return res


def time_to_solution(torch, pmg, dev, refine=4, repeats=3):
    """Q6, kappa = 1 + 0.9 sin(2 pi x) sin(2 pi y) sin(2 pi z), 48^3 affine cells (3^3 coarse
    cells refined 4 times, 24,137,569 DoFs), f = 1, homogeneous Dirichlet; ph-multigrid with
    p 6 -> 3 -> 2 -> 1 and Q1 h-levels 48^3 .. 3^3, Chebyshev degree 4; FP64 CG to a relative
    residual of 1e-10.  The V-cycle runs in FP32 (mixed) or FP64 (all-FP64 method); each
    number is the median of `repeats` solves from x = 0 after one warm-up solve.  Each
    variant's solution is compared with the FP64 ph-multigrid CG run to 1e-12
    (`error_vs_fp64_1e-12`: max-norm difference relative to the max norm of that solution)."""
    box = pmg.Box.make(coarse=(3, 3, 3), refine=refine)
    res = {}
    solutions, x_ref = {}, None
    # fp32_mg / fp64_mg: the ph-multigrid with an FP32 / FP64 V-cycle; fp64_plain_hmg: the
    # all-FP64 plain method (geometric multigrid at degree 6 on every level 48^3 .. 3^3,
    # GeometricTransfer<dim, fe_degree> as in source/geometric_multigrid/program.cc:245-249)
    # fp32_mg_tf32 / fp32_mg_3xtf32: the FP32 V-cycle with its affine levels on the tensor cores
    for name, dt, pseq, hdeg, tc in (("fp32_mg", pmg.F32, [6, 3, 2, 1], 1, 0),
                                     ("fp32_mg_tf32", pmg.F32, [6, 3, 2, 1], 1, 1),
                                     ("fp32_mg_3xtf32", pmg.F32, [6, 3, 2, 1], 1, 3),
                                     ("fp64_mg", pmg.F64, [6, 3, 2, 1], 1, 0),
                                     ("fp64_plain_hmg", pmg.F64, [6], 6, 0)):
        h = pmg.Hierarchy(box, pseq, mg_dtype=dt, cheb_degree=4, h_degree=hdeg, tensor_cores=tc,
                          geometry=pmg.GEOMETRY_AFFINE, coeff_kind=pmg.COEFF_KAPPA, device=dev)
        b = h.fine64.assemble_rhs(0)
        h.estimate()
        h.solve(b, reduce=1e-10)
        times, info = [], None
        for _ in range(repeats):
            x = h.fine64.initialize_dof_vector()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            x, info = h.solve(b, x=x, reduce=1e-10)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        r = h.fine64.initialize_dof_vector()
        h.fine64.vmult(r, x)
        rel = float(torch.linalg.norm(r - b) / torch.linalg.norm(b))
        res[name] = {"seconds": float(np.median(times)), "iterations": info["iterations"],
                     "relative_residual": rel, "reduction_per_step": info["reduction_per_step"]}
        solutions[name] = x
        if name == "fp64_mg":
            x_ref, _ = h.solve(b, x=h.fine64.initialize_dof_vector(), reduce=1e-12, max_iterations=100)
        n = h.fine64.m()
        del h, b, r
        torch.cuda.empty_cache()
    scale = float(x_ref.abs().max())
    for name, x in solutions.items():
        res[name]["error_vs_fp64_1e-12"] = float((x - x_ref).abs().max()) / scale
    del solutions, x_ref
    torch.cuda.empty_cache()
    res["n_dofs"] = n
    res["speedup_fp32_mg_over_fp64"] = res["fp64_mg"]["seconds"] / res["fp32_mg"]["seconds"]
    res["speedup_fp32_mg_over_fp64_plain"] = res["fp64_plain_hmg"]["seconds"] / res["fp32_mg"]["seconds"]
    res["config"] = ("Q6 variable kappa, 48^3 affine cells, Chebyshev(4); ph-multigrid p 6-3-2-1 + Q1 h-levels to "
                     "3^3 (FP32 or FP64 V-cycle) against the plain method (FP64 h-multigrid at Q6 to 3^3)")
    return res


def q6_kernel_rates(torch, pmg, dev, peaks, refine=4, launches=20):
    """The Q6 affine + kappa cell kernels of the config-3 fine level (48^3 cells) alone, FP32
    and FP64: event-timed duration per launch and the algorithmic FLOP rate against the
    same-run FMA peak.  Algorithmic FLOPs per cell: 24 N^4 (twelve 1D passes of N^4
    multiply-adds: interpolation and derivative in three directions, forward and transposed)
    + 6 N^3 (the diagonal cell tensor times weight and coefficient at each point), N = 7.  The
    even/odd form executes about half the passes' multiply-adds, so the rate is an
    algorithmic one, not an instruction count."""
    box = pmg.Box.make(coarse=(3, 3, 3), refine=refine)
    mesh = pmg.Mesh(box)
    N = 7
    flops = mesh.n_cells() * (24 * N ** 4 + 6 * N ** 3)
    res = {"algorithmic_flops_per_launch": flops}
    for name, dt, tdt, peak_key, tc in (("fp32", pmg.F32, torch.float32, "fp32_fma_tflops", 0),
                                        ("fp32_tf32", pmg.F32, torch.float32, "fp32_fma_tflops", 1),
                                        ("fp32_3xtf32", pmg.F32, torch.float32, "fp32_fma_tflops", 3),
                                        ("fp64", pmg.F64, torch.float64, "fp64_fma_tflops", 0)):
        op = pmg.LaplaceOperator(mesh, 6, dt, pmg.GEOMETRY_AFFINE, pmg.COEFF_KAPPA, device=dev)
        if tc:
            op.set_tensor_cores(tc)
        src = torch.rand(op.m(), dtype=tdt, device=f"cuda:{dev}")
        dst = torch.empty_like(src)
        for _ in range(3):
            op.vmult(dst, src)
        torch.cuda.synchronize()
        pmg.profile_reset()
        pmg.profile_enable(True)
        for _ in range(launches):
            op.vmult(dst, src)
        torch.cuda.synchronize()
        pmg.profile_enable(False)
        ms, n = pmg.profile_query("vmult_cell")
        t = ms / max(n, 1) * 1e-3
        tflops = flops / t / 1e12
        res[name] = {"cell_kernel_us": t * 1e6, "algorithmic_tflops": tflops,
                     "frac_of_same_run_fma": tflops / peaks[peak_key] if peaks else None}
        del op, src, dst
    del mesh
    torch.cuda.empty_cache()
    return res


# the reference's logged GH200 figures for the doubling-mesh solve (seconds, CG iterations)
REFERENCE_LOGS = {
    # one GH200: tests/poisson_cube_bk3_fp64/results/single-gpu-batched.out:1172-1184 and
    # tests/poisson_cube_bk3/results/signle-gpu-batched-mixed-precision.out:1262-1281
    20: {"gpus": 1, "fp64_mg_seconds": 0.5695, "fp32_mg_seconds": 0.4902, "iterations": 5,
         "fp64_mg_setup_seconds": 129.87, "fp32_mg_setup_seconds": 194.33},
    # four GH200 (MPI): tests/poisson_cube_bk3_fp64/results/1-node-batched.out:1388,1417,1463 and
    # tests/poisson_cube_bk3/results/1-node-batched-mixed-precision.out:1485,1514,1560
    22: {"gpus": 4, "fp64_mg_seconds": 0.77931, "fp32_mg_seconds": 0.61183, "iterations": 5,
         "fp64_mg_setup_seconds": 136.41, "fp32_mg_setup_seconds": 206.83},
}


def reference_problem(torch, pmg, dev, cycle=20, repeats=3):
    """The reference's own logged solve: Q4, f = 1, homogeneous Dirichlet on the "doubling" mesh
    of `cycle` (cycle 20: 2 x 2 x 1 coarse cells refined 6 times, 67,634,433 DoFs; cycle 22:
    269,748,225 DoFs), ph-multigrid with p 4 -> 3 -> 2 -> 1 and Q1 h-levels, Chebyshev(5), CG to
    a reduction of 1e-9, all-FP64 and with the FP32 V-cycle; setup (hierarchy, right-hand side,
    eigenvalue estimates) and solve times on this one GPU next to the GH200 figures the
    reference logged for the same problem (REFERENCE_LOGS: one GH200 at cycle 20, four at
    cycle 22)."""
    box = pmg.doubling_box(cycle)
    res = {}
    for name, dt in (("fp64_mg", pmg.F64), ("fp32_mg", pmg.F32)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = pmg.Hierarchy(box, [4, 3, 2, 1], mg_dtype=dt, cheb_degree=5, device=dev)
        b = h.fine64.assemble_rhs(0)
        h.estimate()
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        h.solve(b)
        times, info = [], None
        for _ in range(repeats):
            x = h.fine64.initialize_dof_vector()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            x, info = h.solve(b, x=x)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        res[name] = {"seconds": float(np.median(times)), "iterations": info["iterations"],
                     "reduction_per_step": info["reduction_per_step"], "setup_seconds": setup}
        n = h.fine64.m()
        del h, b, x
        torch.cuda.empty_cache()
    res["n_dofs"] = n
    ref = REFERENCE_LOGS[cycle]
    res["reference_gh200"] = ref
    res["speedup_vs_reference"] = {"fp64_mg": ref["fp64_mg_seconds"] / res["fp64_mg"]["seconds"],
                                   "fp32_mg": ref["fp32_mg_seconds"] / res["fp32_mg"]["seconds"]}
    res["config"] = (f"Q4 doubling mesh cycle {cycle}, p 4-3-2-1 + Q1 h-levels, Chebyshev(5), CG to 1e-9; "
                     f"one B200 against {ref['gpus']} GH200")
    return res


def dg_time_to_solution(torch, pmg, dev, refine=6, repeats=3):
    """DG-SIPG Q3 on 64^3 Cartesian cells (16,777,216 DoFs), penalty 2 (p+1)^2 / h,
    u = exp(x) sin(pi y) cos(pi z) with the Dirichlet data imposed weakly; multigrid
    DG Q3 -> continuous Q3 -> Q1 -> Q1 h-levels to 1^3, Chebyshev degree 5, inside FP64 CG to
    a relative residual of 1e-10; FP32 and FP64 V-cycles, median of `repeats` solves."""
    p = 3
    box = pmg.Box.make(refine=refine)
    res = {}
    for name, dt in (("fp32_mg", pmg.F32), ("fp64_mg", pmg.F64)):
        h = pmg.Hierarchy(box, [3, 1], mg_dtype=dt, cheb_degree=5, dg=True, penalty=2.0 * (p + 1) ** 2,
                          device=dev)
        b = h.fine64.assemble_rhs(2, p + 2)
        h.estimate()
        h.solve(b, reduce=1e-10, max_iterations=300)
        times, info = [], None
        for _ in range(repeats):
            x = h.fine64.initialize_dof_vector()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record()
            x, info = h.solve(b, x=x, reduce=1e-10, max_iterations=300)
            e1.record()
            e1.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        res[name] = {"seconds": float(np.median(times)), "iterations": info["iterations"],
                     "reduction_per_step": info["reduction_per_step"]}
        n = h.fine64.m()
        del h, b, x
        torch.cuda.empty_cache()
    res["n_dofs"] = n
    res["speedup_fp32_mg_over_fp64"] = res["fp64_mg"]["seconds"] / res["fp32_mg"]["seconds"]
    res["config"] = "DG-SIPG Q3, 64^3 cells, DG Q3 -> CG Q3 -> Q1 -> h-levels, Chebyshev(5)"
    res["dg_vmult"] = dg_vmult_rates(torch, pmg, dev, refine)
    return res


def dg_vmult_rates(torch, pmg, dev, refine=6, launches=20, peak=None):
    """The DG-SIPG Q3 vmult of config 4 alone (64^3 cells), FP32 and FP64: CUDA-event time per
    vmult (all its kernels: the fused tile kernel where the mesh allows it), GDoF/s and the
    algorithmic bytes 2 s N + 6 s C (src read and dst written once, six geometry values per
    cell; DG indices are implicit) over that time as a fraction of the HBM peak."""
    p = 3
    mesh = pmg.Mesh(pmg.Box.make(refine=refine))
    peak = peak or measured_peaks()[0]
    out = {}
    for name, dt, tdt in (("fp32", pmg.F32, torch.float32), ("fp64", pmg.F64, torch.float64)):
        op = pmg.DGLaplaceOperator(mesh, p, dt, 2.0 * (p + 1) ** 2, device=dev)
        src = torch.rand(op.m(), dtype=tdt, device=f"cuda:{dev}")
        dst = torch.empty_like(src)
        for _ in range(3):
            op.vmult(dst, src)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(launches):
            op.vmult(dst, src)
        e1.record()
        e1.synchronize()
        t = e0.elapsed_time(e1) / launches * 1e-3
        s = 8 if dt == pmg.F64 else 4
        alg = 2 * s * op.m() + 6 * s * mesh.n_cells()
        units, par = op.last_launch(pmg.KERNEL_DG_FACES)
        out[name] = {"vmult_us": t * 1e6, "gdofs": op.m() / t / 1e9, "algorithmic_bytes": alg,
                     "frac_of_hbm": alg / t / 1e9 / peak, "tiles": units, "blocks": par}
        del op, src, dst
    del mesh
    torch.cuda.empty_cache()
    out["peak_gbs"] = peak
    return out


def adjoint_check(torch, pmg, dev, refine=5, n_dirs=8, eps=1e-6):
    """-div(exp(m) grad u) = 1 on the unit cube, Q4 on 32^3 cells (2,146,689 DoFs); m and the
    target's m_B are sums of 16 random Fourier modes (seeds 1 and 2) with std 0.5 over the
    quadrature points; u_d = u(m_B); J = 1/2 ||u - u_d||^2_{L2}.  Times one gradient (coefficient
    load on all levels, forward solve, adjoint solve, per-point kernel; solves to 1e-13 with the
    FP32 V-cycle inside FP64 CG) and checks <g, d> against central differences in n_dirs
    directions (seeds 100..), eps = 1e-6."""
    from pmg.adjoint import AdjointPoisson, fourier_field
    box = pmg.Box.make(refine=refine)
    prob = AdjointPoisson(box, degree=4, reduce=1e-13, device=dev)
    xq = prob.quadrature_points()
    u_d = prob.solve(fourier_field(xq, seed=2))
    m = fourier_field(xq, seed=1)
    prob.gradient(m, u_d)
    times = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        J, g, _ = prob.gradient(m, u_d)
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
    errs = []
    for k in range(n_dirs):
        d = fourier_field(xq, seed=100 + k)
        fd = (prob.objective(m + eps * d, u_d)[0] - prob.objective(m - eps * d, u_d)[0]) / (2 * eps)
        ad = float((g * d).sum())
        errs.append(abs(fd - ad) / abs(ad))
    out = {"n_dofs": prob.A.m(), "J": J, "gradient_seconds": float(np.median(times)),
           "forward_iterations": prob.last_info["forward"]["iterations"],
           "adjoint_iterations": prob.last_info["adjoint"]["iterations"],
           "fd_rel_err_max": max(errs), "fd_directions": n_dirs, "eps": eps,
           "config": "Q4, 32^3 cells, p 4-2-1 + Q1 h-levels, FP32 V-cycle in FP64 CG to 1e-13"}
    del prob, xq, u_d, m, g
    torch.cuda.empty_cache()
    return out


def gpu_arm(args):
    import torch
    import pmg
    rank, world, local = dist_env()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.cuda.current_device()
    # same-run peaks (copy bandwidth, FMA rates) before anything else holds device memory
    peaks = pmg.measure_peaks(dev, 1 << 30) if rank == 0 else None
    dt = pmg.F64 if args.dtype == "f64" else pmg.F32
    tdt = torch.float64 if dt == pmg.F64 else torch.float32
    refine = box_for(args.cells)
    box = pmg.Box.make(refine=refine, deform=1, amp=0.1)
    t_setup = time.perf_counter()
    mesh = pmg.Mesh(box)
    op = pmg.LaplaceOperator(mesh, 4, dt, pmg.GEOMETRY_FULL, device=dev)
    torch.cuda.synchronize()
    t_setup = time.perf_counter() - t_setup
    N = op.m()
    src_host = torch.from_numpy(np.random.default_rng(1234).uniform(-1.0, 1.0, N)).to(tdt)
    src = src_host.to(f"cuda:{dev}")
    dst = torch.empty_like(src)
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(max(args.warmup, 3)):
        op.vmult(dst, src)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(dev)
    clocks.start()
    total_ms, cell_ms, cell_n, cons_n = time_vmults(op, dst, src, args.steps, torch, stream)
    clk = clocks.stop()
    torch.cuda.synchronize()
    barrier()
    # slowest rank
    t_max = slowest_rank_ms([total_ms], f"cuda:{dev}")[0]
    ms_per_step = t_max / args.steps
    value = replica_rate(N, world, args.steps, t_max)

    # end to end through the same C-ABI call, host buffers, copies inside the timed region
    e2e_steps = max(3, min(args.steps // 10, 20))
    e2e_ms, e2e_serial_ms = e2e_vmults(op, src_host, e2e_steps, torch, dev, barrier)
    e2e_ms, e2e_serial_ms = slowest_rank_ms([e2e_ms, e2e_serial_ms], f"cuda:{dev}")
    e2e_value = replica_rate(N, world, e2e_steps, e2e_ms)
    e2e_serial = replica_rate(N, world, e2e_steps, e2e_serial_ms)
    bytes_elem = 8 if dt == pmg.F64 else 4

    # roofline of the cell kernel: algorithmic bytes per launch over its event-timed duration
    alg_bytes = op.bytes_per_vmult()
    cell_avg_s = (cell_ms / max(cell_n, 1)) * 1e-3
    achieved = alg_bytes / cell_avg_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic_per_dof = ncu_traffic(f"vmult_q4_{args.dtype}_bytes_per_dof")
    traffic = traffic_per_dof * N if traffic_per_dof else None

    extra = {}
    if rank == 0 and args.dtype == "f64":
        # the FP32 variant of the same workload (not the headline value)
        op32 = pmg.LaplaceOperator(mesh, 4, pmg.F32, pmg.GEOMETRY_FULL, device=dev)
        s32, d32 = src.float(), torch.empty(N, dtype=torch.float32, device=f"cuda:{dev}")
        for _ in range(max(args.warmup, 3)):
            op32.vmult(d32, s32)
        torch.cuda.synchronize()
        t32, c32, n32, _ = time_vmults(op32, d32, s32, args.steps, torch, stream)
        bw32 = op32.bytes_per_vmult() / (c32 / max(n32, 1) * 1e-3) / 1e9
        extra["fp32_vmult"] = {"value": N * args.steps / (t32 * 1e-3) / 1e9, "unit": "GDoF/s",
                               "ms_per_step": t32 / args.steps, "cell_kernel_gbs": bw32,
                               "frac_of_hbm": bw32 / peak,
                               "algorithmic_bytes_per_launch": op32.bytes_per_vmult()}
        del op32, s32, d32

    tts = None
    if not args.skip_solve and world == 1:  # the solver figures are single-GPU measurements
        del op, src, dst
        torch.cuda.empty_cache()
        extra["vmult_sweep"] = vmult_sweep(torch, pmg, dev, peak)
        extra["plain_method_q2_time_to_1e-10"] = plain_method(torch, pmg, dev)
        tts = time_to_solution(torch, pmg, dev)
        tts["q6_cell_kernels"] = q6_kernel_rates(torch, pmg, dev, peaks)
        extra["dg_time_to_1e-10"] = dg_time_to_solution(torch, pmg, dev)
        extra["reference_problem"] = reference_problem(torch, pmg, dev)
        extra["reference_problem_4gpu"] = reference_problem(torch, pmg, dev, cycle=22, repeats=2)
        extra["adjoint_gradient"] = adjoint_check(torch, pmg, dev)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate, info = cpu_vmult_rate(seconds=12.0)
        cpu = {"value": rate, "unit": "GDoF/s", "cores": info["cores"], "kind": "port",
               "sample": (f"oracle CPU restatement, {info['vmults']} vmults of the 32^3-cell "
                          f"deformed cube (Q4, {info['n_dofs']} DoFs), OpenMP over "
                          f"{info['cores']} threads, {info['seconds']:.1f} s")}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.dtype, "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": args.cells ** 3, "n_dofs": N, "degree": 4,
                       "geometry": "full G per quadrature point (6 x 125 per cell)",
                       "parallelism": f"replicas{world}" if world > 1 else "single",
                       "l2": "inputs > L2 (geometry 12.6 GB at 128^3), no flush",
                       "setup_s": t_setup},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": ("measured MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured"
                                         else "fallback 6650 GB/s (MEASURED_PEAKS.json absent)"),
                         "frac_of_same_run_copy": achieved / peaks["copy_gbs"] if peaks else None,
                         "kernel": "vmult_slab_kernel<5,double,0>",
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel_ms_avg": cell_avg_s * 1e3},
            "e2e": {"value": e2e_value, "unit": "GDoF/s",
                    "h2d_bytes_per_step": N * bytes_elem, "d2h_bytes_per_step": N * bytes_elem,
                    "steps": e2e_steps,
                    "schedule": "per step: H2D of the input from pinned host memory, vmult, D2H of "
                                "the result; consecutive steps overlap on copy-in / compute / "
                                "copy-out streams with two device buffer pairs",
                    "serial_value": e2e_serial},
            "gpu_launches": int(cell_n + cons_n),
            "time_to_1e-10": tts,
            "clocks": clk,
            "cpu_baseline": cpu,
            "peaks_same_run": peaks,
        }
        line.update(extra)
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# ----------------------------------------------------------------------------------------
# profiling cases (--case): operators are set up outside the NVTX range "prof", the launches
# to profile run inside it (ncu --nvtx --nvtx-include prof/ ...); the V-cycle runs as plain
# launches (PMG_MG_GRAPH=0), so every kernel is visible
#   q6_kappa   one FP64 CG iteration of the Q6 variable-coefficient problem (3^3 coarse cells
#              refined R times, default 4 = 48^3) preconditioned by one FP32 V-cycle
#   dg_q3      one FP64 CG iteration of DG-SIPG Q3 on 2^R cells per axis (default 6) with the
#              FP32 DG -> CG Q3 -> Q1 -> h multigrid
#   adjoint_q4 the mass-matrix vmult and the per-point form of the adjoint gradient, Q4 FP64
#              on 2^R cells per axis (default 6)
#   vmult_q4   one Q4 FP64 vmult on the deformed cube with 2^R cells per axis (default 5)
#   vmult_q6 / vmult_q6_tc
#              one FP32 Q6 affine + kappa vmult (the config-3 fine operator) on 3^3 coarse
#              cells refined R times (default 3 = 24^3), on CUDA cores / on the tensor cores
#              (TF32 mma, one product)
#   dg_vmult_q3 / dg_vmult_q3_f32
#              one FP64 / FP32 DG-SIPG Q3 vmult (cell and face kernels) on 2^R cells per axis
#              (default 6)
# ----------------------------------------------------------------------------------------
def _prof_range(torch, fn):
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("prof")
    fn()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_pop()


def _one_cg_iteration(pmg, h, b):
    x = h.fine64.initialize_dof_vector()
    pmg.solve_cg(h.fine64, x, b, h.mg, 1e-10, 1e-16, 1, raise_on_noconv=False)


def _case_q6_kappa(torch, pmg, refine):
    box = pmg.Box.make(coarse=(3, 3, 3), refine=refine)
    h = pmg.Hierarchy(box, [6, 3, 2, 1], mg_dtype=pmg.F32, cheb_degree=4, geometry=pmg.GEOMETRY_AFFINE,
                      coeff_kind=pmg.COEFF_KAPPA)
    b = h.fine64.assemble_rhs(0)
    h.estimate()
    _one_cg_iteration(pmg, h, b)
    _prof_range(torch, lambda: _one_cg_iteration(pmg, h, b))


def _case_dg_q3(torch, pmg, refine):
    p = 3
    h = pmg.Hierarchy(pmg.Box.make(refine=refine), [3, 1], mg_dtype=pmg.F32, cheb_degree=5, dg=True,
                      penalty=2.0 * (p + 1) ** 2)
    b = h.fine64.assemble_rhs(2, p + 2)
    h.estimate()
    _one_cg_iteration(pmg, h, b)
    _prof_range(torch, lambda: _one_cg_iteration(pmg, h, b))


def _case_adjoint_q4(torch, pmg, refine):
    mesh = pmg.Mesh(pmg.Box.make(refine=refine))
    op = pmg.LaplaceOperator(mesh, 4, pmg.F64, pmg.GEOMETRY_AFFINE, pmg.COEFF_VALUES)
    xq = op.quadrature_points()
    op.set_coefficient(torch.exp(0.5 * torch.sin(3.0 * xq[..., 0]) * torch.cos(2.0 * xq[..., 1])))
    M = pmg.MassOperator(mesh, 4, pmg.F64)
    u = torch.rand(M.m(), dtype=torch.float64, device="cuda")
    v = torch.rand_like(u)
    out = torch.empty_like(u)
    g = op.qp_form(u, v, -1.0)

    def run():
        M.vmult(out, u)
        op.qp_form(u, v, -1.0, out=g)

    run()
    _prof_range(torch, run)


def _case_vmult_q4(torch, pmg, refine):
    op = pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(refine=refine, deform=1, amp=0.1)), 4, pmg.F64,
                             pmg.GEOMETRY_FULL)
    src = torch.from_numpy(np.random.default_rng(1234).uniform(-1.0, 1.0, op.m())).cuda()
    dst = torch.empty_like(src)
    for _ in range(3):
        op.vmult(dst, src)
    _prof_range(torch, lambda: op.vmult(dst, src))


def _vmult_case(torch, op):
    src = torch.from_numpy(np.random.default_rng(1234).uniform(-1.0, 1.0, op.m())).to(op.torch_dtype).cuda()
    dst = torch.empty_like(src)
    for _ in range(3):
        op.vmult(dst, src)
    _prof_range(torch, lambda: op.vmult(dst, src))


def _case_vmult_q6(torch, pmg, refine, tensor_cores=0):
    op = pmg.LaplaceOperator(pmg.Mesh(pmg.Box.make(coarse=(3, 3, 3), refine=refine)), 6, pmg.F32,
                             pmg.GEOMETRY_AFFINE, pmg.COEFF_KAPPA)
    if tensor_cores:
        op.set_tensor_cores(tensor_cores)
    _vmult_case(torch, op)


def _case_dg_vmult_q3(torch, pmg, refine, dtype=None):
    p = 3
    _vmult_case(torch, pmg.DGLaplaceOperator(pmg.Mesh(pmg.Box.make(refine=refine)), p,
                                             pmg.F64 if dtype is None else dtype, 2.0 * (p + 1) ** 2))


PROFILE_CASES = {"q6_kappa": (_case_q6_kappa, 4), "dg_q3": (_case_dg_q3, 6),
                 "adjoint_q4": (_case_adjoint_q4, 6), "vmult_q4": (_case_vmult_q4, 5),
                 "vmult_q6": (_case_vmult_q6, 3),
                 "vmult_q6_tc": (lambda torch, pmg, r: _case_vmult_q6(torch, pmg, r, 1), 3),
                 "dg_vmult_q3": (_case_dg_vmult_q3, 6),
                 "dg_vmult_q3_f32": (lambda torch, pmg, r: _case_dg_vmult_q3(torch, pmg, r, pmg.F32), 6)}


def profile_case(args):
    os.environ.setdefault("PMG_MG_GRAPH", "0")
    import torch
    import pmg
    fn, default_refine = PROFILE_CASES[args.case]
    fn(torch, pmg, default_refine if args.refine is None else args.refine)
    print(f"{args.case}: done", flush=True)


def main():
    args = parse()
    if args.case:
        profile_case(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()

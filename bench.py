#!/usr/bin/env python
"""Benchmark of the ALP/GraphBLAS hot path on B200.

Headline workload: FP64 plus-times grb::mxv on an R-MAT graph of scale 22
(4,194,304 vertices, edge factor 16, a/b/c/d = .57/.19/.19/.05, seeded,
duplicates merged, edge weights U(0,1)), dense x ~ U(0,1), y accumulated.
One step = one product u += A x over the whole matrix.

value   algorithmic GB/s = (12 nnz + 8 (m+1) + 8 n + 16 m) / step time, inputs
        resident in HBM (the matrix, 0.8 GB, exceeds the 126 MB L2, so no
        flush is needed between steps; x stays L2-resident by design).
e2e     the same metric through the C-ABI with host buffers: each step copies
        x from pinned host memory, runs alpb_mxv, copies u back (pipelined over
        three streams: one step's copies overlap its neighbours' products).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --only batched_cg|hpcg|adjoint_cg|ppr [size options]   (one workload)

--impl reference runs the unmodified ALP reference_omp backend (compiled
from the reference sources into oracle/_ref) on the host cores, on the same
workload, metric and unit.  Under torchrun every rank runs an independent
replica (scaling "weak"); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = ("mxv GB/s vs HBM peak; batched CG solves/s & adjoint grads/s vs plain, 1 B200")
SCALE = 22
EDGE_FACTOR = 16
SEED = 42


def algorithmic_bytes(m: int, n: int, nnz: int, val_bytes: int = 8, vec_bytes: int = 8) -> int:
    """Bytes one mxv must move at least: values + indices once, offsets,
    x once, u read + written."""
    return nnz * (val_bytes + 4) + (m + 1) * 8 + n * vec_bytes + 2 * m * vec_bytes


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(kernel_tag: str):
    """DRAM bytes per launch recorded by the ncu summary of the kernel
    (profiles/<tag>.md, line `traffic_bytes_per_launch: N`), else None."""
    f = ROOT / "profiles" / f"{kernel_tag}.md"
    if not f.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", f.read_text())
    return float(m.group(1)) if m else None


def max_over_ranks(ms: float, world: int, device) -> float:
    """The slowest rank's time (every rank calls this the same number of
    times); one rank returns its own."""
    if world == 1:
        return ms
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(bytes_per_step: int, ms_per_step: float, world: int) -> float:
    """Whole-job GB/s of `world` replicas that each moved bytes_per_step per
    step, timed by the slowest rank."""
    return world * bytes_per_step / (ms_per_step * 1e-3) / 1e9


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> list[dict]:
        if self.proc is None:
            return []
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append({"sm": float(parts[1]), "sm_max": float(parts[2]),
                             "power": float(parts[3]) if parts[3] not in ("[N/A]", "") else None,
                             "hw_slowdown": parts[5], "hw_thermal": parts[6],
                             "sw_thermal": parts[7], "sw_power_cap": parts[8]})
            except ValueError:
                continue
        return rows

    @staticmethod
    def summary(rows: list[dict]) -> dict:
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        load = [r for r in rows if r["power"] is None or r["power"] > 300] or rows
        reasons = set()
        for r in load:
            if r["hw_slowdown"] == "Active":
                reasons.add("hw_slowdown")
            if r["hw_thermal"] == "Active":
                reasons.add("hw_thermal_slowdown")
            if r["sw_thermal"] == "Active":
                reasons.add("sw_thermal_slowdown")
            if r["sw_power_cap"] == "Active":
                reasons.add("sw_power_cap")
        return {"sm_mhz": statistics.median(r["sm"] for r in load),
                "sm_max_mhz": max(r["sm_max"] for r in rows),
                "reasons": sorted(reasons), "samples": len(load)}


# ------------------------------------------------------------------ GPU arm --
def gpu_arm(args, rank: int, world: int, local_rank: int) -> dict | None:
    import ctypes as C
    import torch
    import torch.distributed as dist
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev

    torch.cuda.set_device(local_rank)
    abi.call("alpb_init", local_rank)
    stream = torch.cuda.current_stream()
    sp = dev.stream_ptr(stream)

    A = dev.rmat(args.scale, EDGE_FACTOR, seed=SEED, vtype=abi.FP64)
    x = dev.gen_values(A.n, abi.FP64, seed=SEED + 7)
    u = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    if args.hot_slots is None:
        plan = dev.Plan(A, sched=abi.SCHED_AUTO)
        plan.autotune(abi.RING_PLUS_TIMES_F64, x, u)
    else:
        # the autotuner's choice pinned (profiling: under ncu its event timings
        # are not the kernels' own, so it may choose otherwise)
        plan = dev.Plan(A, sched=abi.SCHED_MERGE_PATH)
        abi.call("alpb_spmv_plan_hot", plan.h, abi.RING_PLUS_TIMES_F64, A.n, dev.ptr(A.indices),
                 args.hot_slots, dev.stream_ptr())
    sched, vw, tiles = plan.info()
    hot_slots, hot_cover = C.c_int64(), C.c_double()
    abi.call("alpb_spmv_plan_hot_info", plan.h, C.byref(hot_slots), C.byref(hot_cover))
    hot = hot_slots.value > 0
    nbytes = algorithmic_bytes(A.m, A.n, A.nnz)

    def step():
        dev.mxv(abi.RING_PLUS_TIMES_F64, A, u, x, plan=plan, stream=stream)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    barrier()
    l0 = abi.launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    barrier()
    launches = abi.launches() - l0
    ms = e0.elapsed_time(e1) / args.steps
    # keep the GPU under the same load long enough for the clock sampler
    t_hold = time.time()
    while time.time() - t_hold < 1.0:
        for _ in range(50):
            step()
        torch.cuda.synchronize()
    clock_rows = clocks.stop()
    ms = max_over_ranks(ms, world, "cuda")
    value = replica_rate(nbytes, ms, world)

    # end to end through the C-ABI with host buffers, pipelined over three
    # streams: step k copies its x from pinned host memory (copy-in stream),
    # accumulates u += A x (compute stream: u carried forward by a device copy
    # into the step's u buffer) and copies that u back to pinned host memory
    # (copy-out stream); the copy-in of step k+1 and the copy-out of step k
    # overlap the products, so PCIe's two directions run concurrently.  x and
    # u are double-buffered, and every step still moves its own bytes.
    hx = torch.empty(A.n, dtype=torch.float64, pin_memory=True)
    hx.copy_(x.cpu())
    hu = [torch.zeros(A.m, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    dx = [torch.empty_like(x) for _ in range(2)]
    du = [u, torch.empty_like(u)]
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    p_in, p_out = dev.stream_ptr(s_in), dev.stream_ptr(s_out)
    ev_x = [torch.cuda.Event() for _ in range(2)]
    ev_c = [torch.cuda.Event() for _ in range(2)]
    ev_o = [torch.cuda.Event() for _ in range(2)]
    for e in ev_c + ev_o:
        e.record(stream)
    state = {"k": 0}

    def e2e_step():
        k = state["k"]
        bi, prev = k & 1, (k - 1) & 1
        s_in.wait_event(ev_c[bi])        # x buffer free: its last product is done
        abi.call("alpb_memcpy_h2d", dev.ptr(dx[bi]), C.c_void_p(hx.data_ptr()), A.n * 8, p_in)
        ev_x[bi].record(s_in)
        stream.wait_event(ev_x[bi])
        stream.wait_event(ev_o[bi])      # u buffer free: its last copy-out is done
        abi.call("alpb_memcpy_d2d", dev.ptr(du[bi]), dev.ptr(du[prev]), A.m * 8, sp)
        dev.mxv(abi.RING_PLUS_TIMES_F64, A, du[bi], dx[bi], plan=plan, stream=stream)
        ev_c[bi].record(stream)
        s_out.wait_event(ev_c[bi])
        abi.call("alpb_memcpy_d2h", C.c_void_p(hu[bi].data_ptr()), dev.ptr(du[bi]), A.m * 8,
                 p_out)
        ev_o[bi].record(s_out)
        state["k"] = k + 1

    for _ in range(max(3, args.warmup)):
        e2e_step()
    barrier()
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    for _ in range(args.steps):
        e2e_step()
    stream.wait_event(ev_o[(state["k"] - 1) & 1])   # the last step's copy-out
    e1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, "cuda")
    e2e_value = replica_rate(nbytes, e2e_ms, world)

    peaks = measured_peaks()
    kernel_tag = (f"spmv_vector_rmat{args.scale}" if sched != abi.SCHED_MERGE_PATH
                  else f"spmv_wmerge_hot_rmat{args.scale}" if hot
                  else f"spmv_wmerge_rmat{args.scale}")
    traffic = profiled_traffic(kernel_tag)
    achieved = nbytes / (ms * 1e-3) / 1e9
    extra = {}
    cpu = rank == 0 and world == 1 and not args.no_cpu
    # secondary workloads: one GPU only (with replicas the other ranks would
    # wait at the final barrier for as long as they run)
    if rank == 0 and world == 1 and not args.no_extra:
        extra = extra_workloads(args, A, plan, cpu)
    cpu_line = None
    if cpu:
        o, i, v = A.to_host()
        cpu_line = cpu_baseline_sample(o, i, v, x.cpu().numpy(), args.scale)
    result = {
        "metric": METRIC, "value": round(value, 2), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 5),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded R-MAT, counter-based hash)",
        "config": {"workload": f"mxv FP64 plus-times, R-MAT scale {args.scale}", "m": A.m, "n": A.n,
                   "nnz": A.nnz, "edge_factor": EDGE_FACTOR, "rmat_abcd": [0.57, 0.19, 0.19, 0.05],
                   "seed": SEED, "schedule": {1: "merge_path", 2: "vector"}[sched],
                   "vector_width": vw, "tiles": tiles, "bytes_per_step": nbytes,
                   "hot_columns": hot_slots.value, "hot_cover": round(hot_cover.value, 4),
                   "l2": "inputs larger than L2 (matrix 0.8 GB); no flush",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1),
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(achieved / peaks["hbm_gbs"], 4),
                     "peak_source": peaks["source"],
                     "traffic": traffic,
                     "kernel": (f"k_spmv_vector_dense<RingPlusTimesF64,{vw}>" if sched != 1
                                else "k_hot_gather + k_spmv_wmerge_hot<RingPlusTimesF64> + "
                                     "k_wm_fixup" if hot
                                else "k_spmv_wmerge<RingPlusTimesF64> + k_wm_fixup")},
        "e2e": {"value": round(e2e_value, 2), "unit": "GB/s", "h2d_bytes_per_step": A.n * 8,
                "d2h_bytes_per_step": A.m * 8, "ms_per_step": round(e2e_ms, 5),
                "pipelined": "copy-in of step k+1 and copy-out of step k overlap the products"},
        "gpu_launches": int(launches),
        "clocks": ClockSampler.summary(clock_rows),
    }
    if extra:
        result["extra"] = extra
    if cpu_line is not None:
        result["cpu_baseline"] = cpu_line
    return result


def timed(fn, reps: int, stream):
    """Device time of one call of fn (CUDA events on `stream`), mean of reps,
    after a warm-up of at least two calls and half a second: a GPU that sat
    idle (say, while the host ran a reference) takes that long to bring its
    clocks back up, and a short solve timed earlier reads up to 20x slow."""
    import torch
    t0, k = time.time(), 0
    while k < 2 or (time.time() - t0 < 0.5 and k < 200):
        fn()
        torch.cuda.synchronize()
        k += 1
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def semiring_sweeps(stream, A) -> dict:
    """The scale-22 sweep in the two other semirings: boolean lor/land with a
    50% dense output mask (x 50% and 1% true), and int32 min-plus."""
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    out = {}
    # boolean lor/land, value mask with 50% true, dense: the reference reads a
    # non-inverted mask on its CRS gather by structure, so every row runs
    Ab = dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices, None, abi.VOID)
    xb = dev.gen_values(A.n, abi.BOOL, seed=11, p=0.5)
    mk = dev.gen_values(A.m, abi.BOOL, seed=12, p=0.5)
    ub = torch.zeros(A.m, dtype=torch.uint8, device="cuda")
    pb = dev.Plan(Ab, sched=abi.SCHED_MERGE_PATH)

    def lor_step(x):
        # u starts false every step: rows already true would be skipped (the
        # reference's immutable-nonzero shortcut), so a kept u would time less work
        ub.zero_()
        dev.mxv(abi.RING_LOR_LAND_BOOL, Ab, ub, x, u_mask=mk, u_mask_count=A.m, plan=pb)

    nb = A.nnz * 4 + (A.m + 1) * 8 + A.m + A.n + 2 * A.m
    ms = timed(lambda: lor_step(xb), 20, stream)
    out["mxv_lor_land_masked50"] = {
        "ms": round(ms, 4), "GB/s": round(nb / ms / 1e6, 1), "bytes": nb,
        "matrix": "pattern (void)", "x": "50% true",
        "note": "early exit at a row's first true product; GB/s over the full sweep's "
                "bytes; includes zeroing u each step"}
    # the same sweep from a 1%-true x (a BFS frontier): almost no early exits
    xf = dev.gen_values(A.n, abi.BOOL, seed=14, p=0.01)
    ms = timed(lambda: lor_step(xf), 20, stream)
    out["mxv_lor_land_frontier1"] = {
        "ms": round(ms, 4), "GB/s": round(nb / ms / 1e6, 1), "bytes": nb,
        "matrix": "pattern (void)", "x": "1% true", "note": "includes zeroing u each step"}
    del xf
    # int32 min-plus, weights U{1..100}
    Ai = dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices,
                 torch.empty(A.nnz, dtype=torch.int32, device="cuda"), abi.INT32)
    abi.call("alpb_gen_edge_values", dev.ptr(Ai.values), abi.INT32, dev.ptr(A.offsets),
             dev.ptr(A.indices), A.m, A.nnz, SEED + 1, 1, 100, dev.stream_ptr())
    xi = dev.gen_values(A.n, abi.INT32, seed=13, lo=0, hi=1000)
    ui = torch.full((A.m,), 2**31 - 1, dtype=torch.int32, device="cuda")
    ms = timed(lambda: dev.mxv(abi.RING_MIN_PLUS_I32, Ai, ui, xi, plan=pb), 20, stream)
    nb = algorithmic_bytes(A.m, A.n, A.nnz, 4, 4)
    out["mxv_min_plus_i32"] = {"ms": round(ms, 4), "GB/s": round(nb / ms / 1e6, 1), "bytes": nb}
    del Ai, xi, ui
    return out


def extra_workloads(args, A, plan, cpu: bool) -> dict:
    """Secondary workloads of the same sweep, timed the same way (not part of
    `value`): boolean lor/land with a 50% dense output mask, int32 min-plus,
    simple_pagerank on the scale-22 pattern, CG on the 27-point 32^3 grid,
    batched CG, HPCG, the differentiated CG and personalised PageRank.  With
    `cpu`, the unmodified reference_omp backend is timed beside CG, PageRank,
    batched CG and HPCG on the host cores."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    stream = torch.cuda.current_stream()
    later = []     # host reference runs, after the device timings
    out = semiring_sweeps(stream, A)
    out["pagerank_rmat22"] = pagerank_workload(stream, A, cpu, later)
    out["cg_27pt_32"] = cg_workload(stream, 32, cpu, later)
    out["batched_cg"] = batched_cg_workload(stream, cpu=cpu, later=later)
    out["hpcg_256"] = hpcg_workload(stream, cpu=cpu, later=later)
    out["adjoint_cg"] = adjoint_workload(stream)
    out["ppr_rmat24"] = ppr_workload(stream)
    # the host's reference runs come after every device timing: reference_omp's
    # threads keep spinning for a while after a parallel region and would
    # delay the launching thread of a device solve timed next
    for job in later:
        job()
    # each rate next to its fraction of the measured HBM copy bandwidth
    peak = measured_peaks()["hbm_gbs"]
    for v in out.values():
        for k in [k for k in v if k.endswith("GB/s") and isinstance(v[k], (int, float))]:
            v[k.replace("GB/s", "frac_of_measured_hbm")] = round(v[k] / peak, 4)
    return out


def pagerank_workload(stream, A, cpu: bool = False, later: list | None = None) -> dict:
    """simple_pagerank on the pattern of A with unit weights (column-stochastic
    after the out-degree scaling), alpha 0.85, conv 1e-9: one alpb_pagerank
    call with its set-up, and the solve alone (alpb_pagerank_planned with the
    CCS plan and scratch made beforehand)."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    out = {}
    L = dev.CRS(A.m, A.n, A.nnz, A.offsets, A.indices,
                torch.ones(A.nnz, dtype=torch.float64, device="cuda"), abi.FP64)
    LT = dev.transpose(L)
    pr = torch.zeros(A.m, dtype=torch.float64, device="cuda")
    it, res = C.c_int64(), C.c_double()
    prc = [0]

    def pagerank():
        prc[0] = abi.lib().alpb_pagerank(L.m, dev.ptr(L.offsets), dev.ptr(L.indices),
                                         dev.ptr(L.values), dev.ptr(LT.offsets), dev.ptr(LT.indices),
                                         dev.ptr(LT.values), dev.ptr(pr), 0, 0.85, 1e-9, 1000,
                                         C.byref(it), C.byref(res), dev.stream_ptr())
    ms_call = timed(pagerank, 2, stream)   # one call: plan, set-up and every iteration
    # the same solve with the plan of the CCS and the scratch vectors made
    # beforehand (what a caller that solves repeatedly on one graph does):
    # one cooperative launch for the out-degrees and every iteration
    pplan = dev.Plan(LT, sched=abi.SCHED_MERGE_PATH)
    pwork = torch.empty(3 * A.n, dtype=torch.float64, device="cuda")

    def pagerank_planned():
        prc[0] = abi.lib().alpb_pagerank_planned(
            L.m, dev.ptr(L.offsets), dev.ptr(L.indices), dev.ptr(L.values), dev.ptr(LT.offsets),
            dev.ptr(LT.indices), dev.ptr(LT.values), dev.ptr(pr), 0, 0.85, 1e-9, 1000,
            C.byref(it), C.byref(res), dev.ptr(pwork), pplan.h, dev.stream_ptr())
    ms = timed(pagerank_planned, 3, stream)
    per_iter = (A.nnz * 12 + (A.n + 1) * 8 + 6 * A.n * 8)
    out.update({"rc": prc[0], "iterations": it.value, "residual": res.value,
                "ms_per_solve": round(ms, 3), "ms_per_iter": round(ms / max(it.value, 1), 4),
                "ms_per_call_with_setup": round(ms_call, 3),
                "GB/s": round(per_iter * it.value / ms / 1e6, 1),
                "bytes_per_iteration": per_iter})
    if cpu:
        job = (lambda n=L.m, h=L.to_host(), t=ms:
               out.__setitem__("cpu_reference_omp", cpu_pagerank(n, h, t)))
        if later is not None:
            later.append(job)
        else:
            job()
    del pplan, pwork, L, LT, pr
    return out


def cg_workload(stream, side: int = 32, cpu: bool = False, later: list | None = None) -> dict:
    """Plain CG on the 27-point side^3 grid (diagonal 26, off-diagonals -1),
    b = A 1, x0 = 0, tol 1e-10, max 500: the reference's CPU-runnable
    configuration at 32^3, one fused alpb_cg_solve launch per solve."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    out = {}
    it, res = C.c_int64(), C.c_double()
    S = dev.stencil((side, side, side), 26.0, -1.0)
    ones = torch.ones(S.n, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(ones)
    dev.mxv(abi.RING_PLUS_TIMES_F64, S, b, ones)
    ps = dev.Plan(S, sched=abi.SCHED_MERGE_PATH)
    x = torch.zeros_like(b)
    work = torch.empty(4 * S.n, dtype=torch.float64, device="cuda")

    def cg():
        x.zero_()
        abi.call("alpb_cg_solve", S.m, dev.ptr(S.offsets), dev.ptr(S.indices), dev.ptr(S.values),
                 dev.ptr(b), dev.ptr(x), 500, 1e-10, C.byref(it), C.byref(res), dev.ptr(work),
                 ps.h, dev.stream_ptr())
    ms = timed(cg, 5, stream)
    out.update({"iterations": it.value, "residual": res.value, "ms_per_solve": round(ms, 4),
                "us_per_iteration": round(1e3 * ms / max(it.value, 1), 2),
                "err_vs_ones_inf": float((x - 1).abs().max().item())})
    if cpu:
        job = (lambda n=S.m, h=S.to_host(), hb=b.cpu().numpy(), t=ms:
               out.__setitem__("cpu_reference_omp", cpu_cg(n, h, hb, t)))
        if later is not None:
            later.append(job)
        else:
            job()
    del S, ps, work
    return out


def batched_cg_workload(stream, nseg: int = 256, seed: int = 2024, cpu: bool = False,
                        later: list | None = None) -> dict:
    """256 shifted 2-D 5-point Poisson systems, sides log-uniform in [32, 512],
    shift U(0.01, 1), b ~ N(0, 1), relative tolerance 1e-8, FP64: one
    graph-captured persistent launch against one alpb_cg_solve launch per
    instance (plans and buffers prepared outside the timed regions)."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    rng = np.random.default_rng(seed)
    sides = np.round(np.exp(rng.uniform(np.log(32), np.log(512), nseg))).astype(np.int64)
    shifts = rng.uniform(0.01, 1.0, nseg)
    rows = sides * sides
    nnzs = 5 * sides * sides - 4 * sides
    seg_rows = np.concatenate([[0], np.cumsum(rows)]).astype(np.int64)
    seg_nnz = np.concatenate([[0], np.cumsum(nnzs)]).astype(np.int64)
    n, nnz = int(seg_rows[-1]), int(seg_nnz[-1])
    d = torch.device("cuda")
    tL = torch.from_numpy(sides).to(d)
    tS = torch.from_numpy(shifts).to(d)
    tR = torch.from_numpy(seg_rows).to(d)
    tN = torch.from_numpy(seg_nnz).to(d)
    rp = torch.empty(n + 1, dtype=torch.int64, device=d)
    ci = torch.empty(nnz, dtype=torch.int32, device=d)
    va = torch.empty(nnz, dtype=torch.float64, device=d)
    sp = dev.stream_ptr(stream)
    abi.call("alpb_gen_poisson2d_batch", nseg, dev.ptr(tL), dev.ptr(tS), dev.ptr(tR), dev.ptr(tN),
             n, dev.ptr(rp), dev.ptr(ci), dev.ptr(va), sp)
    b = torch.empty(n, dtype=torch.float64, device=d)
    abi.call("alpb_gen_normal", dev.ptr(b), n, seed, 1, sp)
    x = torch.zeros_like(b)
    tol, max_iter = 1e-8, 20000
    h = C.c_void_p()
    abi.call("alpb_batched_cg_create", C.byref(h), n, nnz, dev.ptr(rp), dev.ptr(ci), dev.ptr(va),
             nseg, dev.ptr(tR), sp)
    abi.call("alpb_batched_cg_capture", h, dev.ptr(b), dev.ptr(x), max_iter, tol, sp)

    def batched():
        x.zero_()
        abi.call("alpb_batched_cg_replay", h, sp)
    ms_b = timed(batched, 3, stream)
    it = np.zeros(nseg, np.int64)
    rr = np.zeros(nseg)
    conv = np.zeros(nseg, np.int32)
    rc = abi.lib().alpb_batched_cg_results(h, it.ctypes.data_as(C.c_void_p),
                                           rr.ctypes.data_as(C.c_void_p),
                                           conv.ctypes.data_as(C.c_void_p), sp)
    xb = x.clone()
    abi.lib().alpb_batched_cg_destroy(h)
    # plain path: one alpb_cg_solve launch per instance, on its own CRS
    systems = []
    for L, sh in zip(sides, shifts):
        A = dev.poisson2d(int(L), float(sh))
        systems.append((A, dev.Plan(A, sched=abi.SCHED_MERGE_PATH),
                        torch.empty(4 * A.n, dtype=torch.float64, device=d)))
    xp = torch.zeros_like(b)
    itp = np.zeros(nseg, np.int64)
    i1, r1 = C.c_int64(), C.c_double()

    def plain():
        xp.zero_()
        for k, (A, pl, wk) in enumerate(systems):
            o = int(seg_rows[k])
            rcs = abi.lib().alpb_cg_solve(A.m, dev.ptr(A.offsets), dev.ptr(A.indices),
                                          dev.ptr(A.values), C.c_void_p(b.data_ptr() + 8 * o),
                                          C.c_void_p(xp.data_ptr() + 8 * o), max_iter, tol,
                                          C.byref(i1), C.byref(r1), dev.ptr(wk), pl.h, sp)
            assert rcs == abi.SUCCESS, abi.last_error()
            itp[k] = i1.value
    ms_p = timed(plain, 1, stream)
    diff = float(((xb - xp).abs().max() / xp.abs().max()).item())
    # algorithmic bytes of one CG iteration of instance i: the matrix once
    # (12 B per nonzero + offsets) and 10 vector passes of 8 B per row (phase
    # A reads r, u_old and writes temp, u_new; phase B reads x, u_new, r,
    # temp and writes x, r)
    per_iter = 12 * nnzs + 8 * (rows + 1) + 80 * rows
    moved = float((it * per_iter).sum())
    out = {"systems": nseg, "rows": n, "nnz": nnz, "tol": tol, "rc": rc,
           "all_converged": bool(conv.all()), "iterations_max": int(it.max()),
           "iterations_sum": int(it.sum()), "plain_iterations_sum": int(itp.sum()),
           "batched_ms": round(ms_b, 3), "plain_ms": round(ms_p, 3),
           "batched_solves_per_s": round(nseg / (ms_b * 1e-3), 1),
           "plain_solves_per_s": round(nseg / (ms_p * 1e-3), 1),
           "speedup": round(ms_p / ms_b, 2),
           "batched_GB/s": round(moved / ms_b / 1e6, 1),
           "plain_GB/s": round(moved / ms_p / 1e6, 1),
           "max_rel_diff_batched_vs_plain": diff}
    if cpu:
        hrp, hci, hva = rp.cpu().numpy(), ci.cpu().numpy().view(np.uint32), va.cpu().numpy()
        hb = b.cpu().numpy()

        def cpu_batched():
            # reference_omp solving the 256 systems one after the other (the
            # same matrices and right-hand sides, copied from the device)
            from oracle.oracle import crs_to_coo
            ref = reference_omp()
            if ref is None:
                out["cpu_reference_omp"] = _cpu_unavailable()
                return
            tot, its = 0.0, 0
            for k in range(nseg):
                r0, r1 = int(seg_rows[k]), int(seg_rows[k + 1])
                srp = hrp[r0:r1 + 1] - hrp[r0]
                I, J = crs_to_coo(srp, (hci[hrp[r0]:hrp[r1]].astype(np.int64) - r0)
                                  .astype(np.uint32))
                rcs, _, itk, _, ms_k = ref.cg(r1 - r0, I, J, hva[hrp[r0]:hrp[r1]], hb[r0:r1],
                                              np.zeros(r1 - r0), max_iter, tol)
                tot += ms_k
                its += itk
            out["cpu_reference_omp"] = {
                "ms": round(tot, 1), "iterations_sum": its, "threads": ref.threads(),
                "solves_per_s": round(nseg / (tot * 1e-3), 1),
                "gpu_batched_speedup": round(tot / ms_b, 1),
                "sample": "the whole workload: conjugate_gradient on each of the 256 "
                          "systems in turn, solves alone timed"}
        if later is not None:
            later.append(cpu_batched)
        else:
            cpu_batched()
    return out


def _hpcg_gpu(stream, side, coarse_levels, nrhs, seed):
    """One device HPCG solve of `nrhs` right-hand sides ~ N(0, 1) on the
    side^3 system; returns (ms, iterations, residuals, rows, nnz, levels, fused)."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    sp = dev.stream_ptr(stream)
    h = C.c_void_p()
    abi.call("alpb_hpcg_create", C.byref(h), side, side, side, 26.0, -1.0, 27, 4, coarse_levels,
             nrhs, sp)
    lv, n, nnz, fused = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int()
    abi.call("alpb_hpcg_info", h, C.byref(lv), C.byref(n), C.byref(nnz), C.byref(fused))
    b = torch.empty(n.value * nrhs, dtype=torch.float64, device="cuda")
    abi.call("alpb_gen_normal", dev.ptr(b), n.value * nrhs, seed, 1, sp)
    x = torch.zeros_like(b)
    it = (C.c_int64 * nrhs)()
    res = (C.c_double * nrhs)()

    def solve():
        x.zero_()
        abi.call("alpb_hpcg_solve", h, dev.ptr(b), dev.ptr(x), 1, 1, 1, 500, 1e-9, it, res, sp)
    ms = timed(solve, 1, stream)
    abi.lib().alpb_hpcg_destroy(h)
    return ms, list(it), [float(r) for r in res], n.value, nnz.value, lv.value, fused.value


def hpcg_workload(stream, side: int = 256, coarse_levels: int = 3, nrhs: int = 8,
                  cpu: bool = False, later: list | None = None) -> dict:
    """HPCG on the 27-point 256^3 system (diagonal 26, off-diagonals -1) with
    three coarser levels (128^3, 64^3, 32^3), 27 static colours, one pre- and
    one post-smoothing step, 8 right-hand sides ~ N(0, 1) solved together,
    relative tolerance 1e-9, FP64 (alpb_hpcg_solve).  With `cpu`, ALP's own
    hpcg on reference_omp at 64^3 (one right-hand side; 256^3 takes the host
    minutes) beside the device at 64^3 with 8 right-hand sides."""
    ms, it, res, n, nnz, lv, fused = _hpcg_gpu(stream, side, coarse_levels, nrhs, 31)
    iters = max(it)
    # algorithmic bytes of one CG iteration.  A smoother sweep must read the
    # matrix once, x once, r once and write x once (8 nrhs n bytes per vector
    # pass); per V-cycle the finest level runs four sweeps (forward and
    # backward, before and after the coarse correction), the CG adds one
    # product and about ten vector passes, and each coarser level adds about
    # 1/8 of the finest.  The device's colour steps gather x at the rows'
    # neighbours once per colour (26 of the 27 colours neighbour each row),
    # so they move about 27 copies of x per sweep: that delivered rate is
    # reported apart.
    vec = 8 * nrhs * n
    mat = 12 * nnz + 8 * (n + 1)
    fine = 4 * (mat + 3 * vec) + (mat + 3 * vec) + 10 * vec
    per_iter = fine * 8 / 7
    gathered = (4 * (mat + 30 * vec) + (mat + 3 * vec) + 10 * vec) * 8 / 7
    out = {"rows": n, "nnz": nnz, "levels": lv, "rhs": nrhs,
           "fused_smoother": bool(fused), "iterations": it,
           "residuals": res, "ms_per_solve": round(ms, 2),
           "ms_per_iteration": round(ms / max(iters, 1), 3),
           "solves_per_s": round(nrhs / (ms * 1e-3), 3),
           "GB/s": round(per_iter * iters / ms / 1e6, 1),
           "bytes_per_iteration": int(per_iter),
           "gathered_GB/s": round(gathered * iters / ms / 1e6, 1)}
    if cpu:
        ms64, it64, _, _, _, _, _ = _hpcg_gpu(stream, 64, 3, 8, 32)

        def cpu_hpcg():
            ref = reference_omp()
            if ref is None:
                out["cpu_reference_omp"] = _cpu_unavailable()
                return
            b = np.random.default_rng(64).standard_normal(64 ** 3)
            rc, _, itc, _, msc, _ = ref.hpcg(64, 3, 27, b, 500, 1e-9)
            out["cpu_reference_omp"] = {
                "rc": rc, "iterations": itc, "ms_per_rhs": round(msc, 1),
                "threads": ref.threads(),
                "gpu_64_ms_per_rhs": round(ms64 / 8, 2), "gpu_64_iterations": it64,
                "gpu_speedup_64": round(msc / (ms64 / 8), 1),
                "sample": "grb::algorithms::hpcg on 64^3 with 3 coarser levels, one right-hand "
                          "side (the device at 64^3 solves 8 together; ms per right-hand side)"}
        if later is not None:
            later.append(cpu_hpcg)
        else:
            cpu_hpcg()
    return out


def adjoint_workload(stream, side: int = 64) -> dict:
    """Differentiated CG on the 27-point 64^3 pattern: off-diagonals -U(0.5, 1.5)
    (symmetric), diagonal 1.05 |row sum|, b, x* ~ N(0, 1), L = 0.5 |x - x*|^2.
    Forward solve (alpb_cg_solve) against the gradient (alpb_cg_adjoint: CG on
    the CCS for lambda, then the SDDMM -lambda_i x_j), relative tolerance 1e-12."""
    import ctypes as C
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    sp = dev.stream_ptr(stream)
    A = dev.stencil((side, side, side), 1.0, 1.0, ref_order=False)
    abi.call("alpb_gen_sym_dd_values", dev.ptr(A.offsets), dev.ptr(A.indices), A.m, 11, 0.5, 1.5,
             1.05, dev.ptr(A.values), sp)
    At = dev.transpose(A)
    pa, pt = dev.Plan(A, sched=abi.SCHED_MERGE_PATH), dev.Plan(At, sched=abi.SCHED_MERGE_PATH)
    b = torch.empty(A.m, dtype=torch.float64, device="cuda")
    xs = torch.empty_like(b)
    abi.call("alpb_gen_normal", dev.ptr(b), A.m, 5, 1, sp)
    abi.call("alpb_gen_normal", dev.ptr(xs), A.m, 6, 1, sp)
    x = torch.zeros_like(b)
    lam = torch.zeros_like(b)
    g = torch.empty_like(b)
    gv = torch.empty_like(A.values)
    work = torch.empty(4 * A.m, dtype=torch.float64, device="cuda")
    tol = 1e-12
    itf, ita, res = C.c_int64(), C.c_int64(), C.c_double()

    def forward():
        x.zero_()
        abi.call("alpb_cg_solve", A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(A.values),
                 dev.ptr(b), dev.ptr(x), 5000, tol, C.byref(itf), C.byref(res), dev.ptr(work),
                 pa.h, sp)
    ms_f = timed(forward, 3, stream)
    torch.sub(x, xs, out=g)

    def gradient():
        lam.zero_()
        abi.call("alpb_cg_adjoint", A.m, dev.ptr(A.offsets), dev.ptr(A.indices), dev.ptr(A.values),
                 dev.ptr(At.offsets), dev.ptr(At.indices), dev.ptr(At.values), dev.ptr(x),
                 dev.ptr(g), dev.ptr(lam), dev.ptr(gv), 5000, tol, C.byref(ita), C.byref(res),
                 pa.h, pt.h, sp)
    ms_g = timed(gradient, 3, stream)
    return {"rows": A.m, "nnz": A.nnz, "tol": tol, "forward_iterations": itf.value,
            "adjoint_iterations": ita.value, "forward_ms": round(ms_f, 3),
            "gradient_ms": round(ms_g, 3), "gradient_over_forward": round(ms_g / ms_f, 3),
            "forward_solves_per_s": round(1e3 / ms_f, 2), "grads_per_s": round(1e3 / ms_g, 2)}


def ppr_workload(stream, scale: int = 24, nseeds: int = 64) -> dict:
    """Differentiable personalised PageRank on R-MAT scale 24 (edge factor 16,
    U(0, 1) edge weights), 64 one-hot seeds, alpha 0.85, L1 tolerance 1e-9 per
    seed: the forward solve (alpb_ppr_solve), the adjoint for dL/dx ~ N(0, 1)
    (alpb_ppr_adjoint) and the gradient with respect to every edge weight
    (alpb_ppr_grad_weights), each timed once after a two-iteration warm-up."""
    import ctypes as C
    import numpy as np
    import torch
    from alp_b200 import _abi as abi
    from alp_b200 import device as dev
    sp = dev.stream_ptr(stream)
    A = dev.rmat(scale, vtype=abi.FP64, seed=42)
    n, nnz, S = A.n, A.nnz, nseeds
    h = C.c_void_p()
    abi.call("alpb_ppr_create", C.byref(h), n, nnz, dev.ptr(A.offsets), dev.ptr(A.indices),
             dev.ptr(A.values), S, sp)
    seeds = np.ascontiguousarray(np.random.default_rng(scale).integers(0, n, S), np.int64)
    x = torch.empty(n * S, dtype=torch.float64, device="cuda")
    g = torch.empty_like(x)
    abi.call("alpb_gen_normal", dev.ptr(g), n * S, 41, 1, sp)
    lam = torch.empty_like(x)
    grad = torch.empty(nnz, dtype=torch.float64, device="cuda")
    itf, ita = (C.c_int64 * S)(), (C.c_int64 * S)()
    res = (C.c_double * S)()
    sd = seeds.ctypes.data_as(C.c_void_p)
    abi.call("alpb_ppr_solve", h, sd, 0.85, 0.0, 2, dev.ptr(x), 0, itf, res, sp)   # warm-up
    ms_f = timed(lambda: abi.call("alpb_ppr_solve", h, sd, 0.85, 1e-9, 1000, dev.ptr(x), 0, itf,
                                  res, sp), 1, stream)
    ms_a = timed(lambda: abi.call("alpb_ppr_adjoint", h, dev.ptr(g), dev.ptr(lam), 1e-9, 1000,
                                  ita, res, sp), 1, stream)
    ms_g = timed(lambda: abi.call("alpb_ppr_grad_weights", h, dev.ptr(x), dev.ptr(lam),
                                  dev.ptr(grad), sp), 1, stream)
    mass = float(x.view(n, S).sum(0).sub(1).abs().max())
    abi.lib().alpb_ppr_destroy(h)
    kf, ka = max(itf), max(ita)
    # algorithmic bytes per iteration: the storage once (12 nnz + offsets),
    # the gathered vector once, and the row-wise vector passes (forward: x
    # read and written, next input written; adjoint: dL/dx read, next lambda
    # written); the gathers themselves move 8 S bytes per nonzero, reported
    # apart as the delivered rate
    vec = 8 * n * S
    b_f = 12 * nnz + 8 * (n + 1) + 4 * vec
    b_a = 12 * nnz + 8 * (n + 1) + 3 * vec
    b_g = (12 * nnz + 8 * (n + 1) + 2 * vec) + (12 * nnz + 2 * vec)
    gathered = 8 * S * nnz
    del A
    return {"rows": n, "nnz": nnz, "seeds": S, "alpha": 0.85, "tol": 1e-9,
            "forward_iterations_max": kf, "forward_iterations_min": min(itf),
            "adjoint_iterations_max": ka, "forward_ms": round(ms_f, 2),
            "adjoint_ms": round(ms_a, 2), "grad_ms": round(ms_g, 2),
            "forward_ms_per_iteration": round(ms_f / kf, 3),
            "adjoint_ms_per_iteration": round(ms_a / ka, 3),
            "forward_GB/s": round(b_f * kf / ms_f / 1e6, 1),
            "adjoint_GB/s": round(b_a * ka / ms_a / 1e6, 1),
            "grad_GB/s": round(b_g / ms_g / 1e6, 1),
            "forward_gathered_GB/s": round((b_f + gathered) * kf / ms_f / 1e6, 1),
            "gradient_over_forward": round((ms_a + ms_g) / ms_f, 3),
            "max_abs_mass_error": mass}


# ------------------------------------------------------------ reference arm --
def reference_arm(args) -> dict:
    """The unmodified reference_omp backend on the host cores: grb::mxv on the
    same R-MAT scale-22 matrix (generated by the seeded C generator that the
    device generator mirrors bit for bit)."""
    from oracle.oracle import FP64, REF_OMP_SO, Reference, Restatement, crs_to_coo
    if not REF_OMP_SO.exists():
        return {"impl": "reference", "unavailable": "oracle/_ref/libalp_ref_omp.so not built"}
    os.environ.setdefault("OMP_PROC_BIND", "true")
    R = Restatement()
    rp, col, vals = R.rmat(SCALE, EDGE_FACTOR, seed=SEED, vtype=FP64)
    n = len(rp) - 1
    I, J = crs_to_coo(rp, col)
    x = R.values(n, FP64, SEED + 7)
    u = np.zeros(n)
    ref = Reference(omp=True)
    nbytes = algorithmic_bytes(n, n, len(col))
    # one call builds the reference matrix and runs warmup + timed steps
    reps = args.warmup + args.steps
    ms_list = []
    rc, ms = ref.mxv(0, 0, 0, n, n, I, J, vals, u, None, x, reps=reps)
    if rc != 0:
        return {"impl": "reference", "unavailable": f"reference mxv returned rc={rc}"}
    value = nbytes / (ms * 1e-3) / 1e9
    cores = ref.threads()
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": "GB/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded R-MAT, counter-based hash)",
        "config": {"workload": f"mxv FP64 plus-times, R-MAT scale {SCALE}", "m": n, "n": n,
                   "nnz": int(len(col)), "bytes_per_step": nbytes},
        "cpu_baseline": {"value": round(value, 2), "unit": "GB/s", "cores": cores,
                         "kind": "reference",
                         "sample": f"grb::mxv (reference_omp, {cores} threads) on the full "
                                   f"R-MAT scale-{SCALE} matrix, mean of {reps} calls"},
        "e2e": {"value": round(value, 2), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def reference_omp():
    """The unmodified reference_omp backend (oracle/_ref), or None."""
    try:
        from oracle.oracle import REF_OMP_SO, Reference
        if not REF_OMP_SO.exists():
            return None
        os.environ.setdefault("OMP_PROC_BIND", "true")
        return Reference(omp=True)
    except Exception:  # a missing checker must not break the GPU line
        return None


def _cpu_unavailable():
    return {"ms": None, "sample": "unavailable: oracle/_ref/libalp_ref_omp.so not built"}


def cpu_pagerank(n, host_crs, gpu_ms) -> dict:
    """grb::algorithms::simple_pagerank on reference_omp, same graph and
    parameters (alpha 0.85, conv 1e-9); the solve alone is timed."""
    from oracle.oracle import crs_to_coo
    ref = reference_omp()
    if ref is None:
        return _cpu_unavailable()
    o, i, v = host_crs
    I, J = crs_to_coo(o, i)
    rc, pr, it, ms = ref.pagerank(n, I, J, v, alpha=0.85, conv=1e-9, max_iter=1000)
    return {"rc": rc, "iterations": it, "ms": round(ms, 1), "threads": ref.threads(),
            "gpu_speedup": round(ms / gpu_ms, 1),
            "sample": "the whole workload: simple_pagerank on the same scale-22 graph, one solve"}


def cpu_cg(n, host_crs, hb, gpu_ms) -> dict:
    """grb::algorithms::conjugate_gradient on reference_omp, same system and
    parameters (x0 = 0, tol 1e-10, max 500); mean of 5 solves."""
    from oracle.oracle import crs_to_coo
    ref = reference_omp()
    if ref is None:
        return _cpu_unavailable()
    o, i, v = host_crs
    I, J = crs_to_coo(o, i)
    tot, it = 0.0, 0
    for _ in range(5):
        rc, _, it, _, ms = ref.cg(n, I, J, v, hb, np.zeros(n), 500, 1e-10)
        tot += ms
    return {"rc": rc, "iterations": it, "ms": round(tot / 5, 3), "threads": ref.threads(),
            "gpu_speedup": round(tot / 5 / gpu_ms, 1),
            "sample": "the whole workload (27-point 32^3), mean of 5 solves"}


def cpu_baseline_sample(o, i, v, xh, scale) -> dict:
    """reference_omp grb::mxv on the benchmark's own matrix (copied from the
    device), all host threads, mean of 20 calls (about 1-2 s of CPU work after
    the reference's matrix build)."""
    from oracle.oracle import crs_to_coo
    ref = reference_omp()
    if ref is None:
        return {"value": None, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                "sample": "unavailable: oracle/_ref/libalp_ref_omp.so not built"}
    n = len(o) - 1
    I, J = crs_to_coo(o, i)
    u = np.zeros(n)
    rc, ms = ref.mxv(0, 0, 0, n, n, I, J, v, u, None, xh, reps=20)
    if rc != 0:
        return {"value": None, "unit": "GB/s", "cores": ref.threads(), "kind": "reference",
                "sample": f"reference mxv returned rc={rc}"}
    nb = algorithmic_bytes(n, n, len(i))
    return {"value": round(nb / (ms * 1e-3) / 1e9, 2), "unit": "GB/s", "cores": ref.threads(),
            "kind": "reference", "ms_per_step": round(ms, 3),
            "sample": f"grb::mxv (reference_omp, {ref.threads()} threads) on the full R-MAT "
                      f"scale-{scale} matrix ({len(i)} nnz, the same matrix copied from the "
                      "device), mean of 20 calls"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--scale", type=int, default=SCALE,
                    help="R-MAT scale (22 is the benchmark; smaller for profiling captures)")
    ap.add_argument("--only", choices=["batched_cg", "hpcg", "adjoint_cg", "ppr", "pagerank", "cg",
                                       "sweeps"],
                    help="run one secondary workload alone and print its line (profiling)")
    ap.add_argument("--hot-slots", type=int, default=None,
                    help="merge path with this many hot-column slots instead of the autotuner")
    ap.add_argument("--hpcg-side", type=int, default=256)
    ap.add_argument("--hpcg-levels", type=int, default=3)
    ap.add_argument("--ppr-scale", type=int, default=24)
    ap.add_argument("--ppr-seeds", type=int, default=64)
    ap.add_argument("--cg-side", type=int, default=32)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(reference_arm(args)), flush=True)
        return

    if args.only:
        import torch
        from alp_b200 import _abi as abi
        from alp_b200 import device as dev
        torch.cuda.set_device(local_rank)
        abi.call("alpb_init", local_rank)
        stream = torch.cuda.current_stream()
        run = {"batched_cg": lambda: batched_cg_workload(stream),
               "hpcg": lambda: hpcg_workload(stream, args.hpcg_side, args.hpcg_levels),
               "adjoint_cg": lambda: adjoint_workload(stream),
               "ppr": lambda: ppr_workload(stream, args.ppr_scale, args.ppr_seeds),
               "pagerank": lambda: pagerank_workload(
                   stream, dev.rmat(args.scale, EDGE_FACTOR, seed=SEED, vtype=abi.FP64)),
               "cg": lambda: cg_workload(stream, args.cg_side),
               "sweeps": lambda: semiring_sweeps(
                   stream, dev.rmat(args.scale, EDGE_FACTOR, seed=SEED, vtype=abi.FP64))}[args.only]
        if rank == 0:
            print(json.dumps({"workload": args.only, **run()}), flush=True)
        return

    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = gpu_arm(args, rank, world, local_rank)
    if rank == 0:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark of the per-block Godunov update (Mcell-updates/s).

Workload (default): batched AMR blast snapshot -- 8^3 root blocks of 16^3,
5 refinement levels, ~11.6k leaf blocks (uneven per level), FP64 HLLC +
minmod, CFL 0.4, viscosity 5e-3.  One step = one full time step of the
reference's main loop without AMR/output (dt reduction, two Godunov stages
with ghost fill, viscous step), i.e. source/main.f90:81-100.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl wx3d|reference]

--impl reference times the CPU restatement of the reference (oracle/, the
reference's own Fortran cannot be built here: no Fortran compiler) on all host
threads for the same workload.  Under torchrun (N>1) every rank runs an
independent replica of the workload on its GPU (the graded path does not
shard: one GPU, no MPI) and the job throughput is the sum.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    "blast-amr": dict(desc="batched AMR blast: 8^3 root blocks of 16^3, 5 levels, shell-refined snapshot, "
                           "FP64 HLLC+minmod, CFL 0.4, eta 5e-3"),
    "sedov256": dict(desc="Sedov blast 16^3 root blocks of 16^3 (256^3 cells), single level, FP64 HLLC+minmod"),
    "sedov64": dict(desc="Sedov blast 4^3 root blocks of 16^3 (64^3 cells), single level, FP64 HLLC+minmod"),
    "brio-wu": dict(desc="Brio-Wu MHD shock tube 256x16x16 cells, FP64 HLLD+minmod, 8-wave source"),
    "snr-h": dict(desc="radiative SNR, H-rate EOS + COOL_H, 8^3 roots, 4 levels (4,712 blocks), FP64 HLLC+minmod"),
    "winds": dict(desc="colliding stellar winds: 2 sources re-imposed every stage, EOS_H_RATE + 200-row "
                       "COOL_TABLE, 8^3 roots, 6 levels (20,896 blocks), FP64 HLLC+minmod"),
    "snr-h-small": dict(desc="radiative SNR, H-rate EOS + COOL_H, 8^3 roots, 3 levels (1,184 blocks), FP64 HLLC+minmod"),
    "snr-h-c4": dict(desc="radiative SNR, H-rate EOS + COOL_H, 4^3 roots (64^3 root cells), 4 levels (960 blocks), "
                          "FP64 HLLC+minmod"),
}


def build_problem(name: str):
    from walicxe3d_b200 import problems
    if name == "blast-amr":
        return problems.blast_amr()
    if name == "sedov256":
        return problems.sedov(16)
    if name == "sedov64":
        return problems.sedov(4)
    if name == "brio-wu":
        return problems.brio_wu(16)
    if name == "snr-h":
        return problems.snr_h(nroot=8, maxlev=4)
    if name == "snr-h-small":
        return problems.snr_h(nroot=8, maxlev=3)
    if name == "snr-h-c4":
        return problems.snr_h(nroot=4, maxlev=4)
    if name == "winds":
        return problems.colliding_winds()
    raise SystemExit(f"unknown workload {name}")


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([v.strip() for v in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_time_oracle(prob, steps_max: int, budget_s: float, threads: int):
    """Times the CPU oracle on the workload: whole steps, stopping once the
    budget is spent.  Returns (Mcell-updates/s, steps timed, seconds)."""
    import oracle
    o = oracle.from_problem(prob, threads=threads)
    o.step()  # warm the caches and the thread pool
    n, t0 = 0, time.perf_counter()
    while n < steps_max:
        o.step()
        n += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    o.close()
    return prob.cells * n / dt / 1e6, n, dt


def stage_figures(neq: int, fused: bool):
    """Per-cell DRAM bytes and FP64 flops of the corrector from the committed
    ncu summary (profiles/stage_kernels.json, measured on Sedov 256^3 at
    neq 5, with the DRAM bytes also measured on a four-level AMR mesh);
    None for other equation counts, which those captures do not cover."""
    f = ROOT / "profiles" / "stage_kernels.json"
    if neq != 5 or not f.exists():
        return None
    try:
        d = json.loads(f.read_text())
        return d["corrector_fused" if fused else "corrector"]
    except Exception:
        return None


def fp64_peak_tflops(lib):
    import ctypes
    g = ctypes.c_double()
    return g.value / 1e3 if lib.wx3d_measure_fp64_peak(ctypes.byref(g)) == 0 else None


def run_reference(args, rank, world):
    if rank != 0:   # one CPU run per job: the other ranks exit without work
        return
    prob = build_problem(args.workload)
    threads = os.cpu_count() or 1
    budget = float(os.environ.get("WX3D_REF_BUDGET_S", "90"))
    # warm-up steps are whole oracle steps too, bounded by a share of the budget
    import oracle
    o = oracle.from_problem(prob, threads=threads)
    tw = time.perf_counter()
    for _ in range(args.warmup):
        o.step()
        if time.perf_counter() - tw > budget / 4:
            break
    n, t0 = 0, time.perf_counter()
    while n < args.steps:
        o.step()
        n += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    value = prob.cells * n / el / 1e6
    line = {
        "impl": "reference",
        "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s",
        "n_gpus": world, "steps": n, "warmup": args.warmup, "ms_per_step": el / n * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "blocks": prob.nblocks, "cells": prob.cells,
                   "description": WORKLOADS[args.workload]["desc"]},
        "cpu_baseline": {"value": value, "unit": "Mcell-updates/s", "cores": threads, "kind": "port",
                         "sample": f"{n} whole steps of the workload (of {args.steps} requested; "
                                   f"{budget:.0f}s budget) by the C++ FP64 restatement of the reference, "
                                   f"OpenMP over blocks"},
        "e2e": {"value": value, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def live_mesh_leg(prob, args, stream):
    """Throughput with a live mesh (main.f90:79-103 with admesh after every
    step): a fresh context with room for 3x the snapshot's blocks runs W
    warm-up and K timed iterations of wx3d_step followed by wx3d_admesh,
    timed with CUDA events on the library's stream around the K iterations.
    The cells of each step are the leaves of the mesh that step ran on."""
    import torch
    from walicxe3d_b200._lib import WxError
    from walicxe3d_b200.solver import from_problem
    w = from_problem(prob, extra_slots=2 * prob.nblocks)
    w.set_stream(stream.cuda_stream)
    nblocks = prob.nblocks
    out = {"unit": "Mcell-updates/s", "steps": args.steps, "blocks_start": nblocks}
    try:
        for _ in range(args.warmup):
            w.step()
            w.admesh()
        nblocks = int((w.local_blocks != -1).sum())
        out["blocks_after_warmup"] = nblocks
        torch.cuda.synchronize()
        cells, ref, crs, t_ad = 0, 0, 0, 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            cells += nblocks * 4096
            w.step()
            t0 = time.perf_counter()
            r, c = w.admesh()
            t_ad += time.perf_counter() - t0
            ref, crs = ref + r, crs + c
            nblocks = int((w.local_blocks != -1).sum())
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out.update({"value": cells / (ms / 1e3) / 1e6, "ms_per_step": ms / args.steps,
                    "admesh_ms_per_call": 1e3 * t_ad / args.steps, "blocks_end": nblocks,
                    "refined": ref, "coarsened_families": crs,
                    "note": "each step: wx3d_step (synchronous) then wx3d_admesh (device marking, proximity rule "
                            "and slot registry on the host, batched refine/coarsen copies, neighbour-table "
                            "rebuild)"})
    except WxError as e:
        out["error"] = str(e)
    finally:
        w.close()
    return out


def cooling_workload() -> str:
    """The cooling AMR workload of the metric's comparison: colliding winds
    (table cooling + ionisation surrogate, 20,896 blocks) when the host can
    hold the CPU port's arrays (~45 GB), else the radiative SNR at 64^3 root
    cells (COOL_H + surrogate, 960 blocks).  WX3D_COOLING_WORKLOAD overrides."""
    name = os.environ.get("WX3D_COOLING_WORKLOAD")
    if name:
        return name
    try:
        with open("/proc/meminfo") as f:
            avail = next(int(l.split()[1]) * 1024 for l in f if l.startswith("MemAvailable:"))
    except (OSError, StopIteration):
        avail = 0
    return "winds" if avail > 64 * 2**30 else "snr-h-c4"


def cooling_leg(args, stream):
    """The metric's three-way comparison on a cooling AMR workload, timed past
    the 10-step dt ramp of main.f90 (whose dt lies below the surrogate's
    training box): the batched form with the learned surrogate attached
    (autotuned launch shape, replayed CUDA graph, MLP for trusted cells), the
    same batched form without it, the plain GPU path (one synchronous
    wx3d_step per step, launch shape from the mesh size, no graph, plain FP64
    integrator), and the CPU port on a bounded sample.  Device times are CUDA
    events on the library's stream; the CPU port is wall clock."""
    import torch
    from walicxe3d_b200.autotune import tune
    from walicxe3d_b200.solver import from_problem
    name = cooling_workload()
    prob = build_problem(name)
    ramp, K = 12, args.steps
    out = {"workload": name, "description": WORKLOADS[name]["desc"], "blocks": prob.nblocks, "cells": prob.cells,
           "unit": "Mcell-updates/s", "steps": K, "untimed_steps_first": ramp}

    def timed(n, fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(n)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        return {"value": prob.cells * n / (ms / 1e3) / 1e6, "ms_per_step": ms / n}

    w = from_problem(prob)
    w.set_stream(stream.cuda_stream)
    tuned = tune(w, prob, cache=None, reps=1)
    w.attach_surrogate()
    w.run(ramp)
    w.reset_status()
    b = timed(K, w.run_async)
    st = w.status()
    sc, fc = int(st.surrogate_cells), int(st.fallback_cells)
    b.update({"surrogate_cells": sc, "fallback_cells": fc, "share": sc / max(1, sc + fc),
              "autotune": {"zsplit": tuned["zsplit"], "fused_viscous": tuned.get("fused")}})
    out["batched_surrogate"] = b
    w.detach_surrogate()
    w.run(2)
    out["batched"] = timed(K, w.run_async)
    w.close()

    wp = from_problem(prob)
    wp.set_stream(stream.cuda_stream)
    for _ in range(ramp):
        wp.step()

    def plain(n):
        for _ in range(n):
            wp.step()
    out["plain"] = timed(K, plain)
    wp.close()
    out["surrogate_gain_vs_plain"] = out["batched_surrogate"]["value"] / out["plain"]["value"]
    out["batched_gain_vs_plain"] = out["batched"]["value"] / out["plain"]["value"]
    if not args.no_cpu_baseline:
        v, n, secs = cpu_time_oracle(prob, 1000, float(os.environ.get("WX3D_CPU_BUDGET_S", "20")),
                                     os.cpu_count() or 1)
        out["cpu_port"] = {"value": v, "cores": os.cpu_count(), "kind": "port",
                           "sample": f"{n} whole steps from the initial state in {secs:.1f}s, C++ FP64 "
                                     f"restatement of the reference, OpenMP over blocks"}
    return out


def run_partition(args, prob, rank, world, dist):
    """One mesh shared by the ranks (walicxe3d_b200.partition): each owns a
    Hilbert share plus halo copies whose face slabs are exchanged over NCCL
    between the stages;
    timed with CUDA events on the library stream, max over ranks."""
    import torch
    from walicxe3d_b200.partition import Rank, TorchDist, make_plan
    plans = make_plan(prob.local_blocks, prob.cfg.nbroot, prob.cfg.maxlev, world)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    r = Rank(prob, plans[rank], stream.cuda_stream)
    if dist is None:
        class _Local:   # one rank: the parts without exchanges
            def __init__(self, r):
                self.r = r

            def step(self):
                self.r.set_dtmin(self.r.dtmin())
                for p in range(4):
                    self.r.part(p)
        tr = _Local(r)
    else:
        tr = TorchDist(r)
    for _ in range(args.warmup):
        tr.step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        tr.step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    if rank == 0:
        line = {"metric": "Mcell-updates/s", "value": prob.cells * args.steps / (ms / 1e3) / 1e6,
                "unit": "Mcell-updates/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": args.workload, "description": WORKLOADS[args.workload]["desc"],
                           "blocks": prob.nblocks, "cells": prob.cells,
                           "parallelism": f"block partition x{world} (Hilbert shares, halo face slabs over NCCL)",
                           "halo_blocks": [len(p.halo) for p in plans],
                           "halo_face_slabs": [sum(len(v) for v in p.recv_faces.values()) for p in plans],
                           "exchange_bytes_per_step": 2 * sum(sum(len(v) for v in p.recv_faces.values())
                                                              for p in plans) * prob.cfg.neqtot * 1024 * 8}}
        print(json.dumps(line), flush=True)
    r.w.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="wx3d", choices=["wx3d", "reference"])
    ap.add_argument("--workload", default="blast-amr", choices=sorted(WORKLOADS))
    ap.add_argument("--zsplit", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-live-mesh", action="store_true", help="skip the live-mesh (admesh every step) leg")
    ap.add_argument("--no-cooling", action="store_true",
                    help="skip the cooling-workload leg (batched + surrogate vs batched vs plain GPU vs CPU port)")
    ap.add_argument("--partition", action="store_true",
                    help="strong scaling: the ranks share one mesh (halo exchange over NCCL) instead of replicas")
    ap.add_argument("--surrogate", action="store_true",
                    help="attach the trained surrogate (EOS_H_RATE workloads: with COOL_H both outputs, "
                         "with table cooling its ionisation output)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank, world, local = dist_env()
    if args.impl == "reference":
        if world > 1:
            import torch.distributed as dist
            dist.init_process_group("gloo", timeout=__import__("datetime").timedelta(seconds=600))
        run_reference(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from walicxe3d_b200.solver import from_problem

    prob = build_problem(args.workload)
    if args.partition:
        return run_partition(args, prob, rank, world, dist)
    w = from_problem(prob)
    # a dedicated stream: the library runs on it and the timing events are
    # recorded on it (the default stream's handle 0 would select the
    # library's own stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    w.set_stream(stream.cuda_stream)
    tuned = None
    if args.zsplit:
        w.set_zsplit(args.zsplit)
    else:
        from walicxe3d_b200.autotune import tune
        tuned = tune(w, prob, cache=None, reps=2)
    if args.surrogate:
        w.attach_surrogate()
    w.set_timing(True)

    # --- warm-up (graph capture happens here) ---
    w.run(args.warmup - args.warmup % 2 if args.warmup >= 2 else 2)
    torch.cuda.synchronize()

    # --- device-resident timed region ---
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    k0 = w.kernels_launched
    w.reset_status()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    w.run_async(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = w.kernels_launched - k0
    kt_ms, kt_n = w.kernel_times()
    wst = w.status()
    sur_cells, fb_cells = int(wst.surrogate_cells), int(wst.fallback_cells)
    clocks = sampler.stop()
    st = w.state
    if dist is not None:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        if dist is not None:
            dist.barrier()
    value = prob.cells * args.steps * world / (ms / 1e3) / 1e6

    # --- roofline of the dominant kernel (corrector stage) ---
    try:
        peak, peak_src = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except Exception:
        peak, peak_src = 6650.0, "fallback"
    neq = prob.cfg.neqtot
    stage2_ms = kt_ms[1] / max(kt_n[1], 1)
    fused = kt_n[2] == 0          # no separate viscous launch: the corrector carries it
    alg_bytes = 3 * neq * 8 * prob.cells     # reads UP and U, writes the stage result
    achieved = alg_bytes / (stage2_ms / 1e3) / 1e9 if stage2_ms > 0 else None
    step_bytes = 40 * neq * prob.cells       # 5 compulsory state passes per step
    step_achieved = step_bytes * args.steps * world / (ms / 1e3) / 1e9
    fig = stage_figures(neq, fused)
    multilevel = len({int(prob.tree.level(int(b))) for b in prob.local_blocks}) > 1
    per_cell = fig and (fig.get("dram_bytes_per_cell_amr") if multilevel and "dram_bytes_per_cell_amr" in fig
                        else fig["dram_bytes_per_cell"])
    traffic = per_cell * prob.cells if fig else None
    fp64 = None
    if fig and "fp64_flops_per_cell" in fig and stage2_ms > 0:
        pk = fp64_peak_tflops(w.lib)
        ach = fig["fp64_flops_per_cell"] * prob.cells / (stage2_ms / 1e3) / 1e12
        inst = fig.get("fp64_inst_per_cell")
        fp64 = {"achieved_tflops": ach, "peak_tflops": pk, "frac": (ach / pk) if pk else None,
                "flops_per_cell": fig["fp64_flops_per_cell"],
                "inst_per_cell": inst,
                # FP64 instructions issued over the rate of DFMA chains (a DADD
                # or DMUL takes the issue slot of a DFMA)
                "inst_frac": (inst * prob.cells / (stage2_ms / 1e3) / (pk * 1e12 / 2)) if (pk and inst) else None,
                "peak_source": "measured in this run (wx3d_measure_fp64_peak, DFMA chains)",
                "note": "per-cell figures from the ncu capture on Sedov 256^3; the stage kernels are "
                        "latency-bound, below both their FP64 instruction bound and the HBM bound"}

    # --- the plain GPU path: the same kernels, one synchronous wx3d_step per
    # step (host round trip each step), default launch shape, no graph ---
    plain = None
    if rank == 0:
        from walicxe3d_b200.solver import from_problem as _fp
        wp = _fp(prob)
        wp.set_stream(stream.cuda_stream)
        for _ in range(args.warmup):
            wp.step()
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(args.steps):
            wp.step()
        p1.record(stream)
        torch.cuda.synchronize()
        pms = p0.elapsed_time(p1)
        wp.close()
        plain = {"value": prob.cells * args.steps / (pms / 1e3) / 1e6, "unit": "Mcell-updates/s",
                 "ms_per_step": pms / args.steps, "batched_gain": value / world / (prob.cells * args.steps / (pms / 1e3) / 1e6),
                 "note": "wx3d_step per step (returns time/dt/status to the host), launch shape from the mesh "
                         "size alone, no CUDA graph; batched = the timed wx3d_run graph replay with the autotuned shape"}

    # --- end to end through the C-ABI with host buffers ---
    U_host = torch.from_numpy(prob.U).pin_memory()
    U_out = torch.empty_like(U_host).pin_memory()
    import ctypes
    lib, ctx = w.lib, w.ctx
    uptr = ctypes.cast(U_host.data_ptr(), ctypes.POINTER(ctypes.c_double))
    optr = ctypes.cast(U_out.data_ptr(), ctypes.POINTER(ctypes.c_double))
    from walicxe3d_b200.config import WxState
    w.set_timing(False)
    sst = WxState()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = lib.wx3d_upload_blocks(ctx, prob.nblocks, uptr)
    for _ in range(args.steps):
        rc |= lib.wx3d_step(ctx, ctypes.byref(sst))
    rc |= lib.wx3d_download_blocks(ctx, prob.nblocks, optr)
    e2e_s = time.perf_counter() - t0
    if rc:
        raise SystemExit(f"e2e leg failed with status {rc}")
    if dist is not None:
        t = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = prob.cells * args.steps * world / e2e_s / 1e6
    state_bytes = prob.U.nbytes

    w.close()
    live = None
    if rank == 0 and not args.no_live_mesh and not args.surrogate and prob.tree.maxlev > 1 and not prob.winds:
        live = live_mesh_leg(prob, args, stream)

    cooling = None
    if rank == 0 and world == 1 and not args.no_cooling:
        cooling = cooling_leg(args, stream)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, n, secs = cpu_time_oracle(prob, 1000, float(os.environ.get("WX3D_CPU_BUDGET_S", "20")), os.cpu_count() or 1)
        cpu = {"value": v, "unit": "Mcell-updates/s", "cores": os.cpu_count(), "kind": "port",
               "sample": f"{n} whole steps of the same workload in {secs:.1f}s by the C++ FP64 restatement "
                         f"of the reference (OpenMP over blocks)"}

    if rank == 0:
        line = {
            "metric": "Mcell-updates/s", "value": value, "unit": "Mcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload]["desc"],
                       "blocks": prob.nblocks, "cells": prob.cells, "neq": neq,
                       "levels": sorted({int(prob.tree.level(int(b))) for b in prob.local_blocks}),
                       "l2": "state arrays larger than L2 (%.2f GB each)" % (state_bytes / 1e9),
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "path": "wx3d_run: CUDA graph of 2 steps replayed",
                       "autotune": tuned and {"zsplit": tuned["zsplit"], "fused_viscous": tuned.get("fused"),
                                              "ms_per_pass": tuned["ms_per_pass"], "key": tuned.get("key"),
                                              "note": "one shape for all levels: every level's block is the same "
                                                      "16^3 tile of one persistent launch"}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                         "kernel": "stage_kernel<ORDER=2> (corrector%s)" % (" + viscous step" if fused else ""),
                         "peak_source": peak_src, "fp64": fp64,
                         "alg_bytes_per_launch": alg_bytes, "launch_ms": stage2_ms,
                         "step_alg_gbs": step_achieved, "step_frac": step_achieved / peak},
            "kernel_ms_per_launch": {k: (m / n if n else None) for k, m, n in
                                     zip(["stage1", "stage2", "viscous", "sources"], kt_ms, kt_n)},
            "e2e": {"value": e2e_value, "unit": "Mcell-updates/s",
                    "h2d_bytes_per_step": state_bytes / args.steps + 32,
                    "d2h_bytes_per_step": state_bytes / args.steps + 128,
                    "note": "timed: upload of the state from pinned host memory, K wx3d_step calls (each "
                            "returns time/dt/status to the host), download of the final state"},
            "gpu_launches": launches,
            "live_mesh": live,
            "cooling": cooling,
            "plain_steps": plain,
            "surrogate": ({"attached": True, "surrogate_cells": sur_cells, "fallback_cells": fb_cells,
                           "share": sur_cells / max(1, sur_cells + fb_cells)} if args.surrogate else None),
            "clocks": clocks,
            "cpu_baseline": cpu,
            "final_state": {"time": st.time, "dt": st.dt, "it": st.it},
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

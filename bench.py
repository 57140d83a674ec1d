#!/usr/bin/env python
"""Benchmark of the SME time step (cell-steps/s and fraction of the HBM
roofline).

Workload (default): SME level 4 (12 FP64 state slots) on the Hilbert-
renumbered Delaunay mesh of a 1400x1400 jittered grid (3.91M triangles),
16-Gaussian bathymetry, Navier-slip source; order 2 (Green-Gauss + Vacuum/
TVD limiting), SSP-RK2, CFL 0.45.  A "step" is one full time step (two SSP
stages, constraints, implicit source, CFL dt).  Inputs (375 MB of state +
1.1 GB of face states) exceed the 126 MB L2, so no flush is needed between
steps.  The K timed steps run as CUDA graphs; a second, profiled pass of K
steps (one CUDA event pair per kernel launch) gives the per-kernel times
behind the roofline.

``--workload ensemble``: SME level-2 instances on their own meshes (grid
side log-uniform in [40, 400]) advanced by the batched path, then by a loop
of single-instance solvers over the same instances; reports both times, the
speed-up and the largest relative L2 difference between the two results.

Launch: ``python bench.py [--gpus N --steps K --warmup W]``; for N > 1 one
rank per GPU under torchrun, each rank advancing its own replica (the single
mesh is not partitioned: replicas, weak scaling).  ``--impl reference`` times
the CPU restatement of the reference step (the oracle) on the host cores.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SME cell-steps/s & % HBM roofline"
UNIT = "cell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--side", type=int, default=0, help="jittered grid side of the mesh (0: the case's own)")
    ap.add_argument("--case", default="roofline_l4", choices=["roofline_l4", "level2", "plain_l0"],
                    help="plain-step case: SME level 4 on 1400^2 (default), level 2 on 240^2, level 0 on 60^2")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="the CPU baseline (oracle on the same mesh) steps until this much time has passed")
    ap.add_argument("--ref-seconds", type=float, default=240.0,
                    help="--impl reference: the timed oracle steps end once this much time has passed")
    ap.add_argument("--lsq-steps", type=int, default=5,
                    help="steps timed with the least-squares gradient beside the default Green-Gauss (0: none)")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = same as --steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch configuration")
    ap.add_argument("--workload", choices=["roofline", "ensemble", "adjoint", "implicit"], default="roofline")
    ap.add_argument("--imp-side", type=int, default=240, help="grid side of the implicit workload")
    ap.add_argument("--imp-cfl", type=float, default=4.5, help="CFL number of the implicit workload")
    ap.add_argument("--launch", default="", help="launch configuration as JSON (keys of solver.LAUNCH_KEYS); "
                    "skips the autotuner")
    ap.add_argument("--instances", type=int, default=512,
                    help="ensemble size in all, split across the ranks (--workload ensemble)")
    ap.add_argument("--adj-side", type=int, default=200, help="grid side of the adjoint workload")
    ap.add_argument("--adj-steps", type=int, default=400, help="steps of the adjoint workload")
    ap.add_argument("--adj-limiter", default="tvd", choices=["tvd", "none"], help="limiter of the adjoint workload")
    ap.add_argument("--adj-fd", type=int, default=32, help="finite-difference directions of the adjoint check (0: none)")
    ap.add_argument("--positivity", default="none", choices=["none", "zhang_shu", "mood"],
                    help="positivity variant of the roofline workload")
    return ap.parse_args()


CASE_SIDE = {"roofline_l4": 1400, "level2": 240, "plain_l0": 60}
CASE_TEXT = {"roofline_l4": ("sme2d_l4 SME level 4", "Navier-slip Newton source"),
             "level2": ("sme2d_l2 SME level 2", "Navier-slip Newton source"),
             "plain_l0": ("sme2d_l0 SME level 0 (shallow water)", "Manning friction Newton source")}
GRAD_TEXT = {"green_gauss": "order 2 Green-Gauss + Vacuum/TVD",
             "least_squares": "order 2 least squares + Vacuum/TVD (Barth-Jespersen)"}
POS_TEXT = {"none": "", "zhang_shu": ", eta-well-balanced reconstruction + Zhang-Shu theta (CFL clamped to 1/6)",
            "mood": ", eta-well-balanced reconstruction + local MOOD"}


# ------------------------------------------------------------------ roofline
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def algorithmic_bytes(kind, C, F, nq, na, K, stages, fused=False):
    """Compulsory HBM bytes of one launch of each kernel when every array it
    touches is read or written exactly once (neighbour re-reads are free).
    fused: "flux" is the fused face + gather tile kernel (face states,
    geometry and support in, the stage's state in and out; no face
    contributions in device memory)."""
    d = 2
    if kind == "prep":      # state + aux + slot tables in, two face states per face out
        return C * (8 * nq + 8 * na + 12 * K + 16 * d * K) + F * 16 * nq
    if kind == "flux" and fused:
        state_passes = (2 * (stages - 1) + 3) / stages      # FIRST/MID: in+out (+ clamped copy), FINAL: in+base+out
        return F * (16 * nq + 8 * (2 * d + 1) + 12) + C * (8 * na + 4 * K + 8 + 8 * nq * state_passes)
    if kind == "flux":      # face kernel: two face states + geometry + support in, 3 NQ contributions out
        return F * (16 * nq + 8 * (2 * d + 1) + 12 + 24 * nq) + C * 8 * na
    if kind == "gather":    # 3 NQ contributions per face in, state in/out
        state_passes = (2 * (stages - 1) + 3) / stages      # FIRST/MID: in+out, FINAL: in+base+out
        return F * 24 * nq + C * (12 * K + 4 + 8 + 8 * nq * state_passes)
    if kind == "finalize":
        return C * (16 * nq + 16 * na + 8)
    return 0.0


def step_bytes_fused(nq):
    """Per cell-step bytes of a fully fused SSP-RK2 step (5 m_e + 2 state
    arrays + 304 B of geometry, m_e = evolving variables)."""
    me = nq - 1
    return 8 * (5 * me + 2) + 304


# DRAM bytes (read + write) per cell of one launch, from the ncu captures of
# profiles/sme2d_l4_kernels_900.md (900x900 grid, 1,616,402 cells; mean of
# two launches) in the launch configuration the autotuner picks at level 4:
# separate face and gather kernels, the face-state kernel split over four
# threads per cell, the last stage's gather inside finalize (register cap 4).
# The streams scale with the cell count, so a 1400x1400 launch moves these
# figures times its cells.
NCU_DRAM_BYTES_PER_CELL = {
    "sme2d_l4/prep": (436.6 + 425.4) * 1e6 / 1616402,
    "sme2d_l4/flux": (544.7 + 652.4) * 1e6 / 1616402,
    "sme2d_l4/gather": (1143.8 + 282.5) * 1e6 / 1616402,
    "sme2d_l4/finalize+gather": (1125.9 + 422.2) * 1e6 / 1616402,
}
NCU_LAUNCH = {"tile_faces": 0, "fuse_final": 1, "prep_lean": 4}


def traffic_per_cell_step(model, launch, stages):
    """Measured DRAM bytes per cell-step of the whole step (every launch's
    ncu traffic summed), for the launch configuration the table was captured
    in; None for any other."""
    if model != "sme2d_l4" or any(launch.get(k) != v for k, v in NCU_LAUNCH.items()) or stages != 2:
        return None
    t = NCU_DRAM_BYTES_PER_CELL
    return 2 * t["sme2d_l4/prep"] + 2 * t["sme2d_l4/flux"] + t["sme2d_l4/gather"] + t["sme2d_l4/finalize+gather"]


# Algorithmic FP64 operations per unit of each kernel: +, -, *, /, sqrt,
# cbrt and pow on state and parameter values (selects, min / max and fabs
# are not counted), counted by the CPU restatement of the reference step on
# an operation-counting scalar over 2 steps of each configuration's 40x40
# grid (tests/test_flop_count.py recounts them).  prep and gather: per cell
# and stage; flux: per face and stage (the grid's mean over interior and
# wall faces); finalize: per cell and step (constraints, Newton source,
# CFL dt).
FP64_FLOPS = {
    "sme2d_l4": {"prep": 579.524, "flux": 1256.84, "gather": 126.0, "finalize": 2841.0},
    "sme2d_l2": {"prep": 392.726, "flux": 528.504, "gather": 84.0, "finalize": 1280.0},
    "sme2d_l0": {"prep": 183.089, "flux": 204.168, "gather": 42.0, "finalize": 127.0},   # least squares
    "sme2d_l1": {"prep": 311.716, "flux": 332.336, "gather": 63.0, "finalize": 531.129},
}


def fp64_flops(kind, model, C, F, stages, fused=False):
    """Algorithmic FP64 operations of one launch of a step kernel (None
    where the table has no figure); fused: "flux" is the fused face + gather
    tile kernel, which does both kernels' work."""
    t = FP64_FLOPS.get(model, {})
    if kind not in t:
        return None
    if kind == "flux" and fused:
        return t["flux"] * F + t["gather"] * C
    return t[kind] * (F if kind == "flux" else C)


def fp64_flops_per_cell_step(model, C, F, stages):
    t = FP64_FLOPS[model]
    return stages * (t["prep"] + t["gather"] + t["flux"] * F / C) + t["finalize"]


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clock, power and clock-event reasons of the timed GPU, sampled
    while the timed region runs: NVML every 10 ms (the GPU found by its UUID,
    so CUDA_VISIBLE_DEVICES does not matter; start() returns after the
    first sample and stop() takes a last one), else nvidia-smi every 200 ms.
    Read-only queries."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.nv = None
        self.lines = []
        self.samples = []

    def _nvml_handle(self, nv):
        import torch

        pr = torch.cuda.get_device_properties(self.index)
        try:
            return nv.nvmlDeviceGetHandleByUUID("GPU-" + str(pr.uuid))
        except Exception:
            return nv.nvmlDeviceGetHandleByPciBusId_v2("%08X:%02X:%02X.0" % (
                pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id))

    def _nvml_sample(self):
        nv, h = self.nv, self.h
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
        self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), nv.nvmlDeviceGetPowerUsage(h) / 1e3,
                             tuple(n for n, b in zip(self.NAMES, bits) if r & b)))

    def _poll(self):
        while not self.done.is_set():
            try:
                self._nvml_sample()
            except Exception:
                break
            self.first.set()
            self.done.wait(0.01)
        self.first.set()

    def start(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            self.nv = nv
            self.h = self._nvml_handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.done, self.first = threading.Event(), threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            self.first.wait(2.0)
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.nv is not None:
            self.done.set()
            self.t.join(timeout=2.0)
            try:
                self._nvml_sample()
            except Exception:
                pass
            if not self.samples:
                return None
            return {"sm_mhz": statistics.median(x[0] for x in self.samples), "sm_max_mhz": self.max_mhz,
                    "power_w_median": statistics.median(x[1] for x in self.samples),
                    "reasons": sorted({n for x in self.samples for n in x[2]}), "samples": len(self.samples),
                    "source": "NVML, 10 ms"}
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for ln in self.lines:
            v = [x.strip() for x in ln.split(",")]
            if len(v) >= 9:
                rows.append(v)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms"}


# ------------------------------------------------------------------ cases
def params_of(case):
    from zoomy_dmplex_b200 import models

    names, vals = models.parameter_table(case.model)
    for k, v in case.params.items():
        vals[names.index(k)] = v
    return np.array(vals)


def cpu_sample(side, steps=0, warm=1, seconds=0.0, positivity="none", case="roofline_l4", built=None,
               max_seconds=0.0):
    """The oracle (CPU restatement of the reference step) on the workload's
    own mesh (`built`: the case already built by the GPU arm; else the case
    on a side x side grid): `steps` steps, or (steps = 0) one step at a time
    until `seconds` have passed; max_seconds > 0 ends a `steps` run early once
    that much time has passed (the run stays bounded on slow hosts).
    Returns (cell-steps/s, threads, cells, seconds, steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py as O
    from zoomy_dmplex_b200 import cases

    c = built if built is not None else getattr(cases, case)(side)
    c.settings.positivity = positivity
    nt = O.set_threads(0)
    o = O.Oracle(c.model, c.mesh.as_abi_arrays(), c.settings.to_struct(), params_of(c))
    o.set_state(c.q0)
    o.step(warm)
    t0 = time.perf_counter()
    n = 0
    while True:
        el = time.perf_counter() - t0
        if steps:
            if n >= steps or (max_seconds > 0 and n > 0 and el >= max_seconds):
                break
        elif n > 0 and el >= seconds:
            break
        o.step(1)
        n += 1
    dt = time.perf_counter() - t0
    return c.mesh.n_cells * n / dt, nt, c.mesh.n_cells, dt, n


def run_ensemble(a, dev, torch, dist, rank, world):
    """Batched ensemble against the loop of single-instance solvers over the
    same instances (each rank advances its own shard of instances)."""
    import ctypes as ct

    from zoomy_dmplex_b200 import autotune, cases, native
    from zoomy_dmplex_b200.solver import BatchSolver, Solver, set_launch

    def barrier():
        if dist:
            dist.barrier()

    # the configuration's a.instances instances in all, dealt to the ranks in
    # greedy size-balanced shards (total work fixed as N grows)
    shard = cases.ensemble_shard(a.instances, world, rank)
    n = len(shard)
    t0 = time.perf_counter()
    members = cases.ensemble(indices=shard)
    build_s = time.perf_counter() - t0
    model, st = members[0].model, members[0].settings
    meshes = [c.mesh for c in members]
    params = [params_of(c) for c in members]
    C = sum(m.n_cells for m in meshes)
    F = sum(m.n_faces for m in meshes)
    B = BatchSolver(model, meshes, st, params, device=dev)

    def reset_batch():
        for i, c in enumerate(members):
            B.set_state(i, c.q0)

    reset_batch()
    tuned = None
    if not a.no_tune:
        tuned = autotune.tune(B, model, C, steps=2, use_cache=False, write_cache=False)
        reset_batch()
    B.step(a.warmup)
    B.sync()
    reset_batch()
    stream = torch.cuda.ExternalStream(B.stream, device=dev)
    clk = ClockSampler(dev)
    clk.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    B.step(a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    batch_wall = time.perf_counter() - w0
    barrier()
    clocks = clk.stop()
    ms_batch = e0.elapsed_time(e1)
    diag = B.sync(check=True)
    got = [B.get_state(i) for i in range(n)]
    t_batch = [B.time(i)[0] for i in range(n)]
    launches = a.steps * B.launches_per_step()

    # the same instances, one single-instance solver each, stepped one after the other
    singles = [Solver(model, c.mesh, st, p, device=dev) for c, p in zip(members, params)]
    for s, c in zip(singles, members):
        if tuned:
            set_launch(s.h, tuned)
        s.set_state(c.q0)
        s.step(a.warmup)
    torch.cuda.synchronize()
    for s, c in zip(singles, members):
        s.set_state(c.q0)
    torch.cuda.synchronize()
    barrier()
    w0 = time.perf_counter()
    for s in singles:
        s.step(a.steps)
    torch.cuda.synchronize()          # every solver stream
    loop_wall = time.perf_counter() - w0
    barrier()
    rel, t_diff = 0.0, 0.0
    for i, s in enumerate(singles):
        ref = s.get_state()
        rel = max(rel, float(np.linalg.norm(got[i] - ref) / max(np.linalg.norm(ref), 1e-300)))
        t_diff = max(t_diff, abs(s.time()[0] - t_batch[i]))
    # the same loop, waiting for each instance before starting the next
    for s, c in zip(singles, members):
        s.set_state(c.q0)
    torch.cuda.synchronize()
    barrier()
    w0 = time.perf_counter()
    for s in singles:
        s.step(a.steps)
        s.sync(check=False)
    sync_loop_wall = time.perf_counter() - w0
    barrier()
    loop_launches = a.steps * sum(s.launches_per_step() for s in singles)
    for s in singles:
        s.close()

    t = torch.tensor([ms_batch, loop_wall, batch_wall, sync_loop_wall], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max, loop_max, bwall_max, sloop_max = (float(x) for x in t.tolist())
    # the whole job: every rank's cells over the slowest rank's time
    tc = torch.tensor([float(C), float(F), rel, t_diff], dtype=torch.float64, device="cuda")
    if dist:
        tc0 = tc[:2].clone()
        dist.all_reduce(tc0, op=dist.ReduceOp.SUM)
        tc1 = tc[2:].clone()
        dist.all_reduce(tc1, op=dist.ReduceOp.MAX)
        tc = torch.cat([tc0, tc1])
    C_all, F_all, rel_all, t_diff_all = (float(x) for x in tc.tolist())
    identical = rel_all == 0.0 and t_diff_all == 0.0
    value = C_all * a.steps / (ms_max / 1e3)

    # end to end through the public API: every instance's state from pinned host
    # memory, one batched step, every state back
    ne = min(a.steps, 3)
    nq = B.nq
    hosts = [torch.from_numpy(np.ascontiguousarray(c.q0)).pin_memory() for c in members]
    outs = [torch.empty_like(h).pin_memory() for h in hosts]
    lib = native.load()
    P = ct.POINTER(ct.c_double)
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(ne):
        for i in range(n):
            native.check(lib.zsme_batch_set_state(B.h, i, ct.cast(hosts[i].data_ptr(), P), 0.0))
        native.check(lib.zsme_step(B.h, 1))
        for i in range(n):
            native.check(lib.zsme_batch_get_state(B.h, i, ct.cast(outs[i].data_ptr(), P)))
    e3.record(stream)
    torch.cuda.synchronize()
    t2 = torch.tensor([e2.elapsed_time(e3)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_value = C_all * ne / (float(t2.item()) / 1e3)
    B.close()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True,
            "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "ensemble of %d SME level-2 instances (%d on rank 0), jittered-Delaunay grid "
                                   "side log-uniform in [40, 400] (%d cells, %d faces in all), order 2 Green-Gauss + "
                                   "Vacuum/TVD, SSP-RK2, CFL 0.45 per instance, Navier-slip Newton source"
                                   % (a.instances, n, int(C_all), int(F_all)),
                       "model": model, "instances": a.instances, "instances_rank0": n, "cells": int(C_all),
                       "faces": int(F_all),
                       "parallelism": "instance shards x%d" % world if world > 1 else "single GPU",
                       "l2_flush": "not needed: state %.0f MB > 126 MB L2" % (C * nq * 8 / 1e6),
                       "timing": "CUDA events on the batch stream around K graph-launched steps",
                       "launch": tuned or "default", "mesh_build_s": build_s},
            "ensemble": {"batched_ms_per_step": ms_max / a.steps,
                         "batched_wall_ms_per_step": 1e3 * bwall_max / a.steps,
                         "loop_wall_ms_per_step": 1e3 * loop_max / a.steps,
                         "speedup_vs_loop": loop_max / bwall_max,
                         "sync_loop_wall_ms_per_step": 1e3 * sloop_max / a.steps,
                         "speedup_vs_sync_loop": sloop_max / bwall_max,
                         "loop": "one single-instance solver per instance (own stream, CUDA graph per step), "
                                 "K steps each, instances one after the other; host wall clock around the "
                                 "loop and a device synchronize (the batched time beside it is taken the same way); "
                                 "sync loop: the same, waiting for each instance's K steps before the next",
                         "max_rel_l2_vs_loop": rel_all, "max_time_diff_vs_loop": t_diff_all,
                         "bit_identical_to_loop": identical,
                         "loop_gpu_launches": loop_launches},
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": C * nq * 8,
                    "d2h_bytes_per_step": C * nq * 8, "steps": ne,
                    "api": "zsme_batch_set_state x n (pinned host) + zsme_step(1) + zsme_batch_get_state x n"},
            "gpu_launches": launches,
            "diag": {"nonfinite": diag.n_nonfinite, "negative_depth": diag.n_negative_depth,
                     "newton_unconverged": diag.n_newton_unconverged, "mood_cells": diag.n_mood_cells},
            "clocks": clocks}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    # every instance must end bit-identical (state and time) to its own plain solve
    return 0 if identical else 3


def run_implicit(a, dev, torch, dist, rank, world):
    """The fully implicit strategy (BDF2, Newton-Krylov) on the level-2 case
    of configuration 1 at first order in space and a CFL number ten times the
    explicit one, against the explicit splitting step (order 1, CFL 0.45) over
    the same simulated time.  Reported: implicit cell-steps/s, and both
    strategies' simulated time per second of device time.  Each rank runs its
    own replica."""
    import dataclasses

    from zoomy_dmplex_b200 import cases
    from zoomy_dmplex_b200.solver import Solver

    def barrier():
        if dist:
            dist.barrier()

    c = cases.level2(a.imp_side)
    C = c.mesh.n_cells
    p = params_of(c)
    st_imp = dataclasses.replace(c.settings, time_integration="implicit", reconstruction_order=1, cfl=a.imp_cfl)
    st_exp = dataclasses.replace(c.settings, reconstruction_order=1)
    gi = Solver(c.model, c.mesh, st_imp, p, device=dev)
    ge = Solver(c.model, c.mesh, st_exp, p, device=dev)
    stream_i = torch.cuda.ExternalStream(gi.stream, device=dev)
    stream_e = torch.cuda.ExternalStream(ge.stream, device=dev)
    gi.set_state(c.q0)
    gi.step(max(1, a.warmup))
    gi.set_state(c.q0)
    clk = ClockSampler(dev)
    clk.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    newton, gmres = [], []
    t_sim0 = gi.time()[0]
    e0.record(stream_i)
    for _ in range(a.steps):
        gi.step(1)
        s4 = gi.implicit_stats()
        newton.append(s4[0])
        gmres.append(s4[1])
    e1.record(stream_i)
    torch.cuda.synchronize()
    imp_ms = e0.elapsed_time(e1)
    t_sim = gi.time()[0] - t_sim0
    # the explicit step over the same simulated time
    ge.set_state(c.q0)
    ge.step(max(1, a.warmup))
    ge.set_state(c.q0)
    torch.cuda.synchronize()
    n_exp = 0
    e0.record(stream_e)
    while ge.time()[0] < t_sim and n_exp < 100000:
        ge.step(10)
        n_exp += 10
    e1.record(stream_e)
    torch.cuda.synchronize()
    exp_ms = e0.elapsed_time(e1)
    clocks = clk.stop()
    t = torch.tensor([imp_ms, exp_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    imp_ms, exp_ms = (float(x) for x in t.tolist())
    line = {"metric": METRIC, "value": C * a.steps * world / (imp_ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": imp_ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "fully implicit strategy (BDF2, Newton with matrix-free Jacobian, GMRES(30) "
                                   "with block-Jacobi preconditioner) on the level-2 case, jittered-Delaunay %dx%d "
                                   "grid (%d cells), order 1, CFL %.2f; against the splitting step at CFL 0.45"
                                   % (a.imp_side, a.imp_side, C, a.imp_cfl),
                       "model": c.model, "cells": C, "parallelism": "replicas x%d" % world if world > 1
                       else "single GPU",
                       "timing": "CUDA events around the host-driven implicit steps (the GMRES inner products "
                                 "synchronise) and around the explicit graph steps",
                       "l2_flush": "none: the timed work is the whole solve"},
            "implicit": {"simulated_time": t_sim, "newton_per_step": float(np.mean(newton)),
                         "gmres_per_step": float(np.mean(gmres)),
                         "simulated_time_per_device_second": t_sim / (imp_ms / 1e3),
                         "explicit_steps_same_time": n_exp, "explicit_ms": exp_ms,
                         "explicit_simulated_time_per_device_second": ge.time()[0] / (exp_ms / 1e3)},
            "e2e": None, "gpu_launches": None, "clocks": clocks}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def run_adjoint(a, dev, torch, dist, rank, world):
    """SME level 1 on the 200x200 jittered grid, 400 steps; misfit of the depth
    at 64 seeded gauge cells every 10th step against a run whose bathymetry
    is raised by 0.02 exp(-|x - (0.6, 0.4)|^2 / 0.01); gradients with respect
    to the per-cell bathymetry and the Manning coefficient, checkpoints every
    20 steps.  Times the forward run and the adjoint call, and checks the
    gradient against central differences (eps = 1e-6) of the forward run at the
    recorded dts along 32 seeded smooth directions and the Manning direction.
    Each rank runs its own replica."""
    from zoomy_dmplex_b200 import adjoint as adj
    from zoomy_dmplex_b200 import cases, models
    from zoomy_dmplex_b200.solver import Solver

    def barrier():
        if dist:
            dist.barrier()

    side, N, every, ngauge = a.adj_side, a.adj_steps, 20, 64
    c = cases.adjoint_l1(side)
    tgt = cases.adjoint_l1(side, target=True)
    c.settings.limiter = tgt.settings.limiter = a.adj_limiter
    p = params_of(c)
    names, _ = models.parameter_table(c.model)
    C, F = c.mesh.n_cells, c.mesh.n_faces
    g = Solver(c.model, c.mesh, c.settings, p, device=dev)
    tuned = None
    if not a.no_tune:   # the forward's launch configuration (the replay runs the same kernels)
        from zoomy_dmplex_b200 import autotune

        g.set_state(c.q0)
        # ten timed steps per trial: at 79k cells a step is about 0.1 ms, and two
        # left the choice to timing noise
        tuned = autotune.tune(g, c.model, C, steps=10, use_cache=False, write_cache=False)
    cells = adj.gauges(C, ngauge, seed=0)
    steps = list(range(10, N + 1, 10))
    targets = adj.observe_run(g, tgt.q0, N, steps, cells)
    obs = adj.depth_observations(cells, steps, targets)
    stream = torch.cuda.ExternalStream(g.stream, device=dev)
    # warm-up: forward graph, one adjoint call (allocations)
    g.set_state(c.q0)
    g.step(max(1, a.warmup))
    g.set_state(c.q0)
    g.adjoint(N, *obs, checkpoint_every=every)
    # forward: N steps on the graph path
    g.set_state(c.q0)
    clk = ClockSampler(dev)
    clk.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(N)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    # the adjoint call (it synchronises): host wall clock
    g.set_state(c.q0)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    loss, gq, gp, dts = g.adjoint(N, *obs, checkpoint_every=every)
    adj_s = time.perf_counter() - w0
    phases = g.adjoint_phases()
    overlapped = g.adjoint_overlapped()
    # end to end: initial state from the host, adjoint, gradients back
    w0 = time.perf_counter()
    g.set_state(c.q0)
    g.adjoint(N, *obs, checkpoint_every=every)
    e2e_s = time.perf_counter() - w0
    clocks = clk.stop()
    barrier()

    # central differences of the forward run at the recorded dts
    def misfit(q0, pp):
        g.set_params(pp)
        v = adj.observe_run(g, q0, N, steps, cells, dts=dts)
        return float(np.sum((v - targets) ** 2))

    rng = np.random.default_rng(2024)
    eps = 1e-6
    errs, pairs = [], []
    for _ in range(a.adj_fd):
        dq = np.zeros_like(c.q0)
        dq[:, 0] = adj.smooth_direction(c.mesh, rng) * 1e-2
        fd = (misfit(c.q0 + eps * dq, p) - misfit(c.q0 - eps * dq, p)) / (2 * eps)
        ad = float(np.sum(gq * dq))
        errs.append(abs(ad - fd) / max(abs(fd), 1e-300))
        pairs.append((ad, fd))
    ni = names.index("n_manning")
    dp = np.zeros_like(p)
    dp[ni] = 1.0
    fd_n = float("nan")
    if a.adj_fd > 0:
        fd_n = (misfit(c.q0, p + eps * dp) - misfit(c.q0, p - eps * dp)) / (2 * eps)
        g.set_params(p)
    man_err = abs(gp[ni] - fd_n) / max(abs(fd_n), 1e-300)

    t = torch.tensor([fwd_ms, adj_s, e2e_s], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    fwd_ms, adj_s, e2e_s = (float(x) for x in t.tolist())
    s = c.settings.ssp_stages
    lps = g.launches_per_step()
    # per reverse step: finalize; per stage face VJP, cell, combine; the clamps of
    # the stages after the first (odd s adds axpby, copy and seed kernels)
    rev_launches = 1 + 3 * s + (s - 1) + (3 if s % 2 else 0)
    nv = C * g.nq * 8
    line = {"metric": METRIC, "value": C * N * world / adj_s, "unit": UNIT, "n_gpus": world, "steps": N,
            "warmup": a.warmup, "ms_per_step": 1e3 * adj_s / N, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "discrete adjoint of SME level 1 on the jittered-Delaunay %dx%d grid (%d cells, "
                                   "%d faces), %d steps, depth misfit at %d gauge cells every 10th step, gradients "
                                   "w.r.t. per-cell b and Manning n, checkpoints every %d steps, order 2 Green-Gauss "
                                   "+ limiter %s, SSP-RK2, CFL 0.45" % (side, side, C, F, N, ngauge, every,
                                                                        "Vacuum/TVD" if a.adj_limiter == "tvd" else
                                                                        "none"),
                       "model": c.model, "cells": C, "faces": F, "parallelism": "replicas x%d" % world if world > 1
                       else "single GPU",
                       "l2_flush": "not needed for the ratio: both runs see the same cache state",
                       "timing": "forward: CUDA events around N graph-launched steps; adjoint: host wall clock "
                                 "around the (synchronising) zsme_adjoint call, forward pass with checkpoints, "
                                 "segment replays and reverse sweep included",
                       "launch": tuned or "default"},
            "adjoint": {"forward_ms_per_step": fwd_ms / N, "adjoint_call_ms_per_step": 1e3 * adj_s / N,
                        "adjoint_call_over_forward": 1e3 * adj_s / fwd_ms,
                        "phases_ms_per_step": {k: v / N for k, v in phases.items()},
                        "reverse_step_over_forward_step": phases["reverse"] / fwd_ms,
                        "replay_plus_reverse_over_forward": (phases["replay"] + phases["reverse"]) / fwd_ms,
                        "replays_overlap_reverse": overlapped,
                        "phases_note": ("replays on a side stream into a second tape buffer, overlapping the "
                                        "reverse sweep: 'replay' is the first (exposed) replay, 'reverse' the rest "
                                        "of the reverse phase" if overlapped else
                                        "replay and reverse sweep in sequence per segment"),
                        "loss": loss, "grad_n_manning": float(gp[ni]), "grad_b_norm": float(np.linalg.norm(gq[:, 0])),
                        "fd": {"directions": len(errs), "eps": eps, "kind": "smooth random b directions",
                               "max_rel_err": float(max(errs)) if errs else None,
                               "median_rel_err": float(np.median(errs)) if errs else None,
                               "manning_rel_err": float(man_err), "first_pairs_adjoint_fd": pairs[:4],
                               "manning_adjoint_fd": [float(gp[ni]), fd_n]}},
            "e2e": {"value": C * N * world / e2e_s, "unit": UNIT, "h2d_bytes_per_step": nv / N,
                    "d2h_bytes_per_step": nv / N,
                    "api": "zsme_set_state(host) + zsme_adjoint (host observations in, host gradients out)"},
            "gpu_launches": N * (2 * lps + rev_launches) + 2 * len(steps) + 1,
            "clocks": clocks}
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if a.impl == "reference":
        if rank != 0:
            return 0
        from zoomy_dmplex_b200 import cases

        # the GPU arm's own workload (same mesh, model, settings); warm-up and
        # timed steps of the oracle, the timed loop bounded to --ref-seconds
        side = a.side or CASE_SIDE[a.case]
        built = getattr(cases, a.case)(side)
        warm = max(1, min(a.warmup, 2))
        v, nt, C, dt, n = cpu_sample(side, max(1, a.steps), warm=warm, positivity=a.positivity, built=built,
                                     max_seconds=a.ref_seconds)
        line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": a.gpus,
                "steps": n, "warmup": warm, "ms_per_step": 1e3 * dt / n,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": "%s, jittered-Delaunay %dx%d grid (%d cells, %d faces), Hilbert-renumbered, "
                                       "%s, SSP-RK2, CFL 0.45, %s%s"
                                       % (CASE_TEXT[a.case][0], side, side, C, built.mesh.n_faces,
                                          GRAD_TEXT[built.settings.gradient], CASE_TEXT[a.case][1],
                                          POS_TEXT[a.positivity]),
                           "model": built.model, "cells": C, "parallelism": "host threads",
                           "same_config_as_gpu_arm": True},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": nt, "kind": "port",
                                 "sample": "%d timed steps (after %d warm-up) of the CPU restatement (oracle) on the "
                                           "GPU arm's own %dx%d-grid mesh (%d cells), %.1f s; requested %d steps, "
                                           "bounded to %.0f s" % (n, warm, side, side, C, dt, a.steps,
                                                                 a.ref_seconds)},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist_mod

        dist = dist_mod
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local
    torch.cuda.set_device(dev)

    from zoomy_dmplex_b200 import cases, native
    from zoomy_dmplex_b200.solver import Solver

    if a.workload == "ensemble":
        return run_ensemble(a, dev, torch, dist, rank, world)
    if a.workload == "implicit":
        return run_implicit(a, dev, torch, dist, rank, world)
    if a.workload == "adjoint":
        return run_adjoint(a, dev, torch, dist, rank, world)

    side = a.side or CASE_SIDE[a.case]
    case = getattr(cases, a.case)(side)
    case.settings.positivity = a.positivity
    tune_trace = None
    C, F = case.mesh.n_cells, case.mesh.n_faces
    g = Solver(case.model, case.mesh, case.settings, params_of(case), device=dev)
    g.set_state(case.q0)
    tuned = None
    if a.launch:
        from zoomy_dmplex_b200.solver import set_launch

        tuned = json.loads(a.launch)
        set_launch(g.h, tuned)
    elif not a.no_tune:
        from zoomy_dmplex_b200 import autotune

        tuned = autotune.tune(g, case.model, case.mesh.n_cells, steps=2, use_cache=False, write_cache=False)
        tune_trace = autotune.last_trace
        g.set_state(case.q0)          # tuning advanced the state: start again from the initial condition
    nq, na = g.nq, g.naux
    stream = torch.cuda.ExternalStream(g.stream, device=dev)

    def barrier():
        if dist:
            dist.barrier()

    # warm-up on the graph path
    g.step(a.warmup)
    g.sync()

    clk = ClockSampler(dev)
    clk.start()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    g.step(a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    diag = g.sync(check=True)
    # per-kernel durations: a second pass of K steps with one event pair per launch
    g.set_profiling(True)
    g.step(a.steps)
    g.sync()
    prof = g.read_profile()
    g.set_profiling(False)
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = C * a.steps * world / (ms_max / 1e3)

    # roofline of the dominant kernel (algorithmic bytes / live average duration)
    hbm, peak_src = peaks()
    from zoomy_dmplex_b200.solver import get_launch

    launch_cfg = get_launch(g.h)
    fused = launch_cfg["tile_faces"] > 0
    dom = max((k for k in prof if prof[k][1] > 0), key=lambda k: prof[k][0])
    dom_ms = prof[dom][0] / prof[dom][1]
    alg = algorithmic_bytes(dom, C, F, nq, na, case.mesh.max_faces, case.settings.ssp_stages, fused)
    achieved = alg / (dom_ms / 1e3) / 1e9
    same_cfg = all(launch_cfg.get(k) == v for k, v in NCU_LAUNCH.items())
    traffic = NCU_DRAM_BYTES_PER_CELL.get("%s/%s" % (case.model, dom)) \
        if a.positivity == "none" and same_cfg else None
    tps = traffic_per_cell_step(case.model, launch_cfg, case.settings.ssp_stages) if a.positivity == "none" else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                "frac": achieved / hbm, "peak_source": peak_src,
                "algorithmic_bytes_per_launch": alg,
                "traffic": traffic * C if traffic else None,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per cell on the 900x900 grid, "
                                  "scaled to this launch's cells" if traffic else None,
                "traffic_per_cell_step": tps,
                "algorithmic_bytes_per_cell_step": step_bytes_fused(nq),
                "kernel_ms": dom_ms}
    step_ms = ms_max / a.steps
    sb = step_bytes_fused(nq)
    roofline_step = {"bytes_per_cell_step": sb, "achieved": sb * C / (step_ms / 1e3) / 1e9, "peak": hbm,
                     "unit": "GB/s", "frac": sb * C / (step_ms / 1e3) / 1e9 / hbm}
    kernel_share = {k: {"ms_per_launch": v[0] / v[1], "launches": v[1], "share": v[0] / max(1e-30, sum(
        x[0] for x in prof.values()))} for k, v in prof.items() if v[1]}

    # FP64 roofline: the step does ~10 algorithmic flops per algorithmic byte,
    # above the FP64 ridge, so its kernels are also held against the measured
    # FP64 rate (FMA chains, 2 flops per FMA).  The kernels compile without
    # FMA contraction (bit-identical rounding), one add or multiply per
    # instruction: half that rate is their ceiling ("unfused").
    roofline_fp64 = None
    fp64_step = None
    if case.model in FP64_FLOPS and a.positivity == "none":
        pk = ctypes.c_double()
        native.check(native.load().zsme_fp64_fma_peak(dev, ctypes.byref(pk)))
        peak_tf = pk.value
        s_ = case.settings.ssp_stages
        for k, v in kernel_share.items():
            fl = fp64_flops(k, case.model, C, F, s_, fused)
            if fl is not None:
                v["fp64_tflops"] = fl / (v["ms_per_launch"] / 1e3) / 1e12
        fk = max((k for k in kernel_share if "fp64_tflops" in kernel_share[k]),
                 key=lambda k: kernel_share[k]["fp64_tflops"])
        fl = fp64_flops(fk, case.model, C, F, s_, fused)
        ach = kernel_share[fk]["fp64_tflops"]
        roofline_fp64 = {"bound": "fp64", "kernel": fk, "achieved": ach, "peak": peak_tf, "unit": "TFLOP/s",
                         "frac": ach / peak_tf, "frac_of_unfused": ach / (peak_tf / 2),
                         "flops_per_launch": fl,
                         "peak_source": "measured on this GPU: zsme_fp64_fma_peak (FMA chains, 2 flops per FMA)"}
        fc = fp64_flops_per_cell_step(case.model, C, F, s_)
        ach_s = fc * C / (step_ms / 1e3) / 1e12
        fp64_step = {"flops_per_cell_step": fc, "flop_per_byte": fc / sb, "achieved": ach_s, "peak": peak_tf,
                     "unit": "TFLOP/s", "frac": ach_s / peak_tf, "frac_of_unfused": ach_s / (peak_tf / 2)}

    # the other gradient of the same workload (least squares where the case
    # runs Green-Gauss, and the reverse), same launch configuration
    variants = {}
    if a.lsq_steps > 0 and a.positivity == "none":
        import dataclasses

        from zoomy_dmplex_b200.solver import set_launch

        other = "least_squares" if case.settings.gradient == "green_gauss" else "green_gauss"
        g2 = Solver(case.model, case.mesh, dataclasses.replace(case.settings, gradient=other), params_of(case),
                    device=dev)
        if tuned:
            set_launch(g2.h, tuned)
        g2.set_state(case.q0)
        g2.step(2)
        g2.sync()
        s2 = torch.cuda.ExternalStream(g2.stream, device=dev)
        barrier()
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(s2)
        g2.step(a.lsq_steps)
        f1.record(s2)
        torch.cuda.synchronize()
        d2 = g2.sync(check=False)
        t4 = torch.tensor([f0.elapsed_time(f1)], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(t4, op=dist.ReduceOp.MAX)
        ms2 = float(t4.item()) / a.lsq_steps
        variants[other] = {"ms_per_step": ms2, "value": C * world / (ms2 / 1e3), "unit": UNIT,
                           "steps": a.lsq_steps, "gradient": GRAD_TEXT[other],
                           "timing": "CUDA events around graph-launched steps after 2 warm-up steps",
                           "diag": {"nonfinite": d2.n_nonfinite, "negative_depth": d2.n_negative_depth}}
        g2.close()

    # end to end through the public API: pinned host state in, one step, state out
    ne = a.e2e_steps or a.steps
    q_host = torch.from_numpy(np.ascontiguousarray(case.q0)).pin_memory()
    out_host = torch.empty_like(q_host).pin_memory()
    lib = native.load()
    import ctypes as ct

    qp = ct.cast(q_host.data_ptr(), ct.POINTER(ct.c_double))
    op = ct.cast(out_host.data_ptr(), ct.POINTER(ct.c_double))
    native.check(lib.zsme_set_state(g.h, qp, 0.0))
    g.step(1)
    native.check(lib.zsme_get_state(g.h, op))
    barrier()
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(ne):
        native.check(lib.zsme_set_state(g.h, qp, 0.0))
        native.check(lib.zsme_step(g.h, 1))
        native.check(lib.zsme_get_state(g.h, op))
    e3.record(stream)
    torch.cuda.synchronize()
    barrier()
    t2 = torch.tensor([e2.elapsed_time(e3)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    blocking_value = C * ne * world / (float(t2.item()) / 1e3)
    ref_out = out_host.numpy().copy()
    nbytes = C * nq * 8

    # the same, pipelined through the asynchronous state calls: the read-back
    # of one problem, the upload of the next and its step overlap (two output
    # buffers in turn; the copies run on the handle's two copy streams)
    outs = [torch.empty_like(q_host).pin_memory() for _ in range(2)]
    ops = [ct.cast(o.data_ptr(), ct.POINTER(ct.c_double)) for o in outs]
    native.check(lib.zsme_set_state_async(g.h, qp, 0.0))       # allocates the staging buffers
    native.check(lib.zsme_step(g.h, 1))
    native.check(lib.zsme_get_state_async(g.h, ops[0]))
    native.check(lib.zsme_sync(g.h))
    barrier()
    torch.cuda.synchronize()
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    for k in range(ne):
        native.check(lib.zsme_set_state_async(g.h, qp, 0.0))
        native.check(lib.zsme_step(g.h, 1))
        native.check(lib.zsme_get_state_async(g.h, ops[k % 2]))
    native.check(lib.zsme_stream_wait_copies(g.h))
    e5.record(stream)
    torch.cuda.synchronize()
    native.check(lib.zsme_sync(g.h))
    barrier()
    t3 = torch.tensor([e4.elapsed_time(e5)], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t3, op=dist.ReduceOp.MAX)
    e2e_value = C * ne * world / (float(t3.item()) / 1e3)
    same = all(np.array_equal(o.numpy(), ref_out) for o in outs[:min(ne, 2)])   # the buffers the loop wrote

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "%s, jittered-Delaunay %dx%d grid (%d cells, %d faces), "
                                   "Hilbert-renumbered, %s, SSP-RK2, CFL 0.45, "
                                   "%s%s" % (CASE_TEXT[a.case][0], side, side, C, F,
                                             GRAD_TEXT[case.settings.gradient], CASE_TEXT[a.case][1],
                                             POS_TEXT[a.positivity]),
                       "model": case.model, "cells": C, "faces": F, "n_dof_q": nq, "positivity": a.positivity,
                       "parallelism": "replicas x%d" % world if world > 1 else "single GPU",
                       "l2_flush": ("not needed: state %.0f MB + face states %.0f MB > 126 MB L2"
                                    % (C * nq * 8 / 1e6, C * nq * 3 * 8 / 1e6)) if C * nq * 32 > 126e6 else
                                   ("not flushed: state %.1f MB and face states fit in L2 (a latency-bound size)"
                                    % (C * nq * 8 / 1e6)),
                       "timing": "CUDA events on the solver stream around K graph-launched steps; "
                                 "per-kernel events in a second, profiled pass of K steps",
                       "launch": launch_cfg, "tuning_trace": tune_trace},
            "roofline": roofline, "roofline_step": roofline_step, "roofline_fp64": roofline_fp64,
            "variants": variants,
            "fp64_step": fp64_step, "kernels": kernel_share,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "steps": ne,
                    "api": "per step: zsme_set_state_async(pinned host) + zsme_step(1) + "
                           "zsme_get_state_async(pinned host), pipelined; CUDA events around the loop and "
                           "zsme_stream_wait_copies",
                    "blocking_value": blocking_value,
                    "blocking_api": "zsme_set_state(pinned host) + zsme_step(1) + zsme_get_state(pinned host)",
                    "outputs_match_blocking": same},
            "gpu_launches": a.steps * g.launches_per_step(),
            "diag": {"nonfinite": diag.n_nonfinite, "negative_depth": diag.n_negative_depth,
                     "newton_unconverged": diag.n_newton_unconverged, "mood_cells": diag.n_mood_cells,
                     "newton_deferred_cells": diag.n_newton_deferred},
            "clocks": clocks}
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        v, nt, Cs, dts, ns = cpu_sample(side, seconds=a.cpu_seconds, positivity=a.positivity, built=case)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nt, "kind": "port",
                                "sample": "%d steps of the CPU restatement (oracle) on the same %dx%d-grid mesh "
                                          "(%d cells), state and settings, %.1f s" % (ns, side, side, Cs, dts)}
    if rank == 0:
        print(json.dumps(line))
    g.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""Benchmark of the gell_b200 hot path on the large plain-method workload.

Workload: 400^3 voxels of 10 um, two FP32 substrates (oxygen: boundary 38, D 1e5, decay 0.1,
uptake 10/min; drug: boundary 1, D 5e4, decay 0.05, uptake 1/min), 10^6 cells on a seeded
jittered lattice spheroid (radius ~590 um, radii N(5, 0.5) um clipped to [4, 6]).  One step is one
mechanics step as the reference host loop runs it: FM_update, PreLOD, then 10 LOD substeps of
both substrates.

  value      cell-updates/s of whole steps (live cells x steps / device time of the steps)
  components cell-updates/s of FM_update + PreLOD alone, voxel-updates/s of the LOD substeps
             (voxels x substrates x substeps / LOD device time)
  e2e        the same rate through the C ABI with host buffers: every step imports the cells
             from pinned host memory and exports them back, copies inside the timed region; the
             copies are the ABI's queued transfers, which overlap the LOD substeps
  roofline   the kernel with the largest device time in the timed region, against HBM

`--impl reference` times the reference's own CUDA build on the same GPU: its kernels and facades
compiled from its unmodified sources (oracle/_ref), whole steps of the same workload, with the
same e2e contract.  `cpu_baseline` times the reference's kernel bodies compiled for the host with
OpenMP (oracle/_ref/libgellref_host_*), two whole steps on the host cores.

Multi-GPU: every rank runs its own replica (the path has no exchange step); value = cells of all
ranks / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-updates/s + voxel-updates/s @1M cells/400³; surrogate vs plain LOD @≤1% err"
N, LENGTH, NCELLS, SUBSTEPS, CAP = 400, 10.0, 1_000_000, 10, 2_000_000
NSUB = 2
WORKLOAD = ("plain method, large: 400^3 voxels at 10 um, oxygen + drug (FP32), 10^6 cells, "
            "1 mechanics step = FM_update + PreLOD + 10 LOD substeps")
# algorithmic bytes per voxel-update of each sweep: read p once and write it once (8 B).  The
# uptake source (read rate) runs before the x sweep in k_source_lines, on the x-lines that hold
# cells only, so the x sweep itself moves no rate bytes.
ALGO_BYTES = {"k_sweep_x": 8.0, "k_sweep_y": 8.0, "k_sweep_z": 8.0}
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = "k_sweep_400cube_2sub.md"


def config(extra=None):
    c = {"workload": WORKLOAD, "voxels": N ** 3, "substrates": NSUB, "cells": NCELLS,
         "substeps_per_step": SUBSTEPS, "voxel_um": LENGTH,
         "l2": "inputs larger than L2: each field is 256 MB, 2 fields + 2 uptake maps",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


def make_cells():
    from gell_b200.cells import lattice_spheroid
    return lattice_spheroid(NCELLS, N * LENGTH / 2, 0, LENGTH, N)


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel):
    """DRAM bytes (read + write) of one launch of `kernel` at this workload, from the committed ncu
    summary (lines `traffic <kernel>: <bytes>`), or None when no capture is recorded."""
    path = os.path.join(ROOT, "profiles", PROFILE_SUMMARY)
    try:
        for line in open(path):
            if line.startswith(f"traffic {kernel}:"):
                return int(line.split(":", 1)[1].split()[0]), f"profiles/{PROFILE_SUMMARY}"
    except OSError:
        pass
    return None, None


# ---------------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons while the work runs."""

    FIELDS = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid: str | None):
        self.uuid = uuid
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 10:
                continue
            if self.uuid and p[1] != self.uuid:
                continue
            rows.append(p)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        mx = [float(r[3]) for r in rows if r[3].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[6 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[4]) for r in rows if r[4].replace(".", "").isdigit())
                if any(r[4].replace(".", "").isdigit() for r in rows) else None}


# ---------------------------------------------------------------------------- GPU arm

def reduce_over_ranks(times, cells, device):
    """Replicas: device times take the max over ranks, processed cells the sum."""
    import torch
    import torch.distributed as td
    tt = torch.tensor(np.asarray(times, np.float64), device=device)
    td.all_reduce(tt, op=td.ReduceOp.MAX)
    cc = torch.tensor(np.asarray(cells, np.float64), device=device)
    td.all_reduce(cc, op=td.ReduceOp.SUM)
    return tt.cpu().numpy(), cc.cpu().numpy()


def run_gell(args, rank, world, local_rank):
    import torch
    import gell_b200 as gb

    torch.cuda.set_device(local_rank)
    dist = world > 1
    if dist:
        import torch.distributed as td
    cells = make_cells()
    sim = gb.Simulation(voxel_num=N, voxel_length=LENGTH, max_cell_num=CAP)
    sim.add_substrate(gb.oxygen())
    sim.add_substrate(gb.drug())
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    sim.import_cells(cells)
    ncell = sim.count()

    def step():
        sim.FM_update()
        sim.PreLOD()
        sim.LODsolver(SUBSTEPS)

    # warm-up through the driver the timed region uses: its calls capture the step graphs (one per
    # double-buffer assignment; the final two-step call leaves the one the timed region starts on)
    sim.run_mechanics(args.warmup - 2, SUBSTEPS)
    sim.run_mechanics(2, SUBSTEPS)
    sim.sync()

    props = torch.cuda.get_device_properties(local_rank)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else uuid
    sampler = ClockSampler(str(uuid) if uuid else None)
    sampler.start()
    time.sleep(0.3)

    # timed region: K whole steps through gell_run_mechanics (pairs replayed from a CUDA graph)
    K = args.steps
    t0e, t1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = sim.launch_count()
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    t0e.record(stream)
    sim.run_mechanics(K, SUBSTEPS)
    t1e.record(stream)
    torch.cuda.synchronize()
    if dist:
        td.barrier()
    launches = sim.launch_count() - launches0
    sampler.stop()
    t_all = t0e.elapsed_time(t1e)

    # breakdown: the same steps launched one call at a time, with events between the phases
    kc = max(1, min(K, 20))
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(kc)]
    torch.cuda.synchronize()
    for k in range(kc):
        ev[k][0].record(stream)
        sim.FM_update()
        ev[k][1].record(stream)
        sim.PreLOD()
        ev[k][2].record(stream)
        sim.LODsolver(SUBSTEPS)
        ev[k][3].record(stream)
    torch.cuda.synchronize()
    t_fm = sum(ev[k][0].elapsed_time(ev[k][1]) for k in range(kc)) * K / kc
    t_pre = sum(ev[k][1].elapsed_time(ev[k][2]) for k in range(kc)) * K / kc
    t_lod = sum(ev[k][2].elapsed_time(ev[k][3]) for k in range(kc)) * K / kc

    # per-kernel device times: a separate pass with an event pair around every launch, on the
    # stream the kernels run on, so the timed region above carries no profiling events
    kp = max(1, min(K, 10))
    sim.profile(True)
    sim.profile_read(reset=True)
    for _ in range(kp):
        step()
    sim.sync()
    prof = sim.profile_read(reset=True)
    sim.profile(False)

    alive = int(sim.export_cells()["sign"].sum())

    # e2e: the same steps through the C ABI with host buffers
    import torch as _t
    host = _t.empty(ncell * 72, dtype=_t.uint8, pin_memory=True).numpy().view(gb.CELL_DTYPE)
    host[:] = sim.export_cells()
    ke = max(1, min(K, 20))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        td.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(ke):
        # the step's cells in from pinned host memory and its result out: queued transfers that
        # overlap the LOD substeps (which do not use the cells)
        sim.import_cells_async(host)
        step()
        sim.export_cells_async(host)
    sim.wait_transfers()
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1)

    times = np.array([t_all, t_fm + t_pre, t_lod, t_e2e], np.float64)
    cells_all = np.array([alive * K, alive * ke], np.float64)
    if dist:
        times, cells_all = reduce_over_ranks(times, cells_all, "cuda")
    t_all, t_mech, t_lod, t_e2e = times
    value = cells_all[0] / (t_all / 1e3)
    mech_rate = cells_all[0] / (t_mech / 1e3)
    vox_rate = world * N ** 3 * NSUB * SUBSTEPS * K / (t_lod / 1e3)
    e2e_rate = cells_all[1] / (t_e2e / 1e3)

    # roofline of the kernel with the largest device time
    top = max(prof.items(), key=lambda kv: kv[1][1])
    name, (nl, ms) = top
    avg_ms = ms / nl
    peak, peak_kind = hbm_peak()
    algo = ALGO_BYTES.get(name)
    traffic, traffic_src = ncu_traffic(name)
    roof = {"kernel": name, "bound": "hbm", "launches": nl, "avg_ms": avg_ms, "peak": peak,
            "peak_source": f"{peak_kind} hbm_gbs", "unit": "GB/s", "traffic": traffic,
            "traffic_source": traffic_src}
    if algo is not None:
        per_launch = algo * N ** 3 * NSUB
        roof.update(achieved=per_launch / (avg_ms / 1e3) / 1e9, bytes_per_launch=per_launch,
                    bytes_per_unit=algo, unit_name="voxel-update")
        roof["frac"] = roof["achieved"] / peak
    shares = {k: {"launches": v[0], "ms": round(v[1], 4), "share": round(v[1] / sum(x[1] for x in prof.values()), 4)}
              for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}

    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": t_all / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded jittered-lattice spheroid of 10^6 cells, fields start at the boundary values",
            "config": config(),
            "components": {"cell_updates_per_s_fm_prelod": mech_rate, "voxel_updates_per_s_lod": vox_rate,
                           "ms_fm_update": t_fm / K, "ms_prelod": t_pre / K, "ms_lod_10_substeps": t_lod / K},
            "roofline": roof,
            "kernels": shares,
            "e2e": {"value": e2e_rate, "unit": "cell-updates/s", "steps": ke,
                    "h2d_bytes_per_step": int(ncell * 72), "d2h_bytes_per_step": int(ncell * 72)},
            "gpu_launches": int(launches),
            "clocks": sampler.summary(),
        }
    sim.close()
    return line


# ---------------------------------------------------------------------------- birth/death workload

C3_N, C3_CELLS, C3_CAP, C3_BIO = 600, 5_000_000, 10_000_000, 60
C3_WORKLOAD = ("plain method with stochastic birth/death: 600^3 voxels at 10 um, oxygen + drug (FP32), "
               "5*10^6 cells, Philox draws; every 60 mechanics steps (one 6-min biology step) birth "
               "before and death after, as the reference loop runs them")


def run_c3(args, rank, world, local_rank):
    """--workload c3: K mechanics steps in biology periods of 60 (birth, 60 steps, death)."""
    import torch
    import gell_b200 as gb

    torch.cuda.set_device(local_rank)
    length = LENGTH
    cells = gb.lattice_spheroid(C3_CELLS, C3_N * length / 2, 3, length, C3_N)
    gb.seed_ki67_states(cells, 11)
    sim = gb.Simulation(voxel_num=C3_N, voxel_length=length, max_cell_num=C3_CAP, rng_mode=gb.GELL_RNG_PHILOX,
                        seed=20260101)
    sim.add_substrate(gb.oxygen())
    sim.add_substrate(gb.drug())
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    sim.import_cells(cells)
    sim.run_mechanics(args.warmup, SUBSTEPS)
    sim.sync()
    n0 = sim.count()

    props = torch.cuda.get_device_properties(local_rank)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else uuid
    sampler = ClockSampler(str(uuid) if uuid else None)
    sampler.start()
    time.sleep(0.3)
    K = args.steps
    ev = []
    cell_steps = 0
    births = deaths = 0
    t_bio = 0.0
    if world > 1:
        import torch.distributed as td
        td.barrier()
    torch.cuda.synchronize()
    e_start = torch.cuda.Event(enable_timing=True)
    e_start.record(stream)
    done = 0
    while done < K:
        m = min(C3_BIO, K - done)
        a, b, c2, d = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        a.record(stream)
        nb = sim.CellBirth_kernel()
        b.record(stream)
        sim.run_mechanics(m, SUBSTEPS)
        c2.record(stream)
        nd = sim.CellDeath_kernel()
        d.record(stream)
        ev.append((a, b, c2, d))
        births += nb - (n0 if done == 0 else last)
        deaths += nb - nd
        cell_steps += nb * m
        last = nd
        done += m
    e_end = torch.cuda.Event(enable_timing=True)
    e_end.record(stream)
    torch.cuda.synchronize()
    sampler.stop()
    t_all = e_start.elapsed_time(e_end)
    for a, b, c2, d in ev:
        t_bio += a.elapsed_time(b) + c2.elapsed_time(d)
    times = np.array([t_all, t_bio], np.float64)
    cnt = np.array([cell_steps], np.float64)
    if world > 1:
        times, cnt = reduce_over_ranks(times, cnt, "cuda")
    t_all, t_bio = times
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": cnt[0] / (t_all / 1e3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": t_all / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded jittered-lattice spheroid of 5*10^6 cells (radius ~1 mm) with seeded Ki-67 "
                    "phases and clocks, fields start at the boundary values",
            "config": {"workload": C3_WORKLOAD, "voxels": C3_N ** 3, "substrates": 2, "cells": C3_CELLS,
                       "substeps_per_step": SUBSTEPS, "voxel_um": length, "biology_period_steps": C3_BIO,
                       "l2": "inputs larger than L2: each field is 864 MB", "parallelism": "replicas",
                       "cells_per_step": "array slots after the period's birth (cells dead since then included)"},
            "components": {"ms_birth_plus_death_per_period": t_bio / max(len(ev), 1),
                           "births": int(births), "removed": int(deaths), "cells_end": int(last)},
            "gpu_launches": None, "clocks": sampler.summary(),
        }
    sim.close()
    return line


# ---------------------------------------------------------------------------- ensemble workload

C4_MEMBERS, C4_BIO = 64, 60
C4_WORKLOAD = ("batched ensemble: 64 independent instances, grid edge log-uniform in [64, 200] voxels of 10 um, "
               "cells log-uniform in [2,000, 200,000], D U(5e4, 2e5), uptake U(5, 20)/min (seed 7), one FP32 "
               "substrate each, Philox birth/death; one graph of parallel branches (LOD per member or batched "
               "over all members), tuned")


def c4_members(gb, stream):
    rng = np.random.Generator(np.random.Philox(7))
    edges = np.floor(np.exp(rng.uniform(np.log(64), np.log(200), C4_MEMBERS))).astype(int)
    cells = np.floor(np.exp(rng.uniform(np.log(2e3), np.log(2e5), C4_MEMBERS))).astype(int)
    D = rng.uniform(5e4, 2e5, C4_MEMBERS)
    up = rng.uniform(5.0, 20.0, C4_MEMBERS)
    sims = []
    for i in range(C4_MEMBERS):
        N = int(edges[i])
        # at most 35% of the domain's volume packed at 0.6, so the spheroid (radius 0.44 of the
        # edge) stays inside the grid
        n = int(min(cells[i], 0.35 * (N * LENGTH) ** 3 / 873.0))
        sim = gb.Simulation(voxel_num=N, voxel_length=LENGTH, max_cell_num=2 * n + 1024,
                            rng_mode=gb.GELL_RNG_PHILOX, seed=1000 + i)
        sim.add_substrate(gb.Substrate(38.0, float(D[i]), 0.1, -float(up[i]), 38.0))
        c = gb.lattice_spheroid(n, N * LENGTH / 2, i, LENGTH, N)
        gb.seed_ki67_states(c, 2000 + i)
        sim.import_cells(c)
        sim.set_stream(stream)
        sims.append(sim)
    return sims, edges


# ---------------------------------------------------------------------------- surrogate workload

C5_N, C5_CELLS, C5_WARM = 256, 300_000, 1000
C5_WORKLOAD = ("learned surrogate (pattern 4): 256^3 grid of 10 um, oxygen, 300,000 cells (seeded jittered-lattice "
               "spheroid with the large workload's statistics and seeded Ki-67 states); one block = FM_update + PreLOD "
               "+ K = 50 LOD substeps, the substeps either plain or replaced by the judged 3-D conv operator "
               "(4 residual blocks, 32 channels, 3^3 kernels, bf16 operands, fp32 sums) from the same state")
C5_WEIGHTS = os.path.join(ROOT, "gell_b200", "data", "o2_surrogate_256.gsur")


def bf16_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"]), "measured bf16_tflops (cuBLAS burst)"
    except Exception:
        return 1590.0, "fallback"


def run_c5(args, rank, world, local_rank):
    """--workload c5: blocks of a quasi-steady spheroid; per block the same state is advanced by the
    plain solver and by the judged surrogate, each timed with CUDA events on the context's stream;
    the simulation continues from the judged result, as a surrogate-driven run would."""
    import torch
    import gell_b200 as gb
    from gell_b200 import surrogate as gs

    torch.cuda.set_device(local_rank)
    sw = gs.load_weights(args.surrogate_weights or C5_WEIGHTS)
    K = sw.substeps
    cells = gb.lattice_spheroid(C5_CELLS, C5_N * LENGTH / 2, 5, LENGTH, C5_N)
    gb.seed_ki67_states(cells, 13)
    sim = gb.Simulation(voxel_num=C5_N, voxel_length=LENGTH, max_cell_num=C5_CELLS)
    sim.add_substrate(gb.oxygen())
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    sim.import_cells(cells)
    sim.PreLOD()
    sim.LODsolver(C5_WARM, 0)  # from the boundary value to a quasi-steady field
    sim.set_conv_ring(not args.no_conv_ring)
    sim.surrogate_load(0, sw.weights, K, sw.rate_scale, sw.threshold, sw.input_kind)
    b = float(gb.oxygen().boundary)
    inner = ~gs.shell_mask(C5_N)
    for _ in range(args.warmup):  # untimed: kernels loaded, buffers touched
        sim.FM_update()
        sim.PreLOD()
        p = sim.field(0)
        sim.lod_surrogate(0)
        sim.set_field(0, p)
        sim.LODsolver(K, 0)
    sim.sync()

    props = torch.cuda.get_device_properties(local_rank)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else uuid
    sampler = ClockSampler(str(uuid) if uuid else None)
    sampler.start()
    time.sleep(0.3)
    t_plain, t_sur, errs, res, acc = [], [], [], [], []
    for _ in range(args.steps):
        sim.FM_update()
        sim.PreLOD()
        p = sim.field(0)
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        torch.cuda.synchronize()
        e0.record(stream)
        sim.LODsolver(K, 0)
        e1.record(stream)
        ref = sim.field(0)
        sim.set_field(0, p)
        torch.cuda.synchronize()
        e2.record(stream)
        ok, r = sim.lod_surrogate(0)
        e3.record(stream)
        q = sim.field(0)
        t_plain.append(e0.elapsed_time(e1))
        t_sur.append(e2.elapsed_time(e3))
        errs.append(float(np.abs(q - ref)[inner].max() / b))
        res.append(r)
        acc.append(ok)
    sampler.stop()
    # operator kernels alone, from the per-kernel event profile of a few inferences
    sim.profile(True)
    sim.profile_read(reset=True)
    p = sim.field(0)
    for _ in range(3):
        sim.surrogate_infer(0)
        sim.set_field(0, p)
    prof = sim.profile_read(reset=True)
    sim.profile(False)
    sim.close()
    tp, ts = float(np.mean(t_plain)), float(np.mean(t_sur))
    hid = prof.get("k_conv3_hidden", (0, 0.0))
    infer_ms = sum(v[1] for k, v in prof.items() if k.startswith("k_conv3") or k == "k_pack_input") / 3
    flops_hidden = 2.0 * C5_N ** 3 * 32 * 32 * 27
    peak, peak_src = bf16_peak()
    avg_hidden = hid[1] / max(hid[0], 1)
    achieved = flops_hidden / (avg_hidden / 1e3) / 1e12 if hid[0] else None
    acc_errs = [e for e, a in zip(errs, acc) if a]
    line = {
        "metric": "oxygen LOD substeps/s with the judged surrogate (256^3, 300k cells)",
        "value": K / (ts / 1e3), "unit": "substeps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ts, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
        "data": "synthetic: seeded jittered-lattice spheroid of 300,000 cells; weights fitted on 2,000 pairs from the "
                "plain solver (gell_b200.surrogate)",
        "config": {"workload": C5_WORKLOAD, "voxels": C5_N ** 3, "substeps_per_block": K,
                   "conv_ring": not args.no_conv_ring,
                   "warm_substeps": C5_WARM, "judge_threshold": sw.threshold, "l2": "each field is 67 MB; the "
                   "operator's activations are 1.07 GB per 32-channel tensor"},
        "plain": {"value": K / (tp / 1e3), "ms_per_block": tp},
        "speedup_vs_plain": tp / ts,
        "accuracy": {"linf_err_max": max(errs), "linf_err_max_accepted": max(acc_errs) if acc_errs else None,
                     "linf_err_mean": float(np.mean(errs)), "accepted": int(sum(acc)), "blocks": len(acc),
                     "judge_residual_max": max(res), "unit": "max |q - p_plain| / boundary value inside the shell"},
        "components": {"ms_inference": infer_ms, "ms_conv_hidden_per_launch": avg_hidden,
                       "kernels": {k: [v[0] / 3, v[1] / 3] for k, v in prof.items()}},
        "roofline": {"kernel": "k_conv3_hidden (32 -> 32, 256^3)", "bound": "tensor", "achieved": achieved,
                     "peak": peak, "peak_source": peak_src, "unit": "TFLOP/s",
                     "frac": achieved / peak if achieved else None, "traffic": None,
                     "flops_per_launch": flops_hidden},
        "gpu_launches": None, "clocks": sampler.summary(),
    }
    return line


def run_c4(args, rank, world, local_rank):
    """--workload c4: K mechanics steps of all members in biology periods of 60."""
    import torch
    import gell_b200 as gb

    torch.cuda.set_device(local_rank)
    stream = torch.cuda.Stream()
    sims, edges = c4_members(gb, stream)
    ens = gb.Ensemble(sims)
    if args.c4_form == "tuned":
        taken, branches, warps = ens.tune(SUBSTEPS)
    else:
        taken, branches, warps = 0, 4, 0
        ens.configure(branches, warps)
        ens.set_batched(args.c4_form == "batched")
    batched = ens.batched()
    ens.run_mechanics(max(0, args.warmup - taken) + 2, SUBSTEPS)
    ens.sync()
    ncells0 = sum(s.count() for s in sims)

    # the same members stepped one after another (per-member calls), for comparison
    torch.cuda.synchronize()
    q0, q1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0.record(stream)
    for sim in sims:
        sim.mechanics_step(SUBSTEPS)
    q1.record(stream)
    torch.cuda.synchronize()
    t_seq_step = q0.elapsed_time(q1)

    props = torch.cuda.get_device_properties(local_rank)
    uuid = getattr(props, "uuid", None)
    uuid = f"GPU-{uuid}" if uuid is not None and not str(uuid).startswith("GPU-") else uuid
    sampler = ClockSampler(str(uuid) if uuid else None)
    sampler.start()
    time.sleep(0.3)
    K = args.steps
    cell_steps = 0
    launches0 = sum(s.launch_count() for s in sims)
    if world > 1:
        import torch.distributed as td
        td.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    done = 0
    while done < K:
        m = min(C4_BIO, K - done)
        n_after_birth = sum(s.CellBirth_kernel() for s in sims)
        ens.run_mechanics(m, SUBSTEPS)
        for s in sims:
            s.CellDeath_kernel()
        cell_steps += n_after_birth * m
        done += m
    e1.record(stream)
    torch.cuda.synchronize()
    sampler.stop()
    t_all = e0.elapsed_time(e1)
    launches = sum(s.launch_count() for s in sims) - launches0
    times = np.array([t_all], np.float64)
    cnt = np.array([cell_steps], np.float64)
    if world > 1:
        times, cnt = reduce_over_ranks(times, cnt, "cuda")
    line = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": cnt[0] / (times[0] / 1e3), "unit": "cell-updates/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": times[0] / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: 64 seeded jittered-lattice spheroids with seeded Ki-67 states",
            "config": {"workload": C4_WORKLOAD, "members": C4_MEMBERS, "voxels_total": int((edges ** 3).sum()),
                       "cells_total_start": int(ncells0), "substeps_per_step": SUBSTEPS,
                       "biology_period_steps": C4_BIO, "tuned_branches": branches, "tuned_sweep_warps": warps,
                       "tuned_batched_lod": batched, "form": args.c4_form,
                       "cells_cap": "each member's draw capped at 0.35 of its domain volume at packing 0.6, so the "
                                    "spheroid (radius 0.44 of the edge) fits its grid",
                       "tuning_steps": taken, "parallelism": "replicas"},
            "components": {"ms_per_step_members_one_by_one": t_seq_step,
                           "speedup_vs_members_one_by_one": t_seq_step / (times[0] / K)},
            "gpu_launches": int(launches), "clocks": sampler.summary(),
        }
    ens.close()
    for sim in sims:
        sim.close()
    return line


# ---------------------------------------------------------------------------- LOD only

def run_lod(args, rank, world, local_rank):
    """--workload lod: LOD substeps alone on an N^3 grid (--lod-n) with one or two substrates
    (--lod-subs) and a 10^6-cell lattice spheroid's uptake map; K timed substeps.  For kernel studies
    of the sweeps at other sizes than the headline's (the line tiles or, for N > 416, the ring
    kernels, as the library picks them)."""
    import torch
    import gell_b200 as gb

    torch.cuda.set_device(local_rank)
    n_lod = args.lod_n
    cells = gb.lattice_spheroid(NCELLS, n_lod * LENGTH / 2, 0, LENGTH, n_lod)
    sim = gb.Simulation(voxel_num=n_lod, voxel_length=LENGTH, max_cell_num=NCELLS + 1024)
    sim.add_substrate(gb.oxygen())
    if args.lod_subs > 1:
        sim.add_substrate(gb.drug())
    stream = torch.cuda.Stream()
    sim.set_stream(stream)
    sim.import_cells(cells)
    sim.PreLOD()
    sim.LODsolver(args.warmup)
    sim.sync()
    K = args.steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.LODsolver(K)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1)
    sim.profile(True)
    sim.profile_read(reset=True)
    sim.LODsolver(max(1, min(K, 10)))
    sim.sync()
    prof = sim.profile_read(reset=True)
    sim.profile(False)
    sim.close()
    peak, peak_kind = hbm_peak()
    per_launch = 8.0 * n_lod ** 3 * args.lod_subs
    kern = {k: {"avg_ms": v[1] / v[0], "achieved_gbs": per_launch / (v[1] / v[0] / 1e3) / 1e9,
                "frac": per_launch / (v[1] / v[0] / 1e3) / 1e9 / peak}
            for k, v in prof.items() if k.startswith("k_sweep")}
    return {"metric": "voxel-updates/s (LOD substeps alone)", "value": n_lod ** 3 * args.lod_subs * K / (t / 1e3),
            "unit": "voxel-updates/s", "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": t / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: uptake map of a seeded 10^6-cell lattice spheroid, fields at the boundary values",
            "config": {"workload": f"LOD substeps, {n_lod}^3 voxels x {args.lod_subs} substrate(s)"},
            "kernels": kern, "peak": {"hbm_gbs": peak, "source": peak_kind}}


# ---------------------------------------------------------------------------- other workloads

def other_workloads(args, local_rank):
    """Short runs of the other workloads, after the headline measurement (single GPU only), so that
    their figures travel with the headline line: the birth/death workload for one biology period
    (60 mechanics steps), the ensemble for 20 steps, the surrogate for 5 blocks.  Each is the same
    code as its own --workload line, with fewer steps; a failure is reported in place of its
    figures."""
    import gc

    out = {}
    runs = (("c3_600cube_5M_cells_birth_death", run_c3, 60),
            ("c4_ensemble_64", run_c4, 20),
            ("c5_surrogate_256cube", run_c5, 5))
    for name, fn, steps in runs:
        a = argparse.Namespace(**vars(args))
        a.steps, a.warmup = steps, 3
        t0 = time.time()
        try:
            r = fn(a, 0, 1, local_rank)
            keep = {k: r[k] for k in ("value", "unit", "ms_per_step", "steps", "components", "clocks")
                    if k in r}
            for k in ("plain", "speedup_vs_plain", "accuracy", "roofline"):
                if k in r:
                    keep[k] = r[k]
            keep["workload"] = r["config"]["workload"]
            out[name] = keep
        except Exception as e:  # the headline line is printed regardless
            out[name] = {"error": f"{type(e).__name__}: {e}"}
        out[name]["wall_s"] = round(time.time() - t0, 1)
        gc.collect()
    return out


# ---------------------------------------------------------------------------- CPU baseline

CPU_STEPS = 2


def cpu_baseline():
    """The reference's own FM and LOD kernel bodies compiled for the host with OpenMP
    (oracle/_ref/libgellref_host_c2{,d}.so, see oracle/ref_host_harness.cpp), on this machine's
    host cores: CPU_STEPS whole steps of the same workload (FM_update, PreLOD of both substrates,
    10 LODsolver substeps of both), after one untimed FM_update and substep that touch every array.
    Where the host build is missing, the oracle's restatement runs the same steps (kind "port")."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference_build as rb

    cells = make_cells()
    if rb.host_available("c2") and rb.host_available("c2d"):
        o2 = rb.HostRefSim("c2", 38.0, 1e5, 0.1)
        dr = rb.HostRefSim("c2d", 1.0, 5e4, 0.05)
        o2.set_cells(cells)
        o2.fm_update()
        o2.prelod()
        dr.prelod_on(o2)
        o2.lodsolver(1)
        dr.lodsolver(1)
        o2.set_cells(cells)
        t = [0.0, 0.0, 0.0]
        for _ in range(CPU_STEPS):
            t0 = time.perf_counter()
            o2.fm_update()
            t1 = time.perf_counter()
            o2.prelod()
            dr.prelod_on(o2)
            t2 = time.perf_counter()
            o2.lodsolver(SUBSTEPS)
            dr.lodsolver(SUBSTEPS)
            t3 = time.perf_counter()
            t[0] += t1 - t0
            t[1] += t2 - t1
            t[2] += t3 - t2
        alive = int(o2.cells()["sign"].sum())
        cores = o2.threads
        o2.close()
        dr.close()
        kind = "reference"
        what = ("the reference's FM and LOD kernel bodies compiled for the host (g++ -O3 -fopenmp, "
                "oracle/_ref/libgellref_host_c2{,d}.so)")
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_lib as ol
        P = ol.params(N=N, len=LENGTH, cap=CAP)
        subs = [(38.0, 1e5, 0.1, -10.0), (1.0, 5e4, 0.05, -1.0)]
        EF = [ol.mesh_init(N, LENGTH, D, dec, 0.01) for (_, D, dec, _) in subs]
        fields = [np.full(N ** 3, b, np.float32) for (b, _, _, _) in subs]
        c = cells.copy()
        t = [0.0, 0.0, 0.0]
        for _ in range(CPU_STEPS):
            t0 = time.perf_counter()
            ol.fm_update(c, P)
            t1 = time.perf_counter()
            rates = [ol.prelod(c, N, LENGTH, coef) for (_, _, _, coef) in subs]
            t2 = time.perf_counter()
            for k in range(NSUB):
                fields[k] = ol.lod_substeps(fields[k], rates[k], EF[k][0], EF[k][1], N, 0.01, subs[k][0], SUBSTEPS)
            t3 = time.perf_counter()
            t[0] += t1 - t0
            t[1] += t2 - t1
            t[2] += t3 - t2
        alive = int(c["sign"].sum())
        cores = int(ol.lib().go_get_threads())
        kind = "port"
        what = "the oracle's C restatement of the reference (OpenMP)"
    step = sum(t) / CPU_STEPS
    return {"value": alive / step, "unit": "cell-updates/s", "cores": cores, "kind": kind,
            "sample": f"{CPU_STEPS} whole steps of the large workload on {what}: {step:.2f} s per step",
            "s_per_step": step, "cell_updates_per_s_fm_prelod": alive * CPU_STEPS / (t[0] + t[1]),
            "voxel_updates_per_s_lod": N ** 3 * NSUB * SUBSTEPS * CPU_STEPS / t[2]}


def reference_unavailable(why):
    return {"impl": "reference", "unavailable": why}


def run_reference(args, local_rank, world):
    """The reference's own CUDA build on this GPU: its kernels and facades compiled from its
    unmodified sources (oracle/_ref/libgellref_c2.so for oxygen, libgellref_c2d.so for the drug,
    nvcc -O3 for sm_100a), driven as its host loop drives them (Main.cu:108-128) with integer
    counts.  One step = FM_update (include/FMkernel.cuh:181-202), PreLOD of both substrates
    (include/LODkernel.cuh:270-278) and 10 LODsolver substeps of both (:280-300); every facade
    synchronises the device, as the reference does.  Whole steps are timed with CUDA events on the
    legacy default stream the facades launch on.  e2e repeats the steps with the 72-byte cell
    records copied in from pinned host memory before each step and back out after it.  Under
    torchrun only rank 0 runs it, on one GPU (the line says n_gpus 1)."""
    if world > 1:
        # the reference selects no device: use this rank's before any CUDA call
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local_rank)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import reference_build as rb

    missing = [n for n in ("c2", "c2d") if not rb.available(n)]
    if missing:
        return reference_unavailable(f"reference build oracle/_ref/libgellref_{missing[0]}.so is missing "
                                     "(make -C oracle ref needs the reference sources)")
    cells = make_cells()
    o2 = rb.RefSim("c2", 38.0, 1e5, 0.1)
    drug = rb.RefSim("c2d", 1.0, 5e4, 0.05)
    o2.set_cells(cells)
    ncell = len(cells)

    def step():
        o2.fm_update()
        o2.prelod()
        drug.prelod_on(o2)
        o2.lodsolver(SUBSTEPS)
        drug.lodsolver(SUBSTEPS)

    for _ in range(args.warmup):
        step()
    assert rb.lib("c2").gref_sync() == 0
    sampler = ClockSampler(gpu_uuid_from_smi(local_rank))
    sampler.start()
    time.sleep(0.3)
    ev = [rb.RefEvent("c2") for _ in range(2)]
    se = [rb.RefEvent("c2") for _ in range(2)]
    K = args.steps
    per_step = []
    ev[0].record()
    for _ in range(K):
        # every facade ends in a device synchronisation, so these events do not perturb the steps
        se[0].record()
        step()
        se[1].record()
        per_step.append(se[0].elapsed_ms(se[1]))
    ev[1].record()
    t_all = ev[0].elapsed_ms(ev[1])
    sampler.stop()
    alive = int(o2.cells()["sign"].sum())

    # breakdown by facade, a separate pass with events between the facades
    kc = max(1, min(K, 5))
    pe = [rb.RefEvent("c2") for _ in range(4)]
    t_fm = t_pre = t_lod = 0.0
    for _ in range(kc):
        pe[0].record()
        o2.fm_update()
        pe[1].record()
        o2.prelod()
        drug.prelod_on(o2)
        pe[2].record()
        o2.lodsolver(SUBSTEPS)
        drug.lodsolver(SUBSTEPS)
        pe[3].record()
        t_fm += pe[0].elapsed_ms(pe[1])
        t_pre += pe[1].elapsed_ms(pe[2])
        t_lod += pe[2].elapsed_ms(pe[3])
    t_fm, t_pre, t_lod = t_fm * K / kc, t_pre * K / kc, t_lod * K / kc

    # e2e: the cell records in from pinned host memory and back out, every step
    host = rb.PinnedCells("c2", ncell)
    host.cells[:] = o2.cells()
    ke = max(1, min(K, 20))
    ev[0].record()
    for _ in range(ke):
        o2.set_cells(host.cells)
        step()
        o2.get_cells_into(host.cells)
    ev[1].record()
    t_e2e = ev[0].elapsed_ms(ev[1])
    alive_e2e = int(host.cells["sign"].sum())
    host.close()
    for e in ev + pe + se:
        e.close()
    drug.close()
    o2.close()

    cnt = (alive * K, alive_e2e * ke)
    t_mech = t_fm + t_pre
    c5 = reference_lod_256(rb) if rb.available("c5") else None
    return {
        "impl": "reference", "metric": METRIC, "value": cnt[0] / (t_all / 1e3), "unit": "cell-updates/s",
        "n_gpus": 1, "ranks_launched": world, "steps": K, "warmup": args.warmup, "ms_per_step": t_all / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded jittered-lattice spheroid of 10^6 cells, fields start at the boundary values",
        "config": config(),
        "reference_build": {
            "what": "the reference's own kernels and facades, compiled from its unmodified sources",
            "libraries": ["oracle/_ref/libgellref_c2.so", "oracle/_ref/libgellref_c2d.so"],
            "compile": "nvcc -O3 -gencode arch=compute_100a,code=sm_100a (oracle/Makefile, oracle/ref_harness.cu)",
            "step": "FM_update, PreLOD x 2 substrates, 10 x LODsolver x 2 substrates; integer loop counts"},
        "components": {"cell_updates_per_s_fm_prelod": cnt[0] / (t_mech / 1e3),
                       "voxel_updates_per_s_lod": N ** 3 * NSUB * SUBSTEPS * K / (t_lod / 1e3),
                       "ms_fm_update": t_fm / K, "ms_prelod": t_pre / K, "ms_lod_10_substeps": t_lod / K,
                       "lod_256cube_surrogate_workload": c5,
                       # every facade synchronises the device, so a step's time includes any host-side
                       # pause between its launches; the spread shows how much of the mean that is
                       "ms_per_step_each": {"min": float(np.min(per_step)),
                                            "p10": float(np.percentile(per_step, 10)),
                                            "median": float(np.median(per_step)),
                                            "p90": float(np.percentile(per_step, 90)),
                                            "max": float(np.max(per_step)),
                                            "steps_over_twice_the_median":
                                                int(np.sum(np.asarray(per_step) > 2 * np.median(per_step)))}},
        "e2e": {"value": cnt[1] / (t_e2e / 1e3), "unit": "cell-updates/s", "steps": ke,
                "h2d_bytes_per_step": int(ncell * 72), "d2h_bytes_per_step": int(ncell * 72)},
        "clocks": sampler.summary(),
    }


def reference_lod_256(rb, blocks=3):
    """The reference's own LODsolver (oracle/_ref/libgellref_c5.so: 256^3 voxels of 10 um, oxygen)
    on the surrogate workload's state: the same 300,000-cell spheroid and Ki-67 states as
    `--workload c5`, the field relaxed by the same 1000 substeps; then per block FM_update, PreLOD
    and the 50 timed substeps the surrogate replaces.  Returns ms per block of 50 substeps."""
    import gell_b200.cells as gc

    cells = gc.lattice_spheroid(C5_CELLS, C5_N * LENGTH / 2, 5, LENGTH, C5_N)
    gc.seed_ki67_states(cells, 13)
    ref = rb.RefSim("c5", 38.0, 1e5, 0.1)
    ref.set_cells(cells)
    ref.prelod()
    ref.lodsolver(C5_WARM)
    a, b = rb.RefEvent("c5"), rb.RefEvent("c5")
    ms = []
    for _ in range(blocks):
        ref.fm_update()
        ref.prelod()
        a.record()
        ref.lodsolver(50)
        b.record()
        ms.append(a.elapsed_ms(b))
    a.close()
    b.close()
    ref.close()
    return {"ms_per_50_substeps": float(np.mean(ms)), "blocks": blocks,
            "what": "the reference's LODsolver x 50 at 256^3 (oracle/_ref/libgellref_c5.so), same state as "
                    "--workload c5"}


def gpu_uuid_from_smi(index):
    """UUID of GPU `index` as nvidia-smi prints it (None when unavailable)."""
    try:
        out = subprocess.run(["nvidia-smi", "--query-gpu=index,uuid", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=20).stdout
        for line in out.splitlines():
            i, u = [x.strip() for x in line.split(",", 1)]
            if int(i) == int(index):
                return u
    except Exception:
        pass
    return None


# ---------------------------------------------------------------------------- main

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("gell", "reference"), default="gell")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=("large", "c3", "c4", "c5", "lod"), default="large",
                    help="large: 400^3, 10^6 cells (the headline line); c3: 600^3, 5*10^6 cells with "
                         "birth/death; c4: ensemble of 64 small instances; c5: the learned oxygen surrogate "
                         "against the plain solver at 256^3; lod: LOD substeps alone (--lod-n, --lod-subs)")
    ap.add_argument("--surrogate-weights", default=None, help="c5: weight file (default: the packaged one)")
    ap.add_argument("--no-conv-ring", action="store_true", help="c5: convolutions without the row ring")
    ap.add_argument("--c4-form", choices=("tuned", "members", "batched"), default="tuned",
                    help="c4: the tuner's choice, or 4 branches with LOD per member or batched over all members")
    ap.add_argument("--lod-n", type=int, default=400, help="lod: grid edge")
    ap.add_argument("--lod-subs", type=int, choices=(1, 2), default=2, help="lod: substrates")
    ap.add_argument("--no-extras", action="store_true",
                    help="large: skip the short runs of the other workloads reported under components")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # rank 0 alone runs the reference build (on its GPU); the other ranks exit without work
        if rank == 0:
            print(json.dumps(run_reference(args, local_rank, world)), flush=True)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as td
        torch.cuda.set_device(local_rank)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.workload in ("c3", "c4", "c5", "lod"):
        line = {"c3": run_c3, "c4": run_c4, "c5": run_c5, "lod": run_lod}[args.workload](args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            import torch.distributed as td
            td.destroy_process_group()
        return
    line = run_gell(args, rank, world, local_rank)
    if rank == 0:
        if world == 1 and not args.no_extras:
            line["components"]["other_workloads"] = other_workloads(args, local_rank)
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline()
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as td
        td.destroy_process_group()


if __name__ == "__main__":
    main()

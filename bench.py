#!/usr/bin/env python
"""ns/day of the FEN ZI MD step on one B200 (230,400-atom workload).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fenzi|reference]

A "step" is one velocity-Verlet + SHAKE/RATTLE MD time step (1 fs) of the whole
system: device-side neighbour maintenance, real-space pair kernel, bonded terms,
PME (spread, R2C/C2R FFT with the influence function, gather) and integration.
Workload (seeded synthetic, the reference ships no benchmark set): 72,000 TIP3P
waters + 480 linear 30-atom chains = 230,400 atoms in a 130 A cubic box, 128^3 PME,
beta 0.34, rc 10 / switch from 8, pair-list radius 11, 1 fs.

Timing: W untimed warm-up steps, then K steps each bracketed by CUDA events on the
library's stream, with a 256 MB write between steps so every timed step starts with
a cold L2 (the step's working set, ~80 MB, would otherwise stay in the 126 MB L2).
With --gpus N each rank runs an independent replica (one system does not shard:
replicas only); value = N x ns/day of the slowest rank.
e2e: the same metric through the C ABI with host buffers: per chunk of --chunk
steps, host->device copy of positions+velocities from pinned memory, fz_step(chunk),
device->host copy of positions+velocities, wall clock.
--impl reference: the FP64 CPU oracle (the reference's own CUDA build does not
compile with CUDA 12.9; it has no CPU path) on the same system, all host threads.
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

WORKLOAD = ("large230k: 72,000 TIP3P + 480 x 30-atom chains = 230,400 atoms, 130 A cubic box, 128^3 PME, "
            "beta 0.34, rc 10 / ron 8, pair list 11, SHAKE, 1 fs")
FLOP_PER_PAIR = 60  # algorithmic FP32 work per in-cutoff pair (FMA = 2)


def args_():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=30)
    ap.add_argument("--impl", default="fenzi", choices=["fenzi", "reference"])
    ap.add_argument("--workload", default="large230k")
    ap.add_argument("--chunk", type=int, default=100, help="MD steps per e2e call")
    ap.add_argument("--e2e-chunks", type=int, default=3)
    ap.add_argument("--equil", type=int, default=2000,
                    help="input preparation: MD steps with 300 K velocity reassignment every 100 steps "
                         "(relaxes the seeded lattice start; untimed, before the warm-up)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", action="store_true",
                    help="only run warm-up + steps (no timing/report): a clean target for ncu")
    return ap.parse_args()


def build_inputs(workload, seed):
    from fenzi_b200 import gen_system
    s = gen_system.build(name=workload, seed=seed)
    d = tempfile.mkdtemp(prefix=f"fzbench_{workload}_")
    return s, gen_system.write(s, d)


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None
        self.lines = []

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.p = None

    def _read(self):
        for ln in self.p.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
            except ValueError:
                continue
            for k, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(k)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def traffic_from_profiles(kernel_file):
    p = os.path.join(ROOT, "profiles", kernel_file)
    if not os.path.exists(p):
        return None
    try:
        return json.load(open(p)).get("dram_bytes_per_launch")
    except Exception:
        return None


def cpu_baseline(path, nsteps):
    """The FP64 oracle on the same system: nsteps MD steps on all host threads."""
    import fenzi_b200 as fz
    from oracle.oracle import Oracle
    s = fz.FenZi.ReadInput(path).LoadSystem()
    top = s.topology()
    orc = Oracle(top)
    pos = top["pos"]
    vel = orc.reassign_velocities(pos, 300.0, 2345, 0)
    t0 = time.perf_counter()
    orc.forces(pos)
    tf = time.perf_counter() - t0
    t0 = time.perf_counter()
    orc.md(pos, vel, nsteps, dt_ps=0.001, tol=1e-10, traces=False)
    tmd = time.perf_counter() - t0
    per_step = max(1e-9, (tmd - tf) / nsteps)
    s.close()
    return per_step, os.cpu_count()


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    _, path = build_inputs(a.workload, 2345)
    nsteps = max(1, min(a.steps, 4))
    per_step, cores = cpu_baseline(path, nsteps)
    nsd = 86.4 / (per_step * 1e3)
    natom = 230400 if a.workload == "large230k" else None
    line = {"metric": "ns/day @230K atoms (MD step, 1 fs)", "value": nsd, "unit": "ns/day", "impl": "reference",
            "n_gpus": a.gpus, "steps": nsteps, "warmup": 0, "ms_per_step": per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded generator, CHARMM file formats)",
            "config": {"workload": WORKLOAD, "parallelism": "host threads"},
            "cpu_baseline": {"value": nsd, "unit": "ns/day", "cores": cores, "kind": "port",
                             "sample": f"{nsteps} full MD steps (forces + velocity Verlet + SHAKE/RATTLE) of the "
                                       f"230,400-atom system after one force evaluation; FP64 oracle, OpenMP"},
            "e2e": {"value": nsd, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference CUDA build does not compile with CUDA 12.9 (legacy texture references); "
                    "timed arm is the FP64 CPU restatement of its algorithm"}
    if natom:
        line["atom_steps_per_s"] = natom / per_step
    print(json.dumps(line))
    return 0


def main():
    a = args_()
    if a.impl == "reference":
        return run_reference(a)
    import torch
    import fenzi_b200 as fz
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    s_gen, path = build_inputs(a.workload, 2345 + rank)
    sysm = fz.FenZi.ReadInput(path).LoadSystem()
    sysm.InitMem(local)
    sysm.InitVelocity(T=300.0, seed=2345 + rank, counter=0)
    for k in range(a.equil // 100):
        sysm.SingleStep(100)
        sysm.InitVelocity(T=300.0, seed=2345 + rank, counter=k + 1)
    natom = sysm.n
    dt_fs = sysm.cfg.timestep_ps * 1000.0
    stream = torch.cuda.ExternalStream(sysm.stream(), device=local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{local}")  # 256 MB > L2

    if a.profile:
        sysm.SingleStep(a.warmup)
        sysm.SingleStep(a.steps)
        sysm.sync()
        sysm.close()
        return 0
    # warm-up
    sysm.SingleStep(max(3, a.warmup))
    torch.cuda.synchronize()
    launches0 = sysm.counters()["launches"]
    rebuilds0 = sysm.counters()["rebuilds"]
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    clk = Clocks(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    for i in range(a.steps):
        flush.add_(1.0)  # cold L2 for every timed step (not timed)
        torch.cuda.synchronize()
        evs[i][0].record(stream)
        sysm.SingleStep(1)
        evs[i][1].record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clk.stop()
    total_ms = sum(b.elapsed_time(e) for b, e in evs)
    launches = sysm.counters()["launches"] - launches0
    rebuilds = sysm.counters()["rebuilds"] - rebuilds0
    if dist:
        t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_step = total_ms / a.steps
    nsd = 86.4 * dt_fs / ms_step
    value = nsd * world

    # per-stage breakdown (separate, untimed run with events between stages)
    sysm.stage_timing(True)
    sysm.SingleStep(50)
    stages = sysm.stage_times()
    sysm.stage_timing(False)

    # e2e through the C ABI with host buffers (wall clock)
    pin_p = torch.empty((natom, 3), dtype=torch.float32).pin_memory()
    pin_v = torch.empty((natom, 3), dtype=torch.float32).pin_memory()
    pos_h, vel_h = pin_p.numpy(), pin_v.numpy()
    sysm.get_state_f32(pos_h, vel_h)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.e2e_chunks):
        sysm.set_state_f32(pos_h, vel_h)
        sysm.SingleStep(a.chunk)
        sysm.get_state_f32(pos_h, vel_h)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / (a.e2e_chunks * a.chunk)
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_nsd = 86.4 * dt_fs / (e2e_s * 1e3) * world

    line = None
    if rank == 0:
        # roofline of the dominant kernel (real-space pairs): algorithmic FLOPs / measured duration
        from oracle.oracle import Oracle
        top = sysm.topology()
        orc = Oracle(top)
        pairs = orc.count_pairs(sysm.positions(), sysm.cfg.cutoff)
        nb_ms = stages["nonbonded"]
        achieved = FLOP_PER_PAIR * pairs / (nb_ms * 1e-3) / 1e12
        peak = fz.fp32_peak_tflops(local)
        roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic_from_profiles("nonbonded_large230k.json"),
                "kernel": "k_nonbonded", "kernel_ms": nb_ms,
                "work": f"{FLOP_PER_PAIR} FLOP x {pairs} non-excluded pairs within rc per launch",
                "peak_source": "measured FP32 FMA microbenchmark (fz_measure_fp32_peak); "
                               "MEASURED_PEAKS.json has no FP32 figure"}
        # whole-step roofline: T_ideal = W_nb/P_fp32 + (B_pme + B_int)/BW_hbm
        hbm = None
        try:
            hbm = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]
        except Exception:
            hbm = 6650.0
        K = list(sysm.cfg.pme_grid)
        bytes_ = 56 * natom + 24 * K[0] * K[1] * K[2] + 120 * natom
        t_ideal = FLOP_PER_PAIR * pairs / (peak * 1e12) + bytes_ / (hbm * 1e9)
        cpu = None
        if not a.no_cpu_baseline and world == 1:
            per, cores = cpu_baseline(path, 4)
            cpu = {"value": 86.4 * dt_fs / (per * 1e3), "unit": "ns/day", "cores": cores, "kind": "port",
                   "sample": "4 full MD steps of the 230,400-atom system (FP64 oracle, OpenMP, all host threads)"}
        line = {"metric": "ns/day @230K atoms (MD step, 1 fs)", "value": value, "unit": "ns/day",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (seeded generator written as CHARMM crd/psf/prm/rtf + .in)",
                "config": {"workload": WORKLOAD, "natom": natom, "parallelism": f"replicas x{world}",
                           "preparation": f"{a.equil} untimed MD steps with 300 K velocity reassignment every 100",
                           "l2": "flushed (256 MB write) before every timed step",
                           "pairs_within_cutoff": pairs},
                "atom_steps_per_s": natom * world / (ms_step * 1e-3),
                "step_roofline": {"t_ideal_ms": t_ideal * 1e3, "frac": t_ideal * 1e3 / ms_step,
                                  "model": "60 FLOP/pair / FP32 peak + (56N + 24K^3 + 120N) B / HBM"},
                "stages_ms": stages, "rebuilds_in_timed_steps": rebuilds,
                "pair_tiles": sysm.counters()["tiles"],
                "prunes_total": sysm.counters()["prunes"],
                "pair_slot_efficiency": pairs / (sysm.counters()["tiles"] * 1024.0),
                "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e_nsd, "unit": "ns/day", "h2d_bytes_per_step": 24 * natom,
                        "d2h_bytes_per_step": 24 * natom,
                        "step": f"one C-ABI call chain per {a.chunk} MD steps: fz_set_state_f32 + fz_step + "
                                f"fz_get_state_f32 (pinned host buffers, wall clock)"},
                "gpu_launches": launches, "clocks": clocks}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    sysm.close()
    if line:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())

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
compile with CUDA 12.9; it has no CPU path) on the same system, all host threads, W
untimed and K timed full MD steps (about 0.6 s a step on 16 host cores), rank 0 only.
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
    ap.add_argument("--ensemble", type=int, default=256,
                    help="batched-ensemble measurement (256 uneven TIP3P boxes of 648-6,000 atoms) with this many boxes; 0 skips it")
    ap.add_argument("--served", type=int, default=256,
                    help="served-job measurement (Poisson arrivals of 1.5k-30k-atom jobs) with this many jobs; 0 skips it")
    ap.add_argument("--precision", type=int, default=100000,
                    help="precision study: NVE steps of the 17,280-atom system, then NPT; 0 skips it")
    ap.add_argument("--small", type=int, default=2000,
                    help="9,000-atom water box: timed product-path steps (plus plain path and CPU oracle); 0 skips it")
    ap.add_argument("--profile", action="store_true",
                    help="only run warm-up + steps (no timing/report): a clean target for ncu")
    ap.add_argument("--profile-ensemble", action="store_true",
                    help="only prepare the batched ensemble (--ensemble boxes) and run --steps batched steps")
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
                                       "-lms", "20", "-i", str(self.device)], stdout=subprocess.PIPE,
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


def step_ideal_s(pairs, natom, K, peak_tflops, hbm_gbs):
    """Step roofline time: 60 FLOP per pair within rc at the FP32 peak plus the PME and
    integration bytes (56 N + 24 K^3 + 120 N) at the HBM bandwidth."""
    return FLOP_PER_PAIR * pairs / (peak_tflops * 1e12) + (176.0 * natom + 24.0 * K[0] * K[1] * K[2]) / (hbm_gbs * 1e9)


def measured_hbm_gbs():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def oracle_force_error(sy):
    """Relative RMS of the system's GPU forces at its current positions against the FP64 oracle."""
    from oracle.oracle import Oracle
    sy.ComputeAccelGPU()
    f = sy.forces()
    f0, _ = Oracle(sy.topology()).forces(sy.positions())
    return float(np.sqrt(((f - f0) ** 2).sum() / (f0 ** 2).sum()))


def traffic_from_profiles(kernel_file):
    p = os.path.join(ROOT, "profiles", kernel_file)
    if not os.path.exists(p):
        return None
    try:
        return json.load(open(p)).get("dram_bytes_per_launch")
    except Exception:
        return None


def bench_ensemble(nsys, device, steps=200, dist=None, peak_tflops=None, profile_steps=0):
    """Aggregate atom-steps/s of nsys independent water boxes advanced together (one
    graph launch per step) versus the same boxes stepped one at a time; wall clock with
    a device synchronisation on both sides of each timed region.  Under a process group
    the boxes are sharded over the ranks (longest-processing-time-first on atoms), each
    rank runs its shard as one batch, and the time is that of the slowest rank."""
    import torch
    import fenzi_b200 as fz
    from fenzi_b200 import gen_system
    from fenzi_b200.shard import lpt_assign, max_over_ranks
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    sizes = gen_system.ensemble_sizes(nsys)
    natoms_all = int(3 * sizes.sum())
    mine = lpt_assign(list(3 * sizes), world)[rank]
    boxes = gen_system.ensemble(nsys, only=set(mine))
    root = tempfile.mkdtemp(prefix="fzens_")
    systems = []
    for i, b in enumerate(boxes):
        sy = fz.FenZi.ReadInput(gen_system.write(b, os.path.join(root, f"b{i:03d}"))).LoadSystem()
        sy.InitMem(device)
        sy.InitVelocity(T=300.0, seed=100 + i)
        systems.append(sy)
    natoms = sum(s.n for s in systems)
    batch = fz.Batch(systems)
    for k in range(3):  # relax the lattice starts
        batch.step(100)
        for i, sy in enumerate(systems):
            sy.InitVelocity(T=300.0, seed=100 + i, counter=k + 1)
    batch.step(10)
    torch.cuda.synchronize()
    if profile_steps:
        batch.step(profile_steps)
        torch.cuda.synchronize()
        batch.close()
        for sy in systems:
            sy.close()
        return None
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    batch.step(steps)
    torch.cuda.synchronize()
    tb = max_over_ranks((time.perf_counter() - t0) / steps, dist, device=f"cuda:{device}")
    if world > 1:
        batch.close()
        for sy in systems:
            sy.close()
        return {"metric": "batched aggregate atom-steps/s", "value": natoms_all / tb, "unit": "atom-steps/s",
                "systems": nsys, "atoms": natoms_all, "ms_per_batched_step": tb * 1e3, "n_gpus": world,
                "scaling": "strong", "sharding": "longest-processing-time-first on atoms, one batch per rank",
                "timing": f"wall clock over {steps} batched steps (100-step graphs), max over ranks"}
    seq_steps = max(3, steps // 3)
    for sy in systems:  # warm each system's own graph
        sy.SingleStep(1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for sy in systems:
        sy.SingleStep(seq_steps)
    torch.cuda.synchronize()
    ts = (time.perf_counter() - t0) / seq_steps
    plain_rate, plain_atoms, plain_boxes = plain_one_at_a_time(systems, device)
    batch.close()
    # step roofline of the whole batch, oracle force error and the FP64 oracle one box
    # at a time on the host cores (samples)
    from oracle.oracle import Oracle
    hbm, hbm_src = measured_hbm_gbs()
    t_ideal = 0.0
    for sy in systems:
        orc = Oracle(sy.topology())
        t_ideal += step_ideal_s(orc.count_pairs(sy.positions(), sy.cfg.cutoff), sy.n, list(sy.cfg.pme_grid),
                                peak_tflops or 71.8, hbm)
    errs = [oracle_force_error(sy) for sy in systems[:: max(1, len(systems) // 4)][:4]]
    cpu_atoms, cpu_s = 0, 0.0
    for sy in systems[:: max(1, len(systems) // 8)][:8]:
        orc = Oracle(sy.topology())
        p0, v0 = sy.positions(), sy.velocities()
        orc.forces(p0)
        t0 = time.perf_counter()
        orc.md(p0, v0, 3, dt_ps=sy.cfg.timestep_ps, tol=1e-10, traces=False)
        cpu_s += (time.perf_counter() - t0) / 3
        cpu_atoms += sy.n
    for sy in systems:
        sy.close()
    return {"metric": "batched aggregate atom-steps/s", "value": natoms / tb, "unit": "atom-steps/s",
            "systems": nsys, "atoms": natoms, "ms_per_batched_step": tb * 1e3,
            "sequential_atom_steps_per_s": natoms / ts, "ms_per_sequential_sweep": ts * 1e3,
            "speedup_vs_one_at_a_time": ts / tb,
            "step_roofline": {"t_ideal_ms": t_ideal * 1e3, "frac": t_ideal / tb,
                              "model": "sum over boxes of 60 FLOP/pair / FP32 peak + (176 N + 24 K^3) B / HBM "
                                       f"({hbm_src} HBM)"},
            "force_rel_rms_vs_fp64_oracle": {"max": max(errs), "boxes_checked": len(errs)},
            "cpu_baseline": {"value": cpu_atoms / cpu_s, "unit": "atom-steps/s", "cores": os.cpu_count(),
                             "kind": "port", "sample": "FP64 oracle MD, 3 steps of each of 8 boxes one after "
                                                       "another (all host threads inside each box)"},
            "plain_one_at_a_time_atom_steps_per_s": plain_rate,
            "speedup_vs_plain_one_at_a_time": natoms / tb / plain_rate,
            "plain_sample": f"{plain_boxes} of the {len(systems)} boxes (every 4th, {plain_atoms} atoms), each on "
                            f"its own plain-path engine from its current state, 3 warm-up + 10 timed steps",
            "workload": f"{nsys} TIP3P boxes, 216-2000 waters each at 0.0334/A^3, grids 16^3-36^3 (smallest "
                        f"2^a3^b5^c >= L/1.2), rc 9 / ron 7.5, beta 0.34, SHAKE, NVE, 1 fs; seeded",
            "timing": f"wall clock over {steps} batched steps (100-step graphs) vs a sweep of {seq_steps}-step runs "
                      "of each box alone, device synchronised around each; working set > L2"}


def bench_small(device, peak_tflops, steps=2000):
    """The 9,000-atom water box (3,000 TIP3P, 44.8 A, 48^3 PME, rc 10): the product path
    (CUDA events around `steps` steps after 1,100 prepared ones), the plain path from the
    same state, the FP64 oracle on the host cores, the step roofline and the force error
    against the oracle."""
    import torch
    import fenzi_b200 as fz
    from fenzi_b200.plain import Plain
    from oracle.oracle import Oracle
    s_gen, path = build_inputs("water3000", 2345)
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(device)
    s.InitVelocity(T=300.0, seed=2345)
    for k in range(10):
        s.SingleStep(100)
        s.InitVelocity(T=300.0, seed=2345, counter=k + 1)
    s.SingleStep(100)
    stream = torch.cuda.ExternalStream(s.stream(), device=f"cuda:{device}")
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    s.SingleStep(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) * 1e-3 / steps
    p = Plain(s, device)
    p.set_positions(s.positions())
    p.set_velocities(s.velocities())
    p.SingleStep(20)
    t0 = time.perf_counter()
    p.SingleStep(300)
    tp = (time.perf_counter() - t0) / 300
    p.close()
    orc = Oracle(s.topology())
    pairs = orc.count_pairs(s.positions(), s.cfg.cutoff)
    hbm, hbm_src = measured_hbm_gbs()
    t_ideal = step_ideal_s(pairs, s.n, list(s.cfg.pme_grid), peak_tflops, hbm)
    err = oracle_force_error(s)
    per, cores = cpu_baseline(s_gen, 10)
    dt_fs = s.cfg.timestep_ps * 1000.0
    out = {"workload": "water3000: 3,000 TIP3P = 9,000 atoms, 44.8 A, 48^3 PME, beta 0.34, rc 10 / ron 8, "
                       "SHAKE, 1 fs (1,100 prepared steps with 300 K reassignment every 100)",
           "ns_per_day": 86.4 * dt_fs / (t * 1e3), "ms_per_step": t * 1e3, "atom_steps_per_s": s.n / t,
           "step_roofline": {"t_ideal_ms": t_ideal * 1e3, "frac": t_ideal / t, "hbm": hbm_src},
           "force_rel_rms_vs_fp64_oracle": err,
           "plain_path": {"ns_per_day": 86.4 * dt_fs / (tp * 1e3), "ms_per_step": tp * 1e3,
                          "product_speedup": tp / t, "timing": "wall clock over 300 steps"},
           "cpu_baseline": {"value": 86.4 * dt_fs / (per * 1e3), "unit": "ns/day", "cores": cores, "kind": "port",
                            "sample": "10 MD steps of the same system, FP64 oracle, all host threads"},
           "timing": f"CUDA events on the system's stream around {steps} steps (graph replay; the 2.2 us "
                     "roofline step is launch-latency bound)"}
    s.close()
    return out


def plain_one_at_a_time(systems, device, every=4, steps=10, warm=3):
    """Boxes one at a time on the plain path (every `every`-th box), each on its own
    engine started from the box's current state.  The plain step synchronises with the
    host every step, so each box is timed by wall clock.  Returns (atom-steps/s of the
    sample run one after another, atoms in the sample, boxes in the sample)."""
    from fenzi_b200.plain import Plain
    atoms, secs, nb = 0, 0.0, 0
    for sy in systems[::every]:
        p = Plain(sy, device)
        p.set_positions(sy.positions())
        p.set_velocities(sy.velocities())
        p.SingleStep(warm)
        t0 = time.perf_counter()
        p.SingleStep(steps)
        secs += (time.perf_counter() - t0) / steps
        atoms += sy.n
        nb += 1
        p.close()
    return atoms / secs, atoms, nb


def bench_plain_single(sysm, device, t_ideal_s, ms_ours, steps=60, warm=10):
    """The 230,400-atom system on the plain path (FP32, the reference's method) from the
    product path's current state: wall clock per step (it synchronises with the host
    every step), its fraction of the step roofline, and the product path's speed-up."""
    from fenzi_b200.plain import Plain
    p = Plain(sysm, device, fp64=False)
    p.set_positions(sysm.positions())
    p.set_velocities(sysm.velocities())
    p.SingleStep(warm)
    c0 = p.counters()
    t0 = time.perf_counter()
    p.SingleStep(steps)
    sec = (time.perf_counter() - t0) / steps
    c1 = p.counters()
    p.close()
    return {"method": "plain path, FP32: cell list + per-atom full neighbour list (no Newton-3), thread-per-atom "
                      "nonbonded, per-grid-point atom lists + gather-style spread, complex cuFFT, thread-per-atom "
                      "gather, one launch per stage, host synchronisation every step",
            "ms_per_step": sec * 1e3, "ns_per_day": 86.4 * sysm.cfg.timestep_ps * 1e3 / (sec * 1e3),
            "atom_steps_per_s": sysm.n / sec, "step_roofline_frac": t_ideal_s / sec,
            "product_speedup": sec * 1e3 / ms_ours,
            "rebuilds_in_timed_steps": c1["rebuilds"] - c0["rebuilds"],
            "launches_per_step": (c1["launches"] - c0["launches"]) / steps,
            "list_entries": c1["list_entries"], "timing": f"wall clock over {steps} steps after {warm} warm-up"}


def served_jobs(njobs, seed):
    """The served-job stream: sizes U[1,500, 30,000] atoms with 0-40 chains (rest TIP3P),
    steps log-uniform in [1,000, 20,000], half NVE and half NVT (300 K reassignment
    every 1,000 steps), Poisson arrivals at 200 jobs/s; all from one seed."""
    rng = np.random.default_rng(seed)
    jobs = []
    t = 0.0
    for i in range(njobs):
        natom = int(rng.integers(1500, 30001))
        nch = min(int(rng.integers(0, 41)), natom // 120)  # chains at most a quarter of the atoms
        nw = (natom - 30 * nch) // 3
        steps = int(round(float(np.exp(rng.uniform(np.log(1000), np.log(20000))))))
        nvt = bool(rng.integers(0, 2))
        t += float(rng.exponential(1.0 / 200.0))
        jobs.append(dict(nw=nw, nchains=nch, steps=steps, nvt=nvt, arrival=t, seed=seed + 1 + i))
    return jobs


def bench_served(device, njobs=256, seed=4242, check=4, sample=32, max_running=64, dist=None):
    """Served jobs through the serving loop (fz_server): each job of the seeded stream
    is submitted at its Poisson arrival time and admitted in FIFO order while fewer
    than `max_running` jobs run and their device bytes fit the 150 GB HBM budget, so
    later arrivals queue and are admitted as running jobs finish and free their slots
    (continuous batching); running jobs advance together in the batch graph.
    Per job: queue wait = start - submission, service = end - start, latency = end -
    submission, all on the server's steady clock.  The one-at-a-time comparisons time
    a seeded sample of `sample` jobs alone (200 steps on the product path, 30 on the
    plain path, each scaled to the job's step count).
    Under a process group the stream is routed online (each arrival to the rank with
    the least atoms x steps routed so far, the same on every rank) and each rank serves
    its jobs on its GPU; latencies are pooled over the ranks and the aggregate rate is
    all atom-steps over the slowest rank's makespan (no one-at-a-time comparison)."""
    import torch
    import fenzi_b200 as fz
    from fenzi_b200 import gen_system
    from fenzi_b200.shard import route_online
    from oracle.oracle import Oracle
    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    stream = served_jobs(njobs, seed)
    costs = [(3 * j["nw"] + 30 * j["nchains"]) * j["steps"] for j in stream]
    mine = route_online(costs, world)[rank]
    jobs = [stream[i] for i in mine]
    root = tempfile.mkdtemp(prefix="fzserve_")
    paths, gens = [], []
    for i, j in enumerate(jobs):
        box = (j["nw"] / 0.0334 + 15.0 * 30 * j["nchains"]) ** (1.0 / 3.0)  # ~15 A^3 per chain atom
        g = gen_system.build(name=f"job{i:03d}", nw=j["nw"], nchains=j["nchains"], chain_len=30, box=box, rc=10.0,
                             ron=8.0, seed=j["seed"])
        gens.append(g)
        paths.append(gen_system.write(g, os.path.join(root, f"j{i:03d}")))

    def load(i):
        s = fz.FenZi.ReadInput(paths[i])
        if jobs[i]["nvt"]:
            s.cfg.temp_reset_every = 1000
        return s.LoadSystem()

    # one at a time, on a seeded sample of the stream (one GPU only)
    from fenzi_b200.plain import Plain
    pick = sorted(np.random.default_rng(seed + 1).choice(len(jobs), min(sample, len(jobs)), replace=False)) \
        if world == 1 else []
    seq_s, plain_s, sample_work = 0.0, 0.0, 0.0
    for i in pick:
        j = jobs[i]
        s = load(i)
        s.InitMem(device)
        s.InitVelocity(T=300.0, seed=j["seed"])
        s.SingleStep(20)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.SingleStep(200)
        torch.cuda.synchronize()
        seq_s += (time.perf_counter() - t0) / 200 * j["steps"]
        sample_work += s.n * j["steps"]
        pl = Plain(s, device)
        pl.set_positions(s.positions())
        pl.set_velocities(s.velocities())
        pl.SingleStep(5)
        t0 = time.perf_counter()
        pl.SingleStep(30)
        plain_s += (time.perf_counter() - t0) / 30 * j["steps"]
        pl.close()
        s.close()
    systems = [load(i) for i in range(len(jobs))]
    total = sum(sy.n * j["steps"] for sy, j in zip(systems, jobs))
    server = fz.Server(device, hbm_budget_bytes=150e9, chunk_steps=100, max_running=max_running)
    ids = []
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for i, j in enumerate(jobs):
        d = j["arrival"] - (time.perf_counter() - t0)
        if d > 0:
            time.sleep(d)
        ids.append(server.submit(systems[i], j["steps"]))
    infos = [server.wait(k) for k in ids]
    wall = time.perf_counter() - t0
    stats = server.stats()
    lat = np.array([x["latency_s"] for x in infos])
    wait = np.array([x["start_s"] - x["submit_s"] for x in infos])
    serv = np.array([x["end_s"] - x["start_s"] for x in infos])
    # final-frame force error against the FP64 oracle (generator topology), smallest jobs
    errs = []
    for i in sorted(range(len(jobs)), key=lambda k: systems[k].n)[:check]:
        pos = server.positions(ids[i])
        s = load(i)
        s.InitMem(device)
        s.set_positions(pos)
        s.ComputeAccelGPU()
        f = s.forces()
        f0, _ = Oracle(gen_system.topology(gens[i])).forces(s.positions())
        errs.append(float(np.sqrt(((f - f0) ** 2).sum() / (f0 ** 2).sum())))
        s.close()
    server.close()
    pct = lambda a, q: float(np.percentile(a, q))
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, (lat.tolist(), wait.tolist(), serv.tolist(), total, wall, errs,
                                       stats["peak_running"]))
        lat = np.array([x for p in parts for x in p[0]])
        wait = np.array([x for p in parts for x in p[1]])
        serv = np.array([x for p in parts for x in p[2]])
        total = sum(p[3] for p in parts)
        wall = max(p[4] for p in parts)
        errs = [e for p in parts for e in p[5]]
        return {"metric": "served p50/p99 job latency", "p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "unit": "s",
                "jobs": len(stream), "n_gpus": world,
                "queue_wait_s": {"p50": pct(wait, 50), "p99": pct(wait, 99), "max": float(wait.max())},
                "service_s": {"p50": pct(serv, 50), "p99": pct(serv, 99)},
                "aggregate_atom_steps_per_s": total / wall, "makespan_s": wall, "max_running_per_gpu": max_running,
                "peak_running_jobs_per_gpu": [p[6] for p in parts],
                "routing": "online: each arrival to the rank with the least atoms x steps routed so far",
                "final_frame_force_rel_rms_vs_oracle": {"max": max(errs), "jobs_checked": len(errs)},
                "timing": "wall clock from a barrier before the first submission to each rank's last "
                          "completion; the aggregate uses the slowest rank"}
    return {"metric": "served p50/p99 job latency", "p50_s": pct(lat, 50), "p99_s": pct(lat, 99), "unit": "s",
            "jobs": len(jobs), "queue_wait_s": {"p50": pct(wait, 50), "p99": pct(wait, 99), "max": float(wait.max())},
            "service_s": {"p50": pct(serv, 50), "p99": pct(serv, 99)},
            "aggregate_atom_steps_per_s": total / wall, "makespan_s": wall,
            "max_running": max_running, "peak_running_jobs": stats["peak_running"],
            "jobs_that_queued": int((wait > 0.05).sum()),
            "one_at_a_time_atom_steps_per_s": sample_work / seq_s,
            "speedup_vs_one_at_a_time": (total / wall) / (sample_work / seq_s),
            "plain_one_at_a_time_atom_steps_per_s": sample_work / plain_s,
            "speedup_vs_plain_one_at_a_time": (total / wall) / (sample_work / plain_s),
            "one_at_a_time_sample": f"{len(pick)} seeded jobs of the stream",
            "final_frame_force_rel_rms_vs_oracle": {"max": max(errs), "jobs_checked": len(errs)},
            "workload": f"{len(jobs)} jobs of a Poisson(200/s) stream (seed {seed}): 1.5k-30k atoms, 0-40 30-atom "
                        f"chains + TIP3P, 1k-20k steps log-uniform, half NVT (reassignment every 1,000), rc 10, "
                        f"beta 0.34, SHAKE, 1 fs; HBM budget 150 GB, at most {max_running} running, 100-step chunks",
            "timing": "wall clock from the first submission to the last completion; per-job times on the "
                      "server's steady clock"}


def drift_fit(t_ns, etot, natom):
    """Least-squares slope of the total energy (kcal/mol/ns/atom) and its standard error."""
    t, e = np.asarray(t_ns, float), np.asarray(etot, float)
    if len(t) < 2:
        return 0.0, None
    if len(t) < 4:
        return float(np.polyfit(t, e, 1)[0]) / natom, None
    c, cov = np.polyfit(t, e, 1, cov=True)
    return float(c[0]) / natom, float(np.sqrt(cov[0, 0])) / natom


def plain_fp64_drift(s, device, pos0, vel0, nsteps, chunk):
    """NVE energy drift of the all-FP64 GPU variant (the plain path with every quantity
    in FP64) from the given state: total energy every `chunk` steps, slope per ns per atom."""
    from fenzi_b200.plain import Plain
    p = Plain(s, device, fp64=True)
    p.set_positions(pos0)
    p.set_velocities(vel0)
    t, tot = [], []
    t0 = time.perf_counter()
    for k in range(nsteps // chunk + 1):
        if k:
            p.SingleStep(chunk)
        e = p.EvalProps()
        t.append(k * chunk * s.cfg.timestep_ps * 1e-3)
        tot.append(e["potential"] + e["kinetic"])
    wall = time.perf_counter() - t0
    p.close()
    slope, err = drift_fit(t, tot, s.n)
    return {"method": "plain path in FP64 (positions, velocities, forces, PME mesh and FFT, SHAKE/RATTLE)",
            "nve_steps": nsteps, "nve_wall_s": wall, "nve_drift_kcal_per_mol_per_ns_per_atom": slope,
            "nve_drift_stderr": err,
            "nve_total_energy_std_kcal_per_mol": float(np.std(tot)), "t_ns": t}


def bench_precision(device, nve_steps=100000, npt_steps=2000, fp64_steps=20000):
    """The 17,280-atom precision study: NVE energy drift per ns per atom over nve_steps
    (after 2,000 thermalised steps), total-force error against the FP64 oracle, run-to-
    run bit-equality of the int64 force buffer (SHA-256 of two evaluations), the drift
    of the all-FP64 GPU variant over fp64_steps from the same state (the product path's
    drift over the same span beside it), then an Andersen leg of npt_steps at 1 atm
    (conserved-quantity excursion, volume change).  Drifts are least-squares slopes of
    the total energy sampled every 1,000 steps, with their standard errors."""
    import hashlib
    import fenzi_b200 as fz
    from fenzi_b200 import gen_system
    from oracle.oracle import Oracle
    g = gen_system.build(name="chain17k", seed=2345)
    path = gen_system.write(g, tempfile.mkdtemp(prefix="fzprec_"))
    s = fz.FenZi.ReadInput(path).LoadSystem()
    s.InitMem(device)
    s.InitVelocity(T=300.0, seed=2345, counter=0)
    for k in range(20):
        s.SingleStep(100)
        s.InitVelocity(T=300.0, seed=2345, counter=k + 1)
    s.SingleStep(100)
    pos0, vel0 = s.positions(), s.velocities()
    per, cores = cpu_baseline(g, 3)
    cpu = {"value": 86.4 * s.cfg.timestep_ps * 1e3 / (per * 1e3), "unit": "ns/day", "cores": cores, "kind": "port",
           "sample": "3 MD steps of the same system, FP64 oracle, all host threads"}
    chunk = 1000
    t, tot = [], []
    t0 = time.perf_counter()
    for k in range(nve_steps // chunk + 1):
        if k:
            s.SingleStep(chunk)
        e = s.EvalProps()
        t.append(k * chunk * s.cfg.timestep_ps * 1e-3)  # ns
        tot.append(e["potential"] + e["kinetic"])
    wall = time.perf_counter() - t0
    slope, slope_err = drift_fit(t, tot, s.n)
    # the all-FP64 GPU variant (plain path, FP64 throughout) from the same state
    fp64 = plain_fp64_drift(s, device, pos0, vel0, min(nve_steps, fp64_steps), chunk)
    nspan = len(fp64["t_ns"])
    slope_same, slope_same_err = drift_fit(t[:nspan], tot[:nspan], s.n)
    s.ComputeAccelGPU()
    a = s.forces_fixed()
    s.ComputeAccelGPU()
    b = s.forces_fixed()
    f = s.forces()
    f0, _ = Oracle(s.topology()).forces(s.positions())
    err = float(np.sqrt(((f - f0) ** 2).sum() / (f0 ** 2).sum()))
    s.set_barostat(True, 1.0, 1e-5)
    e0 = s.EvalProps()
    hs, vs = [], []
    for _ in range(npt_steps // 100):
        s.SingleStep(100)
        e = s.EvalProps()
        hs.append(e["conserved"] - e0["conserved"])
        vs.append(e["volume"] / e0["volume"] - 1.0)
    out = {"workload": "chain17k: 5,360 TIP3P + 40 x 30-atom chains = 17,280 atoms, 56 A, 64^3, beta 0.34, rc 10, "
                       "SHAKE, 1 fs",
           "nve_steps": nve_steps, "nve_wall_s": wall,
           "ns_per_day": 86.4 * s.cfg.timestep_ps * 1e3 / (wall / max(1, nve_steps) * 1e3),
           "cpu_baseline": cpu,
           "nve_drift_kcal_per_mol_per_ns_per_atom": slope, "nve_drift_stderr": slope_err,
           "nve_total_energy_std_kcal_per_mol": float(np.std(tot)),
           "force_rel_rms_vs_fp64_oracle": err,
           "force_sha256": [hashlib.sha256(a.tobytes()).hexdigest()[:16], hashlib.sha256(b.tobytes()).hexdigest()[:16]],
           "forces_bit_reproducible": bool(np.array_equal(a, b)),
           "nve_drift_same_span_kcal_per_mol_per_ns_per_atom": slope_same,
           "nve_drift_same_span_stderr": slope_same_err,
           "all_fp64_gpu_variant": {k: v for k, v in fp64.items() if k != "t_ns"},
           "npt": {"steps": npt_steps, "pref_atm": 1.0, "pmass": 1e-5,
                   "conserved_max_excursion_kcal_per_mol": float(np.abs(hs).max()),
                   "kinetic_kcal_per_mol": e0["kinetic"], "volume_change_max": float(np.abs(vs).max()),
                   "final_box_A": e["box"][0], "final_pressure_atm": e["pressure_atm"]}}
    s.close()
    return out


def cpu_baseline(s_gen, nsteps, warmup=0):
    """The FP64 oracle on the same system, on all host threads: `warmup` untimed MD
    steps, then nsteps timed MD steps (forces + velocity Verlet + SHAKE/RATTLE).  The
    oracle's topology comes from the generator (no product library is loaded)."""
    from fenzi_b200 import gen_system
    from oracle.oracle import Oracle
    orc = Oracle(gen_system.topology(s_gen))
    pos = np.asarray(s_gen.pos, np.float64)
    vel = orc.reassign_velocities(pos, 300.0, 2345, 0)
    if warmup > 0:
        st = orc.md(pos, vel, warmup, dt_ps=0.001, tol=1e-10, traces=False)
        pos, vel = st["pos"], st["vel"]
    else:
        orc.forces(pos)  # first-touch of the oracle's buffers, untimed
    t0 = time.perf_counter()
    orc.md(pos, vel, nsteps, dt_ps=0.001, tol=1e-10, traces=False)
    per_step = max(1e-9, (time.perf_counter() - t0) / nsteps)
    return per_step, os.cpu_count()


def pme_error(sysm, s_gen, nsample=2000):
    """PME force error of the product against a converged direct Ewald sum (FP64, on a
    seeded subsample of atoms), relative to the total nonbonded force, beside the error
    of the FP64 order-4 mesh of the same grid (the method's own error)."""
    import fenzi_b200 as fz
    from fenzi_b200 import gen_system
    from oracle import oracle as O
    from oracle.ewald_direct import kmax_for, recip_forces
    pos = sysm.positions()
    sysm.ComputeAccelGPU(terms=fz.TERM_PME)
    f_pme = sysm.forces()
    sysm.ComputeAccelGPU(terms=fz.TERM_NONBONDED | fz.TERM_PAIRS14 | fz.TERM_EXCLUSIONS)
    f_real = sysm.forces()
    atoms = np.random.default_rng(7).choice(len(pos), min(nsample, len(pos)), replace=False)
    fe, _ = recip_forces(pos, s_gen.charge, s_gen.box, s_gen.beta, atoms, kmax_for(s_gen.box, s_gen.beta))
    f64, _ = O.Oracle(gen_system.topology(s_gen)).forces(pos, O.T_PME)
    den = ((f_real[atoms] + fe) ** 2).sum()
    return {"vs_direct_ewald": float(np.sqrt(((f_pme[atoms] - fe) ** 2).sum() / den)),
            "fp64_mesh_vs_direct_ewald": float(np.sqrt(((f64[atoms] - fe) ** 2).sum() / den)),
            "vs_fp64_mesh": float(np.sqrt(((f_pme - f64) ** 2).sum() / (f64 ** 2).sum())),
            "relative_to": "total nonbonded force (real-space pairs + 1-4 + exclusion + reciprocal)",
            "sample": f"{len(atoms)} seeded atoms; direct sum over |m| with exp(-pi^2 m^2/beta^2) > 1e-12"}


def config_block(natom):
    """The `config` object of both arms (the workload only; run details are elsewhere)."""
    return {"workload": WORKLOAD, "natom": natom, "timestep_fs": 1.0,
            "l2": "GPU arm: flushed (256 MB write) before every timed step"}


def run_reference(a):
    """The reference arm: the FP64 CPU restatement of the reference's algorithm (its own
    CUDA build does not compile with CUDA 12.9 and it has no CPU path), W untimed and K
    timed full MD steps of the same 230,400-atom system on all host threads, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    s_gen, _ = build_inputs(a.workload, 2345)
    per_step, cores = cpu_baseline(s_gen, a.steps, a.warmup)
    nsd = 86.4 / (per_step * 1e3)
    natom = s_gen.n
    line = {"metric": "ns/day @230K atoms (MD step, 1 fs)", "value": nsd, "unit": "ns/day", "impl": "reference",
            "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": per_step * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded generator, CHARMM file formats)",
            "config": config_block(natom),
            "parallelism": f"host threads x{cores} (rank 0)",
            "cpu_baseline": {"value": nsd, "unit": "ns/day", "cores": cores, "kind": "port",
                             "sample": f"{a.steps} full MD steps (forces + velocity Verlet + SHAKE/RATTLE) of the "
                                       f"230,400-atom system after {a.warmup} untimed steps; FP64 oracle, OpenMP"},
            "e2e": {"value": nsd, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "atom_steps_per_s": natom / per_step,
            "note": "reference CUDA build does not compile with CUDA 12.9 (legacy texture references); "
                    "timed arm is the FP64 CPU restatement of its algorithm"}
    print(json.dumps(line))
    return 0


def main():
    a = args_()
    if a.impl == "reference":
        return run_reference(a)
    if a.profile_ensemble:
        bench_ensemble(a.ensemble, 0, profile_steps=a.steps)
        return 0
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

    shapes = sysm.launch_shapes()
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

    # batched ensemble sharded over the ranks (every rank takes part)
    batched_multi = bench_ensemble(a.ensemble, local, dist=dist) if a.ensemble > 0 and world > 1 else None
    # served stream routed over the ranks (every rank takes part)
    served_multi = bench_served(local, a.served, dist=dist) if a.served > 0 and world > 1 else None
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
            per, cores = cpu_baseline(s_gen, 4)
            cpu = {"value": 86.4 * dt_fs / (per * 1e3), "unit": "ns/day", "cores": cores, "kind": "port",
                   "sample": "4 full MD steps of the 230,400-atom system (FP64 oracle, OpenMP, all host threads)"}
        plain = bench_plain_single(sysm, local, t_ideal, ms_step) if world == 1 else None
        pme_err = pme_error(sysm, s_gen) if world == 1 else None
        small = bench_small(local, peak, a.small) if a.small > 0 and world == 1 else None
        batched = batched_multi
        if a.ensemble > 0 and world == 1:
            batched = bench_ensemble(a.ensemble, local, peak_tflops=peak)
        served = served_multi
        if a.served > 0 and world == 1:
            served = bench_served(local, a.served)
        precision = None
        if a.precision > 0 and world == 1:
            precision = bench_precision(local, a.precision)
        line = {"metric": "ns/day @230K atoms (MD step, 1 fs)", "value": value, "unit": "ns/day",
                "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
                "data": "synthetic (seeded generator written as CHARMM crd/psf/prm/rtf + .in)",
                "config": config_block(natom),
                "parallelism": f"replicas x{world}",
                "run": {"preparation": f"{a.equil} untimed MD steps with 300 K velocity reassignment every 100",
                        "pairs_within_cutoff": pairs, "launch_shapes": shapes},
                "atom_steps_per_s": natom * world / (ms_step * 1e-3),
                "step_roofline": {"t_ideal_ms": t_ideal * 1e3, "frac": t_ideal * 1e3 / ms_step,
                                  "model": "60 FLOP/pair / FP32 peak + (56N + 24K^3 + 120N) B / HBM"},
                "stages_ms": stages, "rebuilds_in_timed_steps": rebuilds,
                "pair_slots": sysm.counters()["pair_slots"],
                "prunes_total": sysm.counters()["prunes"],
                "pair_slot_efficiency": pairs / float(sysm.counters()["pair_slots"]),
                "roofline": roof, "cpu_baseline": cpu, "plain_path": plain, "small_system": small,
                "e2e": {"value": e2e_nsd, "unit": "ns/day", "h2d_bytes_per_step": 24 * natom / a.chunk,
                        "d2h_bytes_per_step": 24 * natom / a.chunk, "h2d_bytes_per_call": 24 * natom,
                        "d2h_bytes_per_call": 24 * natom,
                        "step": f"one C-ABI call chain per {a.chunk} MD steps: fz_set_state_f32 (positions + "
                                f"velocities from pinned host memory) + fz_step({a.chunk}) + fz_get_state_f32 "
                                f"(wall clock); bytes per MD step are the per-call copies / {a.chunk}"},
                "gpu_launches": launches, "clocks": clocks, "pme_error": pme_err, "batched": batched,
                "served": served,
                "precision": precision}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    sysm.close()
    if line:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""Benchmark of the per-timestep lattice update (D3Q19 colour-gradient MRT).

Default workload ("mix"): the 96 uneven Rayleigh-Plateau domains of the
batched configuration (Nx=Ny in [24,64], Nz in [64,384], half of them with an
on-axis sphere; 45.0 M nodes in all), FP16 shifted storage, stepped as one
batch: one CUDA graph per step holding one phase-field launch for all domains,
one launch per particle/wall subroutine for all domains, and one persistent
collide launch over a work-tile table.  One bench step = one lattice update of
every domain (every node counted, fluid or solid).  `value` is MLUPS of the
graph replay, inputs resident in HBM.  Beside it, on the same box (N=1 only):
  per_kernel   eager steps with CUDA events around each kernel class
  e2e          host buffers through the C ABI: upload both colours'
               populations and rho_N of every domain (pinned, Fortran
               layout), 100 batch steps, download five macroscopic fields
  storages     the same 96 domains batched in FP32 and in FP64 storage
  plain_fp64   the same 96 domains in plain FP64, one domain at a time
  c3_fp64      the 256x256x512 thread in plain FP64 (the roofline run)
  serving      the Poisson job stream through the job server: FP16 batched
               (continuous batching) and plain FP64 one job at a time
  cpu_baseline the oracle (C++ restatement of Source1.f90) on the host cores

  python bench.py [--gpus N --steps K --warmup W] [--workload mix|c3|c2|c1]
  python bench.py --impl reference ...   # the reference algorithm on the host cores

Multi-GPU: the path does not shard (domains are independent); N GPUs run N
replicas of the batch ("replicas only"), value = all ranks' node updates /
max-over-ranks device time.
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
import traceback

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STORE_BYTES = {"fp64": 8, "fp32": 4, "fp16": 2}
PHI_BYTES = {"fp64": 8, "fp32": 4, "fp16": 4}
METRIC = "MLUPS (lattice node updates per second, 1e6) of the per-timestep lattice update"


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def b_collide(storage):
    """Algorithmic bytes per node of the collide kernel: 38 populations read and
    written, phi read once."""
    return 76 * STORE_BYTES[storage] + PHI_BYTES[storage]


def b_phase(storage):
    """Bytes per node the phase kernel must move: FP64 reads the two colour
    densities the collide kernel accumulated, clears them and writes phi;
    the other storages read the 38 populations and write phi."""
    if storage == "fp64":
        return 4 * 8 + PHI_BYTES[storage]
    return 38 * STORE_BYTES[storage] + PHI_BYTES[storage]


# DRAM bytes per node of one collide launch, dram__bytes_read.sum +
# dram__bytes_write.sum from one ncu capture divided by the nodes of the
# launch: profiles/k_collide_batch_fp16_mix24.md (16-bit, batched kernel) and
# profiles/k_collide_fp64_thread_128x128x256.md (FP64, single-domain kernel;
# the batched kernel runs the same tile code).  The traffic per node does not
# depend on the number of nodes, so it scales to a full launch.
COLLIDE_TRAFFIC_B_PER_NODE = {"fp16": 224.7, "fp64": 704.2}


def collide_traffic(storage, nodes):
    b = COLLIDE_TRAFFIC_B_PER_NODE.get(storage)
    return None if b is None else b * nodes


def b_step(storage):
    """Algorithmic bytes per node update of the whole step."""
    return 76 * STORE_BYTES[storage] + 2 * PHI_BYTES[storage]


def workload(name: str, storage: str, size=None):
    from symmetry_b200 import configs
    if size:
        nx, ny, nz = (int(v) for v in size.lower().split("x"))
        if name == "c3":
            return configs.c3_thread(nx=nx, ny=ny, nz=nz, storage=storage, radius=24.0 * nx / 256.0)
        if name == "c1":
            return configs.c1_thread(nx=nx, ny=ny, nz=nz, storage=storage, radius=6.0 * nx / 32.0)
        raise SystemExit("--size applies to the thread workloads (c1, c3)")
    if name == "c3":
        return configs.c3_thread(storage=storage)
    if name == "c2":
        return configs.c2_wall_particle(storage=storage)
    if name == "c1":
        return configs.c1_thread(storage=storage)
    raise SystemExit(f"unknown workload {name}")


def describe(w, storage):
    p = w.params
    return (f"{w.name} {p.nx}x{p.ny}x{p.nz} "
            f"{'walls+%d particle(s)' % p.par if (p.par or p.wall_x) else 'periodic'}, {storage} storage")


MIX_DESC = ("96 uneven Rayleigh-Plateau domains (Nx=Ny in [24,64], Nz in [64,384] in whole wavelengths, "
            "48 with an on-axis sphere R/2), seeded manifest default_rng(4)")


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for k, n in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def leg(name, fn, *a, **kw):
    """Run an auxiliary measurement; a failure is reported in the line, not fatal."""
    try:
        return fn(*a, **kw)
    except Exception as e:  # noqa: BLE001
        traceback.print_exc(file=sys.stderr)
        return {"error": f"{name}: {type(e).__name__}: {e}"}


# ---- reference arm and CPU baseline -------------------------------------------------
def mix_sample(n=4):
    """The first n domains of the batched mix in FP64: the bounded CPU sample."""
    from symmetry_b200 import configs
    return configs.c4_manifest(storage="fp64")[:n]


def thread_sample(w):
    from symmetry_b200 import configs
    p = w.params
    sample = configs.Workload(w.name, p.copy(), w.kind, dict(w.gen), w.steps, list(w.particles))
    if w.kind == "thread":
        sample.params.nz = min(p.nz, 32)
        sample.gen["wavelength"] = float(sample.params.nz)
    return [sample]


def cpu_run(samples, warmup, steps=None, budget_s=None):
    """Step every sample domain once per step through the oracle (all host
    threads); returns (node updates per step, seconds per step, steps)."""
    from oracle import oracle as orc
    os_ = [orc.setup_workload(w) for w in samples]
    for _ in range(warmup):
        for o in os_:
            o.step(1)
    nodes = sum(w.params.n_nodes for w in samples)
    n, t0 = 0, time.perf_counter()
    while True:
        for o in os_:
            o.step(1)
        n += 1
        dt = time.perf_counter() - t0
        if (steps and n >= steps) or (budget_s and dt > budget_s):
            break
    return nodes, dt / n, n


def cpu_baseline(samples, label, budget_s=20.0):
    from oracle import oracle as orc
    nodes, sec, n = cpu_run(samples, 1, budget_s=budget_s)
    return {"value": nodes / sec / 1e6, "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
            "sample": f"{n} steps of {label} ({nodes} nodes per step), FP64; the oracle restating Source1.f90 "
                      "(g++ -O3 -fopenmp; no Fortran compiler on this image), equal bit for bit to the "
                      "reference's own source executed through a mechanical translation"}


def cpu_run_each(samples, warmup, steps):
    """Each domain in turn through the oracle (all host threads): set up,
    `warmup` untimed steps, `steps` timed steps, freed before the next one (the
    whole mix at once would hold ~40 GB of host memory).  Returns (node updates
    per step over all domains, seconds per step over all domains)."""
    from oracle import oracle as orc
    nodes, sec = 0, 0.0
    for w in samples:
        o = orc.setup_workload(w)
        for _ in range(warmup):
            o.step(1)
        t0 = time.perf_counter()
        o.step(steps)
        sec += (time.perf_counter() - t0) / steps
        nodes += w.params.n_nodes
        del o
    return nodes, sec


def run_reference(args):
    """--impl reference: the reference's algorithm on the host cores (the oracle
    port; the Fortran reference cannot be compiled on this image).  The mix
    runs every one of its domains (the GPU arm's configuration), one domain
    at a time."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as orc
    if args.workload == "mix":
        from symmetry_b200 import configs
        samples = configs.c4_manifest(storage="fp64")[:max(1, min(96, args.domains))]
        label = f"all {len(samples)} domains of the batched mix, one at a time"
        cfg = MIX_DESC + ("" if len(samples) == 96 else f" (first {len(samples)} domains only)")
        nodes, sec = cpu_run_each(samples, args.warmup, args.steps)
        same = len(samples) == 96
    else:
        w = workload(args.workload, "fp64", args.size)
        samples, label, cfg = thread_sample(w), "a z-slab of the domain", describe(w, "fp64")
        nodes, sec, n = cpu_run(samples, args.warmup, steps=args.steps)
        same = False
    v = nodes / sec / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "MLUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded phase fields)",
        "config": {"workload": cfg, "nodes_per_step": nodes, "same_config_as_gpu_arm": same},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
                         "sample": f"{label}, {nodes} nodes per step, {args.steps} timed steps each; C++ "
                                   "restatement of Source1.f90 (no Fortran compiler on this image), equal "
                                   "bit for bit to the reference's own source executed through a mechanical "
                                   "translation"},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---- legs -------------------------------------------------------------------------
def pinned(torch, shape):
    import numpy as np
    n = int(np.prod(shape))
    return torch.empty(n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape)


def e2e_batch(torch, lattices, B, inner=100, reps=3):
    """End to end through the C ABI with pinned host buffers, one output
    interval of the reference driver: upload ri, bi and rho_N of every domain
    (Fortran layout), `inner` batch steps, then calmacros of every domain
    downloaded as rho_N, rho, ux, uy, uz (sym_get_macros); `reps` timed
    intervals after one warm-up interval."""
    host = []
    h2d = d2h = 0
    for L in lattices:
        shape = L.shape
        ri, bi, phi = pinned(torch, shape + (19,)), pinned(torch, shape + (19,)), pinned(torch, shape)
        outs = [pinned(torch, shape) for _ in range(5)]
        L.get_into("ri", ri)
        L.get_into("bi", bi)
        L.get_into("rho_N", phi)
        host.append((ri, bi, phi, outs))
        h2d += ri.nbytes + bi.nbytes + phi.nbytes
        d2h += sum(o.nbytes for o in outs)
    nodes = sum(L.p.n_nodes for L in lattices)

    def one():
        for L, (ri, bi, phi, outs) in zip(lattices, host):
            L.set("rho_N", phi)
            L.set_populations(ri, bi)
        B.step(inner)
        for L, (ri, bi, phi, outs) in zip(lattices, host):
            L.macros(dict(zip(["rho_N", "rho", "ux", "uy", "uz"], outs)))

    one()   # warm-up (graph rebuild after the uploads)
    dts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        one()
        dts.append(time.perf_counter() - t0)
    dt = sum(dts) / len(dts)
    return {"value": nodes * inner / dt / 1e6, "unit": "MLUPS", "h2d_bytes_per_step": h2d / inner,
            "d2h_bytes_per_step": d2h / inner, "inner_steps": inner, "repeats": reps,
            "interval_s": {"mean": dt, "min": min(dts), "max": max(dts)},
            "step": f"upload ri+bi+rho_N of all 96 domains (pinned, Fortran layout, {h2d / 1e9:.2f} GB) -> "
                    f"{inner} batch steps -> calmacros -> download rho_N,rho,u ({d2h / 1e9:.2f} GB); "
                    "per-step bytes = interval bytes / inner steps"}


def plain_fp64(ws, steps, local):
    """The same domains in plain FP64, one domain at a time (graph replay)."""
    from symmetry_b200.lib import setup_workload
    tot_nodes, tot_ms, per = 0, 0.0, []
    for w in ws:
        p = w.params.copy()
        p.storage = 0
        w64 = type(w)(w.name, p, w.kind, dict(w.gen), w.steps, list(w.particles))
        L = setup_workload(w64, device=local)
        L.step(2)
        ms = L.step_timed(steps, use_graph=True)[0]
        tot_nodes += w.nodes * steps
        tot_ms += ms
        per.append(w.nodes * steps / ms / 1e3)
        L.close()
    return {"value": tot_nodes / tot_ms / 1e3, "unit": "MLUPS", "steps_per_domain": steps,
            "domain_mlups_min": min(per), "domain_mlups_max": max(per),
            "how": "each domain alone through sym_step (graph replay), CUDA events; aggregate = all node "
                   "updates / summed device time"}


def batched_mix(storage, steps, local):
    """The same 96 domains batched in another storage (graph replay, tiles
    from the autotuner): the precision/speed trade-off beside the headline."""
    from symmetry_b200 import configs
    from symmetry_b200.lib import Batch, setup_workload
    ws = configs.c4_manifest(storage=storage)
    lattices = [setup_workload(w, device=local) for w in ws]
    B = Batch(lattices)
    B.autotune(trial_steps=3)
    B.step(3)
    ms = B.step_timed(steps)
    B.close()
    for L in lattices:
        L.close()
    nodes = sum(w.nodes for w in ws)
    return {"value": nodes * steps / ms / 1e3, "unit": "MLUPS", "storage": storage, "steps": steps,
            "ms_per_step": ms / steps}


def c3_leg(steps, peak, local):
    from symmetry_b200 import configs
    from symmetry_b200.lib import setup_workload
    w = configs.c3_thread(storage="fp64")
    n = w.nodes
    L = setup_workload(w, device=local)
    L.step(3)
    ms = L.step_timed(steps, use_graph=False)
    g = L.step_timed(steps, use_graph=True)[0]
    L.close()
    v = n * steps / g / 1e3
    col = ms[3] / steps
    ph = ms[1] / steps
    return {"workload": describe(w, "fp64"), "value": v, "unit": "MLUPS", "ms_per_step": g / steps,
            "step_gbs": b_step("fp64") * v * 1e6 / 1e9, "step_frac": b_step("fp64") * v * 1e6 / 1e9 / peak,
            "collide_ms": col, "collide_gbs": b_collide("fp64") * n / (col / 1e3) / 1e9,
            "collide_frac": b_collide("fp64") * n / (col / 1e3) / 1e9 / peak,
            "collide_traffic": collide_traffic("fp64", n),
            "phase_ms": ph, "phase_gbs": b_phase("fp64") * n / (ph / 1e3) / 1e9,
            "phase_frac": b_phase("fp64") * n / (ph / 1e3) / 1e9 / peak}


def run_serving(storage, slots, rate, duration, cap, budget, wall_limit, xchunk, local):
    """Open-loop Poisson arrivals through the job server; jobs stop at breakup
    or at `cap` steps."""
    import numpy as np
    from symmetry_b200 import configs
    from symmetry_b200.lib import Server, job_spec
    jobs = configs.c5_jobs(rate=rate, duration=duration, storage=storage, max_steps=cap)
    S = Server(device=local, budget_bytes=budget, slots=slots, check_every=10)
    for c, x in (xchunk or {}).items():
        S.set_xchunk(int(c), int(x))
    ids = []
    clock0 = S.stats()["clock_s"]
    t0 = time.perf_counter()
    k = 0
    while True:
        now = time.perf_counter() - t0
        while k < len(jobs) and jobs[k].t_arrival <= now:
            ids.append(S.submit(job_spec(jobs[k].workload, cap, 1.0, clock0 + jobs[k].t_arrival)))
            k += 1
        r, p = S.tick()
        if k == len(jobs) and r == 0 and p == 0:
            break
        if time.perf_counter() - t0 > wall_limit:
            break
        if r == 0 and p == 0 and k < len(jobs):
            time.sleep(max(0.0, min(0.05, jobs[k].t_arrival - (time.perf_counter() - t0))))
    elapsed = time.perf_counter() - t0
    st = S.stats()
    res = [S.result(i) for i in ids]
    S.close()
    done = [x for x in res if x.status in (2, 3)]
    failed = [x for x in res if x.status == 4]
    lat = np.array([x.t_done - x.t_arrival for x in done]) if done else np.zeros(0)
    latb = np.array([x.t_done - x.t_arrival for x in done if x.status == 2])
    errs = {}
    for i, x in zip(range(len(res)), res):
        if x.status == 4:
            errs.setdefault(int(x.error), []).append(jobs[i].workload.name)
    return {
        "storage": storage, "slots": slots, "offered_jobs": len(jobs), "arrival_rate_jobs_s": rate,
        "arrival_window_s": duration, "step_cap": cap, "submitted": len(ids), "done": len(done),
        "breakup": sum(1 for x in done if x.status == 2), "failed": len(failed),
        "failed_by_error": {str(k2): {"count": len(v), "jobs": v[:8]} for k2, v in errs.items()},
        "backlog_at_end": len(jobs) - len(done) - len(failed),
        "elapsed_s": elapsed, "jobs_per_s": len(done) / elapsed,
        "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
        "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
        "p50_breakup_s": float(np.percentile(latb, 50)) if latb.size else None,
        "p99_breakup_s": float(np.percentile(latb, 99)) if latb.size else None,
        "breakup_step_median": float(np.median([x.breakup_step for x in done if x.status == 2]))
        if latb.size else None,
        "mlups_wall": st["node_updates"] / elapsed / 1e6,
        "mlups_device": st["node_updates"] / (st["device_ms"] / 1e3) / 1e6 if st["device_ms"] > 0 else None,
    }


# ---- main ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mix")
    ap.add_argument("--storage", default=None, help="storage of the timed workload (mix: fp16, others: fp64)")
    ap.add_argument("--size", default=None, help="override domain size NXxNYxNZ (thread workloads)")
    ap.add_argument("--legs", default="kernels,e2e,storages,plain,c3,serve,cpu",
                    help="auxiliary measurements at N=1 (comma list; 'none' for the timed region only)")
    ap.add_argument("--domains", type=int, default=96, help="mix: the first D domains of the manifest "
                                                             "(smaller cases for profiler captures)")
    ap.add_argument("--xchunk", type=int, default=0, help="mix: fixed tile x extent for every domain instead of "
                                                           "the autotuner (profiler captures)")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-cap", type=int, default=6000)
    ap.add_argument("--serve-wall", type=float, default=120.0)
    ap.add_argument("--serve-budget-gb", type=float, default=160.0)
    ap.add_argument("--serve-slots", type=int, default=16,
                    help="resident jobs of the batched server (16 and 48 served the same MLUPS; 16 the shorter "
                         "time to result; 256 left most jobs unfinished at the wall-clock limit)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    legs = set() if world > 1 else set(x for x in args.legs.split(",") if x and x != "none")
    peak, peak_kind = measured_peaks()
    if args.workload == "mix":
        line = mix_main(args, torch, dist, rank, world, local, legs, peak, peak_kind)
    else:
        line = single_main(args, torch, dist, rank, world, local, legs, peak, peak_kind)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def timed_max(torch, dist, ms, local):
    """The slowest rank's device time (symmetry_b200.dist)."""
    from symmetry_b200.dist import max_over_ranks
    return max_over_ranks(torch, dist, ms, device=f"cuda:{local}")


def whole_job_mlups(torch, dist, node_updates, t_max, local):
    """All ranks' node updates over the slowest rank's time (symmetry_b200.dist)."""
    from symmetry_b200.dist import aggregate_mlups, sum_over_ranks
    return aggregate_mlups(sum_over_ranks(torch, dist, node_updates, device=f"cuda:{local}"), t_max)


def mix_main(args, torch, dist, rank, world, local, legs, peak, peak_kind):
    from symmetry_b200 import configs
    from symmetry_b200.lib import Batch, setup_workload
    storage = args.storage or "fp16"
    ws = configs.c4_manifest(storage=storage)[:max(1, min(96, args.domains))]
    nodes = sum(w.nodes for w in ws)
    lattices = [setup_workload(w, device=local) for w in ws]
    B = Batch(lattices)
    if args.xchunk > 0:
        for i in range(len(ws)):
            B.set_xchunk(i, args.xchunk)
        tuned_steps = 0
    else:
        tuned_steps = B.autotune(trial_steps=3)
    cls = lambda nx: 0 if nx <= 32 else (1 if nx <= 48 else 2)  # noqa: E731
    xchunk = {}
    for i, w in enumerate(ws):
        xchunk[cls(w.params.nx)] = B.xchunk(i)
    B.step(args.warmup)
    kps = B.kernels_per_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms = B.step_timed(args.steps)
    torch.cuda.synchronize()
    t_max = timed_max(torch, dist, ms, local)
    value = whole_job_mlups(torch, dist, nodes * args.steps, t_max, local)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32", "fp16": "f16-store/f32"}[storage],
        "data": "synthetic (seeded phase fields, no dataset)",
        "config": {"workload": f"batched mix: {MIX_DESC}, {storage} storage, one CUDA graph per step"
                               + ("" if len(ws) == 96 else f" (first {len(ws)} domains only)"),
                   "nodes": nodes, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 ({2 * 38 * STORE_BYTES[storage] * nodes / 1e9:.1f} GB of "
                         "populations, double buffered)",
                   "xchunk_by_size_class": xchunk, "autotune_steps": tuned_steps},
        "clocks": clk.summary(),
        "gpu_launches": kps * args.steps,
        "gpu_launches_per_step": kps,
    }
    if "kernels" in legs:
        k = leg("kernels", B.step_kernels, min(args.steps, 10))
        if isinstance(k, dict):
            line["roofline"] = k
        else:
            ks = min(args.steps, 10)
            col, ph, sp = k[3] / ks, k[1] / ks, k[2] / ks
            ach = b_collide(storage) * nodes / (col / 1e3) / 1e9
            line["roofline"] = {
                "bound": "hbm", "kernel": "k_collide_batch (fused derivatives+collide+recolour+stream, "
                                          "persistent over the work-tile table)",
                "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                "traffic": collide_traffic(storage, nodes),
                "traffic_source": "ncu dram bytes per node of one captured launch x nodes of this launch",
                "peak_kind": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "algorithmic_bytes_per_node": b_collide(storage), "nodes_per_launch": nodes,
                "ms_per_launch": col}
            line["per_kernel_ms_per_step"] = {
                "eager_total": k[0] / ks, "k_phase_batch": ph, "particle_wall_chains": sp,
                "k_collide_batch": col,
                "phase_gbs": b_phase(storage) * nodes / (ph / 1e3) / 1e9,
                "step_gbs_graph": b_step(storage) * value * 1e6 / world / 1e9,
                "step_frac_graph": b_step(storage) * value * 1e6 / world / 1e9 / peak}
    if "e2e" in legs:
        line["e2e"] = leg("e2e", e2e_batch, torch, lattices, B)
    B.close()
    for L in lattices:
        L.close()
    del lattices, B
    if "storages" in legs:
        line["batched_same_mix_other_storage"] = {
            st: leg("mix_" + st, batched_mix, st, 20, local) for st in ("fp32", "fp64")}
    if "plain" in legs:
        p = leg("plain", plain_fp64, configs.c4_manifest(storage="fp64"), 20, local)
        if "value" in p:
            p["batched_vs_plain"] = value / world / p["value"]
        line["plain_fp64_same_mix"] = p
    if "c3" in legs:
        line["c3_fp64_roofline"] = leg("c3", c3_leg, 20, peak, local)
    if "serve" in legs:
        line["serving"] = {
            "workload": "Poisson arrivals at 20 jobs/s (seed 5): 90% batched-mix domains, 10% 128x128x512 "
                        "threads R=16, 30% with wetting walls (contact angle U[30,150] deg); stop at breakup "
                        f"(min r_eq < 1) or the step cap; arrivals for {args.serve_seconds:.0f} s (the 120 s "
                        f"stream truncated to keep the bench within minutes), step cap {args.serve_cap} (the "
                        "50000 cap lowered; the mix threads with an unstable wavelength break within it), "
                        f"budget {args.serve_budget_gb:.0f} GB, check every 10 steps, wall-clock limit "
                        f"{args.serve_wall:.0f} s per arm: the offered load exceeds capacity, jobs unfinished "
                        "at the limit are the backlog",
            "batched_fp16": leg("serve16", run_serving, "fp16", args.serve_slots, 20.0, args.serve_seconds,
                                args.serve_cap, int(args.serve_budget_gb * 1e9), args.serve_wall, xchunk, local),
            "plain_fp64_one_at_a_time": leg("serve64", run_serving, "fp64", 1, 20.0, args.serve_seconds,
                                            args.serve_cap, int(args.serve_budget_gb * 1e9), args.serve_wall,
                                            None, local),
        }
    if "cpu" in legs:
        line["cpu_baseline"] = leg("cpu", cpu_baseline, mix_sample(4), "the first 4 domains of the batched mix")
    return line


def single_main(args, torch, dist, rank, world, local, legs, peak, peak_kind):
    from symmetry_b200.lib import setup_workload
    storage = args.storage or "fp64"
    w = workload(args.workload, storage, args.size)
    nodes = w.nodes
    L = setup_workload(w, device=local)
    L.step(args.warmup)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms = L.step_timed(args.steps, use_graph=True)[0]
    t_max = timed_max(torch, dist, ms, local)
    value = whole_job_mlups(torch, dist, nodes * args.steps, t_max, local)
    k = L.step_timed(min(args.steps, 20), use_graph=False)
    ks = min(args.steps, 20)
    col, ph = k[3] / ks, k[1] / ks
    ach = b_collide(storage) * nodes / (col / 1e3) / 1e9
    solid = bool(w.params.par or w.params.wall_x)
    line = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": {"fp64": "f64", "fp32": "f32", "fp16": "f16-store/f32"}[storage],
        "data": "synthetic (seeded phase field, no dataset)",
        "config": {"workload": describe(w, storage), "nodes": nodes, "parallelism": f"replicas x{world}",
                   "l2": f"{2 * 38 * STORE_BYTES[storage] * nodes / 1e9:.2f} GB of populations "
                         "(larger than L2 only for the 256x256x512 thread)"},
        "roofline": {"bound": "hbm", "kernel": "k_collide", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": collide_traffic(storage, nodes), "peak_kind": peak_kind,
                     "algorithmic_bytes_per_node": b_collide(storage), "ms_per_launch": col},
        "per_kernel_ms_per_step": {"k_phase": ph, "sparse": k[2] / ks, "k_collide": col,
                                   "step_frac_graph": b_step(storage) * value * 1e6 / world / 1e9 / peak},
        "clocks": clk.summary(),
        "gpu_launches": None if solid else 2 * args.steps,
    }
    if "cpu" in legs:
        line["cpu_baseline"] = leg("cpu", cpu_baseline, thread_sample(w), "a z-slab of the domain")
    L.close()
    return line


if __name__ == "__main__":
    main()

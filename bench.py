#!/usr/bin/env python
"""Benchmark of the per-timestep lattice update (D3Q19 colour-gradient MRT).

One bench step = one lattice update of the whole domain (every node counted,
fluid or solid).  Prints one JSON line (rank 0).

  python bench.py [--gpus N --steps K --warmup W] [--workload c3|c2|c1] [--storage fp64|fp32|fp16]
  python bench.py --impl reference ...   # CPU restatement of the reference (all host threads)

Multi-GPU: the path does not shard (one domain per job); N GPUs run N
independent replicas ("replicas only"), value = all ranks' node updates /
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

STORE_BYTES = {"fp64": 8, "fp32": 4, "fp16": 2}
PHI_BYTES = {"fp64": 8, "fp32": 4, "fp16": 4}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


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


def cpu_baseline(w, steps=None, budget_s=20.0):
    """The oracle (C++ restatement of Source1.f90, all host threads) on a bounded
    sample of the same workload: the full x-y extent with a shorter z."""
    import numpy as np
    from oracle import oracle as orc
    from symmetry_b200 import configs
    p = w.params
    nz = min(p.nz, 32)
    if w.kind == "thread":
        sample = configs.Workload(w.name, p.copy(), "thread", dict(w.gen), w.steps, list(w.particles))
        sample.params.nz = nz
        sample.gen["wavelength"] = float(nz)
    else:
        sample = w
        nz = p.nz
    o = orc.setup_workload(sample)
    o.step(1)
    n = 0
    t0 = time.perf_counter()
    while True:
        o.step(1)
        n += 1
        if time.perf_counter() - t0 > budget_s or (steps and n >= steps):
            break
    dt = time.perf_counter() - t0
    nodes = sample.params.n_nodes
    return {"value": nodes * n / dt / 1e6, "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
            "sample": f"{n} steps of {sample.params.nx}x{sample.params.ny}x{nz} "
                      f"({describe(sample, 'fp64')}), oracle restating Source1.f90, g++ -O3 -fopenmp"}


def run_reference(args):
    """--impl reference: the reference's algorithm on the host cores (the oracle
    port; the Fortran reference cannot be compiled on this image)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = workload(args.workload, "fp64")
    times = []
    from oracle import oracle as orc
    from symmetry_b200 import configs
    p = w.params
    sample = configs.Workload(w.name, p.copy(), w.kind, dict(w.gen), w.steps, list(w.particles))
    if w.kind == "thread":
        sample.params.nz = min(p.nz, 32)
        sample.gen["wavelength"] = float(sample.params.nz)
    o = orc.setup_workload(sample)
    for _ in range(args.warmup):
        o.step(1)
    for _ in range(args.steps):
        t0 = time.perf_counter()
        o.step(1)
        times.append(time.perf_counter() - t0)
    nodes = sample.params.n_nodes
    ms = 1e3 * sum(times) / len(times)
    v = nodes / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": "MLUPS (lattice node updates per second, 1e6)", "value": v,
        "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded phase field)",
        "config": {"workload": describe(w, "fp64"), "nodes_per_step_sample": nodes},
        "cpu_baseline": {"value": v, "unit": "MLUPS", "cores": orc.threads(), "kind": "port",
                         "sample": f"{sample.params.nx}x{sample.params.ny}x{sample.params.nz} slab of the "
                                   "workload per step; C++ restatement of Source1.f90 (no Fortran compiler)"},
        "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def e2e_measure(L, w, reps: int, inner: int):
    """End to end through the public C ABI with pinned host buffers: upload both
    colours' populations and rho_N (Fortran layout), run `inner` lattice steps,
    run calmacros and download the five macroscopic fields."""
    import numpy as np
    import torch
    n = w.params.n_nodes
    shape = (w.params.nx, w.params.ny, w.params.nz)
    ri = torch.empty(19 * n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape + (19,))
    bi = torch.empty(19 * n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape + (19,))
    phi = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape)
    outs = [torch.empty(n, dtype=torch.float64, pin_memory=True).numpy().reshape(shape) for _ in range(5)]
    L.get_into("ri", ri)
    L.get_into("bi", bi)
    L.get_into("rho_N", phi)
    h2d = ri.nbytes + bi.nbytes + phi.nbytes
    d2h = sum(o.nbytes for o in outs)

    def one():
        L.set("rho_N", phi)
        L.set_populations(ri, bi)
        L.step(inner)
        L.call("calmacros")
        for name, o in zip(["rho_N", "rho", "ux", "uy", "uz"], outs):
            L.get_into(name, o)

    one()  # warm-up
    t0 = time.perf_counter()
    for _ in range(reps):
        one()
    dt = time.perf_counter() - t0
    return {"value": n * inner * reps / dt / 1e6, "unit": "MLUPS", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h,
            "step": f"upload ri+bi+rho_N (pinned, Fortran layout) -> {inner} lattice steps -> calmacros -> "
                    "download rho_N,rho,u (one output interval of the reference driver)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3")
    ap.add_argument("--storage", default="fp64")
    ap.add_argument("--size", default=None, help="override domain size NXxNYxNZ (profiling captures)")
    ap.add_argument("--modes", default="fp32,fp16", help="extra storage modes timed on the same workload")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--e2e-inner", type=int, default=100)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from symmetry_b200.lib import setup_workload

    w = workload(args.workload, args.storage, args.size)
    peak, peak_kind = measured_peaks()
    nodes = w.params.n_nodes
    sp, sf = STORE_BYTES[args.storage], PHI_BYTES[args.storage]

    L = setup_workload(w, device=local)
    L.step(args.warmup)
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms = L.step_timed(args.steps, use_graph=False)
    ms_graph = L.step_timed(args.steps, use_graph=True)[0]
    t_max = ms[0]
    if dist:
        t = torch.tensor([ms[0]], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    ms_step = t_max / args.steps
    value = world * nodes * args.steps / (t_max / 1e3) / 1e6
    collide_ms = ms[3] / args.steps
    phase_ms = ms[1] / args.steps
    b_collide = (76 * sp + sf) * nodes          # read+write 38 populations, read phi once
    b_phase = (38 * sp + sf) * nodes            # read 38 populations, write phi
    b_alg = (76 * sp + 2 * sf)                  # per node update (whole step)
    ach = b_collide / (collide_ms / 1e3) / 1e9
    line = {
        "metric": "MLUPS (lattice node updates per second, 1e6) of the per-timestep lattice update",
        "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": {"fp64": "f64", "fp32": "f32", "fp16": "f16-store/f32"}[args.storage],
        "data": "synthetic (seeded phase field, no dataset)",
        "config": {"workload": describe(w, args.storage), "nodes": nodes, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 ({2 * 38 * sp * nodes / 1e9:.1f} GB of populations)"},
        "roofline": {"bound": "hbm", "kernel": "k_collide (fused derivatives+collide+recolour+stream)",
                     "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": None,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_node": 76 * sp + sf,
                     "ms_per_launch": collide_ms},
        "step_roofline": {"b_alg_per_node": b_alg, "achieved_gbs": b_alg * value * 1e6 / world / 1e9,
                          "frac": b_alg * value * 1e6 / world / 1e9 / peak,
                          "phase_kernel_gbs": b_phase / (phase_ms / 1e3) / 1e9 if phase_ms > 0 else None,
                          "phase_ms": phase_ms, "particles_ms": ms[2] / args.steps},
        "graph_replay": {"value": world * nodes * args.steps / (ms_graph / 1e3) / 1e6,
                         "ms_per_step": ms_graph / args.steps},
        "clocks": clk.summary(),
        "gpu_launches": (2 + (0 if not w.params.par else 0)) * args.steps if not (w.params.par or w.params.wall_x)
        else None,
    }
    if w.params.par or w.params.wall_x:
        line["gpu_launches_note"] = "walls/particles add sparse kernels per step"
        line["gpu_launches"] = 2 * args.steps
    # other storage modes on the same workload
    extra = {}
    for m in [x for x in args.modes.split(",") if x and x not in (args.storage, "none")]:
        wm = workload(args.workload, m, args.size)
        Lm = setup_workload(wm, device=local)
        Lm.step(args.warmup)
        mm = Lm.step_timed(args.steps, use_graph=False)
        vm = nodes * args.steps / (mm[0] / 1e3) / 1e6
        spm, sfm = STORE_BYTES[m], PHI_BYTES[m]
        cm = mm[3] / args.steps
        extra[m] = {"value": vm, "unit": "MLUPS", "ms_per_step": mm[0] / args.steps,
                    "speedup_vs_" + args.storage: vm / (value / world),
                    "collide_gbs": (76 * spm + sfm) * nodes / (cm / 1e3) / 1e9,
                    "step_frac": (76 * spm + 2 * sfm) * vm * 1e6 / 1e9 / peak}
        Lm.close()
        del Lm
    if extra:
        line["modes"] = extra
    if not args.no_e2e and rank == 0:
        line["e2e"] = e2e_measure(L, w, reps=2, inner=args.e2e_inner)
    if not args.no_cpu and rank == 0:
        line["cpu_baseline"] = cpu_baseline(w)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

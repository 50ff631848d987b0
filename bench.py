#!/usr/bin/env python
"""bench.py -- grid cells/s of the AVISM hot path (particles -> void catalogue).

Workload (the 512^3 configuration the metric is quoted on): 2^27 particles
Poisson-sampled from a lognormal field (Gaussian random field with P(k) ~ k^-1.2,
sigma_ln = 1) in a periodic L = 500 cMpc box, linear-theory velocities (350 km/s
rms), equal masses; grid 512^3 (ext 640^3), k = 32, SPH density and velocity,
README thresholds.  Synthetic, seeded (1004 + rank).

A step is one pass of the whole level on the GPU: kNN / SPH particle-to-grid,
normalisation, divergence, flags, candidate ordering, cube growth, merging and
post-processing, ending with the catalogue on the host.  The timed path is the
learned one (params.learned = 1: the trained MLP proposes every bin's starting
kNN radius); the plain path (learned = 0) is timed beside it and must give the
identical catalogue.
  value  -- inputs already resident in HBM (device pointers through the C-ABI)
  e2e    -- the same call with pinned host buffers: H2D of the particles and the
            D2H of the catalogue inside the timed region
Inputs (3.5 GB of particles, GBs of grids) exceed the 126 MB L2, so no flush is
needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank processes its own snapshot (iterations of the
reference's FIRST..LAST loop are independent): replicas, weak scaling.
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

METRIC = "grid cells/s end-to-end at 512³, learned+batched vs plain GPU, exact catalogue"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--log2n", type=int, default=27)
    ap.add_argument("--box", type=float, default=500.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stages", action="store_true", help="print per-stage device times to stderr")
    return ap.parse_args()


# ---- clocks sampled during the timed region ----------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and s[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---- distributed plumbing -----------------------------------------------------
def dist_setup(n_gpus: int, backend: str | None = None):
    """(rank, world, local rank) from the torchrun environment; joins the
    process group when world > 1 (NCCL on GPUs, gloo otherwise)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return rank, world, local


def replica_seed(rank: int) -> int:
    """Seed of rank's snapshot: each rank runs its own iteration."""
    return 1004 + rank


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda" if dist.get_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload_params(a):
    from avism_b200._abi import Params
    return Params(nx=a.nx, periodic=1, lado0=a.box, kneighbours=32, flag_vel_interp=1, flag_dens_interp=1,
                  nvoid_max=4_000_000)


def config_dict(a, world):
    return {"workload": f"particles->void catalogue, {a.nx}^3 grid (ext {a.nx + 2 * (a.nx // 8)}^3), "
                        f"2^{a.log2n} particles, L={a.box:g} cMpc periodic, k=32, SPH/SPH",
            "grid": a.nx, "particles": 2 ** a.log2n, "box_cmpc": a.box, "kneighbours": 32,
            "field": "lognormal GRF P(k)~k^-1.2 sigma_ln=1, linear-theory v 350 km/s rms",
            "l2": "inputs > L2 (126 MB); no flush", "parallelism": f"replicas x{world} (one snapshot per rank)"}


# ---- CPU baseline: the oracle on a bounded sample of the same workload -------
def cpu_sample_run(steps: int, warmup: int, seed: int = 1004, nx: int = 128):
    """The C oracle (restatement of the reference's algorithms: k-d tree kNN,
    scatter SPH, serial growth and merge) on a sub-box of the workload with the
    same cell size and particle density: nx^3 cells, L = nx * 500/512 cMpc,
    2^27 (nx/512)^3 particles, periodic.  Returns (cells/s, cores, s per level,
    sample description)."""
    from avism_b200 import synth
    from avism_b200._abi import Params
    from oracle import oracle as O
    box = nx * 500.0 / 512
    n = int(round(2 ** 27 * (nx / 512) ** 3))
    parts = synth.to_reader_units(synth.lognormal(n=n, ng=nx, box=box, index=-1.2, sigma_ln=1.0,
                                                  vrms=350.0, seed=seed))
    p = Params(nx=nx, periodic=1, lado0=box, kneighbours=32, nvoid_max=4_000_000)
    g, _ = O.grid_setup(p)
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        O.run_level(p, parts)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    t = statistics.mean(times)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return nx ** 3 / t, cores, t, (f"oracle port (k-d tree kNN, scatter SPH, serial growth and merge), one full "
                                   f"level per step on a {nx}^3 sub-box ({n} particles, L={box:g} cMpc periodic, "
                                   f"ext {g.ne}^3) with the cell size and particle density of the 512^3 workload; "
                                   f"{t:.2f} s per level; cells/s = {nx}^3 / that time, a per-cell rate "
                                   f"extrapolated to 512^3")


REF_NX = 96     # reference-arm sub-box: one level takes a few seconds on 16 host cores


def run_reference(a):
    """The reference arm: the oracle port on the host cores, every one of the
    --warmup + --steps steps a full level on a REF_NX^3 sub-box of the workload
    (rank 0 only; other ranks exit without work)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    value, cores, t, sample = cpu_sample_run(a.steps, a.warmup, nx=REF_NX)
    box = REF_NX * 500.0 / 512
    cfg = {"workload": f"particles->void catalogue on a {REF_NX}^3 sub-box of the 512^3 workload "
                       f"(L={box:g} cMpc periodic, same cell size and particle density, k=32, SPH/SPH); "
                       f"cells/s is extrapolated per cell to the 512^3 level",
           "grid": REF_NX, "particles": int(round(2 ** 27 * (REF_NX / 512) ** 3)), "box_cmpc": box,
           "kneighbours": 32, "field": "lognormal GRF P(k)~k^-1.2 sigma_ln=1, linear-theory v 350 km/s rms",
           "parallelism": "host threads (OpenMP)"}
    line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": cfg,
            "cpu_baseline": {"value": value, "unit": "cells/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- our arm ----------------------------------------------------------------
# algorithmic bytes per unit of the dominant stages: compulsory reads and writes
# of each stage's inputs and outputs, counted once
ALG_BYTES = {
    # per cell query: the k neighbours' (x,y,z,m,vx,vy,vz,rho) are compulsory once per
    # particle; per cell 3 velocity components written, per particle h read+written
    "cells_knn": lambda n, nc, ne3: 36 * n + 8 * n + 12 * nc,
    "ppart_dens": lambda n, nc, ne3: 20 * n + 4 * n,
    "ddens_scatter": lambda n, nc, ne3: 24 * n + 16 * nc,
    "fill_h_zeros": lambda n, nc, ne3: 20 * n,
    # stencils: DIVER_UNIFORM reads 3 velocity grids and writes one; the flag
    # stencil reads U1CO and DIVERCO and writes one byte per ext cell
    "divergence": lambda n, nc, ne3: 16 * nc,
    "flags": lambda n, nc, ne3: 9 * ne3,
}
HBM_STAGES = ("divergence", "flags")
# DRAM bytes (read + write) per unit of the dominant stage from one ncu capture
# of k_cells_knn_w on the 256^3 / 2^24-particle case of this workload: 0.857 GB
# read + 0.260 GB written for 2^24 cell queries.  The capture is too large to
# take at 512^3 under the profiling size rule; the queries and particles both
# scale by 8, so the traffic is scaled by the cells of the launch.
TRAFFIC_PER_CELL = {"cells_knn": (0.857047040e9 + 0.260322560e9) / 2 ** 24}


def run_ours(a):
    import numpy as np
    import torch
    from avism_b200 import synth
    from avism_b200._abi import Cubes, Voids, ptr  # noqa: F401
    from avism_b200.avism import AvismGPU

    rank, world, local = dist_setup(a.gpus)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    from avism_b200 import proposal
    p = workload_params(a)
    p.learned = 1
    p_plain = workload_params(a)
    n = 2 ** a.log2n
    ncells = a.nx ** 3
    ne3 = (a.nx + 2 * (a.nx // 8)) ** 3
    with torch.no_grad():
        parts = synth.lognormal_torch(n, min(a.nx, 512), a.box, -1.2, 1.0, 350.0, seed=replica_seed(rank), device=dev)
        parts = synth.to_reader_units(parts)
    dev_parts = {k: parts[k].contiguous() for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    host_parts = {k: v.cpu().pin_memory() for k, v in dev_parts.items()}
    torch.cuda.synchronize()
    ctx = AvismGPU(local)
    ctx.proposal_load(proposal.load_weights())    # the trained network (a model load, not timed)

    def step(src, prm, bufs):
        return ctx.run_level(prm, src, bufs=bufs)

    def timed(src, steps, warmup, prm=p):
        # the caller's cube and catalogue arrays, allocated once and reused by
        # every step (as a driver keeps them); each timed run has its own set
        bufs = ctx.level_buffers(prm, capacity=prm.nvoid_max)
        for _ in range(warmup):
            step(src, prm, bufs)
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = ctx.launches()
        stages = []
        e0.record()
        for _ in range(steps):
            r = step(src, prm, bufs)
            stages.append(ctx.stage_times())
        e1.record()
        torch.cuda.synchronize()
        barrier(world)
        ms = e0.elapsed_time(e1) / steps
        return ms, r, stages, ctx.launches() - l0

    sampler = ClockSampler(local)
    with sampler:
        ms_dev, res, stages, launches = timed(dev_parts, a.steps, a.warmup)
        ms_e2e, res_h, stages_h, _ = timed(host_parts, max(1, a.steps), 1)
        ms_plain, res_p, stages_p, _ = timed(dev_parts, max(1, a.steps), 1, p_plain)
    ms_dev = max_over_ranks(ms_dev, world)
    ms_e2e = max_over_ranks(ms_e2e, world)
    ms_plain = max_over_ranks(ms_plain, world)
    # host- and device-input runs, and the learned and plain paths, give one catalogue
    cat_keys = ("indice", "uvoid", "ncellv", "volnew", "gxc", "gyc", "gzc", "eps", "ip", "umean", "mtot")
    same = all(np.array_equal(res["cat"][k], res_h["cat"][k]) for k in cat_keys)
    same_plain = (res["nvoid"] == res_p["nvoid"] and
                  all(np.array_equal(res["cat"][k], res_p["cat"][k]) for k in cat_keys) and
                  all(np.array_equal(res["cubes"][k], res_p["cubes"][k]) for k in res["cubes"]))
    value = world * ncells / (ms_dev / 1e3)
    e2e = world * ncells / (ms_e2e / 1e3)
    # per-stage mean device time (events on the library's stream)
    keys = stages[0].keys()
    st = {k: statistics.mean(s.get(k, 0.0) for s in stages) for k in keys}
    if a.stages and rank == 0:
        print(json.dumps({"stages_ms": st, "nvoid": res["nvoid"], "nvoidt": res["cat"]["nvoidt"]}), file=sys.stderr)
    dom = max((k for k in st if k in ALG_BYTES), key=lambda k: st[k])
    peaks = json.load(open(PEAKS)) if os.path.exists(PEAKS) else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    alg = ALG_BYTES[dom](n, ncells, ne3)
    achieved = alg / (st[dom] / 1e3) / 1e9
    # the HBM-bound stencil stages against the same peak
    stencils = {}
    for k in HBM_STAGES:
        if st.get(k, 0.0) > 0:
            gbs = ALG_BYTES[k](n, ncells, ne3) / (st[k] / 1e3) / 1e9
            stencils[k] = {"ms": round(st[k], 4), "alg_bytes": ALG_BYTES[k](n, ncells, ne3),
                           "achieved_gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    nvoid = res["nvoid"]
    h2d = 7 * 4 * n
    d2h = nvoid * (17 * 4) + nvoid * (15 * 4 + 3 * 4)
    if rank == 0:
        cpu = None
        if not a.no_cpu_baseline:
            v, cores, t, sample = cpu_sample_run(1, 0)
            cpu = {"value": v, "unit": "cells/s", "cores": cores, "kind": "port", "sample": sample}
        line = {"metric": METRIC, "value": value, "unit": "cells/s", "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_dev, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": config_dict(a, world),
                "e2e": {"value": e2e, "unit": "cells/s", "ms_per_step": ms_e2e,
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                             "unit": "GB/s", "frac": achieved / peak,
                             "traffic": TRAFFIC_PER_CELL[dom] * ncells if dom in TRAFFIC_PER_CELL else None,
                             "alg_bytes_per_launch": alg, "ms_per_launch": st[dom],
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback"},
                "cpu_baseline": cpu,
                "clocks": sampler.summary(),
                "gpu_launches": launches,
                "catalogue": {"cubes": nvoid, "voids": res["cat"]["nvoidt"], "host_vs_device_identical": same,
                              "learned_vs_plain_identical": same_plain},
                "path": "learned (MLP starting kNN radius, params.learned = 1)",
                "plain": {"ms_per_step": ms_plain, "value": world * ncells / (ms_plain / 1e3), "unit": "cells/s",
                          "learned_speedup": ms_plain / ms_dev},
                "roofline_stencils": stencils,
                "particles_per_s": {"value": world * n / (ms_dev / 1e3), "e2e": world * n / (ms_e2e / 1e3)},
                "stages_ms": {k: round(v, 3) for k, v in st.items()},
                "stages_ms_plain": {k: round(statistics.mean(s_.get(k, 0.0) for s_ in stages_p), 3)
                                    for k in stages_p[0].keys()}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()

"""Benchmark: particle-timesteps/s of the DEM time step on the periodic
inclined chute workload (200,000 bidisperse flowing spheres, size ratio 2,
two HGrid levels, rough base of fixed spheres, periodic 100 x 50 small
diameters, 24 deg, LinearViscoelasticSlidingFriction, dt = tc/50).

One bench "step" is one dem_step call that advances the whole system by
STEPS_PER_CALL time steps (inputs resident in HBM). `value` counts moving
particles x time steps over all ranks / the slowest rank's device time.
`e2e` is the same metric through the public C ABI with host buffers: every
bench step uploads the state from pinned host memory, runs the same batch and
downloads the state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank runs an independent replica (the time step does not
shard across GPUs on this path: replicas only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-timesteps/s"
STEPS_PER_CALL = 200
WORKLOAD = dict(workload="periodic_chute_200k", packing="close-packed layers (LLLLS), spacing = mean diameter",
                n_flowing=200_000, size_ratio=2, hgrid_levels=2,
                periodic="xy", domain_small_diameters=[100, 50], angle_deg=24, species="LinearViscoelasticSlidingFriction",
                restitution=0.88, friction=0.5, dt="tc/50", time_steps_per_bench_step=STEPS_PER_CALL,
                verlet_skin="0.8 x smallest radius (engine default 0.4)",
                l2="working set >= L2; 256 MiB L2 flush before every timed dem_step call")
# Verlet skin of the neighbour lists for this workload, in smallest radii:
# the flowing chute moves fast enough that halving the rebuilds (skin 0.8)
# outweighs the longer lists (measured 119 vs 122 us per time step); dense,
# slow beds (drum, heaps) are faster with the engine's default 0.4.
SKIN_OVER_RMIN = 0.8


def max_over_ranks(ms: float, device: str) -> float:
    """The largest of the ranks' times (every rank must call it, in the same
    order); the time itself when there is one rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, max_ms: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return units_per_rank * world / (max_ms / 1e3)


def rank_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0:
                    self.samples.append([x.strip() for x in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if len(s) > 3 + k and s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def workload():
    from mercurydpm_fork_b200 import scenarios
    # dense start: close-packed layers at the mean diameter (about 3.7 contacts per particle)
    return scenarios.periodic_chute(n_flow=200_000, seed=2, packing="layers", spacing_factor=1.0)


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def force_kernel_bytes(n, nwords, entries, contacts, wall_contacts, ncomp=3):
    """Algorithmic bytes of one time-step force evaluation (compulsory traffic
    of k_detect + k_contacts + k_sum).

    per particle: read pr, vm, wi, qo (4 x 32 B) + info (16 B) + caller (4 B),
                  write the same 6 arrays to the other buffer (148 B),
                  active-bit words read + written (8 B x words), wall bits (8 B);
    per neighbour-list entry: its index (4 B);
    per contact (a particle pair once, a wall contact once):
                  spring history read + written (2 x 8 B x ncomp).
    Neighbour state gathers are cache hits (sorted order) and not counted, nor
    is the compact contact list the three kernels pass between them.
    """
    per_particle = (4 * 32 + 16 + 4) + (4 * 32 + 16 + 4) + 8 * nwords + 8
    return n * per_particle + 4 * entries + (contacts + wall_contacts) * 2 * 8 * ncomp


def run_ours(args):
    import torch
    rank, world, local = rank_info()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from mercurydpm_fork_b200 import DemEngine, _abi
    sc = workload()
    n_moving = sc.n_moving
    eng = DemEngine(sc.time_step, [sc.instance], sc.species, sc.walls, rotation=True, device=local,
                    skin=SKIN_OVER_RMIN * float(np.min(sc.radius)))
    eng.upload(sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia, sc.species_index, sc.ids)
    eng.step(0)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        eng.step(STEPS_PER_CALL)
    barrier()
    total_ms = 0.0
    launches = 0
    rebuilds = 0
    t0 = time.perf_counter()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            eng.step(STEPS_PER_CALL)
            st = eng.stats()
            total_ms += st["ms"]
            launches += st["kernel_launches"]
            rebuilds += st["rebuilds"]
    barrier()
    wall = time.perf_counter() - t0
    max_ms = max_over_ranks(total_ms, f"cuda:{local}")
    steps_total = args.steps * STEPS_PER_CALL
    value = job_rate(n_moving * steps_total, world, max_ms)

    # roofline of the dominant kernel (time-step force + integration)
    info = eng.stats()
    cnt = eng.counts()
    nwords = info["max_neighbors"] // 32
    fk_ms = eng.time_force_kernel(20)
    fk_bytes = force_kernel_bytes(sc.n, nwords, cnt["list_entries"], cnt["contacts"], cnt["wall_contacts"])
    peak, peak_kind = measured_peak()
    achieved = fk_bytes / (fk_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "force_kernel_traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            traffic = tj.get("bytes_per_launch_scaled")
        except Exception:
            traffic = None

    # end to end through the public API with host buffers
    # (pinned host memory in both directions; each step uploads the full input
    # state and reads back the evolved state: position, velocity, angular
    # velocity, orientation)
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    inputs = [pinned(a) for a in (sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia,
                                  sc.species_index, sc.ids)]
    outputs = dict(position=pinned(np.zeros((sc.n, 3))), velocity=pinned(np.zeros((sc.n, 3))),
                   angular_velocity=pinned(np.zeros((sc.n, 3))), orientation=pinned(np.zeros((sc.n, 4))))
    h2d = sum(a.nbytes for a in inputs)
    d2h = sum(a.nbytes for a in outputs.values())
    e2e_ms = 0.0
    e2e_steps = max(1, min(args.steps, 3))
    barrier()
    for _ in range(e2e_steps):
        t1 = time.perf_counter()
        eng.upload(*inputs)
        eng.step(STEPS_PER_CALL)
        eng.download(out=outputs)
        e2e_ms += (time.perf_counter() - t1) * 1e3
    e2e_value = job_rate(n_moving * e2e_steps * STEPS_PER_CALL, world, max_over_ranks(e2e_ms, f"cuda:{local}"))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sc)

    line = {
        "metric": METRIC, "value": value, "unit": "particle-timesteps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded periodic-chute packing)",
        "config": dict(WORKLOAD, parallelism=f"replicas{world}", n_total=sc.n, n_moving=n_moving),
        "e2e": {"value": e2e_value, "unit": "particle-timesteps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": "force evaluation: k_detect + k_contacts + k_sum (force + integration)", "peak_source": peak_kind,
                     "bytes_per_launch": fk_bytes, "launch_ms": fk_ms},
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "rebuilds": rebuilds,
        "clocks": clocks.summary(),
        "wall_s": wall,
        "contacts": cnt,
    }
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    eng.close()
    if rank == 0:
        print(json.dumps(line))


def cpu_baseline(sc, target_s: float = 15.0):
    """The reference's own OpenMP build on this host's cores, on a bounded
    sample of the same workload (a few time steps of the full system)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import harness as H
    if not H.reference_available("omp"):
        return None
    threads = os.cpu_count() or 1
    # calibrate on a short window, then time a window of about target_s seconds
    t = H.time_reference(sc, 1, 2, threads, "omp")
    nsteps = int(max(2, min(400, target_s / max(t / 2, 1e-6))))
    t = H.time_reference(sc, 2, nsteps, threads, "omp")
    return {"value": sc.n_moving * nsteps / t, "unit": "particle-timesteps/s", "cores": threads,
            "kind": "reference",
            "sample": f"{nsteps} time steps of the full workload after 2 warm-up steps (MercuryDPM OpenMP build, "
                      f"{threads} threads, std::chrono around computeOneTimeStep)"}


def run_reference(args):
    rank, world, _ = rank_info()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import harness as H
    if not H.reference_available("omp"):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
        return
    sc = workload()
    threads = os.cpu_count() or 1
    per_step = max(1, STEPS_PER_CALL // 20)
    t = H.time_reference(sc, args.warmup, per_step * args.steps, threads, "omp")
    value = sc.n_moving * per_step * args.steps / t
    line = {
        "metric": METRIC, "value": value, "unit": "particle-timesteps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded periodic-chute packing)",
        "config": dict(WORKLOAD, parallelism="cpu", time_steps_per_bench_step=per_step), "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-timesteps/s", "cores": threads, "kind": "reference",
                         "sample": f"{per_step} time steps per bench step of the full workload"},
        "e2e": {"value": value, "unit": "particle-timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_profile_target(args):
    """Small, self-terminating run for ncu captures: the bench workload, a
    few time steps, then `--profile-launches` extra launches of the time-step
    force kernel (dem_time_force_kernel). Prints the kernel-launch plan."""
    from mercurydpm_fork_b200 import DemEngine
    sc = workload()
    # direct launches: every kernel of a time step is its own launch in ncu's list
    eng = DemEngine(sc.time_step, [sc.instance], sc.species, sc.walls, rotation=True, use_graphs=False,
                    skin=SKIN_OVER_RMIN * float(np.min(sc.radius)))
    eng.upload(sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia, sc.species_index, sc.ids)
    eng.step(args.profile_steps)
    st = eng.stats()
    ms = eng.time_force_kernel(args.profile_launches)
    cnt = eng.counts()
    print(json.dumps({"profile_steps": args.profile_steps, "force_launches_before_timing": 1 + args.profile_steps,
                      "timed_force_launches": 1 + args.profile_launches, "force_ms": ms, "stats": st,
                      "counts": cnt}))
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-target", action="store_true", help="run the small ncu capture target and exit")
    ap.add_argument("--profile-steps", type=int, default=20)
    ap.add_argument("--profile-launches", type=int, default=2)
    args = ap.parse_args()
    if args.profile_target:
        run_profile_target(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

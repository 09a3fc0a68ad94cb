"""Benchmark: particle-timesteps/s of the DEM time step on the 1,000,000-sphere
rotating drum (size ratio 3, 10 % large by number, Hertz-Mindlin with rolling
and torsion friction, cylinder of 60 small diameters length rotating at
1 rad/s about x, two flat caps, dt = 0.02 x the Hertz collision time of two
small spheres at 1 m/s), bed started as a lattice whose neighbours overlap by
0.1 % of a diameter (scenarios.dense_drum).

Both arms time the SAME window of time steps from the SAME initial state:
with W warm-up and K timed bench steps of STEPS_PER_CALL time steps each, the
window is time steps W*S+1 .. (W+K)*S after the initial force evaluation
(S = STEPS_PER_CALL). The bed relaxes its initial overlaps over its first
~100 steps and loosens afterwards, so the cost of a step depends on where the
window lies; both arms report the contacts at the window's start and end.

* `value` (ours): moving particles x time steps over all ranks / the slowest
  rank's device time (CUDA events of each dem_step call on the engine's
  stream; inputs resident in HBM; a 256 MiB buffer is written before every
  timed call to flush L2).
* `e2e` (ours): the same metric through the public C ABI with host buffers:
  one e2e step uploads the initial state from pinned host memory, runs the
  initial evaluation and the (W+K)*S time steps of the window, and downloads
  the state into pinned host memory (host wall clock around the calls).
* `--impl reference`: the reference (MercuryDPM's OpenMP build, oracle/_ref,
  every host thread) on the same input and the same window: W*S untimed
  steps, then K*S steps timed with std::chrono around computeOneTimeStep.
  That process maps no library of this repository's engine.

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
STEPS_PER_CALL = 5
# time steps of the reference's CPU baseline sample inside our arm's run
# (about 10-20 s on 16 host cores)
CPU_SAMPLE_STEPS = 12


def workload_config(steps: int, warmup: int) -> dict:
    from mercurydpm_fork_b200 import scenarios
    s = STEPS_PER_CALL
    return dict(workload="rotating_drum_1M_dense_bed", n=1_000_000, small_fraction=0.9, size_ratio=3,
                species="HertzianViscoelasticMindlinRollingTorsion", E_eff=1e7, poisson=0.3,
                shear_modulus="E/2 (1 + nu), the reference's setEffectiveElasticModulusAndPoissonRatio",
                mu=0.4, mu_rolling=0.05, restitution=0.7, density=2000, omega_rad_s=1.0,
                dt="0.02 x getCollisionTime(d_small, rho, 1 m/s)",
                drum_radius_d=scenarios.DRUM_RADIUS_D, drum_length_d=60,
                deviation=("radius 175 d instead of 120 d: 1M spheres of this size mix hold 0.69 of a "
                           "120 d x 60 d cylinder's volume; 0.33 at 175 d"),
                start="lattice bed, neighbour spacing 0.999 d, jitter +-0.005 d, at rest",
                time_steps_per_bench_step=s, window_time_steps=[warmup * s + 1, (warmup + steps) * s],
                l2="working set > L2 (126 MB); 256 MiB written before every timed dem_step call",
                skin="0.4 x smallest radius (engine default)")


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
    return scenarios.dense_drum()


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# Algorithmic bytes per live contact (pair or wall contact) of one time step:
# its 8-byte key read and written, and every spring of its law (3 FP64 each)
# read and written.
CONTACT_BYTES = {1: 64, 2: 160, 3: 64, 4: 160, 0: 16}  # DEM_FRICTION_*: sliding, rolling+torsion, Mindlin, ...
PARTICLE_BYTES = 248


def force_step_bytes(n: int, contacts: int, wall_contacts: int, friction_law: int) -> int:
    """Algorithmic (compulsory) bytes of one time step's force evaluation and
    integration, the model B_step = N B_p + C B_c:

    B_p = 248 B per particle: x, v, omega in FP64 read and written (144 B);
          radius, inverse mass and inertia, species and flags (24 B); force
          and torque written once and read once (48 B); a cell-relative
          float4 position written once and read once (32 B);
    B_c per live contact: its key (8 B) read and written plus each spring of
          the law (3 x 8 B) read and written: 64 B for sliding or Mindlin
          friction, 160 B with rolling and torsion springs.
    The neighbour-list rebuild is a separate kernel, not counted here."""
    return n * PARTICLE_BYTES + (contacts + wall_contacts) * CONTACT_BYTES[friction_law]


def run_ours(args):
    import torch
    rank, world, local = rank_info()
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    torch.cuda.set_device(local)
    from mercurydpm_fork_b200 import DemEngine
    sc = workload()
    n_moving = sc.n_moving
    S = STEPS_PER_CALL
    eng = DemEngine(sc.time_step, [sc.instance], sc.species, sc.walls, rotation=True, device=local)
    eng.upload(sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia, sc.species_index, sc.ids)
    eng.step(0)  # the initial force evaluation (DPMBase::initialiseSolve)
    # launch shapes of the force kernels measured on this state (dem_autotune:
    # spare buffers only, the simulation state does not change)
    tuning = eng.autotune(reps=10)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        eng.step(S)
    barrier()
    cnt_start = eng.counts()
    total_ms = 0.0
    launches = 0
    rebuilds = 0
    t0 = time.perf_counter()
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            eng.step(S)
            st = eng.stats()
            total_ms += st["ms"]
            launches += st["kernel_launches"]
            rebuilds += st["rebuilds"]
    barrier()
    wall = time.perf_counter() - t0
    cnt_end = eng.counts()
    max_ms = max_over_ranks(total_ms, f"cuda:{local}")
    steps_total = args.steps * S
    value = job_rate(n_moving * steps_total, world, max_ms)

    # roofline of the dominant kernel: one time step's force evaluation and
    # integration (k_detect + k_contacts + k_sum), timed with CUDA events on
    # the engine's stream at the state where the timed window ended
    fk_ms = eng.time_force_kernel(20)
    cnt = eng.counts()
    fk_bytes = force_step_bytes(sc.n, cnt["contacts"], cnt["wall_contacts"], sc.species[0].friction_law)
    peak, peak_kind = measured_peak()
    achieved = fk_bytes / (fk_ms / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "force_kernel_traffic.json")
    if os.path.exists(tpath):
        try:
            tj = json.load(open(tpath))
            if tj.get("workload") == "rotating_drum_1M_dense_bed":
                traffic = tj.get("bytes_per_launch_scaled")
        except Exception:
            traffic = None

    # end to end through the public API with host buffers in pinned memory:
    # upload of the initial state, the initial evaluation, the whole window,
    # download of the evolved state
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    inputs = [pinned(a) for a in (sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia,
                                  sc.species_index, sc.ids)]
    outputs = dict(position=pinned(np.zeros((sc.n, 3))), velocity=pinned(np.zeros((sc.n, 3))),
                   angular_velocity=pinned(np.zeros((sc.n, 3))), orientation=pinned(np.zeros((sc.n, 4))))
    h2d = sum(a.nbytes for a in inputs)
    d2h = sum(a.nbytes for a in outputs.values())
    window = (args.warmup + args.steps) * S
    e2e_runs = 2
    e2e_ms = 0.0
    barrier()
    for _ in range(e2e_runs):
        t1 = time.perf_counter()
        eng.upload(*inputs)
        eng.step(0)
        eng.step(window)
        eng.download(out=outputs)
        e2e_ms += (time.perf_counter() - t1) * 1e3
    e2e_value = job_rate(n_moving * e2e_runs * window, world, max_over_ranks(e2e_ms, f"cuda:{local}"))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(sc, args.warmup * S)

    line = {
        "metric": METRIC, "value": value, "unit": "particle-timesteps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": max_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice bed in a rotating drum)",
        "config": dict(workload_config(args.steps, args.warmup), parallelism=f"replicas{world}", n_total=sc.n,
                       n_moving=n_moving, contacts_window_start=cnt_start, contacts_window_end=cnt_end,
                       tuning=tuning),
        "e2e": {"value": e2e_value, "unit": "particle-timesteps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "step": f"upload + initial evaluation + {window} time steps + download, {e2e_runs} runs"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic,
                     "kernel": "one time step's force evaluation + integration: k_detect + k_contacts + k_sum",
                     "peak_source": peak_kind, "bytes_per_launch": fk_bytes, "launch_ms": fk_ms,
                     "bytes_model": "N x 248 B + C x B_c (B_c = 160 B with rolling and torsion springs)"},
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


def cpu_baseline(sc, warmup_steps: int):
    """The reference's own OpenMP build on this host's cores, on a bounded
    sample of the same window: the first CPU_SAMPLE_STEPS time steps after the
    warm-up steps."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import harness as H
    if not H.reference_available("omp"):
        return None
    threads = os.cpu_count() or 1
    r = H.time_reference_window(sc, warmup_steps, CPU_SAMPLE_STEPS, threads, "omp")
    return {"value": sc.n_moving * CPU_SAMPLE_STEPS / r["seconds"], "unit": "particle-timesteps/s", "cores": threads,
            "kind": "reference",
            "sample": f"time steps {warmup_steps + 1}..{warmup_steps + CPU_SAMPLE_STEPS} of the workload "
                      f"(MercuryDPM OpenMP build, {threads} threads, std::chrono around computeOneTimeStep); "
                      f"interactions {r['interactions_start']} -> {r['interactions_end']}"}


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
    S = STEPS_PER_CALL
    r = H.time_reference_window(sc, args.warmup * S, args.steps * S, threads, "omp")
    t = r["seconds"]
    value = sc.n_moving * S * args.steps / t
    line = {
        "metric": METRIC, "value": value, "unit": "particle-timesteps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded lattice bed in a rotating drum)",
        "config": dict(workload_config(args.steps, args.warmup), parallelism="cpu", n_total=sc.n,
                       n_moving=sc.n_moving, interactions_window_start=r["interactions_start"],
                       interactions_window_end=r["interactions_end"]),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "particle-timesteps/s", "cores": threads, "kind": "reference",
                         "sample": f"time steps {args.warmup * S + 1}..{(args.warmup + args.steps) * S} of the "
                                   f"workload, {S} per bench step (MercuryDPM OpenMP build, {threads} threads)"},
        "e2e": {"value": value, "unit": "particle-timesteps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "native_so_loaded": loaded_shared_objects(),
    }
    print(json.dumps(line))


def loaded_shared_objects() -> list:
    """Shared objects of this repository mapped by this process."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so")}
    except OSError:
        return []
    return sorted(os.path.relpath(p, ROOT) for p in paths if p.startswith(ROOT))


def run_profile_target(args):
    """Small, self-terminating run for ncu captures: the drum with
    --profile-n spheres (default 200,000), a few time steps, then
    `--profile-launches` extra launches of the time-step force kernel
    (dem_time_force_kernel). Prints the kernel-launch plan."""
    from mercurydpm_fork_b200 import DemEngine, scenarios
    sc = scenarios.dense_drum(n=args.profile_n)
    # direct launches: every kernel of a time step is its own launch in ncu's list
    eng = DemEngine(sc.time_step, [sc.instance], sc.species, sc.walls, rotation=True, use_graphs=False)
    eng.upload(sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia, sc.species_index, sc.ids)
    eng.step(args.profile_steps)
    st = eng.stats()
    ms = eng.time_force_kernel(args.profile_launches)
    cnt = eng.counts()
    print(json.dumps({"profile_n": sc.n, "profile_steps": args.profile_steps,
                      "force_launches_before_timing": 1 + args.profile_steps,
                      "timed_force_launches": 1 + args.profile_launches, "force_ms": ms, "stats": st,
                      "counts": cnt}))
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-target", action="store_true", help="run the small ncu capture target and exit")
    ap.add_argument("--profile-n", type=int, default=200_000)
    ap.add_argument("--profile-steps", type=int, default=20)
    ap.add_argument("--profile-launches", type=int, default=2)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    if args.profile_target:
        run_profile_target(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

"""Throughput of the workloads other than the headline bench (bench.py):

    python -m mercurydpm_fork_b200.measure chute       # 200k periodic chute, linear + sliding friction, 2 HGrid levels
    python -m mercurydpm_fork_b200.measure drum        # 1M-sphere rotating drum, Hertz-Mindlin (loose start)
    python -m mercurydpm_fork_b200.measure drum_dense  # the same drum started as a touching lattice bed
    python -m mercurydpm_fork_b200.measure heaps       # 4,096 calibration heaps in one handle (steps=40000: the whole run)
    python -m mercurydpm_fork_b200.measure surrogate   # MLP inference / training on the tensor cores
    python -m mercurydpm_fork_b200.measure calibration # calibrations per hour at 2 % response error
    python -m mercurydpm_fork_b200.measure c5          # wall time to 2 %: surrogate-guided / plain batched DEM
    python -m mercurydpm_fork_b200.measure cg          # Gaussian CG of the 200k chute (XZ 100 x 1 x 50)
    python -m mercurydpm_fork_b200.measure triangles   # 200k spheres settling on a 32-triangle mesh floor

Each prints one JSON line. Device time comes from CUDA events (dem_step's own
events for DEM; torch events around the calls for the surrogate).
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np


def _time_dem(e, n_moving, steps_per_call=200, calls=5, warmup=2):
    e.step(0)
    for _ in range(warmup):
        e.step(steps_per_call)
    ms, rebuilds = 0.0, 0
    for _ in range(calls):
        e.step(steps_per_call)
        st = e.stats()
        ms += st["ms"]
        rebuilds += st["rebuilds"]
    return dict(value=n_moving * steps_per_call * calls / (ms / 1e3), unit="particle-timesteps/s",
                ms_per_time_step=ms / (steps_per_call * calls), rebuilds_per_1000_steps=1000.0 * rebuilds /
                (steps_per_call * calls))


def chute(skin_over_rmin=0.8):
    """The periodic inclined chute: 200,000 bidisperse flowing spheres (size
    ratio 2, two HGrid levels) over a rough base of fixed spheres, periodic
    100 x 50 small diameters, 24 deg, LinearViscoelasticSlidingFriction,
    dt = tc/50, started as close-packed layers. Verlet skin 0.8 x the smallest
    radius: the chute flows fast enough that halving the rebuilds outweighs
    the longer lists (measured 119 vs 122 us per time step)."""
    from . import scenarios
    sc = scenarios.periodic_chute(n_flow=200_000, seed=2, packing="layers", spacing_factor=1.0)
    e = sc.engine(skin=skin_over_rmin * float(np.min(sc.radius)))
    out = _time_dem(e, sc.n_moving)
    out["counts"] = e.counts()
    e.close()
    out.update(workload="periodic_chute_200k", n=sc.n, n_moving=sc.n_moving, dt=sc.time_step,
               species="LinearViscoelasticSlidingFriction")
    return out


def drum(n=1_000_000, radius_d=175.0, length_d=60.0, site_spacing=1.02, workload="rotating_drum"):
    from . import scenarios
    sc = scenarios.rotating_drum(n=n, radius_d=radius_d, length_d=length_d, vstd=0.0, site_spacing=site_spacing)
    e = sc.engine()
    out = _time_dem(e, sc.n_moving)
    out["counts"] = e.counts()
    e.close()
    out.update(workload=workload, site_spacing_d=site_spacing, n=sc.n, radius_d=radius_d, length_d=length_d,
               solid_fraction_of_drum=sc.info["solid_fraction_of_drum"], dt=sc.time_step,
               species="HertzianViscoelasticMindlinRollingTorsion")
    return out


def drum_dense():
    """The drum with its bed started as a lattice whose neighbours overlap by
    0.1 % of a diameter: every sphere is in contact from the first step, as in
    a settled bed (the loose start of `drum` spends the timed steps in free
    fall)."""
    return drum(site_spacing=0.999, workload="rotating_drum_dense_bed")


def heaps(n_instances=4096, seed=1, steps=0, max_contacts=6):
    """The calibration batch of heaps in ONE engine handle: n_instances heaps
    of U[500, 8000] spheres (17.4M spheres for 4,096), each with its own
    floor, deletion plane and species. Spring history is stored per contact,
    sized by max_contacts per sphere (a settled heap has about 3). With
    steps = 0: throughput over 1,000 steps of the pouring phase; with
    steps > 0: the whole run of that many steps (40,000 for the heap
    procedure), device time summed over its dem_step calls, then the per-heap
    outputs. Reports the device memory the handle holds."""
    from . import calibration as cal
    n_instances, seed, steps, max_contacts = int(n_instances), int(seed), int(steps), int(max_contacts)
    t0 = time.perf_counter()
    b, params, R = cal.heap_batch(n_instances, seed=seed)
    t1 = time.perf_counter()
    e = b.engine(max_contacts=max_contacts)
    mem = e.memory()
    if steps > 0:
        t2 = time.perf_counter()
        res = cal.run_heaps(b, R, steps=steps, engine=e)
        wall = time.perf_counter() - t2
        counts = e.counts()
        e.close()
        ms = res["device_ms"]
        aor = res["aor_reference"]
        out = dict(value=b.n * steps / (ms / 1e3), unit="particle-timesteps/s", steps=steps,
                   ms_per_time_step=ms / steps, wall_s=wall, device_s=ms / 1e3,
                   heaps_per_hour=n_instances * 3600.0 / wall,
                   aor_reference_deg=dict(median=float(np.nanmedian(aor)), min=float(np.nanmin(aor)),
                                          max=float(np.nanmax(aor)), finite=int(np.isfinite(aor).sum())),
                   remaining_fraction=float(res["n_remaining"].sum() / b.n), counts=counts)
    else:
        out = _time_dem(e, b.n, steps_per_call=200, calls=5)
        out["counts"] = e.counts()
        e.close()
    out.update(workload="calibration_heaps", instances=n_instances, n_total=b.n, build_s=t1 - t0,
               instance_timesteps_per_s=out["value"] / b.n * n_instances, device_bytes=mem["device_bytes"],
               device_bytes_per_sphere=mem["device_bytes"] / b.n, contact_capacity=mem["contact_capacity"],
               max_contacts=max_contacts)
    return out


def heap_pin():
    """The three cased heaps of tests/golden/heap_aor.json through
    CalibrationHeap's procedure on the engine (calibration.heap_procedure):
    angle of repose, casing removal time and particles left, next to the
    reference Kernel's serial and 4-thread results in that file."""
    import os
    from . import calibration as cal
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    gold = json.load(open(os.path.join(root, "tests", "golden", "heap_aor.json")))
    rows = []
    for g in gold["heaps"]:
        sc, R = cal.cased_heap_scenario(cal.HeapParams(**g["params"]))
        t0 = time.perf_counter()
        ours = cal.heap_procedure(sc, R)
        rows.append(dict(params=g["params"], engine=ours, engine_wall_s=time.perf_counter() - t0,
                         reference_serial=g["serial"], reference_omp4=g["omp4"]))
    return dict(workload="calibration_heap_procedure", heaps=rows)


def surrogate(batch=65536, train_batch=1024, reps=20):
    import torch
    from .surrogate import Surrogate
    s = Surrogate(capacity=batch, seed=0)
    rng = np.random.default_rng(0)
    x = rng.uniform(size=(batch, 4)).astype(np.float32)
    y = rng.uniform(size=(batch, 3)).astype(np.float32)
    s.predict(x)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        s.predict(x)
    t_inf = (time.perf_counter() - t0) / reps
    dev_ms = s.time_forward(batch, reps)
    s.train_step(x[:train_batch], y[:train_batch])
    t0 = time.perf_counter()
    for _ in range(reps):
        s.train_step(x[:train_batch], y[:train_batch])
    t_train = (time.perf_counter() - t0) / reps
    s.close()
    flop = 2 * (4 * 256 + 2 * 256 * 256 + 256 * 3)
    return dict(workload="surrogate", inference_batch=batch, inference_ms=t_inf * 1e3,
                inference_tflops=flop * batch / t_inf / 1e12, inference_device_ms=dev_ms,
                inference_device_tflops=flop * batch / (dev_ms / 1e3) / 1e12, train_batch=train_batch,
                train_step_ms=t_train * 1e3,
                note="inference_ms / train_step_ms: host-to-host per call; inference_device_ms: CUDA events")


def calibration(n_train=2048, n_targets=16, tol=0.02, rounds=4, proposals=256, seed=3, chunk=2048):
    """Calibrations per hour at `tol` response error: training heaps from
    batched DEM, the surrogate trained on them, then the held-out targets
    (parameters drawn from the same box, their responses from DEM) calibrated
    together by calibration.calibrate_batch, so each round of all targets'
    proposals is one batched DEM run; timed host to host. Every heap is the
    600-sphere heap of `calibration.heap_responses` (20,000 steps)."""
    from . import calibration as cal
    from .surrogate import Surrogate
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    x = cal.sample_params(rng, n_train)
    y = cal.heap_responses(x)
    t_data = time.perf_counter() - t0
    s = Surrogate(capacity=65536, seed=0)
    s.fit_normalisation(x, y)
    t0 = time.perf_counter()
    s.fit(x, y, epochs=200, batch=1024)
    t_train = time.perf_counter() - t0
    pt = cal.sample_params(rng, n_targets)
    targets = cal.heap_responses(pt)
    t0 = time.perf_counter()
    res = cal.calibrate_batch(targets, lambda p: cal.heap_responses(p, chunk=chunk), s, rounds=rounds,
                              proposals=proposals, candidates=65_536, tol=tol, seed=seed, data=(x, y))
    t_cal = time.perf_counter() - t0
    s.close()
    errors = [r["best_error"] for r in res]
    ok = [e <= tol for e in errors]
    per = t_cal / n_targets
    return dict(workload="calibration", value=3600.0 / per, unit="calibrations/hour", tol=tol,
                succeeded=int(sum(ok)), targets=n_targets, seconds_all_targets=t_cal, seconds_per_calibration=per,
                rounds=[r["rounds"] for r in res], best_errors=[round(e, 5) for e in errors],
                proposals_per_round=proposals, heaps_per_dem_batch=chunk, training_runs=n_train, training_data_s=t_data, training_s=t_train,
                per_hour_with_training_amortised_over_100=3600.0 / (per + (t_data + t_train) / 100.0),
                heap="600 spheres, 20,000 steps, lognormal PSD, rough floor disk (calibration.heap_responses)")


def c5(n=2000, steps=40_000, n_train=1024, n_targets=128, tol=0.02, proposals=64, surrogate_proposals=8, rounds=4,
       plain_rounds=8, seed=3, chunk=4096):
    """The surrogate claim as a wall-time ratio: the same held-out targets
    (responses of DEM heaps at parameters drawn from the box) calibrated to
    `tol` twice on this GPU, timed host to host --
      surrogate-guided: the training heaps (n_train DEM runs), the network's
      training, then calibration.calibrate_batch with the surrogate, each
      target proposing its `surrogate_proposals` best-predicted candidates per
      round;
      plain: calibration.calibrate_batch without it, each target proposing
      `proposals` uniform parameter sets per round, up to plain_rounds rounds.
    Every heap has n spheres (a calibration campaign fixes the sample size;
    C4's heaps range over U[500, 8000]) and runs `steps` time steps; a
    round's proposals for all targets are one batched DEM call. ratio =
    surrogate-guided seconds / plain seconds (if the plain search stopped at
    its round cap before every target reached tol, its time is a lower bound
    and the ratio an upper one)."""
    from . import calibration as cal
    from .surrogate import Surrogate
    n, steps, n_train, n_targets = int(n), int(steps), int(n_train), int(n_targets)
    proposals, surrogate_proposals = int(proposals), int(surrogate_proposals)
    rounds, plain_rounds, seed, chunk, tol = int(rounds), int(plain_rounds), int(seed), int(chunk), float(tol)
    dem = lambda p: cal.heap_responses(p, n=n, steps=steps, chunk=chunk)
    rng = np.random.default_rng(seed)
    pt = cal.sample_params(rng, n_targets)
    targets = dem(pt)
    # surrogate-guided
    t0 = time.perf_counter()
    x = cal.sample_params(rng, n_train)
    y = dem(x)
    t_data = time.perf_counter() - t0
    s = Surrogate(capacity=65536, seed=0)
    s.fit_normalisation(x, y)
    s.fit(x, y, epochs=200, batch=1024)
    t_train = time.perf_counter() - t0 - t_data
    res_s = cal.calibrate_batch(targets, dem, s, rounds=rounds, proposals=surrogate_proposals, candidates=65_536,
                                tol=tol, seed=seed, data=(x, y))
    t_surr = time.perf_counter() - t0
    s.close()
    # plain batched DEM
    t0 = time.perf_counter()
    res_p = cal.calibrate_batch(targets, dem, None, rounds=plain_rounds, proposals=proposals, tol=tol, seed=seed + 1)
    t_plain = time.perf_counter() - t0
    ok_s = [r["best_error"] <= tol for r in res_s]
    ok_p = [r["best_error"] <= tol for r in res_p]
    return dict(workload="calibration_c5", metric="wall-time ratio, surrogate-guided / plain batched DEM",
                value=t_surr / t_plain, tol=tol, targets=n_targets, heap_spheres=n, heap_steps=steps,
                surrogate=dict(seconds=t_surr, training_data_s=t_data, training_s=t_train, succeeded=int(sum(ok_s)),
                               proposals_per_round=surrogate_proposals, rounds_histogram=np.bincount(
                                   [r["rounds"] for r in res_s]).tolist(),
                               dem_runs=n_train + sum(r["dem_runs"] for r in res_s),
                               median_best_error=float(np.median([r["best_error"] for r in res_s]))),
                plain=dict(seconds=t_plain, succeeded=int(sum(ok_p)), proposals_per_round=proposals,
                           rounds_histogram=np.bincount([r["rounds"] for r in res_p]).tolist(),
                           dem_runs=sum(r["dem_runs"] for r in res_p), round_cap=plain_rounds,
                           median_best_error=float(np.median([r["best_error"] for r in res_p]))),
                plain_time_is_lower_bound=not all(ok_p))


def cg(reps=10, steps_between=1000):
    """Gaussian coarse-graining of the 200k periodic chute on an XZ grid of
    100 x 1 x 50 points, width one small diameter, cutoff 3 widths (the
    chute config's CG), evaluated after a flowing phase: ms per evaluation
    host to host (fields copied back), and its share of a 1,000-step
    interval."""
    from . import scenarios
    from ._abi import DEM_CG_XZ
    reps, steps_between = int(reps), int(steps_between)
    sc = scenarios.periodic_chute(n_flow=200_000, seed=2, packing="layers", spacing_factor=1.0)
    e = sc.engine()
    e.step(0)
    e.step(200)
    d_small = 1e-3
    x = e.download()["position"]
    inst = sc.instance
    lo = (inst.periodic_min[0], inst.periodic_min[1], float(inst.domain_min[2]))
    hi = (inst.periodic_max[0], inst.periodic_max[1], float(x[:, 2].max()) + d_small)
    n = (100, 1, 50)
    e.cg(DEM_CG_XZ, n, lo, hi, d_small)
    t0 = time.perf_counter()
    for _ in range(reps):
        f = e.cg(DEM_CG_XZ, n, lo, hi, d_small)
    cg_ms = (time.perf_counter() - t0) / reps * 1e3
    e.step(steps_between)
    step_ms = e.stats()["ms"]
    cnt = e.counts()
    e.close()
    return dict(workload="cg_chute_xz", value=cg_ms, unit="ms per CG evaluation (host to host)", points=list(n),
                fields=int(f.shape[1]), width=d_small, cutoff_widths=3.0, particles=sc.n, contacts=cnt["contacts"],
                steps_between=steps_between, step_loop_ms=step_ms,
                cg_share_of_interval=cg_ms / (cg_ms + step_ms))


def triangles(n=200_000, settle_steps=40_000, drop_d=1.0, v0=0.0):
    """The triangle_floor scenario after `settle_steps` steps (the bed has
    landed on the mesh), then timed; counts of triangle contacts reported."""
    from . import scenarios
    sc = scenarios.triangle_floor(n=int(n), drop_d=float(drop_d), v0=float(v0))
    settle_steps = int(settle_steps)
    e = sc.engine()
    e.step(settle_steps)
    out = _time_dem(e, sc.n_moving)
    c = e.contacts()
    out["counts"] = e.counts()
    out["triangle_contacts"] = int(np.count_nonzero(c["is_wall"]))
    e.close()
    out.update(workload="triangle_floor", n=sc.n, triangles=sc.info["triangles"], group=sc.info["group"],
               layers=sc.info["layers"], settle_steps=settle_steps, dt=sc.time_step,
               species="LinearViscoelasticSlidingFriction")
    return out


if __name__ == "__main__":
    which = sys.argv[1] if len(sys.argv) > 1 else "drum"
    kwargs = dict(a.split("=", 1) for a in sys.argv[2:])  # e.g. triangles n=20000 settle_steps=2000
    fn = dict(chute=chute, drum=drum, drum_dense=drum_dense, heaps=heaps, surrogate=surrogate, calibration=calibration,
              c5=c5, cg=cg, triangles=triangles, heap_pin=heap_pin)[which]
    print(json.dumps(fn(**kwargs)))

"""Batched heap-formation runs for calibration (the reference's
Drivers/Calibration/CalibrationHeap.cpp and Calibration.h, run as thousands of
independent instances in one engine handle).

Each instance: spheres with a lognormal size distribution poured from a
seeded column onto a frictional floor disk (AxisymmetricIntersectionOfWalls,
CalibrationHeap.cpp:86-91) with a DeletionBoundary below the floor
(CalibrationHeap.cpp:129-131); species LinearViscoelasticFrictionSpecies set
up as Calibration::setSpecies does (Calibration.h:147-186): collision time
and restitution for the smallest particle's mass, sliding stiffness and
dissipation 2/7 of the normal ones, rolling and torsion 2/5, time step 0.05
collision times, and a wall species whose mixed sliding and rolling friction
are max(1, rolling) and max(1, sliding).

Outputs per instance:
* the reference's angle of repose, atan(4 COM_z / R_base) in degrees
  (CalibrationHeap.cpp:139-150);
* an angle of repose fitted to the surface particles (the highest particle of
  each radial bin, a least-squares line z(r) over 0.2-0.8 R_base);
* the packing fraction of the heap core (solid volume in r < R_base / 3 up to
  the fitted surface, divided by that volume);
* the kinetic energy trace (one value per trace interval).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import _abi
from .engine import Instance, axisymmetric_wall, species_pair
from .host import PI, linear_collision_time_restitution, sphere_inv_mass_inertia
from .scenarios import Batch, Scenario, batch


@dataclass
class HeapParams:
    n: int
    sigma: float        # lognormal width of the radii
    mu: float           # sliding friction
    mu_r: float         # rolling friction
    restitution: float
    seed: int


def heap_species(tc: float, eps: float, mass_min: float, mu: float, mu_r: float) -> list:
    """Species table of one heap instance: 0 = particles, 1 = the floor's
    frictional wall species (Calibration.h:161-186)."""
    k, g = linear_collision_time_restitution(tc, eps, mass_min)

    def sp(mu_s, mu_roll):
        return species_pair(normal_law=_abi.DEM_NORMAL_LINEAR_VISCOELASTIC, friction_law=_abi.DEM_FRICTION_ROLLING_TORSION,
                            stiffness=k, dissipation=g,
                            sliding_stiffness=2. / 7. * k, sliding_dissipation=2. / 7. * g,
                            sliding_mu=mu_s, sliding_mu_static=mu_s,
                            rolling_stiffness=2. / 5. * k, rolling_dissipation=2. / 5. * g,
                            rolling_mu=mu_roll, rolling_mu_static=mu_roll,
                            torsion_stiffness=2. / 5. * k, torsion_dissipation=2. / 5. * g,
                            torsion_mu=0.0, torsion_mu_static=0.0)
    pp = sp(mu, mu_r)
    pw = sp(max(1.0, mu_r), max(1.0, mu))  # the reference sets them crosswise (Calibration.h:183-184)
    return [pp, pw, pw, pp]


def lognormal_radii(rng, n: int, sigma: float, r50: float, clip: float = 2.0) -> np.ndarray:
    z = np.clip(rng.normal(size=n), -clip, clip)
    return r50 * np.exp(sigma * z)


def heap_scenario(p: HeapParams, d50: float = 1e-3, density: float = 2000.0, tc: float = 1e-4,
                  base_radius_d: float = 30.0, column_radius_d: float = 10.0, spacing: float = 1.05,
                  v0: float = 0.0):
    """One heap: returns (Scenario, deletion planes, base radius). v0 is an
    initial downward speed (0 for a pour from rest)."""
    rng = np.random.Generator(np.random.PCG64(p.seed))
    radius = lognormal_radii(rng, p.n, p.sigma, 0.5 * d50)
    R = base_radius_d * d50
    Rc = column_radius_d * d50
    s = spacing * 2.0 * radius.max()
    # column sites: a square lattice clipped to the column, layer by layer
    m = int(Rc // s)
    g = (np.arange(-m, m + 1) * s)
    X, Y = np.meshgrid(g, g, indexing="ij")
    keep = np.hypot(X, Y) <= Rc - 0.5 * s
    layer = np.stack([X[keep], Y[keep]], 1)
    nl = len(layer)
    layers = (p.n + nl - 1) // nl
    sites = np.concatenate([np.column_stack([layer, np.full(nl, (k + 0.5) * s + 0.5 * s)]) for k in range(layers)])
    pos = sites[: p.n] + rng.uniform(-0.02 * s, 0.02 * s, size=(p.n, 3))
    pos = pos[rng.permutation(p.n)]
    mass_min = 4.0 / 3.0 * PI * radius.min() ** 3 * density
    species = heap_species(tc, p.restitution, mass_min, p.mu, p.mu_r)
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    top = float(pos[:, 2].max()) + 4 * radius.max()
    inst = Instance(domain_min=(-R - 4 * d50, -R - 4 * d50, -2 * d50), domain_max=(R + 4 * d50, R + 4 * d50, top),
                    gravity=(0.0, 0.0, -9.8), n_species=2)
    floor = axisymmetric_wall((0, 0, 1), [((-1, 0, 0), (R, 0, 0)), ((0, 0, -1), (0, 0, 0))], species=1)
    vel = np.zeros((p.n, 3))
    vel[:, 2] = -v0
    sc = Scenario("calibration_heap", 0.05 * tc, inst, species, np.array([density, density]), [floor], pos,
                  vel, radius, inv_mass, inv_inertia, np.zeros(p.n, np.int32),
                  np.arange(p.n, dtype=np.int32), info=dict(params=p, base_radius=R))
    return sc, [((0, 0, -1), 0.0)], R  # DeletionBoundary set({0,0,-1}, 0): z < 0 leaves


def heap_species_cased(tc: float, eps: float, mass_min: float, mu: float, mu_r: float) -> list:
    """Species table of a heap poured inside a casing, as Calibration::
    setSpecies builds it (Calibration.h:147-186): 0 = particles, 1 = the
    casing's frictionless wall species (mixed sliding and rolling friction 0),
    2 = the floor's frictional wall species (mixed rolling friction
    max(1, sliding), sliding max(1, rolling))."""
    k, g = linear_collision_time_restitution(tc, eps, mass_min)

    def sp(mu_s, mu_roll):
        return species_pair(normal_law=_abi.DEM_NORMAL_LINEAR_VISCOELASTIC, friction_law=_abi.DEM_FRICTION_ROLLING_TORSION,
                            stiffness=k, dissipation=g,
                            sliding_stiffness=2. / 7. * k, sliding_dissipation=2. / 7. * g,
                            sliding_mu=mu_s, sliding_mu_static=mu_s,
                            rolling_stiffness=2. / 5. * k, rolling_dissipation=2. / 5. * g,
                            rolling_mu=mu_roll, rolling_mu_static=mu_roll,
                            torsion_stiffness=2. / 5. * k, torsion_dissipation=2. / 5. * g,
                            torsion_mu=0.0, torsion_mu_static=0.0)
    pp = sp(mu, mu_r)
    smooth = sp(0.0, 0.0)
    rough = sp(max(1.0, mu_r), max(1.0, mu))
    return [pp, smooth, rough,
            smooth, pp, pp,
            rough, pp, pp]


def cased_heap_scenario(p: HeapParams, d50: float = 1e-3, density: float = 2000.0, tc: float = 5e-4,
                        base_radius_d: float = 7.5, spacing: float = 1.05):
    """The set-up of Drivers/Calibration/CalibrationHeap.cpp (GranuHeap,
    CalibrationHeap.cpp:70-115) for one heap: spheres in a column of radius
    R_base inside the frictionless casing (AxisymmetricIntersectionOfWalls,
    face (1, 0, 0) at R_base), standing on the frictional floor disk (faces
    (-1, 0, 0) at R_base and (0, 0, -1) at 0), time step 0.05 collision
    times. The reference fills the column by random insertion
    (CubeInsertionBoundary); here the column is a seeded jittered lattice.
    Returns (Scenario, R_base); wall 1 is the casing."""
    rng = np.random.Generator(np.random.PCG64(p.seed))
    radius = lognormal_radii(rng, p.n, p.sigma, 0.5 * d50)
    R = base_radius_d * d50
    s = spacing * 2.0 * radius.max()
    m = int(R // s) + 1
    g = np.arange(-m, m + 1) * s
    X, Y = np.meshgrid(g, g, indexing="ij")
    keep = np.hypot(X, Y) <= R - 0.5 * s
    layer = np.stack([X[keep], Y[keep]], 1)
    nl = len(layer)
    layers = (p.n + nl - 1) // nl
    sites = np.concatenate([np.column_stack([layer, np.full(nl, (k + 0.5) * s + 0.5 * s)]) for k in range(layers)])
    pos = sites[: p.n] + rng.uniform(-0.02 * s, 0.02 * s, size=(p.n, 3))
    pos = pos[rng.permutation(p.n)]
    mass_min = 4.0 / 3.0 * PI * radius.min() ** 3 * density
    species = heap_species_cased(tc, p.restitution, mass_min, p.mu, p.mu_r)
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    top = float(pos[:, 2].max()) + 4 * radius.max()
    inst = Instance(domain_min=(-R - 4 * d50, -R - 4 * d50, -2 * d50), domain_max=(R + 4 * d50, R + 4 * d50, top),
                    gravity=(0.0, 0.0, -9.8), n_species=3)
    floor = axisymmetric_wall((0, 0, 1), [((-1, 0, 0), (R, 0, 0)), ((0, 0, -1), (0, 0, 0))], species=2)
    casing = axisymmetric_wall((0, 0, 1), [((1, 0, 0), (R, 0, 0))], species=1)
    sc = Scenario("cased_heap", 0.05 * tc, inst, species, np.array([density] * 3), [floor, casing], pos,
                  np.zeros((p.n, 3)), radius, inv_mass, inv_inertia, np.zeros(p.n, np.int32),
                  np.arange(p.n, dtype=np.int32), info=dict(params=p, base_radius=R))
    return sc, R


def heap_procedure(sc: Scenario, R: float, casing: int = 1, check_every: int = 1000, max_steps: int = 400_000,
                   engine=None) -> dict:
    """Drivers/Calibration/CalibrationHeap.cpp's run (GranuHeap::
    actionsAfterTimeStep, CalibrationHeap.cpp:119-160) on the engine: every
    `check_every` time steps the reference's hook values -- the time before
    the step's increment, the translational kinetic energy at the step's
    half-kick velocities v - F dt / 2m, the elastic energy of the step's
    contacts -- decide: at the first quiet check (kinetic < 1e-2 elastic) the
    casing is removed and a DeletionBoundary z < 0 added between the steps;
    from twice that time on, every quiet check measures the angle of repose
    atan(4 COM_z / R_base) and the first one ends the run 0.05 s later. (The
    reference keeps the removal time in an uninitialised local variable; the
    time the casing was removed is what its code intends.) Returns the angle
    of repose, the removal and end times and the particles left."""
    from .engine import deletion_boundary
    e = engine if engine is not None else sc.engine()
    dt = sc.time_step
    e.step(0)
    fill, first, removal, aor = True, True, 0.0, float("nan")
    # DPMBase::solve steps while time < timeMax, time accumulated step by
    # step (time_ += timeStep_); the hook sees the time before the increment
    t_max, steps, time_ = float("inf"), 0, 0.0
    while time_ < t_max and steps < max_steps:
        k, t = 0, time_
        while k < check_every - steps % check_every and time_ < t_max:
            t = time_
            time_ += dt
            k += 1
        e.step(k)
        steps += k
        if steps % check_every:
            continue
        st = e.download()
        f, _ = e.forces()
        alive = st["instance"] >= 0
        im = sc.inv_mass[alive]
        vmid = st["velocity"][alive] - f[alive] * (im * 0.5 * dt)[:, None]
        ke = float(np.sum(0.5 / im * np.sum(vmid * vmid, axis=1)))
        g = e.reduce()
        ee = g["elastic_energy"]
        if fill:
            if ke < 1e-2 * ee:
                fill, removal = False, t
                e.remove_wall(casing)
                e.set_deletion_boundaries([deletion_boundary((0, 0, -1), 0.0)])
        elif t > 2.0 * removal and ke < 1e-2 * ee:
            aor = math.degrees(math.atan(4.0 * g["centre_of_mass"][2] / R))
            if first:
                t_max, first = t + 0.05, False
    st = e.download()
    g = e.reduce()
    if engine is None:
        e.close()
    return dict(aor=aor, removal_time=removal, end_time=time_, steps=steps,
                n_remaining=int((st["instance"] >= 0).sum()), com_z=float(g["centre_of_mass"][2]))


def heap_batch(n_instances: int, seed: int = 1, n_range=(500, 8000), sigma_range=(0.0, 0.2), mu_range=(0.1, 0.8),
               mu_r_range=(0.0, 0.3), e_range=(0.3, 0.9), **kw):
    """Batch of heap instances with parameters drawn uniformly from the given
    ranges (the calibration sampling). Returns (Batch, [HeapParams], R_base)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    params, members, dels = [], [], []
    R = None
    for k in range(n_instances):
        p = HeapParams(n=int(rng.integers(n_range[0], n_range[1] + 1)), sigma=float(rng.uniform(*sigma_range)),
                       mu=float(rng.uniform(*mu_range)), mu_r=float(rng.uniform(*mu_r_range)),
                       restitution=float(rng.uniform(*e_range)), seed=int(rng.integers(1 << 31)))
        sc, d, R = heap_scenario(p, **kw)
        params.append(p)
        members.append(sc)
        dels.append(d)
    return batch(members, deletions=dels), params, R


def aor_com(z_com: np.ndarray, base_radius: float) -> np.ndarray:
    """CalibrationHeap.cpp:139-150: height = 4 COM_z (a cone's centre of mass
    sits at a quarter of its height), AoR = atan(height / R_base) in degrees."""
    return np.degrees(np.arctan(4.0 * np.asarray(z_com) / base_radius))


def aor_surface_fit(pos: np.ndarray, radius: np.ndarray, base_radius: float, bins: int = 12) -> tuple:
    """Angle of repose from the heap surface: the top of the highest particle
    in each radial bin over 0.2-0.8 R_base, fitted with a straight line
    z = h0 - tan(a) r. Returns (angle in degrees, h0)."""
    r = np.hypot(pos[:, 0], pos[:, 1])
    top = pos[:, 2] + radius
    edges = np.linspace(0.2 * base_radius, 0.8 * base_radius, bins + 1)
    rc, zc = [], []
    for a, b in zip(edges[:-1], edges[1:]):
        sel = (r >= a) & (r < b)
        if sel.any():
            rc.append(0.5 * (a + b))
            zc.append(top[sel].max())
    if len(rc) < 2:
        return float("nan"), float("nan")
    slope, h0 = np.polyfit(np.array(rc), np.array(zc), 1)
    return float(np.degrees(np.arctan(max(-slope, 0.0)))), float(h0)


def packing_fraction(pos: np.ndarray, radius: np.ndarray, base_radius: float, h0: float, angle_deg: float) -> float:
    """Solid fraction of the heap core: sphere volume with centres inside
    r < R_base/3, 0 < z < the fitted surface at R_base/3 (minus one mean
    diameter), over that cylinder's volume."""
    rc = base_radius / 3.0
    zt = h0 - math.tan(math.radians(angle_deg)) * rc - 2.0 * float(np.mean(radius))
    if not zt > 0:
        return float("nan")
    r = np.hypot(pos[:, 0], pos[:, 1])
    sel = (r < rc) & (pos[:, 2] > 0) & (pos[:, 2] < zt)
    return float(np.sum(4.0 / 3.0 * PI * radius[sel] ** 3) / (PI * rc * rc * zt))


def run_heaps(b: Batch, base_radius: float, steps: int = 40_000, trace_every: int = 1_000, engine=None,
              max_neighbors: int = 0) -> dict:
    """Runs every instance of the batch for `steps` time steps in one handle;
    returns the per-instance outputs, kinetic-energy traces and the device
    time of the time steps (device_ms, summed over the dem_step calls)."""
    e = engine if engine is not None else b.engine(max_neighbors=max_neighbors)
    e.step(0)
    ke = [e.reduce_batch()["kinetic_energy"]]
    done = 0
    device_ms = 0.0
    while done < steps:
        k = min(trace_every, steps - done)
        e.step(k)
        device_ms += e.stats()["ms"]
        done += k
        ke.append(e.reduce_batch()["kinetic_energy"])
    g = e.reduce_batch()
    st = e.download(out=dict(position=np.zeros((b.n, 3)), instance=np.zeros(b.n, np.int32)))
    if engine is None:
        e.close()
    n_inst = len(b.members)
    out = dict(aor_reference=aor_com(g["centre_of_mass"][:, 2], base_radius), aor_surface=np.full(n_inst, np.nan),
               packing_fraction=np.full(n_inst, np.nan), kinetic_energy=np.array(ke).T,
               elastic_energy=g["elastic_energy"], n_remaining=np.zeros(n_inst, np.int64), device_ms=device_ms)
    for k in range(n_inst):
        sl = b.member_slice(k)
        alive = st["instance"][sl] >= 0
        pos = st["position"][sl][alive]
        rad = b.radius[sl][alive]
        out["n_remaining"][k] = int(alive.sum())
        a, h0 = aor_surface_fit(pos, rad, base_radius)
        out["aor_surface"][k] = a
        if a == a:
            out["packing_fraction"][k] = packing_fraction(pos, rad, base_radius, h0, a)
    return out


# ---------------------------------------------------------------------------
# surrogate-guided calibration
# ---------------------------------------------------------------------------
PARAM_NAMES = ("sliding_friction", "rolling_friction", "restitution", "psd_sigma")
RESPONSE_NAMES = ("angle_of_repose", "packing_fraction", "settle_time")
PARAM_BOX = np.array([[0.1, 0.8], [0.0, 0.3], [0.3, 0.9], [0.0, 0.2]])


def heap_responses(params: np.ndarray, n: int = 600, seed: int = 11, steps: int = 20_000, trace_every: int = 500,
                   chunk: int = 1024, **kw) -> np.ndarray:
    """Runs one heap per parameter row (sliding friction, rolling friction,
    restitution, PSD width) in batches of `chunk` instances and returns the
    responses [angle of repose (reference estimator, degrees), packing
    fraction, settle time (s)] per row. All heaps share `n` and the packing
    seed, so the responses are a deterministic function of the parameters.

    packing fraction: solid volume left on the floor over the volume of the
    cone of height 4 COM_z on the floor disk (the cone the reference's AoR
    estimator assumes); settle time: the first trace time at which the
    kinetic energy is below 1e-2 of the elastic energy (the reference's settle
    test, CalibrationHeap.cpp:119-131), or the end of the run."""
    params = np.asarray(params, np.float64).reshape(-1, 4)
    out = np.zeros((len(params), 3))
    for a in range(0, len(params), chunk):
        rows = params[a:a + chunk]
        members, dels, R = [], [], None
        for p in rows:
            hp = HeapParams(n=n, sigma=float(p[3]), mu=float(p[0]), mu_r=float(p[1]), restitution=float(p[2]),
                            seed=seed)
            sc, d, R = heap_scenario(hp, **kw)
            members.append(sc)
            dels.append(d)
        b = batch(members, deletions=dels)
        e = b.engine()
        e.step(0)
        settle = np.full(len(rows), steps * b.time_step)
        done = 0
        g = None
        while done < steps:
            e.step(trace_every)
            done += trace_every
            g = e.reduce_batch()
            quiet = (g["kinetic_energy"] < 1e-2 * g["elastic_energy"]) & (settle >= steps * b.time_step)
            settle[quiet] = done * b.time_step
        e.close()
        com_z = g["centre_of_mass"][:, 2]
        h = np.maximum(4.0 * com_z, 1e-9)
        solid = g["mass"] / 2000.0  # density of every heap species
        out[a:a + len(rows), 0] = aor_com(com_z, R)
        out[a:a + len(rows), 1] = solid / (PI * R * R * h / 3.0)
        out[a:a + len(rows), 2] = settle
    return out


def response_error(resp: np.ndarray, target: np.ndarray) -> np.ndarray:
    """Largest relative error over angle of repose and packing fraction (the
    settle time is quantised by the trace interval and is reported, not
    judged)."""
    resp = np.atleast_2d(resp)
    return np.max(np.abs(resp[:, :2] - target[:2]) / np.abs(target[:2]), axis=1)


def sample_params(rng, n: int) -> np.ndarray:
    return PARAM_BOX[:, 0] + rng.uniform(size=(n, 4)) * (PARAM_BOX[:, 1] - PARAM_BOX[:, 0])


def calibrate(target: np.ndarray, dem, surrogate=None, rounds: int = 4, proposals: int = 256,
              candidates: int = 65_536, tol: float = 0.02, seed: int = 0, data=None, retrain_epochs: int = 30):
    """Searches parameters whose DEM response is within `tol` of `target`.

    Each round proposes `proposals` parameter sets and judges them with
    `dem(params) -> responses` (batched DEM). With a surrogate, the proposals
    are the candidates (of `candidates` uniform samples) whose predicted
    responses are closest to the target; DEM then also judges the surrogate:
    if its median prediction error on the proposals exceeds `tol`, the next
    round falls back to plain proposals, and every DEM result refines the
    network. Without a surrogate every round is plain: uniform proposals
    (plain batched DEM search). Returns the best parameters, their error and
    the per-round history."""
    rng = np.random.default_rng(seed)
    best_err, best_p, best_r = np.inf, None, None
    hist = []
    xs = [] if data is None else [np.asarray(data[0])]
    ys = [] if data is None else [np.asarray(data[1])]
    trust = surrogate is not None
    for r in range(rounds):
        pred = None
        if trust:
            cand = sample_params(rng, candidates)
            pc = surrogate.predict(cand)
            order = np.argsort(response_error(pc, target))[:proposals]
            props, pred, mode = cand[order], pc[order], "surrogate"
        else:
            props, mode = sample_params(rng, proposals), ("fallback" if surrogate is not None else "plain")
        resp = dem(props)
        err = response_error(resp, target)
        k = int(np.argmin(err))
        if err[k] < best_err:
            best_err, best_p, best_r = float(err[k]), props[k], resp[k]
        rec = dict(round=r, mode=mode, best_error=float(err[k]), median_error=float(np.median(err)))
        if surrogate is not None:
            if pred is None:
                pred = surrogate.predict(props)
            surr_err = float(np.median(np.max(np.abs(pred[:, :2] - resp[:, :2]) / np.abs(resp[:, :2]), axis=1)))
            rec["surrogate_error"] = surr_err
            trust = surr_err <= tol
            xs.append(props)
            ys.append(resp)
            surrogate.fit(np.concatenate(xs), np.concatenate(ys), epochs=retrain_epochs)
        hist.append(rec)
        if best_err <= tol:
            break
    return dict(best_error=best_err, params=best_p, response=best_r, history=hist, rounds=len(hist),
                dem_runs=len(hist) * proposals)


def calibrate_batch(targets: np.ndarray, dem, surrogate, rounds: int = 4, proposals: int = 256,
                    candidates: int = 65_536, tol: float = 0.02, seed: int = 0, data=None,
                    retrain_epochs: int = 30) -> list:
    """calibrate() for many targets at once: every round, each target still
    above `tol` proposes `proposals` parameter sets (the surrogate's closest
    candidates, or uniform ones while the surrogate is not trusted for that
    target) and one call of `dem` judges all of them together, so a round of
    many calibrations is one batched DEM run. The surrogate is refined once
    per round on every new DEM result. Returns one result per target, as
    calibrate() does."""
    targets = np.atleast_2d(np.asarray(targets, np.float64))
    nt = len(targets)
    rng = np.random.default_rng(seed)
    best_err = np.full(nt, np.inf)
    best_p, best_r = [None] * nt, [None] * nt
    hist = [[] for _ in range(nt)]
    trust = np.full(nt, surrogate is not None)
    xs = [] if data is None else [np.asarray(data[0])]
    ys = [] if data is None else [np.asarray(data[1])]
    for r in range(rounds):
        active = [k for k in range(nt) if best_err[k] > tol]
        if not active:
            break
        props, preds, modes = [], [], []
        for k in active:
            if trust[k]:
                cand = sample_params(rng, candidates)
                pc = surrogate.predict(cand)
                order = np.argsort(response_error(pc, targets[k]))[:proposals]
                props.append(cand[order])
                preds.append(pc[order])
                modes.append("surrogate")
            else:
                pk = sample_params(rng, proposals)
                props.append(pk)
                preds.append(surrogate.predict(pk) if surrogate is not None else None)
                modes.append("fallback" if surrogate is not None else "plain")
        resp = dem(np.concatenate(props))
        for j, k in enumerate(active):
            rk = resp[j * proposals:(j + 1) * proposals]
            err = response_error(rk, targets[k])
            i = int(np.argmin(err))
            if err[i] < best_err[k]:
                best_err[k], best_p[k], best_r[k] = float(err[i]), props[j][i], rk[i]
            rec = dict(round=r, mode=modes[j], best_error=float(err[i]), median_error=float(np.median(err)))
            if surrogate is not None:
                pe = np.max(np.abs(preds[j][:, :2] - rk[:, :2]) / np.abs(rk[:, :2]), axis=1)
                rec["surrogate_error"] = float(np.median(pe))
                trust[k] = rec["surrogate_error"] <= tol
            hist[k].append(rec)
        if surrogate is not None and any(best_err[k] > tol for k in range(nt)) and r + 1 < rounds:
            # refine only when another round follows: the next round is the one that uses it
            xs.append(np.concatenate(props))
            ys.append(resp)
            surrogate.fit(np.concatenate(xs), np.concatenate(ys), epochs=retrain_epochs)
    return [dict(best_error=float(best_err[k]), params=best_p[k], response=best_r[k], history=hist[k],
                 rounds=len(hist[k]), dem_runs=len(hist[k]) * proposals) for k in range(nt)]

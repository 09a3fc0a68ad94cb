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
    returns the per-instance outputs and kinetic-energy traces."""
    e = engine if engine is not None else b.engine(max_neighbors=max_neighbors)
    e.step(0)
    ke = [e.reduce_batch()["kinetic_energy"]]
    done = 0
    while done < steps:
        k = min(trace_every, steps - done)
        e.step(k)
        done += k
        ke.append(e.reduce_batch()["kinetic_energy"])
    g = e.reduce_batch()
    st = e.download(out=dict(position=np.zeros((b.n, 3)), instance=np.zeros(b.n, np.int32)))
    if engine is None:
        e.close()
    n_inst = len(b.members)
    out = dict(aor_reference=aor_com(g["centre_of_mass"][:, 2], base_radius), aor_surface=np.full(n_inst, np.nan),
               packing_fraction=np.full(n_inst, np.nan), kinetic_energy=np.array(ke).T,
               elastic_energy=g["elastic_energy"], n_remaining=np.zeros(n_inst, np.int64))
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

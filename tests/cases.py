"""Small parity cases shared by the CPU and GPU tests (seeded, sized so the
CPU oracle finishes in well under a second)."""
from __future__ import annotations

import json
import os

import numpy as np

from mercurydpm_fork_b200 import scenarios
from mercurydpm_fork_b200.engine import Instance
from mercurydpm_fork_b200.host import PI, linear_collision_time_restitution, sphere_inv_mass_inertia
from mercurydpm_fork_b200.scenarios import Scenario, linear_sliding_species

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def compressed_box(n=800, seed=3):
    """Settling box on a slightly overlapping lattice: every particle starts
    with contacts, several touch the walls after a few hundred steps."""
    return scenarios.settling_box(n=n, seed=seed, spacing=0.995, jitter=0.003, box=(10, 10, 40), vstd=0.05)


def wall_box(n=400, seed=5):
    """Particles pressed against the bottom and side walls from the start."""
    sc = scenarios.settling_box(n=n, seed=seed, spacing=0.999, jitter=0.002, box=(8, 8, 20), vstd=0.05)
    # shift the lattice so the first layer overlaps the floor and x=0 wall slightly
    sc.position[:, 2] -= sc.position[:, 2].min() - 0.499e-3
    sc.position[:, 0] -= sc.position[:, 0].min() - 0.4995e-3
    return sc


def small_chute(n_flow=3000, seed=7):
    """Periodic chute, 20 x 10 small diameters, bidisperse, with rough base;
    the bed starts pre-compressed so that contacts (also across the periodic
    boundaries and with the base) exist from the first step."""
    sc = scenarios.periodic_chute(n_flow=n_flow, seed=seed, lx=20, ly=10, vstd=0.05, site_scale=0.96,
                                  base_gap=-0.1)
    return sc


def offset_chute(offset=1000.0):
    """small_chute moved `offset` metres along every axis (domain, periodic
    bounds and particles): coordinates are a million particle diameters from
    the origin, where FP32 keeps about 0.1 mm of resolution."""
    import dataclasses
    sc = small_chute()
    inst = sc.instance
    shift = lambda t: tuple(float(v) + offset for v in t)
    sc.instance = dataclasses.replace(inst, domain_min=shift(inst.domain_min), domain_max=shift(inst.domain_max),
                                      periodic_min=shift(inst.periodic_min), periodic_max=shift(inst.periodic_max))
    sc.position = sc.position + offset
    return sc


def cubic_packing(n=5, distance=0.99):
    """Drivers/UnitTests/CG3DPackingUnitTest.cpp: n^3 spheres (r = 0.5) on a
    cubic lattice of spacing 0.99 in a triply periodic box; every contact
    carries a unit force, so CG<O> gives density n^3/V and contact stress
    n^3 0.99 / V on the diagonal."""
    from mercurydpm_fork_b200 import _abi
    from mercurydpm_fork_b200.engine import species_pair
    k = 100.0
    eps = 0.5
    mass = 1.0
    log_eps = np.log(eps)
    diss = -np.sqrt(2.0 * mass * k / (PI * PI + log_eps * log_eps)) * log_eps
    sp = species_pair(normal_law=_abi.DEM_NORMAL_LINEAR_VISCOELASTIC, friction_law=_abi.DEM_FRICTION_NONE,
                      stiffness=k, dissipation=diss)
    density = 6.0 / PI
    ijk = np.array([(i, j, l) for i in range(n) for j in range(n) for l in range(n)], dtype=np.float64)
    pos = distance * (ijk + 0.5)
    m = len(pos)
    radius = np.full(m, 0.5)
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    L = n * distance
    inst = Instance(domain_min=(0, 0, 0), domain_max=(L, L, L), gravity=(0, 0, 0), n_species=1, periodic_mask=0b111,
                    periodic_min=(0, 0, 0), periodic_max=(L, L, L))
    tc = PI / np.sqrt(k / (.5 * mass) - (diss / mass) ** 2)  # getCollisionTime(1.0)
    sc = Scenario("cubic_packing", 0.02 * tc, inst, [sp], np.array([density]), [], pos, np.zeros((m, 3)), radius,
                  inv_mass, inv_inertia, np.zeros(m, np.int32), np.arange(m, dtype=np.int32), rotation=False)
    return sc, dict(n=n, distance=distance, volume=L ** 3)


def tangential_spring():
    """Drivers/UnitTests/TangentialSpringUnitTest.cpp: a sphere rolling off a
    fixed sphere under gravity (0, 0, -1); returns (scenario, steps, golden)."""
    g = json.load(open(os.path.join(GOLDEN, "tangential_spring.json")))
    tc, eps, m = g["collision_time_restitution_mass"]
    k, diss = linear_collision_time_restitution(tc, eps, m)
    sp = linear_sliding_species(tc, eps, m, 1e20)
    sp.sliding_stiffness = k * 2 / 7
    density = 6. / PI
    radius = np.array([0.25, 0.25])
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    inv_mass[0] = 0.0
    inv_inertia[0] = 0.0
    pos = np.array([[0.5, 0.5, 0.25], [0.5, 0.5, 0.75]])
    vel = np.array([[0.0, 0.0, 0.0], [0.1, 0.0, 0.0]])
    inst = Instance(domain_min=(0, 0, 0), domain_max=(1, 1, 1), gravity=tuple(g["gravity"]), n_species=1)
    sc = Scenario("tangential_spring", g["time_step"], inst, [sp], np.array([density]), [], pos, vel, radius,
                  inv_mass, inv_inertia, np.zeros(2, np.int32), np.arange(2, dtype=np.int32))
    t, steps = 0.0, 0
    while t < g["time_max"]:  # DPMBase::solve: while (time < timeMax) { step; time += dt }
        t += g["time_step"]
        steps += 1
    return sc, steps, g["expected"]


def _hertz_mindlin_table(nsp):
    from mercurydpm_fork_b200.scenarios import hertz_mindlin_species
    sp = hertz_mindlin_species(1e7, 1e7 / 2 * 1.3, 0.7, 0.4, 0.05, 0.02, sliding_dissipation=0.3,
                               rolling_dissipation=0.2, torsion_dissipation=0.1)
    return [sp] * (nsp * nsp)


def _rot(q, v):
    q0, q1, q2, q3 = q
    Rm = np.array([[q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                   [2 * (q1 * q2 + q0 * q3), q0 * q0 - q1 * q1 + q2 * q2 - q3 * q3, 2 * (q2 * q3 - q0 * q1)],
                   [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), q0 * q0 - q1 * q1 - q2 * q2 + q3 * q3]])
    return v @ Rm.T


def wall_probe(kind: str, n: int = 300, seed: int = 11, omega=(0.0, 0.0, 0.0)):
    """Spheres (d = 1 mm, Hertz-Mindlin with rolling and torsion) scattered
    without mutual overlap within 0.3-1.1 radii of an intersection wall, so
    that face, edge and corner contacts all occur at the start:

    * "heap_base": CalibrationHeap's floor disk (AxisymmetricIntersectionOfWalls,
      axis z, addObject((-1,0,0),(R,0,0)) and addObject((0,0,-1),(0,0,0)),
      Drivers/Calibration/CalibrationHeap.cpp:86-91), R = 6 mm;
    * "ring_ridge": an axisymmetric ring of triangular cross-section (axis z;
      r > 4 mm, a > 0, r + a < 5.5 mm): near its narrow tip a sphere is
      within reach of all three faces, whose normals are coplanar in the
      (r, a) plane, so the reference's corner point is not finite and its
      corner branch falls through to the edge branch;
    * "box_corner": an IntersectionOfWalls of three orthogonal faces (a solid
      octant) at a seeded random orientation and position: face, edge and
      corner contacts in 3D.
    The wall rotates with angular velocity `omega` about its own position."""
    from mercurydpm_fork_b200.engine import axisymmetric_wall, intersection_wall
    from mercurydpm_fork_b200.scenarios import hertz_collision_time
    rng = np.random.Generator(np.random.PCG64(seed))
    d = 1e-3
    r = 0.5 * d
    R = 6e-3
    q = None
    if kind == "heap_base":
        wall = axisymmetric_wall((0, 0, 1), [((-1, 0, 0), (R, 0, 0)), ((0, 0, -1), (0, 0, 0))], species=1,
                                 angular_velocity=omega)

        def local(m):
            rr = np.sqrt(rng.uniform(0, (R + 2 * r) ** 2, m))
            ph = rng.uniform(0, 2 * PI, m)
            z = rng.uniform(-2 * r, 2 * r, m)
            p = np.stack([rr * np.cos(ph), rr * np.sin(ph), z], 1)
            dist = np.where(rr <= R, z, np.where(z <= 0, rr - R, np.hypot(rr - R, z)))
            return p, dist
    elif kind == "ring_ridge":
        R1, R2 = 4e-3, 5.5e-3
        wall = axisymmetric_wall((0, 0, 1), [((1, 0, 0), (R1, 0, 0)), ((0, 0, 1), (0, 0, 0)),
                                             ((-1, 0, -1), (R2, 0, 0))], species=1, angular_velocity=omega)
        tri = np.array([[R1, 0.0], [R2, 0.0], [R1, R2 - R1]])

        def local(m):
            rr = rng.uniform(R1 - 2 * r, R2 + 2 * r, m)
            a = rng.uniform(-2 * r, R2 - R1 + 2 * r, m)
            ph = rng.uniform(0, 2 * PI, m)
            p = np.stack([rr * np.cos(ph), rr * np.sin(ph), a], 1)
            q2 = np.stack([rr, a], 1)
            dist = np.full(m, np.inf)
            for k in range(3):
                s0, s1 = tri[k], tri[(k + 1) % 3]
                t = np.clip(((q2 - s0) @ (s1 - s0)) / ((s1 - s0) @ (s1 - s0)), 0, 1)
                dist = np.minimum(dist, np.linalg.norm(q2 - (s0 + t[:, None] * (s1 - s0)), axis=1))
            inside = (rr > R1) & (a > 0) & (rr + a < R2)
            return p, np.where(inside, -dist, dist)
    elif kind == "box_corner":
        qv = rng.normal(size=4)
        q = tuple(qv / np.linalg.norm(qv))
        origin = np.array([1e-3, -2e-3, 0.5e-3])
        wall = intersection_wall([((1, 0, 0), (0, 0, 0)), ((0, 1, 0), (0, 0, 0)), ((0, 0, 1), (0, 0, 0))],
                                 position=origin, orientation=q, species=1, angular_velocity=omega)

        def local(m):
            p = rng.uniform(-2 * r, 14 * r, size=(m, 3))
            out = np.maximum(-p, 0.0)
            dist = np.where((p > 0).all(1), -p.min(1), np.sqrt((out ** 2).sum(1)))
            return p, dist
    else:
        raise ValueError(kind)
    pts = []
    for _ in range(50):
        p, dist = local(4000)
        for x in p[(dist > 0.3 * r) & (dist < 1.1 * r)]:
            if len(pts) >= n:
                break
            if not pts or np.min(np.sum((np.array(pts) - x) ** 2, 1)) > (2.05 * r) ** 2:
                pts.append(x)
        if len(pts) >= n:
            break
    pos = np.array(pts)
    if q is not None:
        pos = _rot(q, pos) + origin
    m = len(pos)
    radius = np.full(m, r)
    density = 2000.0
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    vel = rng.normal(0.0, 0.05, size=(m, 3))
    lo, hi = pos.min(0) - 8 * r, pos.max(0) + 8 * r
    inst = Instance(domain_min=tuple(lo), domain_max=tuple(hi), gravity=(0, 0, -9.81), n_species=2)
    dt = 0.02 * hertz_collision_time(d, density, 1e7)
    return Scenario(f"wall_probe_{kind}", dt, inst, _hertz_mindlin_table(2), np.array([density, density]), [wall],
                    pos, vel, radius, inv_mass, inv_inertia, np.zeros(m, np.int32), np.arange(m, dtype=np.int32))


def small_drum(n=600, seed=5):
    """Rotating drum (R = 12 mm, length 12 mm, 5 rad/s), bidisperse 1:3,
    Hertz-Mindlin with rolling and torsion, bed pre-compressed, the outer
    spheres pressed onto the cylinder."""
    return scenarios.rotating_drum(n=n, seed=seed, radius_d=12, length_d=12, site_spacing=0.995, touch_wall=3.0,
                                   omega=5.0, mu_o=0.02, sliding_dissipation=0.3, rolling_dissipation=0.2,
                                   torsion_dissipation=0.1, vstd=0.02)


def point_triangle_distance(p, a, b, c):
    """Distance from each point of p (m x 3) to the triangle abc: the plane
    distance where the projection lies inside, else the distance to the
    nearest edge segment."""
    p = np.atleast_2d(p)
    n = np.cross(b - a, c - a)
    n = n / np.linalg.norm(n)
    sd = (p - a) @ n
    proj = p - sd[:, None] * n
    inside = np.ones(len(p), bool)
    for u, v in ((a, b), (b, c), (c, a)):
        inside &= (np.cross(v - u, proj - u) @ n) >= 0
    seg = np.full(len(p), np.inf)
    for u, v in ((a, b), (b, c), (c, a)):
        t = np.clip(((p - u) @ (v - u)) / ((v - u) @ (v - u)), 0.0, 1.0)
        seg = np.minimum(seg, np.linalg.norm(p - (u + t[:, None] * (v - u)), axis=1))
    return np.where(inside, np.abs(sd), seg)


def triangle_mesh_triangles():
    """A triangulated height field z = h(x) over x in [-4, 4] mm, y in [-3, 3] mm:
    two valleys (x = -2, 2 mm) and a ridge (x = 0), nodes every 2 mm in x and
    3 mm in y, 16 triangles; both diagonals directions occur."""
    xs = np.array([-4e-3, -2e-3, 0.0, 2e-3, 4e-3])
    hs = np.array([2e-3, 0.0, 1.2e-3, 0.0, 2e-3])
    ys = np.array([-3e-3, 0.0, 3e-3])
    tris = []
    for i in range(4):
        for j in range(2):
            p00 = np.array([xs[i], ys[j], hs[i]])
            p10 = np.array([xs[i + 1], ys[j], hs[i + 1]])
            p01 = np.array([xs[i], ys[j + 1], hs[i]])
            p11 = np.array([xs[i + 1], ys[j + 1], hs[i + 1]])
            if (i + j) % 2 == 0:
                tris += [(p00, p10, p11), (p00, p11, p01)]
            else:
                tris += [(p00, p10, p01), (p10, p11, p01)]
    return tris


def triangle_mesh(group: int = 1, n: int = 300, seed: int = 13, velocity=(0.0, 0.0, 0.0), dropped: bool = False):
    """Spheres (d = 0.5 mm, Hertz-Mindlin with rolling and torsion) scattered
    without mutual overlap within 0.3-1.1 radii of the triangulated surface of
    triangle_mesh_triangles() (TriangleWall::setVertices(A, B, C) each, one
    group id for all), so that face, edge and vertex contacts, particles on
    shared edges and in the valleys (two face contacts) all occur; gravity
    pulls them into the surface. `velocity` moves every triangle. With
    `dropped`, the spheres start 0.02-0.2 radii clear of the surface moving
    towards it at 1 m/s under 500 m/s^2 of gravity, so that every triangle
    contact is made during the run and most of them last."""
    from mercurydpm_fork_b200.engine import triangle_wall
    from mercurydpm_fork_b200.scenarios import hertz_collision_time
    rng = np.random.Generator(np.random.PCG64(seed))
    d = 0.5e-3
    r = 0.5 * d
    tris = triangle_mesh_triangles()
    walls = [triangle_wall(a, b, c, species=1, group=group, velocity=velocity) for a, b, c in tris]
    pts = []
    for _ in range(50):
        x = rng.uniform(-4e-3, 4e-3, 4000)
        h = np.interp(x, [-4e-3, -2e-3, 0.0, 2e-3, 4e-3], [2e-3, 0.0, 1.2e-3, 0.0, 2e-3])
        lift = (1.0, 2.6) if dropped else (0.1, 1.6)
        p = np.stack([x, rng.uniform(-3e-3, 3e-3, 4000), h + rng.uniform(lift[0] * r, lift[1] * r, 4000)], 1)
        dist = np.min([point_triangle_distance(p, a, b, c) for a, b, c in tris], axis=0)
        # above the surface: the height field at x, linearly interpolated
        above = p[:, 2] > np.interp(p[:, 0], [-4e-3, -2e-3, 0.0, 2e-3, 4e-3], [2e-3, 0.0, 1.2e-3, 0.0, 2e-3])
        band = (dist > 1.02 * r) & (dist < 1.2 * r) if dropped else (dist > 0.3 * r) & (dist < 1.1 * r)
        for x in p[above & band]:
            if len(pts) >= n:
                break
            if not pts or np.min(np.sum((np.array(pts) - x) ** 2, 1)) > (2.05 * r) ** 2:
                pts.append(x)
        if len(pts) >= n:
            break
    pos = np.array(pts)
    m = len(pos)
    radius = np.full(m, r)
    density = 2000.0
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    vel = rng.normal(0.0, 0.05, size=(m, 3))
    if dropped:
        vel[:, 2] -= 1.0
    lo, hi = pos.min(0) - 8 * r, pos.max(0) + 8 * r
    inst = Instance(domain_min=tuple(lo), domain_max=tuple(hi), gravity=(0, 0, -500.0 if dropped else -9.81),
                    n_species=2)
    dt = 0.02 * hertz_collision_time(d, density, 1e7)
    return Scenario(f"triangle_mesh_g{group}{'_dropped' if dropped else ''}", dt, inst, _hertz_mindlin_table(2), np.array([density, density]), walls,
                    pos, vel, radius, inv_mass, inv_inertia, np.zeros(m, np.int32), np.arange(m, dtype=np.int32))


LAWS = ("linear", "linear_sliding", "linear_sliding_constant_restitution", "linear_rolling_torsion",
        "hertz", "hertz_sliding", "hertz_mindlin", "hertz_mindlin_rolling_torsion")


def drum_with_law(law: str, n: int = 600, seed: int = 5):
    """small_drum (bidisperse 1:3, a rotating AxisymmetricIntersectionOfWalls
    cylinder and two InfiniteWall caps, compressed bed pressed onto the
    cylinder) with every species pair on one contact law, so that each law's
    branches run: normal force, sliding spring with the Coulomb cap (mu 0.2),
    rolling (mu_r 0.05) and torsion (mu_o 0.02) springs, dissipation on every
    spring. Linear laws: tc = 1e-4 s, restitution 0.7 for two small spheres,
    k_t = 2/7 k, k_r = k_o = 2/5 k (Calibration.h's ratios), dt = tc/50
    (constant restitution: the same k and gamma per unit mass). Hertz laws:
    the drum's E, G and restitution, dt 0.02 of the Hertz collision time."""
    import dataclasses
    from mercurydpm_fork_b200 import _abi
    from mercurydpm_fork_b200.engine import species_pair
    from mercurydpm_fork_b200.host import hertz_dissipation_from_restitution
    sc = small_drum(n=n, seed=seed)
    m_small = 4.0 / 3.0 * PI * (0.5e-3) ** 3 * 2000.0
    k, g = linear_collision_time_restitution(1e-4, 0.7, m_small)
    E, G, eps = 1e7, 1e7 / 2 * 1.3, 0.7
    L, H = _abi.DEM_NORMAL_LINEAR_VISCOELASTIC, _abi.DEM_NORMAL_HERTZIAN_VISCOELASTIC
    base = dict(sliding_mu=0.2, sliding_mu_static=0.2, rolling_mu=0.05, rolling_mu_static=0.05, torsion_mu=0.02,
                torsion_mu_static=0.02)
    lin = dict(normal_law=L, stiffness=k, dissipation=g, sliding_stiffness=2 / 7 * k, sliding_dissipation=2 / 7 * g,
               rolling_stiffness=2 / 5 * k, rolling_dissipation=2 / 5 * g, torsion_stiffness=2 / 5 * k,
               torsion_dissipation=2 / 5 * g, **base)
    hz = dict(normal_law=H, elastic_modulus=E, dissipation=hertz_dissipation_from_restitution(eps), shear_modulus=G,
              sliding_dissipation=0.3, rolling_dissipation=0.2, torsion_dissipation=0.1, **base)
    table = {
        "linear": dict(lin, friction_law=_abi.DEM_FRICTION_NONE),
        "linear_sliding": dict(lin, friction_law=_abi.DEM_FRICTION_SLIDING),
        "linear_sliding_constant_restitution": dict(lin, friction_law=_abi.DEM_FRICTION_SLIDING, constant_restitution=1,
                                                    stiffness=k / m_small, dissipation=g / m_small,
                                                    sliding_stiffness=2 / 7 * k / m_small,
                                                    sliding_dissipation=2 / 7 * g / m_small),
        "linear_rolling_torsion": dict(lin, friction_law=_abi.DEM_FRICTION_ROLLING_TORSION),
        "hertz": dict(hz, friction_law=_abi.DEM_FRICTION_NONE),
        "hertz_sliding": dict(hz, friction_law=_abi.DEM_FRICTION_SLIDING, sliding_stiffness=2 / 7 * k),
        "hertz_mindlin": dict(hz, friction_law=_abi.DEM_FRICTION_MINDLIN),
        "hertz_mindlin_rolling_torsion": dict(hz, friction_law=_abi.DEM_FRICTION_MINDLIN_ROLLING_TORSION),
    }[law]
    sp = species_pair(**table)
    dt = 2e-6 if law.startswith("linear") else sc.time_step
    return dataclasses.replace(sc, name=f"drum_{law}", species=[sp] * len(sc.species), time_step=dt)


def recontact(owner_first: bool = True, vy: float = 0.1):
    """Sphere P starts just touching the fixed sphere I (overlap 1e-5) while
    moving away from it, with a tangential velocity vy, so the initial
    evaluation builds a sliding spring. In the first time step P leaves I and
    runs into the fixed sphere J, which throws it back onto I in the second.
    The reference keeps the interaction of the initial evaluation through the
    first time step although nothing touches it then (its time stamp is that
    of the first step, InteractionHandler::eraseOldInteractions), so the
    second step's contact continues from that spring. owner_first: P has the
    lower id of the pair (it owns the pair's spring)."""
    from mercurydpm_fork_b200 import _abi
    from mercurydpm_fork_b200.engine import species_pair
    sp = species_pair(normal_law=_abi.DEM_NORMAL_LINEAR_VISCOELASTIC, friction_law=_abi.DEM_FRICTION_SLIDING,
                      stiffness=4e6, dissipation=10.0, sliding_stiffness=4e6 * 2 / 7, sliding_dissipation=0.0,
                      sliding_mu=1e20, sliding_mu_static=1e20)
    density = 6.0 / PI  # unit mass for r = 0.5
    delta = 1e-5
    pos = np.array([[1.0 - delta, 0.0, 0.0], [0.0, 0.0, 0.0], [2.0 - delta, 0.0, 0.0]]) + 5.0
    vel = np.array([[1.0, vy, 0.0], [0.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    radius = np.full(3, 0.5)
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    inv_mass[1:] = 0.0
    inv_inertia[1:] = 0.0
    ids = np.array([0, 1, 2] if owner_first else [2, 0, 1], np.int32)
    inst = Instance(domain_min=(0, 0, 0), domain_max=(10, 10, 10), gravity=(0, 0, 0), n_species=1)
    return Scenario("recontact", 1e-3, inst, [sp], np.array([density]), [], pos, vel, radius, inv_mass, inv_inertia,
                    np.zeros(3, np.int32), ids)


def pressed_column():
    """400 spheres in a cased heap column (lattice spacing 0.98 diameters)
    whose outer ring presses on the casing, and a deletion plane z < 1.5
    spacings that takes the bottom layer: (Scenario, R_base, [plane]). Wall 1
    is the casing."""
    from mercurydpm_fork_b200 import calibration as cal
    p = cal.HeapParams(n=400, sigma=0.1, mu=0.5, mu_r=0.1, restitution=0.5, seed=3)
    sc, R = cal.cased_heap_scenario(p, spacing=0.98)
    s = 0.98 * 2.0 * float(np.max(sc.radius))
    # the outer ring moved out radially until it overlaps the casing by 1 % of a radius
    rxy = np.hypot(sc.position[:, 0], sc.position[:, 1])
    outer = rxy > R - 1.5 * s
    scale = (R - 0.99 * sc.radius[outer]) / rxy[outer]
    sc.position[outer, 0] *= scale
    sc.position[outer, 1] *= scale
    return sc, R, [((0.0, 0.0, -1.0), -1.5 * s)]


def insertion_box(n_live=300, n_free=800, periodic=False, psd="range", rate=float("inf"), seed=11, max_failed=20,
                  psd_seed=0, chute=False):
    """A box 10 x 10 x 30 diameters whose bottom holds n_live settling spheres
    and a CubeInsertionBoundary over z = 3 .. 12 diameters, overlapping the
    top of that bed (candidates meet particles and, near the sides, walls).
    periodic: x and y are periodic instead of walled (candidates near the
    sides have periodic images). psd: "range" = set(..., rMin, rMax) with
    0.4 d .. 0.6 d; "single" = the default PSD of a 0.5 d template; "bins" =
    setDistributionUniform(0.45 d, 0.55 d, 8) with the PSD seed psd_seed.
    rate: the volume flow rate. chute: a ChuteInsertionBoundary instead,
    feeding the plane x = 0.5 d + r over z = 6 .. 12 d (fixed particle radius
    0.5 d, inflow velocity 0.1 m/s, variance 0.2). The n_free rows after the
    bed have radius 0 and the ids the reference hands out next. Returns
    (scenario, [boundary])."""
    import dataclasses
    from mercurydpm_fork_b200.engine import insertion_boundary
    from mercurydpm_fork_b200.host import psd_uniform
    d = 1e-3
    sc = scenarios.settling_box(n=n_live, seed=seed, box=(10, 10, 30), spacing=1.05, jitter=0.02, vstd=0.05)
    L = 10 * d
    if periodic:
        sc.walls = sc.walls[4:]  # floor and lid only
        sc.instance = dataclasses.replace(sc.instance, periodic_mask=0b011, periodic_min=(0.0, 0.0, 0.0),
                                          periodic_max=(L, L, 0.0))
    m = n_free
    sc.position = np.vstack([sc.position, np.zeros((m, 3))])
    sc.velocity = np.vstack([sc.velocity, np.zeros((m, 3))])
    sc.radius = np.concatenate([sc.radius, np.zeros(m)])
    sc.inv_mass = np.concatenate([sc.inv_mass, np.zeros(m)])
    sc.inv_inertia = np.concatenate([sc.inv_inertia, np.zeros(m)])
    sc.species_index = np.concatenate([sc.species_index, np.zeros(m, np.int32)])
    sc.ids = np.arange(n_live + m, dtype=np.int32)
    if psd == "range":
        kw = dict(psd=psd_uniform(0.4 * d, 0.6 * d, 2))
    elif psd == "single":
        kw = dict(radius=0.5 * d)
    else:
        kw = dict(psd=psd_uniform(0.45 * d, 0.55 * d, 8), psd_seed=psd_seed)
    if chute:
        b = insertion_boundary((0.5 * d, 0.0, 6 * d), (2 * d, L, 12 * d), float(sc.density[0]), max_failed=max_failed,
                               volume_flow_rate=rate, chute=(0.5 * d, 0.1, 0.2), **kw)
    else:
        b = insertion_boundary((0.0, 0.0, 3 * d), (L, L, 12 * d), float(sc.density[0]), max_failed=max_failed,
                               vel_min=(-0.05, -0.05, -1.0), vel_max=(0.05, 0.05, 0.0), volume_flow_rate=rate, **kw)
    return sc, [b]


def chute_fill_case(n_base_free=0, n_free=3000, lx=12, ly=6, height=6, seed=13):
    """A periodic chute (x and y periodic, 12 x 6 diameters, domain z from 0
    to twice the inflow height) whose base is the seeded rough base of fixed
    spheres of scenarios.periodic_chute, and Chute::addFlowParticlesCompactly
    filling it to an inflow height of `height` diameters with radii 0.45 d ..
    0.55 d (fixed particle radius 0.5 d). Returns (scenario, fill)."""
    from mercurydpm_fork_b200.engine import chute_fill
    d = 1e-3
    sc = scenarios.periodic_chute(n_flow=1, seed=seed, lx=lx, ly=ly)
    base = sc.inv_mass == 0.0
    for k in ("position", "velocity", "radius", "inv_mass", "inv_inertia", "species_index"):
        setattr(sc, k, getattr(sc, k)[base])
    nb = int(base.sum())
    m = n_free
    sc.position = np.vstack([sc.position, np.zeros((m, 3))])
    sc.velocity = np.vstack([sc.velocity, np.zeros((m, 3))])
    sc.radius = np.concatenate([sc.radius, np.zeros(m)])
    sc.inv_mass = np.concatenate([sc.inv_mass, np.zeros(m)])
    sc.inv_inertia = np.concatenate([sc.inv_inertia, np.zeros(m)])
    sc.species_index = np.concatenate([sc.species_index, np.zeros(m, np.int32)])
    sc.ids = np.arange(nb + m, dtype=np.int32)
    import dataclasses
    sc.instance = dataclasses.replace(sc.instance, domain_min=(0.0, 0.0, 0.0),
                                      domain_max=(sc.instance.domain_max[0], sc.instance.domain_max[1], 2 * height * d))
    inst = sc.instance
    f = chute_fill(x_max=inst.periodic_max[0], y_max=inst.periodic_max[1], inflow_height=height * d,
                   min_radius=0.45 * d, max_radius=0.55 * d, density=float(sc.density[0]),
                   fixed_particle_radius=0.5 * d, x_min=inst.periodic_min[0], y_min=inst.periodic_min[1],
                   z_min=inst.domain_min[2])
    return sc, f

"""Seeded synthetic DEM workloads with the shapes of the benchmark set-ups.

Each builder returns a :class:`Scenario`: ABI structures (config, instance,
species table, walls) plus particle arrays in the caller order. The same
Scenario feeds the GPU engine, the CPU oracle and the reference build, so
all three start from bit-identical inputs.

* :func:`settling_box` -- monodisperse spheres on a jittered simple-cubic
  lattice in a closed box of six InfiniteWalls under gravity
  (LinearViscoelasticSlidingFrictionSpecies).
* :func:`periodic_chute` -- bidisperse (size ratio 2) spheres over a rough
  base of fixed spheres, periodic in x and y, gravity inclined like
  Chute::setChuteAngleAndMagnitudeOfGravity (Kernel/Chute.cc:789-805).
* :func:`rotating_drum` -- bidisperse (size ratio 3, 90 % small by number)
  spheres in a cylinder (AxisymmetricIntersectionOfWalls) with two flat end
  caps, rotating about x, Hertz-Mindlin with rolling and torsion friction.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .engine import Instance, axisymmetric_wall, infinite_wall, species_pair
from .host import hertz_dissipation_from_restitution, linear_collision_time_restitution, sphere_inv_mass_inertia, PI


@dataclass
class Scenario:
    name: str
    time_step: float
    instance: Instance
    species: list
    density: np.ndarray
    walls: list
    position: np.ndarray
    velocity: np.ndarray
    radius: np.ndarray
    inv_mass: np.ndarray
    inv_inertia: np.ndarray
    species_index: np.ndarray
    ids: np.ndarray
    rotation: bool = True
    info: dict = field(default_factory=dict)
    angular_velocity: np.ndarray | None = None   # None: at rest
    orientation: np.ndarray | None = None        # None: identity quaternions

    @property
    def n(self) -> int:
        return len(self.radius)

    @property
    def n_moving(self) -> int:
        return int(np.count_nonzero(self.inv_mass))

    def config(self, **kw) -> _abi.Config:
        c = _abi.Config()
        c.time_step = self.time_step
        c.background_drag = 0.0
        c.rotation = 1 if self.rotation else 0
        c.device = kw.get("device", 0)
        c.max_neighbors = kw.get("max_neighbors", 0)
        c.use_graphs = kw.get("use_graphs", 1)
        c.skin = kw.get("skin", 0.0)
        c.n_instances = 1
        return c

    def engine(self, **kw):
        from .engine import DemEngine
        e = DemEngine(self.time_step, [self.instance], self.species, self.walls, rotation=self.rotation, **kw)
        e.upload(self.position, self.velocity, self.radius, self.inv_mass, self.inv_inertia, self.species_index,
                 self.ids, angular_velocity=self.angular_velocity, orientation=self.orientation)
        return e


def linear_sliding_species(tc: float, eps: float, mass: float, mu: float, kt_ratio: float = 2.0 / 7.0,
                           gt_ratio: float = 0.0, constant_restitution: bool = False) -> _abi.SpeciesPair:
    k, g = linear_collision_time_restitution(tc, eps, mass)
    return species_pair(normal_law=_abi.DEM_NORMAL_LINEAR_VISCOELASTIC, friction_law=_abi.DEM_FRICTION_SLIDING,
                        constant_restitution=1 if constant_restitution else 0, stiffness=k, dissipation=g,
                        sliding_stiffness=kt_ratio * k, sliding_dissipation=gt_ratio * g, sliding_mu=mu,
                        sliding_mu_static=mu)


def settling_box(n: int = 5000, seed: int = 1, d: float = 1e-3, density: float = 2000.0, tc: float = 1e-4,
                 eps: float = 0.8, mu: float = 0.5, box=(20, 20, 40), spacing: float = 1.1,
                 jitter: float = 0.05, vstd: float = 0.01) -> Scenario:
    """Monodisperse settling box: simple-cubic lattice (spacing 1.1 d), first
    n sites in x-fastest order, positions jittered U[-0.05, 0.05] d,
    velocities N(0, 0.01 m/s), six walls, gravity -9.81 z, dt = tc/50."""
    rng = np.random.Generator(np.random.PCG64(seed))
    r = 0.5 * d
    Lx, Ly, Lz = (b * d for b in box)
    nx = int(Lx / (spacing * d))
    ny = int(Ly / (spacing * d))
    nz = int(Lz / (spacing * d))
    if n > nx * ny * nz:
        raise ValueError("too many particles for the lattice")
    i = np.arange(n)
    ix, iy, iz = i % nx, (i // nx) % ny, i // (nx * ny)
    off = np.array([(Lx - nx * spacing * d) / 2, (Ly - ny * spacing * d) / 2, (Lz - nz * spacing * d) / 2])
    pos = (np.stack([ix, iy, iz], 1) + 0.5) * spacing * d + off
    pos = pos + rng.uniform(-jitter * d, jitter * d, size=(n, 3))
    vel = rng.normal(0.0, vstd, size=(n, 3))
    radius = np.full(n, r)
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    mass = 1.0 / inv_mass[0]
    sp = linear_sliding_species(tc, eps, mass, mu)
    walls = [
        infinite_wall((-1, 0, 0), (0, 0, 0)), infinite_wall((1, 0, 0), (Lx, 0, 0)),
        infinite_wall((0, -1, 0), (0, 0, 0)), infinite_wall((0, 1, 0), (0, Ly, 0)),
        infinite_wall((0, 0, -1), (0, 0, 0)), infinite_wall((0, 0, 1), (0, 0, Lz)),
    ]
    inst = Instance(domain_min=(0, 0, 0), domain_max=(Lx, Ly, Lz), gravity=(0, 0, -9.81), n_species=1)
    return Scenario("settling_box", tc / 50, inst, [sp], np.array([density]), walls, pos, vel, radius, inv_mass,
                    inv_inertia, np.zeros(n, np.int32), np.arange(n, dtype=np.int32),
                    info=dict(n=n, d=d, seed=seed, box=box))


def chute_gravity(angle_deg: float, g: float = 9.81):
    """Chute::setChuteAngleAndMagnitudeOfGravity: (sin a, 0, -cos a) g."""
    a = angle_deg * PI / 180.
    return (math.sin(a) * g, 0.0, -math.cos(a) * g)


def _rough_base(rng, Lx, Ly, r_lo, r_hi, area_fraction):
    """Fixed spheres at random non-overlapping xy positions on z = 0."""
    mean_area = PI * (r_lo * r_lo + r_lo * r_hi + r_hi * r_hi) / 3.0
    target = int(round(area_fraction * Lx * Ly / mean_area))
    cell = 2.0 * r_hi
    nxc, nyc = max(1, int(Lx / cell)), max(1, int(Ly / cell))
    grid = {}
    pos, rad = [], []
    attempts = 0
    while len(pos) < target and attempts < 200 * target:
        attempts += 1
        x, y = rng.uniform(0, Lx), rng.uniform(0, Ly)
        rr = rng.uniform(r_lo, r_hi)
        cx, cy = int(x / Lx * nxc) % nxc, int(y / Ly * nyc) % nyc
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for j in grid.get(((cx + dx) % nxc, (cy + dy) % nyc), ()):
                    ddx = x - pos[j][0]
                    ddy = y - pos[j][1]
                    ddx -= Lx * round(ddx / Lx)
                    ddy -= Ly * round(ddy / Ly)
                    if ddx * ddx + ddy * ddy < (rr + rad[j]) ** 2:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            grid.setdefault((cx, cy), []).append(len(pos))
            pos.append((x, y, 0.0))
            rad.append(rr)
    return np.array(pos), np.array(rad)


def _hcp_layers(rng, Lx, Ly, z0, counts_radii, spacing_factor, pattern):
    """Close-packed triangular layers with ABC stacking, periodic in x and y.

    counts_radii: {"L": (n, sampler), "S": (n, sampler)}; pattern: the layer
    type sequence that repeats ("LLLLS"). A layer's nearest-neighbour spacing
    is spacing_factor x the mean diameter of its type, stretched so that an
    integer number of rows and columns fills the periodic box exactly."""
    left = {k: v[0] for k, v in counts_radii.items()}
    pos, rad = [], []
    z = z0
    prev_r = None
    layer = 0
    while any(v > 0 for v in left.values()):
        kind = pattern[layer % len(pattern)]
        layer += 1
        if left[kind] <= 0:
            continue
        n_kind, sampler, r_mean = counts_radii[kind]
        s = 2.0 * r_mean * spacing_factor
        nx = max(3, int(round(Lx / s)))
        ny = max(4, 2 * int(round(Ly / (s * math.sqrt(3.0) / 2.0) / 2.0)))
        ax, ay = Lx / nx, Ly / ny
        if prev_r is None:
            z = z0 + r_mean
        elif prev_r == r_mean:  # same kind: close-packed layer distance
            z += 2.0 * r_mean * spacing_factor * math.sqrt(2.0 / 3.0)
        else:  # change of kind: centres may sit on top of each other
            z += (prev_r + r_mean) * spacing_factor
        k3 = layer % 3  # ABC stacking: shift by the hollow-site offset (a1 + a2) / 3
        take = min(left[kind], nx * ny)
        j = np.arange(take)
        ix, iy = j % nx, j // nx
        x = (ix + 0.5 * (iy % 2) + 0.5 * k3) * ax
        y = (iy + k3 / 3.0) * ay
        pos.append(np.stack([np.mod(x, Lx), np.mod(y, Ly), np.full(take, z)], 1))
        rad.append(sampler(take))
        left[kind] -= take
        prev_r = r_mean
    return np.concatenate(pos), np.concatenate(rad)


def periodic_chute(n_flow: int = 200_000, seed: int = 2, ds: float = 1e-3, density: float = 2000.0,
                   tc: float = 1e-4, eps: float = 0.88, mu: float = 0.5, angle: float = 24.0,
                   lx: float = 100.0, ly: float = 50.0, base_fraction: float = 0.6, vstd: float = 0.01,
                   site_scale: float = 1.0, base_gap: float = 1.2, packing: str = "sites",
                   spacing_factor: float = 1.0) -> Scenario:
    """Periodic inclined chute: n_flow spheres, 50:50 by number, small radii
    U[0.45, 0.55] ds, large = 2x; periodic 100 x 50 small diameters; rough
    base of fixed small spheres (area fraction 0.6); 24 deg; dt = tc/50.
    Flowing spheres start on a lattice of 2.2 ds sites (times site_scale),
    each holding one large sphere or a 2x2x2 block of small ones, base_gap ds
    above the base; site_scale < 1 starts the bed pre-compressed."""
    rng = np.random.Generator(np.random.PCG64(seed))
    Lx, Ly = lx * ds, ly * ds
    r_lo, r_hi = 0.45 * ds, 0.55 * ds
    bpos, brad = _rough_base(rng, Lx, Ly, r_lo, r_hi, base_fraction)
    n_large = n_flow // 2
    n_small = n_flow - n_large
    site = 2.2 * ds * site_scale
    # a pre-compressed bed also closes the gaps across the periodic boundaries
    fit = math.ceil if site_scale < 1.0 else int
    sx, sy = fit(Lx / site), fit(Ly / site)
    n_small_sites = (n_small + 7) // 8
    n_sites = n_large + n_small_sites
    kinds = np.zeros(n_sites, np.int8)
    kinds[rng.permutation(n_sites)[:n_small_sites]] = 1
    pos, rad = [], []
    small_left = n_small
    z0 = r_hi + base_gap * ds
    if packing == "layers":
        fpos, frad = _hcp_layers(
            rng, Lx, Ly, r_hi * spacing_factor,
            {"L": (n_large, lambda k: 2.0 * rng.uniform(r_lo, r_hi, k), r_lo + r_hi),
             "S": (n_small, lambda k: rng.uniform(r_lo, r_hi, k), 0.5 * (r_lo + r_hi))},
            spacing_factor, "LLLLS")
        n_sites = 0
    for s in range(n_sites):
        ix, iy, iz = s % sx, (s // sx) % sy, s // (sx * sy)
        base = np.array([(ix + 0.5) * (Lx / sx), (iy + 0.5) * (Ly / sy), z0 + (iz + 0.5) * site])
        if kinds[s] == 0:
            pos.append(base)
            rad.append(2.0 * rng.uniform(r_lo, r_hi))
        else:
            for k in range(8):
                if small_left == 0:
                    break
                o = (np.array([k & 1, (k >> 1) & 1, (k >> 2) & 1]) - 0.5) * (site / 2)
                pos.append(base + o)
                rad.append(rng.uniform(r_lo, r_hi))
                small_left -= 1
    if packing != "layers":
        fpos = np.array(pos)
        frad = np.array(rad)
    top = float(fpos[:, 2].max()) + 2 * ds
    position = np.concatenate([bpos, fpos])
    radius = np.concatenate([brad, frad])
    n = len(radius)
    velocity = np.zeros((n, 3))
    velocity[len(brad):] = rng.normal(0.0, vstd, size=(len(frad), 3))
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    inv_mass[: len(brad)] = 0.0
    inv_inertia[: len(brad)] = 0.0
    m_small = 4.0 / 3.0 * PI * (0.5 * ds) ** 3 * density
    sp = linear_sliding_species(tc, eps, m_small, mu)
    inst = Instance(domain_min=(0, 0, -2 * ds), domain_max=(Lx, Ly, top + 20 * ds), gravity=chute_gravity(angle),
                    n_species=1, periodic_mask=0b011, periodic_min=(0, 0, 0), periodic_max=(Lx, Ly, 0))
    return Scenario("periodic_chute", tc / 50, inst, [sp], np.array([density]), [], position, velocity, radius,
                    inv_mass, inv_inertia, np.zeros(n, np.int32), np.arange(n, dtype=np.int32),
                    info=dict(n_flow=len(frad), n_base=len(brad), seed=seed, angle=angle, lx=lx, ly=ly))


def hertz_mindlin_species(E: float, G: float, eps: float, mu: float, mu_r: float = 0.0, mu_o: float = 0.0,
                          sliding_dissipation: float = 0.0, rolling_dissipation: float = 0.0,
                          torsion_dissipation: float = 0.0, rolling_torsion: bool = True) -> _abi.SpeciesPair:
    """HertzianViscoelasticMindlin(RollingTorsion)Species: effective elastic
    modulus E and restitution eps
    (setEffectiveElasticModulusAndRestitutionCoefficient,
    HertzianViscoelasticNormalSpecies.cc:109-140), effective shear modulus G
    (MindlinSpecies::setEffectiveShearModulus), Coulomb coefficients
    mu (sliding), mu_r (rolling), mu_o (torsion), static = dynamic."""
    law = _abi.DEM_FRICTION_MINDLIN_ROLLING_TORSION if rolling_torsion else _abi.DEM_FRICTION_MINDLIN
    return species_pair(normal_law=_abi.DEM_NORMAL_HERTZIAN_VISCOELASTIC, friction_law=law, elastic_modulus=E,
                        dissipation=hertz_dissipation_from_restitution(eps), shear_modulus=G,
                        sliding_dissipation=sliding_dissipation, sliding_mu=mu, sliding_mu_static=mu,
                        rolling_dissipation=rolling_dissipation, rolling_mu=mu_r, rolling_mu_static=mu_r,
                        torsion_dissipation=torsion_dissipation, torsion_mu=mu_o, torsion_mu_static=mu_o)


def hertz_collision_time(d: float, density: float, E: float, v: float = 1.0) -> float:
    """HertzianViscoelasticNormalSpecies::getCollisionTime(d, rho, v)
    (HertzianViscoelasticNormalSpecies.cc:290-300): 2.214 (rho^2/E^2/v)^0.2 d."""
    return 2.214 * ((density / E) ** 2 / v) ** 0.2 * d


def _press_onto_cylinder(position, radius, R, band, overlap, tolerance):
    """Moves spheres whose surface lies within `band` of a cylinder of radius
    R about x radially outwards until they overlap it by `overlap`, outermost
    first, keeping a move only if the sphere then overlaps no other sphere by
    more than `tolerance` (in place)."""
    from scipy.spatial import cKDTree
    rho = np.hypot(position[:, 1], position[:, 2])
    cand = np.nonzero(rho + radius > R - band)[0]
    cand = cand[np.argsort(-(rho[cand] + radius[cand]))]
    tree = cKDTree(position)
    reach = 2.0 * radius.max() + band
    for i in cand:
        new = position[i].copy()
        new[1:] *= (R - radius[i] + overlap) / rho[i]
        near = [j for j in tree.query_ball_point(new, reach) if j != i]
        if near:
            gap = np.linalg.norm(position[near] - new, axis=1) - radius[near] - radius[i]
            if gap.min() < -tolerance:
                continue
        position[i] = new


def rotating_drum(n: int = 1_000_000, seed: int = 3, ds: float = 1e-3, size_ratio: float = 3.0,
                  frac_small: float = 0.9, radius_d: float = 120.0, length_d: float = 60.0, omega: float = 1.0,
                  E: float = 1e7, nu: float = 0.3, mu: float = 0.4, mu_r: float = 0.05, eps: float = 0.7,
                  density: float = 2000.0, dt_factor: float = 0.02, site_spacing: float = 1.02,
                  jitter: float = 0.005, vstd: float = 0.0, touch_wall: float = 0.0, gravity: float = 9.81,
                  mu_o: float = 0.0, sliding_dissipation: float = 0.0, rolling_dissipation: float = 0.0,
                  torsion_dissipation: float = 0.0, wall_contact: bool = False) -> Scenario:
    """Rotating drum: n spheres, frac_small of them small (diameter ds), the
    rest size_ratio x larger, in a cylinder of radius radius_d ds and length
    length_d ds along x (AxisymmetricIntersectionOfWalls with setAxis(1,0,0)
    and one face addObject((1,0,0), (R,0,0))) closed by two InfiniteWall
    caps; the cylinder rotates at omega rad/s about x, gravity -z.

    Species: Hertz-Mindlin with rolling and torsion friction, effective
    E and G = E/2 (1 + nu) (the reference's
    setEffectiveElasticModulusAndPoissonRatio, HertzianViscoelasticNormalSpecies.cc:158),
    restitution eps; dt = dt_factor x the Hertz collision time of two small
    spheres at 1 m/s.

    Packing: cubes of 3 x 3 x 3 lattice sites (site_spacing ds apart), each
    holding one large sphere or up to 27 small ones, filled from the bottom of
    the drum upwards, large cubes chosen in seeded random order, positions
    jittered by +-jitter ds. site_spacing < 1 starts the bed pre-compressed.
    touch_wall > 0 moves every sphere within touch_wall ds of the cylinder
    radially onto it with an overlap of 0.1 touch_wall ds. wall_contact puts
    the bed in contact with both walls the way the lattice's neighbours touch
    each other (overlap 0.001 ds): spheres within 1.5 ds of the cylinder
    is moved radially onto it (see _press_onto_cylinder), and each cap is
    placed 0.001 ds inside the lattice's end face (the outermost sites' centre
    plus radius)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    R, L = radius_d * ds, length_d * ds
    r_s, r_l = 0.5 * ds, 0.5 * ds * size_ratio
    n_small = int(round(frac_small * n))
    n_large = n - n_small
    b = int(math.ceil(size_ratio - 1e-9))
    s = site_spacing * ds
    B = b * s
    per_block = b ** 3
    n_blocks = n_large + (n_small + per_block - 1) // per_block
    nx = int(L // B)
    nyz = int(2 * R // B)
    xs = (np.arange(nx) - (nx - 1) / 2) * B
    ys = (np.arange(nyz) - (nyz - 1) / 2) * B
    X, Y, Z = np.meshgrid(xs, ys, ys, indexing="ij")
    cen = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    reach = np.hypot(np.abs(cen[:, 1]) + B / 2, np.abs(cen[:, 2]) + B / 2)
    cen = cen[reach <= R]
    if len(cen) < n_blocks:
        raise ValueError(f"{n} spheres do not fit: {n_blocks} blocks needed, {len(cen)} available")
    order = np.lexsort((cen[:, 0], cen[:, 1], cen[:, 2]))
    cen = cen[order[:n_blocks]]
    large_block = np.zeros(n_blocks, bool)
    large_block[rng.permutation(n_blocks)[:n_large]] = True
    sub = (np.stack(np.meshgrid(np.arange(b), np.arange(b), np.arange(b), indexing="ij"), -1).reshape(-1, 3)
           - (b - 1) / 2) * s
    small_pos = (cen[~large_block][:, None, :] + sub[None, :, :]).reshape(-1, 3)[:n_small]
    large_pos = cen[large_block]
    position = np.concatenate([small_pos, large_pos])
    radius = np.concatenate([np.full(n_small, r_s), np.full(n_large, r_l)])
    species_index = np.concatenate([np.zeros(n_small, np.int32), np.ones(n_large, np.int32)])
    perm = rng.permutation(n)
    position, radius, species_index = position[perm], radius[perm], species_index[perm]
    position = position + rng.uniform(-jitter * ds, jitter * ds, size=position.shape)
    if touch_wall > 0.0:
        rho = np.hypot(position[:, 1], position[:, 2])
        near = rho + radius > R - touch_wall * ds
        target = R - radius[near] + 0.1 * touch_wall * ds
        position[near, 1:] *= (target / rho[near])[:, None]
    cap = L / 2
    if wall_contact:
        lap = 0.001 * ds
        _press_onto_cylinder(position, radius, R, band=1.5 * ds, overlap=lap, tolerance=0.005 * ds)
        # end face of the lattice: outermost block centre + (b-1)/2 sites + a small radius
        cap = float(np.max(np.abs(cen[:, 0]))) + (b - 1) / 2 * s + r_s - lap
    velocity = rng.normal(0.0, vstd, size=(n, 3)) if vstd > 0 else np.zeros((n, 3))
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    G = E / 2 * (1 + nu)
    sp = hertz_mindlin_species(E, G, eps, mu, mu_r, mu_o, sliding_dissipation, rolling_dissipation,
                               torsion_dissipation)
    table = [sp] * 9  # species 0 small, 1 large, 2 wall; identical mixed entries
    walls = [axisymmetric_wall((1, 0, 0), [((1, 0, 0), (R, 0, 0))], species=2, angular_velocity=(omega, 0, 0)),
             infinite_wall((-1, 0, 0), (-cap, 0, 0), species=2),
             infinite_wall((1, 0, 0), (cap, 0, 0), species=2)]
    m = 2 * R + 4 * r_l
    inst = Instance(domain_min=(-L / 2 - 2 * r_l, -m / 2, -m / 2), domain_max=(L / 2 + 2 * r_l, m / 2, m / 2),
                    gravity=(0.0, 0.0, -gravity), n_species=3)
    dt = dt_factor * hertz_collision_time(ds, density, E, 1.0)
    return Scenario("rotating_drum", dt, inst, table, np.array([density] * 3), walls, position, velocity, radius,
                    inv_mass, inv_inertia, species_index, np.arange(n, dtype=np.int32),
                    info=dict(n=n, n_small=n_small, n_large=n_large, seed=seed, radius_d=radius_d,
                              length_d=length_d, omega=omega, shear_modulus=G,
                              solid_fraction_of_drum=float(np.sum(4 / 3 * PI * radius ** 3) / (PI * R * R * L))))


@dataclass
class Batch:
    """Several independent simulations in one handle (dem_instance_desc per
    member): species tables concatenated with per-instance offsets, walls and
    particles tagged with their instance, particle ids offset so that they are
    unique across the batch (the order within each member is kept, so every
    member's lower-id rule is unchanged)."""
    time_step: float
    instances: list
    species: list
    walls: list
    position: np.ndarray
    velocity: np.ndarray
    radius: np.ndarray
    inv_mass: np.ndarray
    inv_inertia: np.ndarray
    species_index: np.ndarray
    ids: np.ndarray
    instance: np.ndarray
    members: list
    offsets: np.ndarray
    deletions: list = field(default_factory=list)
    rotation: bool = True

    @property
    def n(self) -> int:
        return len(self.radius)

    def engine(self, **kw):
        from .engine import DemEngine
        e = DemEngine(self.time_step, self.instances, self.species, self.walls, rotation=self.rotation,
                      deletions=self.deletions, **kw)
        e.upload(self.position, self.velocity, self.radius, self.inv_mass, self.inv_inertia, self.species_index,
                 self.ids, instance=self.instance)
        return e

    def member_slice(self, k: int) -> slice:
        return slice(int(self.offsets[k]), int(self.offsets[k + 1]))


def batch(members: list, time_step: float | None = None, deletions: list | None = None) -> Batch:
    """Combines Scenarios into one Batch; all members run with one time step
    (the smallest of theirs unless given). `deletions` holds, per member, a
    list of (normal, distance) DeletionBoundary planes."""
    import copy
    from .engine import Instance, deletion_boundary
    dt = min(m.time_step for m in members) if time_step is None else time_step
    instances, species, walls, dels = [], [], [], []
    id_off = 0
    offsets = [0]
    for k, m in enumerate(members):
        inst = copy.copy(m.instance)
        inst.species_offset = len(species)
        instances.append(inst)
        species.extend(m.species)
        for w in m.walls:
            w2 = copy.copy(w)
            w2.instance = k
            walls.append(w2)
        if deletions is not None:
            for nrm, dist in deletions[k]:
                dels.append(deletion_boundary(nrm, dist, instance=k))
        offsets.append(offsets[-1] + m.n)
    cat = lambda f: np.concatenate([getattr(m, f) for m in members])
    ids = np.concatenate([m.ids.astype(np.int64) + sum(mm.n for mm in members[:k]) for k, m in enumerate(members)])
    return Batch(dt, instances, species, walls, cat("position"), cat("velocity"), cat("radius"), cat("inv_mass"),
                 cat("inv_inertia"), cat("species_index").astype(np.int32), ids.astype(np.int32),
                 np.concatenate([np.full(m.n, k, np.int32) for k, m in enumerate(members)]), members,
                 np.array(offsets), dels, rotation=all(m.rotation for m in members))


def triangle_floor(n: int = 200_000, seed: int = 4, d: float = 1e-3, density: float = 2000.0, tc: float = 1e-4,
                   eps: float = 0.8, mu: float = 0.5, l_d: float = 100.0, spacing: float = 1.05,
                   amplitude_d: float = 3.0, group: int = 1, vstd: float = 0.01, drop_d: float = 1.0,
                   v0: float = 0.0) -> Scenario:
    """Spheres (d = 1 mm, linear viscoelastic + sliding friction) on a simple-
    cubic lattice (spacing 1.05 d) falling onto a triangulated floor: a height
    field over the periodic square [0, L]^2 (L = 100 d, periodic in x and y)
    with 5 x 5 nodes, heights amplitude x a seeded pattern, 32 TriangleWalls of
    one group (as a mesh read by WallHandler::readTriangleWall gets). The
    lowest layer starts drop_d diameters above the highest floor node, every
    sphere moving down at v0."""
    from .engine import triangle_wall
    rng = np.random.Generator(np.random.PCG64(seed))
    r = 0.5 * d
    L = l_d * d
    nodes = np.linspace(0.0, L, 5)
    hz = rng.uniform(0.0, amplitude_d * d, size=(5, 5))
    hz[-1, :] = hz[0, :]  # the floor is periodic
    hz[:, -1] = hz[:, 0]
    walls = []
    for i in range(4):
        for j in range(4):
            p = [np.array([nodes[i + a], nodes[j + b], hz[i + a, j + b]]) for a, b in ((0, 0), (1, 0), (0, 1), (1, 1))]
            if (i + j) % 2 == 0:
                walls += [triangle_wall(p[0], p[1], p[3], group=group), triangle_wall(p[0], p[3], p[2], group=group)]
            else:
                walls += [triangle_wall(p[0], p[1], p[2], group=group), triangle_wall(p[1], p[3], p[2], group=group)]
    nx = int(L / (spacing * d))
    nz = -(-n // (nx * nx))
    i = np.arange(n)
    ix, iy, iz = i % nx, (i // nx) % nx, i // (nx * nx)
    z0 = hz.max() + r + drop_d * d
    pos = np.stack([(ix + 0.5) * spacing * d, (iy + 0.5) * spacing * d, z0 + iz * spacing * d], 1)
    vel = rng.normal(0.0, vstd, size=(n, 3))
    vel[:, 2] -= v0
    radius = np.full(n, r)
    inv_mass, inv_inertia = sphere_inv_mass_inertia(radius, density)
    sp = linear_sliding_species(tc, eps, 1.0 / inv_mass[0], mu)
    top = z0 + nz * spacing * d + 10 * d
    inst = Instance(domain_min=(0, 0, -d), domain_max=(L, L, top), gravity=(0, 0, -9.81), n_species=1,
                    periodic_mask=0b011, periodic_min=(0, 0, 0), periodic_max=(L, L, 0))
    return Scenario("triangle_floor", tc / 50, inst, [sp], np.array([density]), walls, pos, vel, radius, inv_mass,
                    inv_inertia, np.zeros(n, np.int32), np.arange(n, dtype=np.int32),
                    info=dict(n=n, d=d, seed=seed, l_d=l_d, layers=nz, triangles=len(walls), group=group))


# The drum workload's radius, in small diameters. The configured drum
# (R = 120 d, L = 60 d) cannot hold 1,000,000 spheres of this size mix: their
# solid volume is 0.69 of the cylinder. At 175 d it is 0.33.
DRUM_RADIUS_D = 175.0


def dense_drum(n: int = 1_000_000, seed: int = 3, radius_d: float = DRUM_RADIUS_D) -> Scenario:
    """The rotating-drum workload (1,000,000 spheres, 10 % of them 3 d,
    Hertz-Mindlin with rolling and torsion friction, cylinder of 60 d length
    rotating at 1 rad/s about x, two flat caps) with its bed started as a
    lattice whose neighbours overlap by 0.1 % of a diameter (jitter
    +-0.005 d), so that nearly every sphere is in contact from the first time
    step. The first ~100 steps relax those overlaps (about 1.6 contacts per
    sphere then); the bed then loosens. The bed touches the cylinder and both
    caps the same way (rotating_drum's wall_contact)."""
    return rotating_drum(n=n, seed=seed, radius_d=radius_d, length_d=60.0, vstd=0.0, site_spacing=0.999,
                         wall_contact=True)

"""Python view of the C ABI: one :class:`DemEngine` per ``dem_handle``.

The engine state lives on the GPU; this class only converts numpy arrays to
the ABI's structure-of-arrays layout and raises :class:`DemError` on any
non-zero status. It is the interface the tests and ``bench.py`` use; C and
C++ callers use ``include/dem_b200.h`` directly.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        _lib = _abi.load()
    return _lib


class DemError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{_abi.STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


def _dp(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _f64(a, shape=None):
    if a is None:
        return None
    out = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        out = out.reshape(shape)
    return out


def _i32(a):
    if a is None:
        return None
    return np.ascontiguousarray(a, dtype=np.int32)


@dataclass
class Instance:
    """One independent simulation inside a handle (dem_instance_desc)."""
    domain_min: tuple
    domain_max: tuple
    gravity: tuple = (0.0, 0.0, -9.81)
    n_species: int = 1
    species_offset: int = 0
    periodic_mask: int = 0
    periodic_min: tuple = (0.0, 0.0, 0.0)
    periodic_max: tuple = (0.0, 0.0, 0.0)

    def to_c(self) -> _abi.InstanceDesc:
        d = _abi.InstanceDesc()
        d.domain_min[:] = list(map(float, self.domain_min))
        d.domain_max[:] = list(map(float, self.domain_max))
        d.gravity[:] = list(map(float, self.gravity))
        d.periodic_mask = int(self.periodic_mask)
        d.species_offset = int(self.species_offset)
        d.n_species = int(self.n_species)
        d.periodic_min[:] = list(map(float, self.periodic_min))
        d.periodic_max[:] = list(map(float, self.periodic_max))
        return d


def deletion_boundary(normal, distance, instance=0) -> _abi.DeletionBoundary:
    """DeletionBoundary::set(normal, distance): particles with
    distance - x . normal < 0 are removed."""
    b = _abi.DeletionBoundary()
    b.instance = instance
    b.normal[:] = list(map(float, normal))
    b.distance = float(distance)
    return b


def insertion_boundary(pos_min, pos_max, density: float, radius: float | None = None, psd=None, species: int = 0,
                       instance: int = 0, max_failed: int = 0, vel_min=(0, 0, 0), vel_max=(0, 0, 0),
                       volume_flow_rate: float = float("inf"), initial_volume: float = 0.0,
                       psd_seed: int = 0, chute=None) -> _abi.InsertionBoundary:
    """CubeInsertionBoundary::set(particleToCopy, maxFailed, posMin, posMax,
    velMin, velMax) for a template particle of `species` (its density given
    here). Radii: `psd` = (radii, cumulative probabilities), e.g.
    host.psd_uniform(rmin, rmax, 2) for the set(..., rMin, rMax) form; with
    psd None the template's `radius` through the PSD InsertionBoundary::
    generateParticle builds when none is set (uniform from radius to radius,
    50 points). chute = (fixedParticleRadius, inflowVelocity,
    inflowVelocityVariance) makes it a ChuteInsertionBoundary instead
    (ChuteInsertionBoundary::set(particleToCopy, maxFailed, posMin, posMax,
    fixedParticleRadius, inflowVelocity, inflowVelocityVariance))."""
    from .host import psd_uniform
    if psd is None:
        if radius is None:
            raise ValueError("give radius or psd")
        psd = psd_uniform(radius, radius, 50)
    radii, probs = psd
    if not 2 <= len(radii) == len(probs) <= _abi.DEM_MAX_PSD_POINTS:
        raise ValueError("a PSD needs 2 to DEM_MAX_PSD_POINTS points")
    b = _abi.InsertionBoundary()
    b.instance, b.species, b.max_failed, b.n_psd = int(instance), int(species), int(max_failed), len(radii)
    b.kind = _abi.DEM_INSERTION_CUBE if chute is None else _abi.DEM_INSERTION_CHUTE
    if chute is not None:
        b.fixed_particle_radius, b.inflow_velocity, b.inflow_velocity_variance = (float(v) for v in chute)
    b.pos_min[:] = list(map(float, pos_min))
    b.pos_max[:] = list(map(float, pos_max))
    b.vel_min[:] = list(map(float, vel_min))
    b.vel_max[:] = list(map(float, vel_max))
    b.density = float(density)
    b.volume_flow_rate = float(volume_flow_rate)
    b.initial_volume = float(initial_volume)
    for k, (r, q) in enumerate(zip(radii, probs)):
        b.psd_radius[k] = float(r)
        b.psd_probability[k] = float(q)
    b.psd_seed = int(psd_seed)
    return b


def chute_fill(x_max: float, y_max: float, inflow_height: float, min_radius: float, max_radius: float,
               density: float, fixed_particle_radius: float = 0.0, x_min: float = 0.0, y_min: float = 0.0,
               z_min: float = 0.0, species: int = 0, instance: int = 0) -> _abi.ChuteFill:
    """Chute::addFlowParticlesCompactly for a chute of length x_max, width
    y_max (getChuteLength / getChuteWidth) with the given inflow height,
    inflow radii and fixed-particle radius (include/dem_b200.h,
    dem_chute_fill)."""
    f = _abi.ChuteFill()
    f.instance, f.species = int(instance), int(species)
    for k, v in dict(density=density, x_min=x_min, x_max=x_max, y_min=y_min, y_max=y_max, z_min=z_min,
                     inflow_height=inflow_height, min_radius=min_radius, max_radius=max_radius,
                     fixed_particle_radius=fixed_particle_radius).items():
        setattr(f, k, float(v))
    return f


def rng_draws(seed: int, n: int) -> np.ndarray:
    """RNG::getRandomNumber(0, 1), n times after RNG::setRandomSeed(seed), from
    the engine's generator (computed on the host; no device needed)."""
    out = np.zeros(n)
    rc = lib().dem_rng_draws(int(seed), int(n), _dp(out))
    if rc:
        raise DemError(rc, "dem_rng_draws failed")
    return out


def psd_draws(boundary: _abi.InsertionBoundary, n: int) -> np.ndarray:
    """The first n radii the boundary's PSD gives (PSD::drawSample), computed on the host."""
    out = np.zeros(n)
    rc = lib().dem_psd_draws(C.byref(boundary), int(n), _dp(out))
    if rc:
        raise DemError(rc, "dem_psd_draws failed")
    return out


def species_pair(**kw) -> _abi.SpeciesPair:
    s = _abi.SpeciesPair()
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def infinite_wall(normal, point, species=0, instance=0, velocity=(0, 0, 0), angular_velocity=(0, 0, 0),
                  orientation=None) -> _abi.Wall:
    """An InfiniteWall with outward normal `normal` through `point`.

    The orientation is the reference's quaternion for that normal
    (BaseInteractable::setOrientationViaNormal); pass it explicitly to reuse
    the exact quaternion a reference object holds.
    """
    from .host import quaternion_from_normal
    w = _abi.Wall()
    w.type = _abi.DEM_WALL_INFINITE
    w.species = species
    w.instance = instance
    w.position[:] = list(map(float, point))
    q = orientation if orientation is not None else quaternion_from_normal(normal)
    w.orientation[:] = list(map(float, q))
    w.velocity[:] = list(map(float, velocity))
    w.angular_velocity[:] = list(map(float, angular_velocity))
    return w


def intersection_wall(faces, position=(0, 0, 0), orientation=(1, 0, 0, 0), species=0, instance=0,
                      velocity=(0, 0, 0), angular_velocity=(0, 0, 0), axisymmetric=False) -> _abi.Wall:
    """IntersectionOfWalls (or, with axisymmetric=True,
    AxisymmetricIntersectionOfWalls) built from `faces`, a list of
    (normal, point) pairs as given to IntersectionOfWalls::addObject, in the
    wall's frame (position, orientation quaternion)."""
    if len(faces) > _abi.DEM_MAX_WALL_FACES:
        raise ValueError(f"at most {_abi.DEM_MAX_WALL_FACES} faces")
    w = _abi.Wall()
    w.type = _abi.DEM_WALL_AXISYMMETRIC if axisymmetric else _abi.DEM_WALL_INTERSECTION
    w.species = species
    w.instance = instance
    w.n_faces = len(faces)
    w.position[:] = list(map(float, position))
    w.orientation[:] = list(map(float, orientation))
    w.velocity[:] = list(map(float, velocity))
    w.angular_velocity[:] = list(map(float, angular_velocity))
    for k, (nrm, pt) in enumerate(faces):
        w.faces[k][:] = list(map(float, nrm)) + list(map(float, pt))
    return w


def triangle_wall(a, b, c, species=0, instance=0, group=0, position=None, orientation=(1, 0, 0, 0),
                  velocity=(0, 0, 0), angular_velocity=(0, 0, 0)) -> _abi.Wall:
    """TriangleWall with vertices a, b, c (lab frame): setVertices(a, b, c),
    whose position is (a + b + c) / 3 computed as Vec3D does, or
    setVertices(a, b, c, position); `group` is the wall's group id
    (WallHandler::readTriangleWall gives every triangle of a mesh one)."""
    a, b, c = (tuple(map(float, v)) for v in (a, b, c))
    if position is None:
        position = tuple((a[k] + b[k] + c[k]) / 3 for k in range(3))
    w = _abi.Wall()
    w.type = _abi.DEM_WALL_TRIANGLE
    w.species = species
    w.instance = instance
    w.n_faces = 3
    w.group = group
    w.position[:] = list(map(float, position))
    w.orientation[:] = list(map(float, orientation))
    w.velocity[:] = list(map(float, velocity))
    w.angular_velocity[:] = list(map(float, angular_velocity))
    for k, v in enumerate((a, b, c)):
        w.faces[k][:] = list(v) + [0.0, 0.0, 0.0]
    return w


def axisymmetric_wall(axis, faces, position=(0, 0, 0), species=0, instance=0, velocity=(0, 0, 0),
                      angular_velocity=(0, 0, 0)) -> _abi.Wall:
    """AxisymmetricIntersectionOfWalls with setAxis(axis), setPosition(position)
    and addObject(normal, point) for each (normal, point) of `faces`, given
    in (r, 0, a) coordinates."""
    from .host import quaternion_from_normal
    return intersection_wall(faces, position, quaternion_from_normal(axis), species, instance, velocity,
                             angular_velocity, axisymmetric=True)


class DemEngine:
    def __init__(self, time_step: float, instances: list[Instance], species: list[_abi.SpeciesPair],
                 walls: list[_abi.Wall] | None = None, rotation: bool = True, background_drag: float = 0.0,
                 max_neighbors: int = 0, skin: float = 0.0, use_graphs: bool = True, device: int = 0,
                 deletions: list | None = None, batch_api: bool = False, max_contacts: int = 0,
                 insertions: list | None = None, insertion_seeds=None, chute_fills: list | None = None):
        self._h = C.c_void_p()
        cfg = _abi.Config()
        cfg.time_step = time_step
        cfg.background_drag = background_drag
        cfg.rotation = 1 if rotation else 0
        cfg.device = device
        cfg.max_neighbors = max_neighbors
        cfg.use_graphs = 1 if use_graphs else 0
        cfg.skin = skin
        cfg.n_instances = len(instances)
        cfg.max_contacts = max_contacts
        arr = (_abi.InstanceDesc * len(instances))(*[i.to_c() for i in instances])
        if batch_api:
            rc = lib().dem_batch_create(C.byref(cfg), len(instances), arr, C.byref(self._h))
        else:
            rc = lib().dem_create(C.byref(cfg), arr, C.byref(self._h))
        if rc:
            raise DemError(rc, "dem_batch_create failed" if batch_api else "dem_create failed")
        self.n_instances = len(instances)
        sp = (_abi.SpeciesPair * len(species))(*species)
        self._check(lib().dem_set_species(self._h, sp, len(species)))
        self._species = list(species)
        self._rmin = self._rmax = 0.0
        walls = walls or []
        wa = (_abi.Wall * max(1, len(walls)))(*walls)
        self._check(lib().dem_set_walls(self._h, wa, len(walls)))
        self._nwalls = len(walls)
        dels = deletions or []
        da = (_abi.DeletionBoundary * max(1, len(dels)))(*dels)
        self._check(lib().dem_set_deletion_boundaries(self._h, da, len(dels)))
        self._n_ins = 0
        self._n_fill = 0
        if insertions or insertion_seeds is not None:
            self.set_insertion_boundaries(insertions or [], insertion_seeds)
        if chute_fills:
            self.set_chute_fills(chute_fills)
        self.n = 0

    def set_insertion_boundaries(self, insertions: list, seeds=None):
        """InsertionBoundary objects (see :func:`insertion_boundary`) and the
        per-instance RNG::setRandomSeed values; they take effect at the next
        upload, whose rows of radius 0 are the free rows they fill."""
        ia = (_abi.InsertionBoundary * max(1, len(insertions)))(*insertions)
        sa = None
        if seeds is not None:
            sa = (C.c_uint64 * self.n_instances)(*[int(x) for x in seeds])
        self._check(lib().dem_set_insertion_boundaries(self._h, ia, len(insertions), sa))
        self._n_ins = len(insertions)

    def set_chute_fills(self, fills: list):
        """Chute fills (:func:`chute_fill`) the next upload performs."""
        fa = (_abi.ChuteFill * max(1, len(fills)))(*fills)
        self._check(lib().dem_set_chute_fills(self._h, fa, len(fills)))
        self._n_fill = len(fills)

    def chute_fill_results(self):
        """(final inflow heights, particles placed) per chute fill of the last upload."""
        n = self._n_fill
        h = np.zeros(n)
        k = np.zeros(n, np.int64)
        self._check(lib().dem_get_chute_fill_results(self._h, _dp(h), k.ctypes.data_as(C.POINTER(C.c_int64)), n))
        return h, k

    def insertion_counts(self):
        """(particles placed, their volume) per insertion boundary."""
        n = self._n_ins
        cnt = np.zeros(n, np.int64)
        vol = np.zeros(n)
        self._check(lib().dem_get_insertion_counts(self._h, cnt.ctypes.data_as(C.POINTER(C.c_int64)), _dp(vol), n))
        return cnt, vol

    def set_deletion_boundaries(self, deletions: list):
        """Replaces the DeletionBoundary planes; between steps they apply from
        the next time step (BoundaryHandler::copyAndAddObject during a run)."""
        da = (_abi.DeletionBoundary * max(1, len(deletions)))(*deletions)
        self._check(lib().dem_set_deletion_boundaries(self._h, da, len(deletions)))

    def remove_wall(self, wall: int):
        """WallHandler::removeObject: wall `wall` (index in the constructor's
        list) makes no contacts from the next time step on."""
        self._check(lib().dem_remove_wall(self._h, int(wall)))

    # ------------------------------------------------------------------
    def _check(self, rc: int):
        if rc:
            msg = lib().dem_last_error(self._h)
            raise DemError(rc, msg.decode() if msg else "")

    def close(self):
        if self._h:
            lib().dem_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ------------------------------------------------------------------
    def upload(self, position, velocity, radius, inv_mass, inv_inertia, species, ids=None, angular_velocity=None,
               orientation=None, instance=None):
        n = len(radius)
        self._keep = dict(
            position=_f64(position, (n, 3)), velocity=_f64(velocity, (n, 3)),
            angular_velocity=_f64(angular_velocity, (n, 3)) if angular_velocity is not None else None,
            orientation=_f64(orientation, (n, 4)) if orientation is not None else None,
            radius=_f64(radius), inv_mass=_f64(inv_mass), inv_inertia=_f64(inv_inertia), species=_i32(species),
            id=_i32(ids if ids is not None else np.arange(n)), instance=_i32(instance))
        k = self._keep
        p = _abi.ParticlesSoA(n, _dp(k["position"]), _dp(k["velocity"]), _dp(k["angular_velocity"]),
                              _dp(k["orientation"]), _dp(k["radius"]), _dp(k["inv_mass"]), _dp(k["inv_inertia"]),
                              _ip(k["species"]), _ip(k["id"]), _ip(k["instance"]))
        self._check(lib().dem_upload_particles(self._h, C.byref(p)))
        self.n = n
        if n:
            self._rmin, self._rmax = float(np.min(k["radius"])), float(np.max(k["radius"]))

    def upload_contacts(self, id_p, id_i, springs, is_wall=None, periodic=None):
        m = len(id_p)
        keep = dict(id_p=_i32(id_p), id_i=_i32(id_i), is_wall=_i32(is_wall) if is_wall is not None else None,
                    periodic=_i32(periodic) if periodic is not None else None,
                    springs=_f64(springs, (m, 9)))
        c = _abi.ContactsSoA(m, _ip(keep["id_p"]), _ip(keep["id_i"]), _ip(keep["is_wall"]), _ip(keep["periodic"]),
                             _dp(keep["springs"]), None, None)
        self._check(lib().dem_upload_contacts(self._h, C.byref(c)))

    def step(self, n: int = 1):
        self._check(lib().dem_step(self._h, int(n)))

    def download(self, out: dict | None = None) -> dict:
        """Particle state in the caller's order. `out` may supply some of the
        arrays (e.g. in pinned memory); only the fields it names are read then."""
        n = self.n
        if out is None:
            out = dict(position=np.zeros((n, 3)), velocity=np.zeros((n, 3)), angular_velocity=np.zeros((n, 3)),
                       orientation=np.zeros((n, 4)), radius=np.zeros(n), inv_mass=np.zeros(n),
                       inv_inertia=np.zeros(n), species=np.zeros(n, np.int32), id=np.zeros(n, np.int32),
                       instance=np.zeros(n, np.int32))
        shapes = dict(position=((n, 3), np.float64), velocity=((n, 3), np.float64),
                      angular_velocity=((n, 3), np.float64), orientation=((n, 4), np.float64),
                      radius=((n,), np.float64), inv_mass=((n,), np.float64), inv_inertia=((n,), np.float64),
                      species=((n,), np.int32), id=((n,), np.int32), instance=((n,), np.int32))
        for k, a in out.items():
            if k not in shapes or a.shape != shapes[k][0] or a.dtype != shapes[k][1] or not a.flags.c_contiguous:
                raise ValueError(f"download: bad output array {k}")
        g = out.get
        p = _abi.ParticlesSoA(n, _dp(g("position")), _dp(g("velocity")), _dp(g("angular_velocity")),
                              _dp(g("orientation")), _dp(g("radius")), _dp(g("inv_mass")), _dp(g("inv_inertia")),
                              _ip(g("species")), _ip(g("id")), _ip(g("instance")))
        self._check(lib().dem_download_particles(self._h, C.byref(p)))
        return out

    def walls(self) -> list:
        """Current wall states (position and orientation after the steps taken)."""
        n = self._nwalls
        arr = (_abi.Wall * max(1, n))()
        self._check(lib().dem_download_walls(self._h, arr, n))
        return [arr[k] for k in range(n)]

    def forces(self):
        f = np.zeros((self.n, 3))
        t = np.zeros((self.n, 3))
        self._check(lib().dem_download_forces(self._h, _dp(f), _dp(t)))
        return f, t

    def contacts(self) -> dict:
        cnt = C.c_int64(0)
        self._check(lib().dem_download_contacts(self._h, None, 0, C.byref(cnt)))
        m = cnt.value
        out = dict(id_p=np.zeros(m, np.int32), id_i=np.zeros(m, np.int32), is_wall=np.zeros(m, np.int32),
                   periodic=np.zeros(m, np.int32), springs=np.zeros((m, 9)), force=np.zeros((m, 3)),
                   overlap=np.zeros(m))
        c = _abi.ContactsSoA(m, _ip(out["id_p"]), _ip(out["id_i"]), _ip(out["is_wall"]), _ip(out["periodic"]),
                             _dp(out["springs"]), _dp(out["force"]), _dp(out["overlap"]))
        self._check(lib().dem_download_contacts(self._h, C.byref(c), m, C.byref(cnt)))
        return out

    def contact_geometry(self) -> dict:
        """dem_download_contact_geometry: contact points, unit normals and
        friction forces of the contacts of contacts(), in the same order."""
        cnt = C.c_int64(0)
        self._check(lib().dem_download_contact_geometry(self._h, None, None, None, 0, C.byref(cnt)))
        m = cnt.value
        out = dict(contact_point=np.zeros((m, 3)), normal=np.zeros((m, 3)), tangential_force=np.zeros((m, 3)))
        self._check(lib().dem_download_contact_geometry(self._h, _dp(out["contact_point"]), _dp(out["normal"]),
                                                        _dp(out["tangential_force"]), m, C.byref(cnt)))
        return out

    def reduce(self, instance: int = 0) -> dict:
        g = _abi.Globals()
        self._check(lib().dem_reduce(self._h, instance, C.byref(g)))
        return dict(kinetic_energy=g.kinetic_energy, rotational_energy=g.rotational_energy,
                    gravitational_energy=g.gravitational_energy, elastic_energy=g.elastic_energy,
                    momentum=np.array(g.momentum[:]), angular_momentum=np.array(g.angular_momentum[:]),
                    mass=g.mass, centre_of_mass=np.array(g.centre_of_mass[:]), n_contacts=g.n_contacts,
                    n_wall_contacts=g.n_wall_contacts, time=g.time, n_steps=g.n_steps)

    def set_periodic(self, instance: int, lo, hi, mask: int):
        """dem_set_periodic (before upload)."""
        a = (C.c_double * 3)(*map(float, lo))
        b = (C.c_double * 3)(*map(float, hi))
        self._check(lib().dem_set_periodic(self._h, instance, a, b, mask))

    def batch_run(self, nsteps: int) -> dict:
        """dem_batch_run: nsteps, then the balances of every instance (as reduce_batch)."""
        arr = (_abi.Globals * max(1, self.n_instances))()
        self._check(lib().dem_batch_run(self._h, nsteps, arr))
        return self._globals_rows(arr, self.n_instances)

    def reduce_batch(self, first: int = 0, count: int | None = None) -> dict:
        """dem_reduce_batch: the balances of instances first..first+count-1 as
        arrays with one row per instance."""
        count = self.n_instances - first if count is None else count
        arr = (_abi.Globals * max(1, count))()
        self._check(lib().dem_reduce_batch(self._h, first, count, arr))
        return self._globals_rows(arr, count)

    @staticmethod
    def _globals_rows(arr, count: int) -> dict:
        g = arr[:count]
        return dict(kinetic_energy=np.array([x.kinetic_energy for x in g]),
                    rotational_energy=np.array([x.rotational_energy for x in g]),
                    gravitational_energy=np.array([x.gravitational_energy for x in g]),
                    elastic_energy=np.array([x.elastic_energy for x in g]),
                    mass=np.array([x.mass for x in g]),
                    momentum=np.array([x.momentum[:] for x in g]).reshape(count, 3),
                    centre_of_mass=np.array([x.centre_of_mass[:] for x in g]).reshape(count, 3),
                    n_contacts=np.array([x.n_contacts for x in g]),
                    n_wall_contacts=np.array([x.n_wall_contacts for x in g]))

    def cg(self, coordinates: int, n, lo, hi, width: float, cutoff_factor: float = 3.0, instance: int = 0):
        g = _abi.CGGrid()
        g.coordinates = coordinates
        g.instance = instance
        g.n[:] = list(map(int, n))
        g.min[:] = list(map(float, lo))
        g.max[:] = list(map(float, hi))
        g.width = width
        g.cutoff_factor = cutoff_factor
        npts = int(np.prod(n))
        out = np.zeros((npts, _abi.DEM_CG_NFIELDS))
        self._check(lib().dem_cg_eval(self._h, C.byref(g), _dp(out)))
        return out

    def cg_time_average(self, coordinates: int, n, lo, hi, width: float, steps_between: int, evaluations: int,
                        cutoff_factor: float = 3.0, instance: int = 0):
        """TimeAveragedCG<Coordinates, Gauss, StandardFields>
        (Kernel/CG/TimeAveragedCG.hcc:80-107): CG evaluated at the current
        state and after every further `steps_between` time steps,
        `evaluations` times in all (advancing the simulation), and averaged.
        The reference sums the raw fields of every evaluation, then divides
        by the averaged volume and by the number of evaluations; this is the
        mean of the volume-averaged fields of each evaluation."""
        total = None
        for k in range(int(evaluations)):
            if k:
                self.step(steps_between)
            f = self.cg(coordinates, n, lo, hi, width, cutoff_factor, instance)
            total = f if total is None else total + f
        return total / float(evaluations)

    def counts(self) -> dict:
        e, c, w = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        self._check(lib().dem_get_counts(self._h, C.byref(e), C.byref(c), C.byref(w)))
        return dict(list_entries=e.value, contacts=c.value, wall_contacts=w.value)

    def time_force_kernel(self, reps: int = 20) -> float:
        """Mean device milliseconds of one time-step force-kernel launch."""
        ms = C.c_double(0)
        self._check(lib().dem_time_force_kernel(self._h, int(reps), C.byref(ms)))
        return ms.value

    def autotune(self, reps: int = 20, cache: dict | None = None, key=None) -> dict:
        """dem_autotune: the fastest launch shape of each force kernel on the
        current state. With a `cache` dict, shapes are looked up and stored
        under `key` (default: workload_class() of this engine), so that
        engines of the same class skip the measurement."""
        t = _abi.Tuning()
        if cache is not None:
            key = key if key is not None else self.workload_class()
            if key in cache:
                t.detect_block, t.contacts_blocks_per_sm, t.sum_block = cache[key]
                self._check(lib().dem_set_tuning(self._h, C.byref(t)))
                return dict(detect_block=t.detect_block, contacts_blocks_per_sm=t.contacts_blocks_per_sm,
                            sum_block=t.sum_block, cached=True)
        self._check(lib().dem_autotune(self._h, int(reps), C.byref(t)))
        out = dict(detect_block=t.detect_block, contacts_blocks_per_sm=t.contacts_blocks_per_sm,
                   sum_block=t.sum_block, ms_before=t.ms_before, ms_after=t.ms_after, cached=False)
        if cache is not None:
            cache[key] = (t.detect_block, t.contacts_blocks_per_sm, t.sum_block)
        return out

    def set_tuning(self, detect_block: int, contacts_blocks_per_sm: int, sum_block: int):
        t = _abi.Tuning(detect_block, contacts_blocks_per_sm, sum_block, 0, 0.0, 0.0)
        self._check(lib().dem_set_tuning(self._h, C.byref(t)))

    def tuning(self) -> dict:
        t = _abi.Tuning()
        self._check(lib().dem_get_tuning(self._h, C.byref(t)))
        return dict(detect_block=t.detect_block, contacts_blocks_per_sm=t.contacts_blocks_per_sm,
                    sum_block=t.sum_block)

    def workload_class(self) -> tuple:
        """(particles to the nearest power of 2, law variant of the species
        table, size ratio to one decimal): the key the autotuner's cache uses."""
        import math
        st = self.stats()
        laws = sorted({(int(p.normal_law), int(p.friction_law)) for p in self._species})
        ratio = round(self._rmax / self._rmin, 1) if self._rmin > 0 else 1.0
        return (int(round(math.log2(max(1, st["n"])))), tuple(laws), ratio)

    def stats(self) -> dict:
        ms = C.c_double(0)
        launches = C.c_int64(0)
        rebuilds = C.c_int64(0)
        self._check(lib().dem_last_step_stats(self._h, C.byref(ms), C.byref(launches), C.byref(rebuilds)))
        n = C.c_int64(0)
        cap = C.c_int64(0)
        cells = C.c_int64(0)
        self._check(lib().dem_get_info(self._h, C.byref(n), C.byref(cap), C.byref(cells)))
        return dict(ms=ms.value, kernel_launches=launches.value, rebuilds=rebuilds.value, n=n.value,
                    max_neighbors=cap.value, n_cells=cells.value)

    def memory(self) -> dict:
        """Device bytes held by the handle's arrays and the contact capacity
        (items of one evaluation) the spring storage was sized for."""
        b = C.c_int64(0)
        cap = C.c_int64(0)
        self._check(lib().dem_get_memory(self._h, C.byref(b), C.byref(cap)))
        return dict(device_bytes=b.value, contact_capacity=cap.value)

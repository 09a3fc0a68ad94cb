"""MercuryDPM restart files (.restart) and the engine.

* :func:`read` parses a restart file the reference writes
  (``DPMBase::write``, Kernel/DPMBase.cc:3550-3680, with the handlers' and
  objects' ``write``) and :meth:`RestartState.scenario` turns it into the
  engine's inputs: species table, walls, periodic boundaries, particles, and
  the contact history (``InteractionHandler::write``,
  Kernel/InteractionHandler.cc:433-451) for ``dem_upload_contacts``. A run
  restarted this way continues as the reference continues after
  ``readRestartFile``: its initialiseSolve evaluates the forces again with the
  stored springs, and so does the engine's first ``dem_step``.
* :func:`write` writes the engine's current state in the same format, for the
  reference's own reader (``DPMBase::read``, DPMBase.cc:3688-3860, which reads
  the header lines by position and the objects by keyword).

Numbers are written with 15 significant digits, like the reference's restart
stream (``std::numeric_limits<double>::digits10``, DPMBase.cc:214-215): a
restart keeps positions to about 1e-15 of their magnitude, not to the bit.
Masses are not taken from the file: the reference recomputes them from the
species density when it restarts (``computeAllMasses`` in initialiseSolve),
and so does :meth:`RestartState.scenario`.

Supported content, as the engine has it: spherical particles; species
``{LinearViscoelastic|HertzianViscoelastic}{|SlidingFriction|Friction|Mindlin|
MindlinRollingTorsion}Species`` and their mixed species; ``InfiniteWall``,
``IntersectionOfWalls``, ``AxisymmetricIntersectionOfWalls``,
``TriangleWall``; ``PeriodicBoundary``. Anything else raises ValueError.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from .engine import Instance, infinite_wall, intersection_wall, species_pair, triangle_wall
from .host import quaternion_from_normal, sphere_inv_mass_inertia

NORMAL_LAWS = {"LinearViscoelastic": _abi.DEM_NORMAL_LINEAR_VISCOELASTIC,
               "HertzianViscoelastic": _abi.DEM_NORMAL_HERTZIAN_VISCOELASTIC}
FRICTION_LAWS = {"": _abi.DEM_FRICTION_NONE, "SlidingFriction": _abi.DEM_FRICTION_SLIDING,
                 "Friction": _abi.DEM_FRICTION_ROLLING_TORSION, "Mindlin": _abi.DEM_FRICTION_MINDLIN,
                 "MindlinRollingTorsion": _abi.DEM_FRICTION_MINDLIN_ROLLING_TORSION}
# the interaction classes' names (getName: normal base name + friction base
# name + "Interaction"; MindlinRollingTorsionInteraction's base name is "Friction")
INTERACTION_FRICTION_NAME = {_abi.DEM_FRICTION_NONE: "", _abi.DEM_FRICTION_SLIDING: "SlidingFriction",
                             _abi.DEM_FRICTION_ROLLING_TORSION: "Friction", _abi.DEM_FRICTION_MINDLIN: "Mindlin",
                             _abi.DEM_FRICTION_MINDLIN_ROLLING_TORSION: "Friction"}
VECTOR_KEYS = {"position": 3, "orientation": 4, "velocity": 3, "angularVelocity": 3, "force": 3, "torque": 3,
               "gravity": 3, "contactPoint": 3, "slidingSpring": 3, "rollingSpring": 3, "torsionSpring": 3,
               "normal": 3, "shift": 3, "particleIds": 2, "particleWallIds": 2}
DIGITS = 15


def _keyvals(tokens: list, start: int) -> dict:
    """key value [value ...] pairs of an object line (vectors by VECTOR_KEYS)."""
    out, i = {}, start
    while i < len(tokens):
        k = tokens[i]
        n = VECTOR_KEYS.get(k, 1)
        vals = tokens[i + 1:i + 1 + n]
        out[k] = [float(v) for v in vals] if n > 1 else vals[0] if vals else None
        i += 1 + n
    return out


def _split_species_name(name: str):
    """('LinearViscoelastic', 'SlidingFriction', mixed) of a species class name."""
    mixed = name.endswith("MixedSpecies")
    core = name[: -len("MixedSpecies")] if mixed else name[: -len("Species")] if name.endswith("Species") else None
    if core is None:
        raise ValueError(f"not a species: {name}")
    for nl in NORMAL_LAWS:
        if core.startswith(nl) and core[len(nl):] in FRICTION_LAWS:
            return nl, core[len(nl):], mixed
    raise ValueError(f"species {name}: the engine has no such contact law")


def _pair(nl: str, fl: str, kv: dict) -> _abi.SpeciesPair:
    g = lambda k: float(kv.get(k, 0.0))
    p = species_pair(normal_law=NORMAL_LAWS[nl], friction_law=FRICTION_LAWS[fl])
    if nl == "LinearViscoelastic":
        p.stiffness, p.dissipation = g("stiffness"), g("dissipation")
    else:
        p.elastic_modulus, p.dissipation = g("elasticModulus"), g("dissipation")
    if fl in ("SlidingFriction", "Friction"):
        p.sliding_stiffness, p.sliding_dissipation = g("slidingStiffness"), g("slidingDissipation")
    if fl in ("Mindlin", "MindlinRollingTorsion"):
        p.shear_modulus, p.sliding_dissipation = g("shearModulus"), g("slidingDissipation")
    if fl:
        p.sliding_mu, p.sliding_mu_static = g("slidingFrictionCoefficient"), g("slidingFrictionCoefficientStatic")
    if fl in ("Friction", "MindlinRollingTorsion"):
        p.rolling_stiffness, p.rolling_dissipation = g("rollingStiffness"), g("rollingDissipation")
        p.rolling_mu, p.rolling_mu_static = g("rollingFrictionCoefficient"), g("rollingFrictionCoefficientStatic")
        p.torsion_stiffness, p.torsion_dissipation = g("torsionStiffness"), g("torsionDissipation")
        p.torsion_mu, p.torsion_mu_static = g("torsionFrictionCoefficient"), g("torsionFrictionCoefficientStatic")
    return p


def quaternion_axis(q) -> tuple:
    """Quaternion::getAxis (Kernel/Math/Quaternion.cc:501-512): the image of
    the x axis, an InfiniteWall's normal."""
    q0, q1, q2, q3 = (float(v) for v in q)
    return (q0 * q0 + q1 * q1 - q2 * q2 - q3 * q3, 2 * (q1 * q2 + q0 * q3), 2 * (q1 * q3 - q0 * q2))


@dataclass
class RestartState:
    name: str
    time_step: float
    time: float
    n_steps: int
    time_max: float
    domain_min: tuple
    domain_max: tuple
    gravity: tuple
    background_drag: float
    species: list                     # n x n table of SpeciesPair (row-major)
    density: np.ndarray
    walls: list                       # dem_wall structures
    periodic: dict                    # axis -> (lo, hi)
    particles: dict                   # arrays: id, species, position, orientation, velocity, angular_velocity, radius, fixed
    interactions: dict                # arrays: id_p, id_i, is_wall, springs, time_stamp
    extra: dict = field(default_factory=dict)

    def scenario(self):
        """(Scenario, contacts) for the engine: the particles in the file's
        order, masses from density and radius (fixed particles: zero inverse
        mass and inertia), the contact history for dem_upload_contacts with
        each pair's periodic flag from the minimum image."""
        from .scenarios import Scenario
        p = self.particles
        n = len(p["radius"])
        inv_mass, inv_inertia = sphere_inv_mass_inertia(p["radius"], self.density[p["species"]])
        inv_mass = np.where(p["fixed"], 0.0, inv_mass)
        inv_inertia = np.where(p["fixed"], 0.0, inv_inertia)
        mask, lo, hi = 0, [0.0] * 3, [0.0] * 3
        dmin, dmax = list(self.domain_min), list(self.domain_max)
        for k, (a, b) in self.periodic.items():
            mask |= 1 << k
            lo[k], hi[k] = a, b
        inst = Instance(domain_min=tuple(dmin), domain_max=tuple(dmax), gravity=tuple(self.gravity),
                        n_species=len(self.density), periodic_mask=mask, periodic_min=tuple(lo), periodic_max=tuple(hi))
        sc = Scenario(self.name, self.time_step, inst, self.species, self.density, self.walls, p["position"],
                      p["velocity"], p["radius"], inv_mass, inv_inertia, p["species"].astype(np.int32),
                      p["id"].astype(np.int32), info=dict(restart_time=self.time, restart_steps=self.n_steps),
                      angular_velocity=p["angular_velocity"], orientation=p["orientation"])
        it = self.interactions
        index = {int(i): k for k, i in enumerate(p["id"])}
        periodic = np.zeros(len(it["id_p"]), np.int32)
        for c in range(len(it["id_p"])):
            if it["is_wall"][c] or not self.periodic:
                continue
            xa, xb = p["position"][index[int(it["id_p"][c])]], p["position"][index[int(it["id_i"][c])]]
            for k, (a, b) in self.periodic.items():
                if abs(xa[k] - xb[k]) > 0.5 * (b - a):
                    periodic[c] = 1
        contacts = dict(id_p=it["id_p"], id_i=it["id_i"], is_wall=it["is_wall"], periodic=periodic,
                        springs=it["springs"])
        return sc, contacts


def read(text: str) -> RestartState:
    """Parses the text of a reference .restart file."""
    lines = [ln for ln in text.splitlines() if ln.strip()]
    head = lines[0].split()
    if head[0] not in ("MercuryDPM", "restart_version") or head[1] not in ("1.0", "0.14"):
        raise ValueError("not a MercuryDPM restart file of version 1.0")
    kv0 = _keyvals(head, 2)
    name = kv0.get("name", "restart")
    i = 1
    while not lines[i].startswith("xMin"):
        i += 1  # the output-file lines
    t = lines[i].split()
    dmin = (float(t[1]), float(t[5]), float(t[9]))
    dmax = (float(t[3]), float(t[7]), float(t[11]))
    t = lines[i + 1].split()
    dt, time, nsteps, tmax = float(t[1]), float(t[3]), int(t[5]), float(t[7])
    t = lines[i + 2].split()
    if int(t[1]) != 3:
        raise ValueError("only three-dimensional systems (systemDimensions 3)")
    gravity = (float(t[5]), float(t[6]), float(t[7]))
    drag = float(t[9])
    i += 3

    def section(title):
        nonlocal i
        t = lines[i].split()
        if t[0] != title:
            raise ValueError(f"expected '{title}', found '{t[0]}'")
        i += 1
        return int(t[1])

    ns = section("Species")
    spec, mixed, density = {}, {}, {}
    while not lines[i].startswith("Walls"):
        t = lines[i].split()
        nl, fl, is_mixed = _split_species_name(t[0])
        kv = _keyvals(t, 1)
        if is_mixed:
            mixed[(int(kv["idA"]), int(kv["idB"]))] = _pair(nl, fl, kv)
        else:
            k = int(kv["id"])
            spec[k] = _pair(nl, fl, kv)
            density[k] = float(kv["density"])
        i += 1
    if len(spec) != ns:
        raise ValueError("species count does not match")
    table = []
    for a in range(ns):
        for b in range(ns):
            table.append(spec[a] if a == b else mixed.get((max(a, b), min(a, b))))
    if any(x is None for x in table):
        raise ValueError("a mixed species is missing")

    nw = section("Walls")
    walls = []
    for _ in range(nw):
        t = lines[i].split()
        i += 1
        walls.append(_wall(t))
    nb = section("Boundaries")
    periodic = {}
    for _ in range(nb):
        t = lines[i].split()
        i += 1
        if t[0] != "PeriodicBoundary":
            raise ValueError(f"boundary {t[0]} is not supported")
        kv = _keyvals(t, 1)
        nrm = kv["normal"]
        axes = [k for k in range(3) if nrm[k] != 0.0]
        if len(axes) != 1:
            raise ValueError("periodic boundaries must be normal to a coordinate axis")
        k = axes[0]
        a, b = float(kv["distanceLeft"]) * nrm[k], float(kv["distanceRight"]) * nrm[k]
        periodic[k] = (min(a, b), max(a, b))
    npart = section("Particles")
    rows = []
    for _ in range(npart):
        t = lines[i].split()
        i += 1
        if t[0] not in ("BaseParticle", "SphericalParticle"):
            raise ValueError(f"particle {t[0]} is not supported (spheres only)")
        rows.append(_keyvals(t, 1))
    particles = dict(
        id=np.array([int(r["id"]) for r in rows], np.int64),
        species=np.array([int(r["indSpecies"]) for r in rows], np.int64),
        position=np.array([r["position"] for r in rows]).reshape(-1, 3),
        orientation=np.array([r["orientation"] for r in rows]).reshape(-1, 4),
        velocity=np.array([r["velocity"] for r in rows]).reshape(-1, 3),
        angular_velocity=np.array([r["angularVelocity"] for r in rows]).reshape(-1, 3),
        radius=np.array([float(r["radius"]) for r in rows]),
        fixed=np.array([float(r["invMass"]) == 0.0 for r in rows]))
    nint = section("Interactions")
    ids_p, ids_i, is_wall, springs, stamps = [], [], [], [], []
    for _ in range(nint):
        t = lines[i].split()
        i += 1
        kv = _keyvals(t, 1)
        wall = "particleWallIds" in kv
        pq = kv["particleWallIds" if wall else "particleIds"]
        ids_p.append(int(pq[0]))
        ids_i.append(int(pq[1]))
        is_wall.append(1 if wall else 0)
        stamps.append(int(kv.get("timeStamp", 0)))
        s = np.zeros(9)
        for j, key in enumerate(("slidingSpring", "rollingSpring", "torsionSpring")):
            if key in kv:
                s[3 * j:3 * j + 3] = kv[key]
        springs.append(s)
    interactions = dict(id_p=np.array(ids_p, np.int32), id_i=np.array(ids_i, np.int32),
                        is_wall=np.array(is_wall, np.int32), springs=np.array(springs).reshape(-1, 9),
                        time_stamp=np.array(stamps, np.int64))
    return RestartState(name, dt, time, nsteps, tmax, dmin, dmax, gravity, drag, table,
                        np.array([density[k] for k in range(ns)]), walls, periodic, particles, interactions)


def _wall(t: list):
    kind = t[0]
    # the wall's own keys end where its faces or vertices begin (the faces
    # repeat the keys position and orientation)
    end = len(t)
    for marker in ("numIntersectionOfWalls", "vertexInLabFrame"):
        if marker in t:
            end = t.index(marker)
    kv = _keyvals(t[:end], 1)
    species = int(kv["indSpecies"])
    pos, q = kv["position"], kv["orientation"]
    vel, ang = kv.get("velocity", [0.0] * 3), kv.get("angularVelocity", [0.0] * 3)
    if kind == "InfiniteWall":
        return infinite_wall(quaternion_axis(q), pos, species=species, velocity=vel, angular_velocity=ang,
                             orientation=q)
    if kind in ("IntersectionOfWalls", "AxisymmetricIntersectionOfWalls"):
        k = t.index("numIntersectionOfWalls")
        nf = int(t[k + 1])
        faces, j = [], k + 2
        for _ in range(nf):
            fkv = _keyvals(t[j:j + 9], 0)  # position x y z orientation q0 q1 q2 q3
            faces.append((quaternion_axis(fkv["orientation"]), tuple(fkv["position"])))
            j += 9
        return intersection_wall(faces, position=pos, orientation=q, species=species, velocity=vel,
                                 angular_velocity=ang, axisymmetric=kind.startswith("Axisymmetric"))
    if kind == "TriangleWall":
        k = t.index("vertexInLabFrame")
        v = [float(x) for x in t[k + 1:k + 10]]
        verts = [tuple(v[3 * j + c] + pos[c] for c in range(3)) for j in range(3)]
        return triangle_wall(*verts, species=species, group=int(kv.get("groupID", 0)), position=pos, orientation=q,
                             velocity=vel, angular_velocity=ang)
    raise ValueError(f"wall {kind} is not supported")


# ---------------------------------------------------------------------------
def _f(x) -> str:
    """C++ ostream << double at precision 15 (%.15g)."""
    x = float(x)
    if math.isnan(x):
        return "nan"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return "%.*g" % (DIGITS, x)


def _v(v) -> str:
    return " ".join(_f(c) for c in v)


def _species_name(p: _abi.SpeciesPair) -> tuple:
    nl = {v: k for k, v in NORMAL_LAWS.items()}[p.normal_law]
    fl = {v: k for k, v in FRICTION_LAWS.items()}[p.friction_law]
    return nl, fl


def _species_params(p: _abi.SpeciesPair) -> str:
    nl, fl = _species_name(p)
    out = [f"stiffness {_f(p.stiffness)} dissipation {_f(p.dissipation)}" if nl == "LinearViscoelastic"
           else f"elasticModulus {_f(p.elastic_modulus)} dissipation {_f(p.dissipation)}"]
    mu = f"slidingFrictionCoefficient {_f(p.sliding_mu)} slidingFrictionCoefficientStatic {_f(p.sliding_mu_static)}"
    if fl in ("SlidingFriction", "Friction"):
        out.append(f"slidingStiffness {_f(p.sliding_stiffness)} slidingDissipation {_f(p.sliding_dissipation)} {mu}")
    if fl in ("Mindlin", "MindlinRollingTorsion"):
        out.append(f"slidingDissipation {_f(p.sliding_dissipation)} {mu} shearModulus {_f(p.shear_modulus)}")
    if fl in ("Friction", "MindlinRollingTorsion"):
        out.append(f"rollingStiffness {_f(p.rolling_stiffness)} rollingDissipation {_f(p.rolling_dissipation)} "
                   f"rollingFrictionCoefficient {_f(p.rolling_mu)} rollingFrictionCoefficientStatic "
                   f"{_f(p.rolling_mu_static)} torsionStiffness {_f(p.torsion_stiffness)} torsionDissipation "
                   f"{_f(p.torsion_dissipation)} torsionFrictionCoefficient {_f(p.torsion_mu)} "
                   f"torsionFrictionCoefficientStatic {_f(p.torsion_mu_static)}")
    return " ".join(out)


def write(engine, scenario, steps: int, name: str = "restart", save_count: int = 1) -> str:
    """The engine's state after `steps` time steps as the reference writes a
    restart file (DPMBase::write): the engine's particles (caller order),
    walls as they have moved, the scenario's species and periodic boundaries,
    and every contact of the last force evaluation with its springs, contact
    point and force (interaction torques and wall forces, which the engine
    does not keep, are written as zero; the reference recomputes both at its
    first evaluation after reading)."""
    from .output import time_after
    inst = scenario.instance
    st = engine.download()
    c = engine.contacts()
    geo = engine.contact_geometry()
    walls = engine.walls()
    n_sp = inst.n_species
    table = scenario.species[inst.species_offset: inst.species_offset + n_sp * n_sp]
    lines = [f"MercuryDPM 1.0 name {name} revision unknown repository unknown"]
    for f in ("dataFile   ", "fStatFile  ", "eneFile    ", "restartFile", "statFile   "):
        lines.append(f"{f} fileType NO_FILE saveCount {save_count} counter 0")
    lines.append("interactionFile fileType NO_FILE saveCount 0 counter 0")
    dmin, dmax = list(inst.domain_min), list(inst.domain_max)
    for k in range(3):
        if (inst.periodic_mask >> k) & 1:
            dmin[k], dmax[k] = inst.periodic_min[k], inst.periodic_max[k]
    lines.append(f"xMin {_f(dmin[0])} xMax {_f(dmax[0])} yMin {_f(dmin[1])} yMax {_f(dmax[1])} "
                 f"zMin {_f(dmin[2])} zMax {_f(dmax[2])}")
    lines.append(f"timeStep {_f(scenario.time_step)} time {_f(time_after(steps, scenario.time_step))} "
                 f"ntimeSteps {int(steps)} timeMax 1e+300")
    lines.append(f"systemDimensions 3 particleDimensions 3 gravity {_v(inst.gravity)} backgroundDrag 0 writeVTK 0 "
                 f"NO_FILE NO_FILE 0 0 0 0 0 random  0 1103515245 12345 1073741824 607 273 784607267")
    lines.append(f"Species {n_sp}")
    for a in range(n_sp):
        nl, fl = _species_name(table[a * n_sp + a])
        lines.append(f"{nl}{fl}Species id {a} density {_f(scenario.density[a])} "
                     f"{_species_params(table[a * n_sp + a])}")
        for b in range(a):
            nl, fl = _species_name(table[a * n_sp + b])
            lines.append(f"{nl}{fl}MixedSpecies idA {a} idB {b} {_species_params(table[a * n_sp + b])}")
    lines.append(f"Walls {len(walls)}")
    for k, w in enumerate(walls):
        common = (f"indSpecies {w.species} position {_v(w.position)} orientation {_v(w.orientation)} "
                  f"velocity {_v(w.velocity)} angularVelocity {_v(w.angular_velocity)} force 0 0 0 torque 0 0 0")
        if w.type == _abi.DEM_WALL_INFINITE:
            lines.append(f"InfiniteWall id {k} {common}")
        elif w.type in (_abi.DEM_WALL_INTERSECTION, _abi.DEM_WALL_AXISYMMETRIC):
            kind = "AxisymmetricIntersectionOfWalls" if w.type == _abi.DEM_WALL_AXISYMMETRIC else "IntersectionOfWalls"
            faces = " ".join(f"position {_v(w.faces[f][3:6])} orientation {_v(quaternion_from_normal(w.faces[f][0:3]))}"
                             for f in range(w.n_faces))
            lines.append(f"{kind} id {k} {common} numIntersectionOfWalls {w.n_faces} {faces}")
        elif w.type == _abi.DEM_WALL_TRIANGLE:
            orig = scenario.walls[k]
            rel = " ".join(_f(orig.faces[j][c] - orig.position[c]) for j in range(3) for c in range(3))
            lines.append(f"TriangleWall id {k} groupID {w.group} {common} vertexInLabFrame  {rel}")
        else:
            raise ValueError("unknown wall type")
    per = [k for k in range(3) if (inst.periodic_mask >> k) & 1]
    lines.append(f"Boundaries {len(per)}")
    for j, k in enumerate(per):
        nrm = [0, 0, 0]
        nrm[k] = 1
        L = inst.periodic_max[k] - inst.periodic_min[k]
        shift = [0.0, 0.0, 0.0]
        shift[k] = L
        lines.append(f"PeriodicBoundary id {j} normal {nrm[0]} {nrm[1]} {nrm[2]} scaleFactor 1 distanceLeft "
                     f"{_f(inst.periodic_min[k])} distanceRight {_f(inst.periodic_max[k])} shift {_v(shift)}")
    f, tq = engine.forces()
    alive = st["instance"] >= 0
    lines.append(f"Particles {int(alive.sum())}")
    for i in np.nonzero(alive)[0]:
        lines.append(f"BaseParticle id {st['id'][i]} indSpecies {st['species'][i]} position {_v(st['position'][i])} "
                     f"orientation {_v(st['orientation'][i])} velocity {_v(st['velocity'][i])} angularVelocity "
                     f"{_v(st['angular_velocity'][i])} force {_v(f[i])} torque {_v(tq[i])} radius "
                     f"{_f(st['radius'][i])} invMass {_f(st['inv_mass'][i])} timeStamp 0")
    sp_of = {int(i): int(s) for i, s in zip(st["id"], st["species"])}
    lines.append(f"Interactions {len(c['id_p'])}")
    for k in range(len(c["id_p"])):
        sa = sp_of[int(c["id_p"][k])]
        sb = walls[int(c["id_i"][k])].species if c["is_wall"][k] else sp_of[int(c["id_i"][k])]
        p = table[sa * n_sp + sb]
        nl, _ = _species_name(p)
        cls = nl + INTERACTION_FRICTION_NAME[p.friction_law] + "Interaction"
        ids = "particleWallIds" if c["is_wall"][k] else "particleIds"
        s = c["springs"][k]
        springs = ""
        if p.friction_law != _abi.DEM_FRICTION_NONE:
            springs = f" slidingSpring {_v(s[0:3])}"
        if p.friction_law in (_abi.DEM_FRICTION_ROLLING_TORSION, _abi.DEM_FRICTION_MINDLIN_ROLLING_TORSION):
            springs += f" rollingSpring {_v(s[3:6])} torsionSpring {_v(s[6:9])}"
        lines.append(f"{cls} {ids} {c['id_p'][k]} {c['id_i'][k]} timeStamp {int(steps)} contactPoint "
                     f"{_v(geo['contact_point'][k])} force {_v(c['force'][k])} torque 0 0 0{springs}")
    return "\n".join(lines) + "\n"

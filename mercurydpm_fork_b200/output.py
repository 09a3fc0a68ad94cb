"""The reference's text outputs, written from the engine's state.

* ``.ene``: ``DPMBase::writeEneHeader`` / ``writeEneTimeStep``
  (Kernel/DPMBase.cc:2010-2033, 2100-2123): time, gravitational energy
  ``-g . sum(m x)``, translational and rotational kinetic energy, elastic
  energy, centre of mass, number of interactions; columns right-aligned to
  ``precision + 6`` characters.
* ``.fstat``: ``DPMBase::writeFstatHeader`` (DPMBase.cc:2039-2089) and
  ``BaseInteraction::writeToFStat`` (Kernel/Interactions/BaseInteraction.cc:
  487-530): three header lines, then per contact one line for P (if P is not
  fixed) and one for I (if I is a particle that is not fixed), with time,
  indices (a wall as ``-index - 1``), contact point, overlap, tangential
  overlap, normal and tangential force magnitudes, normal and tangential
  direction (flipped for walls, as the reference does).
* ``.data``: ``DPMBase::outputXBallsData`` format 14 (DPMBase.cc:2356-2416,
  Kernel/DPMBaseXBalls.icc:36-92): particle count, time and domain, then per
  particle position (15 significant digits), velocity, radius, Euler angles
  (``Quaternion::getEuler``, Kernel/Math/Quaternion.cc:453-471), angular
  velocity and the species index.

Numbers are formatted as the reference's file streams format them: C++
``operator<<`` with precision 10 (DPMBase.cc:211-213), i.e. ``%.10g``.
Particle indices are the caller's order, wall indices the order given to
``dem_set_walls``. The tangential overlap is the reference's for sliding
friction (``-|sliding spring|``, SlidingFrictionInteraction.cc:253-257); the
tangential force is the friction force as the contact law computed it
(``getTangentialForce``).
"""
from __future__ import annotations

import math

import numpy as np

PRECISION = 10
WIDTH = PRECISION + 6


def fmt(x, precision: int = PRECISION) -> str:
    """C++ ``std::ostream << double`` in the default float format."""
    x = float(x)
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    if math.isinf(x):
        return "-inf" if x < 0 else "inf"
    return "%.*g" % (precision, x)


def _vec(v, precision: int = PRECISION) -> str:
    return " ".join(fmt(c, precision) for c in v)


def euler_angles(q) -> np.ndarray:
    """``Quaternion::getEuler`` for quaternions q = (q0, q1, q2, q3), one per row."""
    q = np.atleast_2d(np.asarray(q, np.float64))
    out = np.zeros((len(q), 3))
    for i, (q0, q1, q2, q3) in enumerate(q):
        sinp = 2 * (q0 * q2 - q3 * q1)
        pitch = math.asin(sinp) if abs(sinp) < 1 else math.copysign(math.pi, sinp)
        out[i] = (math.atan2(2 * (q0 * q1 + q2 * q3), 1 - 2 * (q1 * q1 + q2 * q2)), pitch,
                  math.atan2(2 * (q0 * q3 + q1 * q2), 1 - 2 * (q2 * q2 + q3 * q3)))
    return out


def time_after(steps: int, dt: float) -> float:
    """The reference's clock after `steps` time steps (time += dt each step)."""
    t = 0.0
    for _ in range(int(steps)):
        t += dt
    return t


def ene_header() -> str:
    names = ("time ", "gravitEnergy ", "traKineticEnergy ", "rotKineticEnergy ", "elasticEnergy ",
             "centerOfMassX ", "centerOfMassY ", "centerOfMassZ ")
    return "".join(s.rjust(WIDTH) for s in names) + "collisions\n".rjust(WIDTH)


def ene_line(time: float, gravity, globals_: dict, n_interactions: int) -> str:
    """One ``writeEneTimeStep`` line from the balances of ``dem_reduce``."""
    m = float(globals_["mass"])
    com = np.asarray(globals_["centre_of_mass"], np.float64)
    mx = com * m
    grav = -float(np.dot(np.asarray(gravity, np.float64), mx))
    cols = [time, grav, globals_["kinetic_energy"], globals_["rotational_energy"], globals_["elastic_energy"]]
    cols += list(com) if m != 0 else [float("nan")] * 3
    return " ".join(fmt(c).rjust(WIDTH) for c in cols) + " " + str(int(n_interactions)).rjust(WIDTH) + "\n"


def data_text(time: float, domain_min, domain_max, state: dict) -> str:
    """``outputXBallsData`` (3D, format 14) of the particles in `state`
    (engine.download()); deleted particles (instance -1) are left out."""
    keep = np.asarray(state.get("instance", np.zeros(len(state["radius"]))), np.int64) >= 0
    x = state["position"][keep]
    v = state["velocity"][keep]
    w = state["angular_velocity"][keep]
    r = state["radius"][keep]
    e = euler_angles(state["orientation"][keep])
    sp = state["species"][keep]
    lines = [" ".join([str(int(keep.sum())), fmt(time)] + [fmt(a) for a in domain_min] + [fmt(a) for a in domain_max])
             + " \n"]
    for i in range(len(r)):
        lines.append(" ".join([_vec(x[i], 15), _vec(v[i]), fmt(r[i]), _vec(e[i]), _vec(w[i]), fmt(float(sp[i]))])
                     + "\n")
    return "".join(lines)


def fstat_text(time: float, domain_min, domain_max, state: dict, contacts: dict, geometry: dict) -> str:
    """``writeFstatHeader`` + ``writeToFStat`` for every contact of the last
    force evaluation (engine.contacts() and engine.contact_geometry(), same
    order). `state` is engine.download() (ids, radii, inverse masses)."""
    ids = np.asarray(state["id"])
    index_of = {int(i): k for k, i in enumerate(ids)}
    fixed = np.asarray(state["inv_mass"]) == 0.0
    alive = np.asarray(state.get("instance", np.zeros(len(ids))), np.int64) >= 0
    r = np.asarray(state["radius"])[alive]
    rmin = fmt(r.min()) if len(r) else "nan"
    rmax = fmt(r.max()) if len(r) else "nan"
    out = ["# " + fmt(time) + " 1\n",
           "# " + " ".join(fmt(a) for a in list(domain_min) + list(domain_max)) + "\n",
           "# " + rmin + " " + rmax + " 0 0 0 0\n"]
    t = fmt(time)
    for k in range(len(contacts["id_p"])):
        p = index_of[int(contacts["id_p"][k])]
        wall = bool(contacts["is_wall"][k])
        i_index = -int(contacts["id_i"][k]) - 1 if wall else index_of[int(contacts["id_i"][k])]
        f = np.asarray(contacts["force"][k], np.float64)
        n = np.asarray(geometry["normal"][k], np.float64)
        c = np.asarray(geometry["contact_point"][k], np.float64)
        fn = float(np.dot(f, n))
        ft_vec = np.asarray(geometry["tangential_force"][k], np.float64)
        ft = float(np.linalg.norm(ft_vec))
        tdir = ft_vec / ft if ft != 0.0 else np.zeros(3)
        slide = np.asarray(contacts["springs"][k][:3], np.float64)
        tover = -float(np.linalg.norm(slide))
        common = " ".join([_vec(c), fmt(contacts["overlap"][k]), fmt(tover), fmt(fn), fmt(ft)])
        if not fixed[p]:
            nn, tt = (-n, -tdir) if wall else (n, tdir)
            out.append(" ".join([t, str(p), str(i_index), common, _vec(nn), _vec(tt)]) + "\n")
        if not wall and not fixed[i_index]:
            out.append(" ".join([t, str(i_index), str(p), common, _vec(-n), _vec(-tdir)]) + "\n")
    return "".join(out)


def write_outputs(engine, prefix: str, steps: int, dt: float, domain_min, domain_max, gravity, instance: int = 0):
    """Writes prefix.ene, prefix.fstat and prefix.data for the engine's
    current state (the last force evaluation's contacts), as the reference
    writes them after `steps` time steps."""
    t = time_after(steps, dt)
    state = engine.download()
    contacts = engine.contacts()
    geometry = engine.contact_geometry()
    g = engine.reduce(instance)
    with open(prefix + ".ene", "w") as fh:
        fh.write(ene_header())
        fh.write(ene_line(t, gravity, g, len(contacts["id_p"])))
    with open(prefix + ".fstat", "w") as fh:
        fh.write(fstat_text(t, domain_min, domain_max, state, contacts, geometry))
    with open(prefix + ".data", "w") as fh:
        fh.write(data_text(t, domain_min, domain_max, state))

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

"""Host-side set-up helpers that follow MercuryDPM's own formulas.

A driver that builds its inputs with these helpers hands the engine the same
numbers the reference's set-up code would compute, so that the device
evaluates the same expressions on identical operands:

* :func:`quaternion_from_normal` -- Quaternion::setOrientationViaNormal
  (Kernel/Math/Quaternion.cc:543-567), used by InfiniteWall::setNormal.
* :func:`sphere_inv_mass_inertia` -- BaseParticle::computeMass
  (Kernel/Particles/BaseParticle.cc:874-883).
* :func:`linear_collision_time_restitution` --
  LinearViscoelasticNormalSpecies::setCollisionTimeAndRestitutionCoefficient
  (Kernel/Species/NormalForceSpecies/LinearViscoelasticNormalSpecies.cc:225-259).
* :func:`hertz_dissipation_from_restitution` --
  HertzianViscoelasticNormalSpecies::setEffectiveElasticModulusAndRestitutionCoefficient
  (HertzianViscoelasticNormalSpecies.cc:109-132).
* :func:`average` -- BaseSpecies::average (harmonic mean used when two
  species are mixed, Kernel/Species/BaseSpecies.cc:110-115).
* :func:`psd_uniform` -- PSD::setDistributionUniform (Kernel/Math/PSD.cc:
  316-330, with PSD::linspace :1288-1302), the cumulative number distribution
  an InsertionBoundary draws radii from.
"""
from __future__ import annotations

import math

import numpy as np

PI = 3.1415926535897932384626433832795
SQR_PI = 9.8696044010893586188344909998762


def quaternion_from_normal(normal) -> tuple:
    nx, ny, nz = (float(v) for v in normal)
    l = math.sqrt(nx * nx + ny * ny + nz * nz)
    nx, ny, nz = nx / l, ny / l, nz / l
    if nx <= -1 + 1e-14:
        return (0.0, 0.0, 1.0, 0.0)
    hx, hy, hz = 1.0 + nx, 0.0 + ny, 0.0 + nz
    q = [hx, 0.0, -hz, hy]
    l2 = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    return tuple(v / l2 for v in q)


def sphere_inv_mass_inertia(radius, density):
    """Inverse mass and isotropic inverse inertia of spheres (3D)."""
    r = np.asarray(radius, dtype=np.float64)
    inv_mass = 1.0 / (4.0 / 3.0 * PI * r * r * r * density)
    mass = 1.0 / inv_mass
    inv_inertia = 1.0 / (.4 * mass * (r * r))
    return inv_mass, inv_inertia


def linear_collision_time_restitution(tc: float, eps: float, mass: float):
    """(stiffness, dissipation) for collision time tc and restitution eps of two particles of mass `mass`."""
    if eps == 0.0:
        k = .5 * mass * (PI / tc) ** 2
        return k, math.sqrt(2.0 * mass * k)
    diss = -mass / tc * math.log(eps)
    k = .5 * mass * ((PI / tc) * (PI / tc) + (diss / mass) * (diss / mass))
    return k, diss


def hertz_dissipation_from_restitution(eps: float) -> float:
    """Dimensionless damping of the Hertzian law for a constant restitution eps."""
    if eps > 0.0:
        log_rest_squared = math.log(eps) * math.log(eps)
        return math.sqrt(5.0 * log_rest_squared / (log_rest_squared + SQR_PI))
    return math.sqrt(5.0)


def average(a: float, b: float) -> float:
    return 0.0 if (a == 0 or b == 0) else (2. / (1.0 / a + 1.0 / b))


def psd_uniform(rmin: float, rmax: float, bins: int):
    """(radii, cumulative probabilities) of PSD::setDistributionUniform(rmin,
    rmax, bins): both from PSD::linspace (a running sum of the step, the last
    value replaced by the end point); PSD::validateCumulativeDistribution
    leaves such a table as it is (it starts at 0, ends at 1 and rises)."""
    def linspace(lo: float, hi: float, n: int):
        dx = (hi - lo) / float(n - 1)
        out, val = [], lo
        for _ in range(n):
            out.append(val)
            val += dx
        out[-1] = hi
        return out
    return linspace(float(rmin), float(rmax), bins), linspace(0.0, 1.0, bins)

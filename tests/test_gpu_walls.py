"""GPU parity for intersection walls (AxisymmetricIntersectionOfWalls,
IntersectionOfWalls), moving walls and the Hertz-Mindlin rolling-torsion law,
through the C ABI against the CPU oracle.

Tolerances (FP64): at the uploaded state the contact pair set and every
per-contact force, overlap and spring are bit-exact; per-particle totals
agree to 1e-14 of the largest (summation order only); over 10-100 steps
positions agree to 1e-13 of a diameter and forces, torques and springs to
1e-9 relative.
"""
import math

import numpy as np
import pytest

import cases
import harness as H

pytestmark = pytest.mark.gpu

WALL_CASES = {
    "drum": lambda: cases.small_drum(),
    "heap_base": lambda: cases.wall_probe("heap_base", omega=(0.5, 1.0, 3.0)),
    "ring_ridge": lambda: cases.wall_probe("ring_ridge", omega=(0.5, 1.0, 3.0)),
    "box_corner": lambda: cases.wall_probe("box_corner", omega=(0.5, 1.0, 3.0)),
}


@pytest.mark.parametrize("name", list(WALL_CASES))
def test_intersection_walls_initial_evaluation_bit_exact(gpu, name):
    sc = WALL_CASES[name]()
    g = H.run_gpu(sc, 0)
    o = H.run_oracle(sc, 0)
    assert H.pair_set(g["contacts"]) == H.pair_set(o["contacts"])
    assert int(g["contacts"]["is_wall"].sum()) > 80
    for k in ("force", "overlap", "springs"):
        np.testing.assert_array_equal(g["contacts"][k], o["contacts"][k])
    assert H.rel_err(g["force"], o["force"]) < 1e-14
    assert H.rel_err(g["torque"], o["torque"]) < 1e-14


@pytest.mark.parametrize("name", list(WALL_CASES))
@pytest.mark.parametrize("nsteps", [10, 100])
def test_intersection_walls_short_horizon(gpu, name, nsteps):
    sc = WALL_CASES[name]()
    g = H.run_gpu(sc, nsteps)
    o = H.run_oracle(sc, nsteps)
    assert H.pair_set(g["contacts"]) == H.pair_set(o["contacts"])
    assert H.rel_err(g["position"], o["position"], 1e-3) < 1e-13
    assert H.rel_err(g["velocity"], o["velocity"]) < 1e-9
    assert H.rel_err(g["angular_velocity"], o["angular_velocity"]) < 1e-9
    assert H.rel_err(g["force"], o["force"]) < 1e-9
    assert H.rel_err(g["torque"], o["torque"]) < 1e-9
    assert H.rel_err(g["contacts"]["springs"], o["contacts"]["springs"]) < 1e-9


@pytest.mark.parametrize("name", ["drum", "box_corner"])
def test_intersection_walls_match_reference(gpu, name):
    if not H.reference_available("serial"):
        pytest.skip("reference build (oracle/_ref) absent")
    sc = WALL_CASES[name]()
    g = H.run_gpu(sc, 20)
    r = H.run_reference(sc, 20)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    assert H.rel_err(g["position"], r["position"], 1e-3) < 1e-13
    assert H.rel_err(g["force"], r["force"]) < 1e-9


def _rotate_ref(q, w):
    """Quaternion::updateAngularDisplacement (Quaternion.cc:432-438) in Python floats."""
    q0, q1, q2, q3 = q
    wx, wy, wz = w
    d = (0.5 * (-q1 * wx - q2 * wy - q3 * wz), 0.5 * (q0 * wx + q3 * wy - q2 * wz),
         0.5 * (-q3 * wx + q0 * wy + q1 * wz), 0.5 * (q2 * wx - q1 * wy + q0 * wz))
    r = [q0 + d[0], q1 + d[1], q2 + d[2], q3 + d[3]]
    ln = math.sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + r[3] * r[3])
    return [x / ln for x in r]


def test_wall_motion_matches_reference_integration(gpu):
    """Every step moves each wall by v dt and rotates it by omega dt
    (BaseInteractable::integrateBeforeForceComputation), bit for bit."""
    sc = cases.wall_probe("box_corner", omega=(0.5, 1.0, 3.0))
    w0 = sc.walls[0]
    w0.velocity[:] = [1e-3, -2e-3, 0.5e-3]
    e = sc.engine()
    e.step(37)
    w = e.walls()[0]
    e.close()
    dt = sc.time_step
    q = list(w0.orientation)
    x = list(w0.position)
    for _ in range(37):
        x = [x[k] + w0.velocity[k] * dt for k in range(3)]
        q = _rotate_ref(q, [w0.angular_velocity[k] * dt for k in range(3)])
    assert list(w.position) == x
    assert list(w.orientation) == q

"""TriangleWall with the reference's triangle-wall correction (its default
build): TriangleWall::getDistanceAndNormal (TriangleWall.cc:57-104), group
merging (BaseWall.cc:375-409) and overlap weighting (DPMBase.cc:3443-3486),
checked against the reference build itself (oracle/_ref, serial, correction
on). The CPU oracle restatement does not cover triangle walls.

CPU: the reference's initial contacts with an ungrouped triangulated surface
are exactly the (particle, triangle) pairs within one radius by an
independent point-triangle distance, so the scenario exercises face, edge
and vertex contacts.

GPU: at the uploaded state the contact set and every per-contact force,
overlap and spring are bit-exact against the reference; over 20-100 steps
(contacts made, merged, weighted, handed between triangles) positions agree
to 1e-13 of a diameter and forces, torques and springs to 1e-9 relative.
Both start states occur: spheres touching the mesh at the upload, where the
reference's first time step shares its time stamp with the initial
evaluation (both numberOfTimeSteps + 1 = 1) and its group rule sees every
contact of that evaluation, and spheres dropped onto the mesh.
"""
import numpy as np
import pytest

import cases
import harness as H

needs_reference = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")


@needs_reference
def test_reference_triangle_contacts_match_point_triangle_distance():
    sc = cases.triangle_mesh(group=0)
    r = H.run_reference(sc, 0)
    c = r["contacts"]
    walls = {(int(p), int(w)) for p, w, iw in zip(c["id_p"], c["id_i"], c["is_wall"]) if iw}
    tris = cases.triangle_mesh_triangles()
    expect = set()
    for w, (a, b, cc) in enumerate(tris):
        dist = cases.point_triangle_distance(sc.position, a, b, cc)
        for p in np.nonzero(dist < sc.radius)[0]:
            expect.add((int(sc.ids[p]), w))
    assert walls == expect
    per_particle = np.bincount([p for p, _ in walls])
    assert per_particle.max() >= 2  # particles on shared edges and in the valleys
    assert len(walls) > 150


def _triangle_pairs(c):
    return sum(1 for iw in c["is_wall"] if iw)


@pytest.mark.gpu
@needs_reference
@pytest.mark.parametrize("group", [0, 1])
def test_triangle_walls_initial_evaluation_bit_exact(gpu, group):
    sc = cases.triangle_mesh(group=group)
    g = H.run_gpu(sc, 0)
    r = H.run_reference(sc, 0)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    assert _triangle_pairs(g["contacts"]) > 100
    for k in ("force", "overlap", "springs"):
        np.testing.assert_array_equal(g["contacts"][k], r["contacts"][k])
    assert H.rel_err(g["force"], r["force"]) < 1e-14
    assert H.rel_err(g["torque"], r["torque"]) < 1e-14


@pytest.mark.gpu
@needs_reference
@pytest.mark.parametrize("group,dropped", [(0, False), (0, True), (1, False), (1, True)])
@pytest.mark.parametrize("nsteps", [20, 100])
def test_triangle_walls_short_horizon(gpu, group, dropped, nsteps):
    sc = cases.triangle_mesh(group=group, dropped=dropped)
    g = H.run_gpu(sc, nsteps)
    r = H.run_reference(sc, nsteps)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    # touching spheres mostly rebound within 100 steps; dropped ones are pressed on
    assert _triangle_pairs(g["contacts"]) > {(False, 20): 60, (False, 100): 0, (True, 20): 25, (True, 100): 80}[
        (dropped, nsteps)]
    assert H.rel_err(g["position"], r["position"], 1e-3) < 1e-13
    assert H.rel_err(g["velocity"], r["velocity"]) < 1e-9
    assert H.rel_err(g["angular_velocity"], r["angular_velocity"]) < 1e-9
    assert H.rel_err(g["force"], r["force"]) < 1e-9
    assert H.rel_err(g["torque"], r["torque"]) < 1e-9
    assert H.rel_err(g["contacts"]["springs"], r["contacts"]["springs"]) < 1e-9


@pytest.mark.gpu
@needs_reference
def test_moving_triangle_walls_match_reference(gpu):
    """Triangles translating every step: vertices and normals recomputed
    after each move (TriangleWall::move -> updateVertexAndNormal)."""
    sc = cases.triangle_mesh(group=1, velocity=(0.01, -0.02, 0.005), dropped=True)
    g = H.run_gpu(sc, 50)
    r = H.run_reference(sc, 50)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    assert H.rel_err(g["position"], r["position"], 1e-3) < 1e-13
    assert H.rel_err(g["force"], r["force"]) < 1e-9


@pytest.mark.gpu
@needs_reference
def test_periodic_triangle_floor_matches_reference(gpu):
    """Grouped triangles spanning a periodic square (x and y), spheres
    arriving at 1 m/s: contacts near the periodic seams, list rebuilds."""
    from mercurydpm_fork_b200 import scenarios
    sc = scenarios.triangle_floor(n=1500, l_d=20.0, amplitude_d=0.3, drop_d=0.05, v0=1.0)
    g = H.run_gpu(sc, 200)
    r = H.run_reference(sc, 200)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    assert _triangle_pairs(g["contacts"]) > 100
    assert H.rel_err(g["position"], r["position"], 1e-3) < 1e-13
    assert H.rel_err(g["force"], r["force"]) < 1e-9
    assert H.rel_err(g["contacts"]["springs"], r["contacts"]["springs"]) < 1e-9


@pytest.mark.gpu
@needs_reference
def test_static_mesh_box_margin_matches_reference(gpu):
    """k_detect skips the triangle tests of a particle outside the bounding
    box of a static mesh widened by its reach (radius + interaction distance).
    Spheres placed around a 10 x 10 diameter patch at that margin (a hair
    inside and outside it, and exactly on it), others a tenth of a diameter
    out and moving in, others dropping onto the patch's corners: the
    contacts, at the start and as they appear, are the reference's."""
    import dataclasses
    from mercurydpm_fork_b200 import scenarios
    d = 1e-3
    sc = scenarios.triangle_floor(n=1, l_d=10.0, amplitude_d=0.3)
    L = 10 * d
    zs = [w.faces[k][2] for w in sc.walls for k in range(3)]
    lo = np.array([0.0, 0.0, min(zs)])
    hi = np.array([L, L, max(zs)])
    r = 0.5 * d
    pos, vel = [], []
    z = 0.5 * (lo[2] + hi[2])
    # one side per margin offset: a hair inside, exactly on, a hair outside, inside again
    sides = (((lambda s, f: (lo[0] - r * f, s, z)), (0.3, 0, 0), 1.0 - 1e-9),
             ((lambda s, f: (hi[0] + r * f, s, z)), (-0.3, 0, 0), 1.0),
             ((lambda s, f: (s, lo[1] - r * f, z)), (0, 0.3, 0), 1.0 + 1e-9),
             ((lambda s, f: (s, hi[1] + r * f, z)), (0, -0.3, 0), 1.0 - 1e-12))
    for place, v, frac in sides:
        for s in np.linspace(1.0 * d, L - 1.0 * d, 5):  # on the margin, at rest
            pos.append(place(s, frac))
            vel.append((0, 0, 0))
        for s in np.linspace(2.0 * d, L - 2.0 * d, 4):  # a tenth of a diameter out, moving in
            pos.append(place(s, 1.2))
            vel.append(v)
    for cx, cy in ((lo[0], lo[1]), (hi[0], lo[1]), (lo[0], hi[1]), (hi[0], hi[1])):
        pos.append((cx, cy, hi[2] + r * 1.05))
        vel.append((0, 0, -0.3))
    # spheres of one side column would touch their neighbours across the corner: spread them
    n = len(pos)
    sc.position, sc.velocity = pos, vel
    sc.radius = np.full(n, r)
    from mercurydpm_fork_b200.host import sphere_inv_mass_inertia
    sc.inv_mass, sc.inv_inertia = sphere_inv_mass_inertia(sc.radius, float(sc.density[0]))
    sc.species_index = np.zeros(n, np.int32)
    sc.ids = np.arange(n, dtype=np.int32)
    sc.instance = dataclasses.replace(sc.instance, periodic_mask=0, domain_min=(-3 * d, -3 * d, -2 * d),
                                      domain_max=(L + 3 * d, L + 3 * d, 4 * d))
    seen = 0
    for steps in (0, 150, 180, 210, 240, 300):
        g = H.run_gpu(sc, steps)
        r_ = H.run_reference(sc, steps)
        assert H.pair_set(g["contacts"]) == H.pair_set(r_["contacts"]), steps
        assert H.rel_err(g["position"], r_["position"], 1e-3) < 1e-13
        assert H.rel_err(g["force"], r_["force"]) < 1e-9
        seen += _triangle_pairs(r_["contacts"])
    assert seen > 10

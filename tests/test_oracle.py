"""CPU tests of the oracle itself: pinned against the reference's golden
vectors and against the reference build compiled here (oracle/_ref)."""
import numpy as np
import pytest

import cases
import harness as H

needs_ref = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build (oracle/_ref) absent")


def test_oracle_tangential_spring_known_answer():
    """TangentialSpringUnitTest.cpp:89-100 known answers, tolerance 1e-7."""
    sc, steps, exp = cases.tangential_spring()
    o = H.run_oracle(sc, steps)
    np.testing.assert_allclose(o["position"][1], exp["Position"]["value"], atol=exp["Position"]["tol"], rtol=0)
    np.testing.assert_allclose(o["velocity"][1], exp["Velocity"]["value"], atol=exp["Velocity"]["tol"], rtol=0)
    np.testing.assert_allclose(o["angular_velocity"][1], exp["AngularVelocity"]["value"],
                               atol=exp["AngularVelocity"]["tol"], rtol=0)
    # the fixed particle does not move
    np.testing.assert_array_equal(o["position"][0], sc.position[0])


@needs_ref
@pytest.mark.parametrize("nsteps", [0, 1, 10])
def test_oracle_matches_reference_short(nsteps):
    sc = cases.compressed_box()
    o = H.run_oracle(sc, nsteps, report="handler")
    r = H.run_reference(sc, nsteps)
    assert H.pair_set(o["contacts"]) == H.pair_set(r["contacts"])
    assert len(o["contacts"]["id_p"]) > 1000
    # one contact evaluation is bit-identical; totals differ only by summation order
    if nsteps == 0:
        np.testing.assert_array_equal(o["contacts"]["force"], r["contacts"]["force"])
        np.testing.assert_array_equal(o["contacts"]["springs"], r["contacts"]["springs"])
    assert H.rel_err(o["force"], r["force"]) < 1e-14
    assert H.rel_err(o["torque"], r["torque"]) < 1e-14
    assert H.rel_err(o["velocity"], r["velocity"]) < 1e-14
    np.testing.assert_array_equal(o["position"], r["position"]) if nsteps <= 1 else None
    assert H.rel_err(o["position"], r["position"], 1e-3) < 1e-15


@needs_ref
def test_oracle_matches_reference_walls_horizon():
    sc = cases.compressed_box()
    o = H.run_oracle(sc, 300, report="handler")
    r = H.run_reference(sc, 300)
    assert H.pair_set(o["contacts"]) == H.pair_set(r["contacts"])
    assert int(o["contacts"]["is_wall"].sum()) > 100
    assert H.rel_err(o["force"], r["force"]) < 1e-10
    assert H.rel_err(o["position"], r["position"], 1e-3) < 1e-12


@needs_ref
@pytest.mark.parametrize("nsteps", [0, 5])
def test_oracle_matches_reference_periodic_chute(nsteps):
    sc = cases.small_chute(n_flow=1500)
    o = H.run_oracle(sc, nsteps, report="handler")
    r = H.run_reference(sc, nsteps)
    assert H.pair_set(o["contacts"]) == H.pair_set(r["contacts"])
    assert int(o["contacts"]["periodic"].sum()) > 0
    assert (o["contacts"]["periodic"] == r["contacts"]["periodic"]).all()
    assert H.rel_err(o["force"], r["force"]) < 1e-12
    assert H.rel_err(o["position"], r["position"], 1e-3) < 1e-14


WALL_CASES = {
    "drum": lambda: cases.small_drum(),
    "heap_base": lambda: cases.wall_probe("heap_base", omega=(0.5, 1.0, 3.0)),
    "ring_ridge": lambda: cases.wall_probe("ring_ridge", omega=(0.5, 1.0, 3.0)),
    "box_corner": lambda: cases.wall_probe("box_corner", omega=(0.5, 1.0, 3.0)),
}


@needs_ref
@pytest.mark.parametrize("name", list(WALL_CASES))
@pytest.mark.parametrize("nsteps", [0, 10, 100])
def test_oracle_matches_reference_intersection_walls(name, nsteps):
    """AxisymmetricIntersectionOfWalls / IntersectionOfWalls (faces, edges,
    corners, the non-finite-corner fall-through), rotating walls and the
    Hertz-Mindlin rolling-torsion law against the reference build."""
    sc = WALL_CASES[name]()
    o = H.run_oracle(sc, nsteps)
    r = H.run_reference(sc, nsteps)
    assert H.pair_set(o["contacts"]) == H.pair_set(r["contacts"])
    if nsteps == 0:
        assert int(o["contacts"]["is_wall"].sum()) > 80
        np.testing.assert_array_equal(o["contacts"]["force"], r["contacts"]["force"])
        np.testing.assert_array_equal(o["contacts"]["overlap"], r["contacts"]["overlap"])
        np.testing.assert_array_equal(o["contacts"]["springs"], r["contacts"]["springs"])
    assert H.rel_err(o["force"], r["force"]) < 1e-12
    assert H.rel_err(o["torque"], r["torque"]) < 1e-12
    assert H.rel_err(o["position"], r["position"], 1e-3) < 1e-13
    assert H.rel_err(o["contacts"]["springs"], r["contacts"]["springs"]) < 1e-11


@needs_ref
def test_oracle_matches_reference_heap():
    """A CalibrationHeap instance: LinearViscoelasticFrictionSpecies (linear
    rolling and torsion springs), lognormal radii, the floor disk and the
    DeletionBoundary below it."""
    from mercurydpm_fork_b200 import calibration as cal
    p = cal.HeapParams(n=400, sigma=0.15, mu=0.5, mu_r=0.1, restitution=0.5, seed=3)
    sc, dels, _ = cal.heap_scenario(p, base_radius_d=8, column_radius_d=4, v0=0.5)
    o = H.run_oracle(sc, 1200, deletions=dels)
    r = H.run_reference(sc, 1200, deletions=dels)
    assert H.pair_set(o["contacts"]) == H.pair_set(r["contacts"])
    assert len(o["contacts"]["id_p"]) > 20 and int(o["contacts"]["is_wall"].sum()) > 0
    np.testing.assert_array_equal(o["instance"], r["instance"])
    assert H.rel_err(o["force"], r["force"]) < 1e-12
    assert H.rel_err(o["position"], r["position"], 1e-3) < 1e-13
    assert H.rel_err(o["contacts"]["springs"], r["contacts"]["springs"]) < 1e-11


@needs_ref
def test_oracle_matches_reference_periodic_transitions():
    """300 steps of the periodic chute: contacts cross the periodic boundaries,
    turning ordinary pairs into periodic ones and back. The reference keeps
    one real-real interaction (the lower index's view,
    InteractionHandler::removeObjectKeepingPeriodics) and gives the other
    particle's ghost a reversed copy (BaseInteraction::copySwitchPointer)."""
    sc = cases.small_chute()
    o = H.run_oracle(sc, 300)
    r = H.run_reference(sc, 300)
    assert H.pair_set(o["contacts"]) == H.pair_set(r["contacts"])
    assert H.rel_err(o["force"], r["force"]) < 1e-12
    assert H.rel_err(o["position"], r["position"], 1e-3) < 1e-13

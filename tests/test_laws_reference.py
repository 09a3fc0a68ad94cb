"""Every contact law the engine offers (DEM_NORMAL_* x DEM_FRICTION_*, and
the linear law's constant-restitution form) against the reference's own
build, on the small rotating drum (cases.drum_with_law: particle pairs of
two sizes, a rotating axisymmetric cylinder and flat caps, Coulomb caps,
rolling and torsion springs all active). The CPU restatement (oracle) is held
to the reference the same way, so no law is only checked against code that
shares its source.

Tolerances (FP64): at the initial evaluation the contact pairs and, per
contact, force, overlap and springs are bit-exact; after 100 steps the pair
set is exact, positions agree to 1e-12 of a diameter, and velocities,
forces and springs to 1e-9 of their largest magnitude, angular velocities and
torques to 1e-9 of |v|/r and |F| r (frictionless laws exert no torque: there
they are rounding noise).
"""
import numpy as np
import pytest

import cases
import harness as H

pytestmark = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")


def _check(sc, a, r, steps):
    assert H.pair_set(a["contacts"]) == H.pair_set(r["contacts"])
    assert len(r["contacts"]["id_p"]) > (300 if steps == 0 else 100)
    if steps == 0:
        for k in ("force", "overlap", "springs"):
            np.testing.assert_array_equal(a["contacts"][k], r["contacts"][k], err_msg=k)
    else:
        assert H.rel_err(a["position"], r["position"], 1e-3) < 1e-12
        for k in ("velocity", "force"):
            assert H.rel_err(a[k], r[k]) < 1e-9, k
        # without friction the torques and angular velocities are rounding
        # noise (central forces): they are measured on the scales |F| r and |v| / r
        rmin, rmax = float(np.min(sc.radius)), float(np.max(sc.radius))
        w_scale = max(np.abs(r["angular_velocity"]).max(), np.abs(r["velocity"]).max() / rmin)
        t_scale = max(np.abs(r["torque"]).max(), np.abs(r["force"]).max() * rmax)
        assert H.rel_err(a["angular_velocity"], r["angular_velocity"], w_scale) < 1e-9
        assert H.rel_err(a["torque"], r["torque"], t_scale) < 1e-9
        assert H.rel_err(a["contacts"]["springs"], r["contacts"]["springs"]) < 1e-9


@pytest.mark.parametrize("steps", [0, 100])
@pytest.mark.parametrize("law", cases.LAWS)
def test_oracle_law_matches_reference(law, steps):
    sc = cases.drum_with_law(law)
    _check(sc, H.run_oracle(sc, steps), H.run_reference(sc, steps), steps)


@pytest.mark.gpu
@pytest.mark.parametrize("steps", [0, 100])
@pytest.mark.parametrize("law", cases.LAWS)
def test_engine_law_matches_reference(gpu, law, steps):
    sc = cases.drum_with_law(law)
    _check(sc, H.run_gpu(sc, steps), H.run_reference(sc, steps), steps)

"""Parity at the sizes that are measured, against the reference's own build
(oracle/_ref, MercuryDPM's serial Kernel compiled from its sources) rather
than the CPU restatement, so no contact law is checked against itself:

* the 1,000,000-sphere dense drum that bench.py times (Hertz-Mindlin with
  rolling and torsion friction, axisymmetric cylinder and two caps);
* the 200,000-sphere periodic chute of `measure chute` (linear + sliding
  friction, two HGrid levels, rough base, periodic x and y), with the
  engine's configuration of that measurement (Verlet skin 0.8 r_min);
* the 5,000-sphere settling box over its full 20,000 steps, through the
  balances of every 500th step against the .ene file the reference writes.

Tolerances (FP64 throughout):
* contact pair sets, wall contacts included, at identical positions:
  bit-exact; per contact force, overlap and springs at the initial
  evaluation: bit-exact (the same IEEE operations in the same order);
* per-particle totals at the initial evaluation: 1e-14 relative to the
  largest (the sums run in another order);
* a few steps later: positions within 1e-13 of a diameter, velocities,
  forces, torques and springs within 1e-9 of their largest magnitude;
* the settling box's .ene lines: see test_settling_box_balances.
"""
import json
import os

import numpy as np
import pytest

import harness as H
from mercurydpm_fork_b200 import scenarios

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _same_contacts_bit_exact(g, r):
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    for k in ("force", "overlap", "springs"):
        np.testing.assert_array_equal(g["contacts"][k], r["contacts"][k], err_msg=k)


@pytest.fixture(scope="module")
def drum():
    return scenarios.dense_drum()


@pytest.fixture(scope="module")
def chute():
    return scenarios.periodic_chute(n_flow=200_000, seed=2, packing="layers", spacing_factor=1.0)


def _chute_skin(sc):
    return 0.8 * float(np.min(sc.radius))


def test_drum_1m_initial_evaluation_bit_exact(gpu, drum):
    g = H.run_gpu(drum, 0)
    r = H.run_reference(drum, 0)
    assert len(g["contacts"]["id_p"]) > 1_000_000
    assert int(g["contacts"]["is_wall"].sum()) > 1000
    _same_contacts_bit_exact(g, r)
    assert H.rel_err(g["force"], r["force"]) < 1e-14
    assert H.rel_err(g["torque"], r["torque"]) < 1e-14


def test_drum_1m_three_steps(gpu, drum):
    g = H.run_gpu(drum, 3)
    r = H.run_reference(drum, 3)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    d = 1e-3
    assert H.rel_err(g["position"], r["position"], d) < 1e-13
    for k in ("velocity", "angular_velocity", "force", "torque"):
        assert H.rel_err(g[k], r[k]) < 1e-9, k
    assert H.rel_err(g["contacts"]["springs"], r["contacts"]["springs"]) < 1e-9


def test_chute_200k_initial_evaluation_bit_exact(gpu, chute):
    g = H.run_gpu(chute, 0, skin=_chute_skin(chute))
    r = H.run_reference(chute, 0)
    assert len(g["contacts"]["id_p"]) > 300_000
    assert int(g["contacts"]["periodic"].sum()) > 1000
    _same_contacts_bit_exact(g, r)
    assert (g["contacts"]["periodic"] == r["contacts"]["periodic"]).all()
    assert H.rel_err(g["force"], r["force"]) < 1e-14
    assert H.rel_err(g["torque"], r["torque"]) < 1e-14


def test_chute_200k_ten_steps(gpu, chute):
    g = H.run_gpu(chute, 10, skin=_chute_skin(chute))
    r = H.run_reference(chute, 10)
    assert H.pair_set(g["contacts"]) == H.pair_set(r["contacts"])
    assert H.rel_err(g["position"], r["position"], 1e-3) < 1e-13
    for k in ("velocity", "angular_velocity", "force", "torque"):
        assert H.rel_err(g[k], r[k]) < 1e-9, k
    assert H.rel_err(g["contacts"]["springs"], r["contacts"]["springs"]) < 1e-9


def test_settling_box_balances(gpu):
    """The 5,000-sphere settling box (20 x 20 x 40 d, six walls, linear +
    sliding friction, dt = tc/50) over its full 20,000 steps: the engine's
    .ene lines against the .ene file the reference's own solve() writes
    (tests/golden/settling_box_ene.json, made by make_golden.py).

    * While the reference's serial and OpenMP builds still write identical
      lines (they differ only in the order of floating-point sums, and agree
      until multi-contact sums appear ~8,500 steps in), the engine's lines
      agree with them to 1e-8 relative per column and the interaction count
      is exact.
    * Over the whole run, the engine differs from the serial build by at most
      3x the largest difference between the reference's two builds in that
      column (plus 1e-9 of the column's magnitude): its balances lie inside
      the envelope the reference's own rounding produces once the settling
      packing turns chaotic."""
    gold = json.load(open(os.path.join(GOLDEN, "settling_box_ene.json")))
    sc = scenarios.settling_box()
    H.check_ene_against_golden(H.engine_ene(sc, gold["steps"], gold["save_count"]), gold)

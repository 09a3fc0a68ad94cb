"""The reference-side binding: MercuryDPM drivers whose base class is the
engine's drop-in GpuMercury3D / GpuDPMBase (mercurydpm_fork_b200/mercury/
GpuTimeStep.h), compiled against the reference's headers and Kernel by
oracle/ref.mk (target gpu) and run through the reference's own
DPMBase::solve() -> computeOneTimeStep loop.

* The reference's unit test Drivers/UnitTests/TangentialSpringUnitTest.cpp,
  compiled from its own source with only its base class swapped (DPMBase ->
  GpuDPMBase), passes its own golden assertions (position, velocity and
  angular velocity to 1e-7) with every time step on the GPU.
* The checker's Mercury3D driver on GpuMercury3D runs the 5,000-sphere
  settling box through solve() and writes its .ene file with the reference's
  File machinery; the lines equal those of the engine driven directly through
  the C ABI, and lie within the reference's own chaos envelope
  (tests/golden/settling_box_ene.json).
* The host state the driver holds after solve() equals the engine's state
  after the same number of steps, bit for bit, whatever the sync interval:
  on the periodic chute, on the rotating drum (AxisymmetricIntersectionOfWalls
  and InfiniteWall caps), and on a cased column whose driver takes the casing
  out and adds a DeletionBoundary in its actionsAfterTimeStep (the deleted
  particles leave its ParticleHandler); its InteractionHandler holds the
  engine's contacts of the last step, whose elastic energy is the engine's.
"""
import json
import os
import subprocess

import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import scenarios

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not H.gpu_binding_available(), reason="binding drivers not built (make -f oracle/ref.mk gpu)")]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_reference_unit_test_on_gpu_base_class(gpu, tmp_path):
    r = subprocess.run([H.GPU_UNIT_TEST], cwd=tmp_path, capture_output=True, text=True, timeout=900)
    out = r.stdout + r.stderr
    assert r.returncode == 0, out[-3000:]
    assert "error has occured" not in out, out[-3000:]


def test_settling_box_through_solve(gpu, tmp_path):
    gold = json.load(open(os.path.join(GOLDEN, "settling_box_ene.json")))
    sc = scenarios.settling_box()
    rows = H.gpu_binding_ene(sc, gold["steps"], gold["save_count"], str(tmp_path / "box"),
                             sync_interval=gold["save_count"])
    direct = H.engine_ene(sc, gold["steps"], gold["save_count"])
    np.testing.assert_array_equal(rows, direct)
    H.check_ene_against_golden(rows, gold)


@pytest.mark.parametrize("sync_interval", [1, 7])
def test_host_state_after_solve_equals_engine(gpu, sync_interval):
    """Periodic bidisperse chute (two HGrid levels, rough base): the state
    GpuMercury3D leaves in the ParticleHandler after solve() is the engine's."""
    sc = cases.small_chute()
    steps = 40
    host = H.gpu_binding_state(sc, steps, sync_interval=sync_interval)
    g = H.run_gpu(sc, steps)
    for k in ("position", "velocity", "angular_velocity"):
        np.testing.assert_array_equal(host[k], g[k], err_msg=k)


def test_drum_through_solve_equals_engine(gpu):
    """Also the InteractionHandler: after solve() it holds the engine's
    contacts of the last step, and DPMBase::getElasticEnergy over them (the
    reference's sum over interactions of the laws' energies) agrees with the
    engine's own balance."""
    sc = cases.small_drum()
    host = H.gpu_binding_state(sc, 40)
    g = H.run_gpu(sc, 40)
    for k in ("position", "velocity", "angular_velocity"):
        np.testing.assert_array_equal(host[k], g[k], err_msg=k)
    assert host["host_interactions"] == len(g["contacts"]["id_p"]) > 100
    ee = g["globals"]["elastic_energy"]
    assert abs(host["host_elastic_energy"] - ee) <= 1e-9 * ee


@pytest.mark.parametrize("sync_interval", [1, 25])
def test_casing_taken_out_by_the_driver(gpu, sync_interval):
    sc, R, planes = cases.pressed_column()
    event = (10, 1, planes)
    host = H.gpu_binding_state(sc, 110, sync_interval=sync_interval, event=event)
    g = H.run_gpu(sc, 110, event=event)
    gone = g["instance"] < 0
    assert gone.sum() > 20
    np.testing.assert_array_equal(host["instance"] < 0, gone)
    for k in ("position", "velocity", "angular_velocity"):
        np.testing.assert_array_equal(host[k][~gone], g[k][~gone], err_msg=k)

"""The autotuner (dem_autotune / dem_set_tuning): launch shapes of the force
kernels chosen by measurement on the live state.

* On two workloads (the rotating drum with 200,000 spheres, Hertz-Mindlin
  with rolling and torsion, and the periodic chute with 200,000 spheres,
  linear + sliding friction) the chosen shapes are at least as fast as the
  default ones, timed again independently of the tuner (5 % allowed for
  timing noise).
* Shapes change where work runs, never the arithmetic: a run with other
  shapes is bit-identical to one with the defaults.
* The per-workload-class cache hands the shapes to the next engine of the
  same class without measuring; invalid shapes are refused.
"""
import numpy as np
import pytest

import cases
from mercurydpm_fork_b200 import DemError, _abi, scenarios

pytestmark = pytest.mark.gpu

DEFAULT = dict(detect_block=128, contacts_blocks_per_sm=4, sum_block=128)


def _workloads():
    chute = scenarios.periodic_chute(n_flow=200_000, seed=2, packing="layers", spacing_factor=1.0)
    return {"drum_200k": (scenarios.dense_drum(n=200_000), {}),
            "chute_200k": (chute, dict(skin=0.8 * float(np.min(chute.radius))))}


@pytest.mark.parametrize("name", ["drum_200k", "chute_200k"])
def test_tuned_shapes_at_least_as_fast_as_defaults(gpu, name):
    sc, kw = _workloads()[name]
    e = sc.engine(**kw)
    try:
        e.step(0)
        e.step(20)
        assert e.tuning() == DEFAULT
        t = e.autotune(reps=10)
        assert t["ms_after"] <= t["ms_before"]
        chosen = e.tuning()
        tuned = min(e.time_force_kernel(20) for _ in range(3))
        e.set_tuning(**DEFAULT)
        default = min(e.time_force_kernel(20) for _ in range(3))
        e.set_tuning(**chosen)
        assert tuned <= 1.05 * default, (chosen, tuned, default)
    finally:
        e.close()


@pytest.mark.parametrize("case", ["compressed_box", "small_chute", "small_drum"])
def test_results_do_not_depend_on_shapes(gpu, case):
    sc = getattr(cases, case)()
    runs = []
    for shape in (DEFAULT, dict(detect_block=64, contacts_blocks_per_sm=3, sum_block=256),
                  dict(detect_block=256, contacts_blocks_per_sm=6, sum_block=64)):
        e = sc.engine()
        e.set_tuning(**shape)
        e.step(40)
        out = e.download()
        out["force"], out["torque"] = e.forces()
        e.close()
        runs.append(out)
    for other in runs[1:]:
        for k in ("position", "velocity", "angular_velocity", "force", "torque"):
            np.testing.assert_array_equal(other[k], runs[0][k], err_msg=k)


def test_cache_and_validation(gpu):
    sc = cases.small_chute()
    cache = {}
    e1 = sc.engine()
    e1.step(5)
    first = e1.autotune(reps=5, cache=cache)
    e1.close()
    assert not first["cached"] and len(cache) == 1
    e2 = sc.engine()
    e2.step(5)
    second = e2.autotune(reps=5, cache=cache)
    assert second["cached"]
    assert e2.tuning() == {k: first[k] for k in DEFAULT}
    with pytest.raises(DemError) as ex:
        e2.set_tuning(detect_block=96, contacts_blocks_per_sm=4, sum_block=128)
    assert ex.value.code == _abi.DEM_ERR_BAD_INPUT
    e2.close()

"""Spring history stored per contact (a pool indexed by the contact's item in
each evaluation; list entries hold only the pool index of their contact).

* The first time step keeps an interaction of the initial evaluation that
  nothing touches in that step (its spring moves to the top of the pool); a
  contact made again in the second step continues from it, as in the
  reference (cases.recontact): bit-exact against the oracle, which matches
  the reference build on this case exactly.
* The contact capacity (dem_config.max_contacts) only sizes storage: a run
  with a tight capacity is bit-identical to one with the automatic size, one
  below the live contacts fails with DEM_ERR_CAPACITY, and the device memory
  per sphere of a heap batch follows the capacity.
* Springs injected in two dem_upload_contacts calls give the run that one
  call gives.
"""
import dataclasses

import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import DemError, _abi

STEPS = (1, 2, 3)


def _same(a, b):
    for k in ("position", "velocity", "angular_velocity", "force", "torque"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    assert H.pair_set(a["contacts"]) == H.pair_set(b["contacts"])
    np.testing.assert_array_equal(a["contacts"]["springs"], b["contacts"]["springs"])


@pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")
@pytest.mark.parametrize("owner_first", [True, False])
def test_recontact_oracle_matches_reference(owner_first):
    sc = cases.recontact(owner_first)
    for steps in STEPS:
        o, r = H.run_oracle(sc, steps), H.run_reference(sc, steps)
        np.testing.assert_array_equal(o["position"], r["position"])
        np.testing.assert_array_equal(o["force"], r["force"])
    # the spring of the second step's contact continued from the initial one
    # (1e-4 along y); a new contact would start near one step's increment
    o = H.run_oracle(sc, 2)
    assert H.pair_set(o["contacts"]) == ({(0, 1, 0)} if owner_first else {(0, 2, 0)})
    assert np.max(np.abs(o["contacts"]["springs"][:, 1])) > 2.5e-4


@pytest.mark.gpu
@pytest.mark.parametrize("owner_first", [True, False])
def test_recontact_engine_matches_oracle(gpu, owner_first):
    sc = cases.recontact(owner_first)
    for steps in STEPS:
        _same(H.run_gpu(sc, steps), H.run_oracle(sc, steps))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["compressed_box", "small_chute", "small_drum"])
def test_tight_capacity_changes_nothing(gpu, case):
    sc = getattr(cases, case)()
    auto = H.run_gpu(sc, 60)
    tight = H.run_gpu(sc, 60, max_contacts=4)
    _same(tight, auto)


@pytest.mark.gpu
def test_capacity_below_the_contacts_is_an_error(gpu):
    sc = cases.compressed_box()
    e = sc.engine(max_contacts=1)
    try:
        with pytest.raises(DemError) as ex:
            e.step(0)
            e.step(10)
        assert ex.value.code == _abi.DEM_ERR_CAPACITY
    finally:
        e.close()


@pytest.mark.gpu
def test_memory_follows_the_contact_capacity(gpu):
    from mercurydpm_fork_b200 import calibration as cal
    b, _, _ = cal.heap_batch(8, seed=4)
    sizes = {}
    for mc in (0, 6):
        e = b.engine(max_contacts=mc)
        sizes[mc] = e.memory()
        e.close()
    assert sizes[6]["contact_capacity"] == 6 * b.n + 1024
    per = {mc: m["device_bytes"] / b.n for mc, m in sizes.items()}
    # per sphere: up to 96 list slots of 28 bytes, the state, and 6 contacts
    # (two springs, item, shares, record) -- well below the 17 KB that
    # per-slot spring storage took
    assert per[6] < 7_000, per
    assert per[0] > per[6]


@pytest.mark.gpu
def test_contacts_uploaded_in_two_calls(gpu):
    sc = cases.small_chute()
    st = H.run_oracle(sc, 30)
    sc2 = dataclasses.replace(sc, position=st["position"], velocity=st["velocity"],
                              angular_velocity=st["angular_velocity"], orientation=st["orientation"])
    c = st["contacts"]
    assert c["periodic"].any()
    runs = []
    for parts in (1, 2):
        e = sc2.engine()
        cut = np.linspace(0, len(c["id_p"]), parts + 1).astype(int)
        for a, z in zip(cut[:-1], cut[1:]):
            e.upload_contacts(c["id_p"][a:z], c["id_i"][a:z], c["springs"][a:z], c["is_wall"][a:z], c["periodic"][a:z])
        e.step(20)
        out = e.download()
        out["force"], out["torque"] = e.forces()
        out["contacts"] = H.sort_contacts(e.contacts())
        e.close()
        runs.append(out)
    _same(runs[1], runs[0])

"""Batched instances (one handle, many independent simulations) and
DeletionBoundary, through the C ABI against the CPU oracle run on each member
alone.

Tolerances as in test_gpu_parity: pair sets bit-exact, per-contact forces
bit-exact at the initial evaluation; positions 1e-13 of a diameter and forces
1e-9 relative over short horizons; balances from dem_reduce_batch equal to
dem_reduce's to 1e-12 relative (same sums, different order for the records).
"""
import dataclasses

import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import scenarios

pytestmark = pytest.mark.gpu


def _members():
    return [cases.compressed_box(n=300), cases.small_drum(n=400), cases.wall_probe("heap_base", omega=(0.5, 1, 3)),
            cases.small_chute(n_flow=600)]


def _falling_probe():
    sc = cases.wall_probe("heap_base")
    rr = np.hypot(sc.position[:, 0], sc.position[:, 1])
    sc.velocity[rr > 6e-3, 2] = -1.0
    return sc, [((0, 0, -1), 0.9e-3)]  # delete below z = -0.9 mm


def _member_contacts(b, g, k):
    """The batch's contacts of member k in the member's own numbering."""
    c = g["contacts"]
    lo, hi = b.offsets[k], b.offsets[k + 1]
    wall_off = sum(len(m.walls) for m in b.members[:k])
    sel = (c["id_p"] >= lo) & (c["id_p"] < hi)
    out = {key: v[sel].copy() for key, v in c.items()}
    out["id_p"] -= lo
    w = out["is_wall"] != 0
    out["id_i"] = np.where(w, out["id_i"] - wall_off, out["id_i"] - lo)
    return H.sort_contacts(out)


def _run_batch(b, nsteps):
    e = b.engine()
    e.step(nsteps)
    out = e.download()
    out["force"], out["torque"] = e.forces()
    out["contacts"] = e.contacts()
    out["batch"] = e.reduce_batch()
    out["single"] = [e.reduce(k) for k in range(len(b.members))]
    e.close()
    return out


@pytest.mark.parametrize("nsteps", [0, 30])
def test_batch_members_match_oracle(gpu, nsteps):
    members = _members()
    b = scenarios.batch(members)
    g = _run_batch(b, nsteps)
    for k, m in enumerate(members):
        mk = dataclasses.replace(m, time_step=b.time_step)
        o = H.run_oracle(mk, nsteps)
        sl = b.member_slice(k)
        gc = _member_contacts(b, g, k)
        assert H.pair_set(gc) == H.pair_set(o["contacts"]), k
        if nsteps == 0:
            np.testing.assert_array_equal(gc["force"], o["contacts"]["force"])
        assert H.rel_err(g["position"][sl], o["position"], 1e-3) < 1e-13
        assert H.rel_err(g["force"][sl], o["force"]) < 1e-9
        assert H.rel_err(g["torque"][sl], o["torque"]) < 1e-9
        assert (g["instance"][sl] == k).all()


def test_reduce_batch_equals_reduce(gpu):
    b = scenarios.batch(_members())
    g = _run_batch(b, 20)
    for k, s in enumerate(g["single"]):
        for key in ("kinetic_energy", "rotational_energy", "gravitational_energy", "elastic_energy", "mass"):
            assert abs(g["batch"][key][k] - s[key]) <= 1e-12 * max(abs(s[key]), 1e-300), (k, key)
        np.testing.assert_allclose(g["batch"]["centre_of_mass"][k], s["centre_of_mass"], rtol=1e-12, atol=1e-18)
        assert g["batch"]["n_contacts"][k] == s["n_contacts"]
        assert g["batch"]["n_wall_contacts"][k] == s["n_wall_contacts"]


@pytest.mark.parametrize("nsteps", [50, 200])
def test_deletion_boundary_matches_oracle(gpu, nsteps):
    sc, dels = _falling_probe()
    g = H.run_gpu(sc, nsteps, deletions=dels)
    o = H.run_oracle(sc, nsteps, deletions=dels)
    gone = o["instance"] < 0
    assert gone.sum() > 5
    np.testing.assert_array_equal(g["instance"] < 0, gone)
    assert H.pair_set(g["contacts"]) == H.pair_set(o["contacts"])
    assert H.rel_err(g["position"][~gone], o["position"][~gone], 1e-3) < 1e-13
    assert H.rel_err(g["force"][~gone], o["force"][~gone]) < 1e-9
    assert g["globals"]["mass"] > 0


def test_deletion_in_one_batch_member(gpu):
    """A deletion plane of one member leaves the other members untouched."""
    probe, dels = _falling_probe()
    members = [cases.compressed_box(n=300), probe]
    b = scenarios.batch(members, deletions=[[], dels])
    e = b.engine()
    e.step(120)
    out = e.download()
    e.close()
    for k, m in enumerate(members):
        mk = dataclasses.replace(m, time_step=b.time_step)
        o = H.run_oracle(mk, 120, deletions=dels if k == 1 else None)
        sl = b.member_slice(k)
        gone = o["instance"] < 0
        np.testing.assert_array_equal(out["instance"][sl] < 0, gone)
        assert H.rel_err(out["position"][sl][~gone], o["position"][~gone], 1e-3) < 1e-13


def test_heap_batch_matches_oracle_and_runs(gpu):
    """Four calibration heaps in one handle against the oracle per member,
    then the batched pipeline's outputs (AoR estimators, packing fraction,
    kinetic-energy traces)."""
    from mercurydpm_fork_b200 import calibration as cal
    b, params, R = cal.heap_batch(4, seed=5, n_range=(300, 500), base_radius_d=8, column_radius_d=4, v0=0.5)
    e = b.engine()
    e.step(1200)
    out = e.download()
    out["contacts"] = e.contacts()
    e.close()
    for k, m in enumerate(b.members):
        o = H.run_oracle(m, 1200, deletions=[((0, 0, -1), 0.0)])
        sl = b.member_slice(k)
        alive = o["instance"] >= 0
        assert H.pair_set(_member_contacts(b, out, k)) == H.pair_set(o["contacts"])
        np.testing.assert_array_equal(out["instance"][sl] >= 0, alive)
        assert H.rel_err(out["position"][sl][alive], o["position"][alive], 1e-3) < 1e-12
    res = cal.run_heaps(b, R, steps=2000, trace_every=500)
    assert res["kinetic_energy"].shape == (4, 5)
    assert np.isfinite(res["aor_reference"]).all()
    assert (res["n_remaining"] > 0).all()


def test_batch_api_equals_step_and_reduce_batch(gpu):
    """dem_batch_create + dem_batch_run against dem_create + dem_step +
    dem_reduce_batch on the same batch: the same run, the same balances."""
    b = scenarios.batch(_members())
    e1 = b.engine(batch_api=True)
    g1 = e1.batch_run(30)
    x1 = e1.download()["position"]
    e1.close()
    e2 = b.engine()
    e2.step(30)
    g2 = e2.reduce_batch()
    x2 = e2.download()["position"]
    e2.close()
    np.testing.assert_array_equal(x1, x2)
    for key in ("kinetic_energy", "rotational_energy", "gravitational_energy", "mass", "n_contacts", "n_wall_contacts"):
        np.testing.assert_array_equal(g1[key], g2[key])
    np.testing.assert_allclose(g1["elastic_energy"], g2["elastic_energy"], rtol=1e-12)  # atomics: last bits


def test_set_periodic_equals_instance_description(gpu):
    """dem_set_periodic before the upload gives the run that periodic bounds
    in the instance description give."""
    from mercurydpm_fork_b200.engine import DemEngine
    sc = cases.small_chute(n_flow=600)
    inst = sc.instance
    plain = dataclasses.replace(inst, periodic_mask=0, periodic_min=(0.0, 0.0, 0.0), periodic_max=(0.0, 0.0, 0.0))
    e1 = DemEngine(sc.time_step, [plain], sc.species, sc.walls, rotation=sc.rotation)
    e1.set_periodic(0, inst.periodic_min, inst.periodic_max, inst.periodic_mask)
    e1.upload(sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia, sc.species_index, sc.ids)
    e1.step(20)
    e2 = sc.engine()
    e2.step(20)
    np.testing.assert_array_equal(e1.download()["position"], e2.download()["position"])
    np.testing.assert_array_equal(e1.forces()[0], e2.forces()[0])
    e1.close()
    e2.close()

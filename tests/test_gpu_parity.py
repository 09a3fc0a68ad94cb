"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (FP64 everywhere):
* contact pair sets (particle pairs, periodic pairs and wall contacts) at
  identical positions: bit-exact;
* one contact evaluation: per-contact force and springs bit-exact (same
  IEEE operations in the same order, no FMA contraction on either side);
* per-particle totals: 1e-14 relative to the largest force (only the order of
  the sums differs);
* short horizons (<= 50 steps): positions 1e-13 of a diameter, velocities,
  forces and torques 1e-9 relative; longer runs diverge chaotically from
  rounding and are compared through balances.
"""
import numpy as np
import pytest

import cases
import harness as H

pytestmark = pytest.mark.gpu


def _same_pairs(g, o):
    assert H.pair_set(g["contacts"]) == H.pair_set(o["contacts"])


@pytest.mark.parametrize("use_graphs", [True, False])
def test_initial_evaluation_bit_exact(gpu, use_graphs):
    sc = cases.compressed_box()
    g = H.run_gpu(sc, 0, use_graphs=use_graphs)
    o = H.run_oracle(sc, 0)
    _same_pairs(g, o)
    assert len(g["contacts"]["id_p"]) > 1000
    np.testing.assert_array_equal(g["contacts"]["force"], o["contacts"]["force"])
    np.testing.assert_array_equal(g["contacts"]["springs"], o["contacts"]["springs"])
    np.testing.assert_array_equal(g["contacts"]["overlap"], o["contacts"]["overlap"])
    assert H.rel_err(g["force"], o["force"]) < 1e-14
    assert H.rel_err(g["torque"], o["torque"]) < 1e-14
    np.testing.assert_array_equal(g["position"], sc.position)


@pytest.mark.parametrize("nsteps", [1, 7, 50])
def test_short_horizon_box(gpu, nsteps):
    sc = cases.compressed_box()
    g = H.run_gpu(sc, nsteps)
    o = H.run_oracle(sc, nsteps)
    _same_pairs(g, o)
    assert H.rel_err(g["position"], o["position"], 1e-3) < 1e-13
    assert H.rel_err(g["velocity"], o["velocity"]) < 1e-9
    assert H.rel_err(g["angular_velocity"], o["angular_velocity"]) < 1e-9
    assert H.rel_err(g["force"], o["force"]) < 1e-9
    assert H.rel_err(g["torque"], o["torque"]) < 1e-9
    assert H.rel_err(g["orientation"], o["orientation"]) < 1e-12
    assert H.rel_err(g["contacts"]["springs"], o["contacts"]["springs"]) < 1e-9


def test_walls_and_rebuilds(gpu):
    """300 steps: contacts with the walls form, the Verlet list is rebuilt
    several times and history must survive every rebuild."""
    sc = cases.compressed_box()
    g = H.run_gpu(sc, 300, skin=0.02e-3)
    o = H.run_oracle(sc, 300)
    _same_pairs(g, o)
    assert int(g["contacts"]["is_wall"].sum()) > 100
    assert g["stats"]["rebuilds"] >= 2
    assert H.rel_err(g["position"], o["position"], 1e-3) < 1e-11
    assert H.rel_err(g["force"], o["force"]) < 1e-7
    assert H.rel_err(g["contacts"]["springs"], o["contacts"]["springs"]) < 1e-7


@pytest.mark.parametrize("nsteps", [0, 1, 5, 40])
def test_periodic_bidisperse_chute(gpu, nsteps):
    """Two HGrid levels, fixed rough base, periodic x and y, inclined gravity."""
    sc = cases.small_chute()
    g = H.run_gpu(sc, nsteps)
    o = H.run_oracle(sc, nsteps)
    _same_pairs(g, o)
    assert int(g["contacts"]["periodic"].sum()) > 0
    assert (g["contacts"]["periodic"] == o["contacts"]["periodic"]).all()
    if nsteps == 0:
        np.testing.assert_array_equal(g["contacts"]["force"], o["contacts"]["force"])
    assert H.rel_err(g["position"], o["position"], 1e-3) < 1e-13
    assert H.rel_err(g["force"], o["force"]) < 1e-9
    assert H.rel_err(g["torque"], o["torque"]) < 1e-9
    assert H.rel_err(g["contacts"]["springs"], o["contacts"]["springs"]) < 1e-9


def test_large_coordinate_offset(gpu):
    """The chute 1 km from the origin: the neighbour-list prefilter works on
    coordinates relative to the grid, so lists, periodic pairs, contacts and
    forces still match the oracle (FP64 throughout) after rebuilds."""
    sc = cases.offset_chute(1000.0)
    g = H.run_gpu(sc, 60, skin=0.004e-3)
    o = H.run_oracle(sc, 60)
    _same_pairs(g, o)
    assert g["stats"]["rebuilds"] >= 1
    assert int(g["contacts"]["periodic"].sum()) > 0
    assert (g["contacts"]["periodic"] == o["contacts"]["periodic"]).all()
    assert H.rel_err(g["position"], o["position"], 1e-3) < 1e-9  # 1e-12 m: a few units of rounding at 1 km
    assert H.rel_err(g["force"], o["force"]) < 1e-9
    assert H.rel_err(g["contacts"]["springs"], o["contacts"]["springs"]) < 1e-9


def test_tangential_spring_known_answer(gpu):
    """Drivers/UnitTests/TangentialSpringUnitTest.cpp golden values (1e-7)."""
    sc, steps, exp = cases.tangential_spring()
    g = H.run_gpu(sc, steps)
    np.testing.assert_allclose(g["position"][1], exp["Position"]["value"], atol=exp["Position"]["tol"], rtol=0)
    np.testing.assert_allclose(g["velocity"][1], exp["Velocity"]["value"], atol=exp["Velocity"]["tol"], rtol=0)
    np.testing.assert_allclose(g["angular_velocity"][1], exp["AngularVelocity"]["value"],
                               atol=exp["AngularVelocity"]["tol"], rtol=0)


def test_reruns_are_bit_identical(gpu):
    sc = cases.small_chute()
    a = H.run_gpu(sc, 60)
    b = H.run_gpu(sc, 60)
    for k in ("position", "velocity", "angular_velocity", "force", "torque"):
        np.testing.assert_array_equal(a[k], b[k])


def test_split_calls_equal_one_call(gpu):
    """dem_step(a) + dem_step(b) is the same trajectory as dem_step(a+b)."""
    sc = cases.compressed_box()
    e = sc.engine()
    e.step(13)
    e.step(20)
    x1 = e.download()["position"]
    e.close()
    g = H.run_gpu(sc, 33)
    np.testing.assert_array_equal(x1, g["position"])


def test_energy_balance_matches_oracle_state(gpu):
    """Balances from dem_reduce against the same quantities of the oracle state."""
    sc = cases.compressed_box()
    g = H.run_gpu(sc, 20)
    o = H.run_oracle(sc, 20)
    fixed = sc.inv_mass == 0
    m = np.where(fixed, 0.0, 1.0 / np.where(fixed, 1.0, sc.inv_mass))
    ke = 0.5 * np.sum(m * np.sum(o["velocity"] ** 2, 1))
    ge = np.sum(m * (o["position"] @ np.array([0, 0, 9.81])))
    assert abs(g["globals"]["kinetic_energy"] - ke) <= 1e-9 * ke
    assert abs(g["globals"]["gravitational_energy"] - ge) <= 1e-12 * abs(ge)
    np.testing.assert_allclose(g["globals"]["momentum"], (m[:, None] * o["velocity"]).sum(0), rtol=1e-8, atol=1e-14)
    assert g["globals"]["n_contacts"] == int((o["contacts"]["is_wall"] == 0).sum())
    assert g["globals"]["n_wall_contacts"] == int(o["contacts"]["is_wall"].sum())


def test_reupload_same_and_other_size(gpu):
    """A second upload into the same handle starts a new simulation: with the
    same sizes the device arrays and graphs are reused, with other sizes they
    are rebuilt; either way the trajectory equals a fresh handle's."""
    sc = cases.compressed_box()
    ref = H.run_gpu(sc, 40)
    e = sc.engine()
    e.step(25)
    e.upload(sc.position, sc.velocity, sc.radius, sc.inv_mass, sc.inv_inertia, sc.species_index, sc.ids)
    e.step(40)
    out = e.download()
    np.testing.assert_array_equal(out["position"], ref["position"])
    np.testing.assert_array_equal(out["angular_velocity"], ref["angular_velocity"])
    np.testing.assert_array_equal(out["id"], sc.ids)
    small = cases.compressed_box(n=500, seed=4)
    ref2 = H.run_gpu(small, 40)
    e.upload(small.position, small.velocity, small.radius, small.inv_mass, small.inv_inertia, small.species_index,
             small.ids)
    e.step(40)
    out2 = e.download()
    e.close()
    np.testing.assert_array_equal(out2["position"], ref2["position"])
    np.testing.assert_array_equal(out2["velocity"], ref2["velocity"])


def test_periodic_chute_long_horizon(gpu):
    """300 steps of the periodic chute: pairs cross the periodic boundaries
    and back, so a contact changes between a periodic pair (two views, each
    particle P of its own) and an ordinary pair (one interaction, the lower
    id is P); the spring must follow the reference's single interaction."""
    sc = cases.small_chute()
    g = H.run_gpu(sc, 300)
    o = H.run_oracle(sc, 300)
    _same_pairs(g, o)
    assert H.rel_err(g["position"], o["position"], 1e-3) < 1e-11
    assert H.rel_err(g["force"], o["force"]) < 1e-6
    assert H.rel_err(g["contacts"]["springs"], o["contacts"]["springs"]) < 1e-6


def test_upload_rejects_bad_particles(gpu):
    """dem_upload_particles refuses non-finite states, non-positive radii,
    species out of range and negative inverse masses (DEM_ERR_BAD_INPUT with
    a message naming the problem), and accepts the repaired arrays."""
    from mercurydpm_fork_b200 import DemError, _abi
    sc = cases.compressed_box(n=200)
    from mercurydpm_fork_b200.engine import DemEngine
    e = DemEngine(sc.time_step, [sc.instance], sc.species, sc.walls, rotation=sc.rotation)
    base = dict(position=sc.position, velocity=sc.velocity, radius=sc.radius, inv_mass=sc.inv_mass,
                inv_inertia=sc.inv_inertia, species=sc.species_index, ids=sc.ids)
    bad_cases = []
    x = sc.position.copy(); x[17, 1] = np.nan; bad_cases.append(("position", x, "non-finite"))
    v = sc.velocity.copy(); v[3, 2] = np.inf; bad_cases.append(("velocity", v, "non-finite"))
    r = sc.radius.copy(); r[5] = -r[5]; bad_cases.append(("radius", r, "radius"))
    s = sc.species_index.copy(); s[9] = 7; bad_cases.append(("species", s, "species"))
    m = sc.inv_mass.copy(); m[11] = -1.0; bad_cases.append(("inv_mass", m, "inverse mass"))
    for key, arr, word in bad_cases:
        kw = dict(base)
        kw[key] = arr
        with pytest.raises(DemError) as ex:
            e.upload(kw["position"], kw["velocity"], kw["radius"], kw["inv_mass"], kw["inv_inertia"], kw["species"],
                     kw["ids"])
        assert ex.value.code == _abi.DEM_ERR_BAD_INPUT
        assert word in str(ex.value), (key, str(ex.value))
    e.upload(**base)
    e.step(1)
    e.close()


def test_bounded_wait_expires_and_reports(gpu):
    """The rebuild's grid-barrier wait is bounded: a barrier that can never
    complete (one arrival short) makes every block give up after its poll
    limit and report DEM_ERR_TIMEOUT in the status word, without a trap; the
    engine keeps working afterwards."""
    import ctypes as C
    from mercurydpm_fork_b200 import _abi
    from mercurydpm_fork_b200.engine import lib
    sc = cases.compressed_box(n=200)
    e = sc.engine()
    st = C.c_uint32(0)
    assert lib().dem_selftest_wait_expiry(e._h, 1 << 14, C.byref(st)) == 0
    assert st.value == (1 << _abi.DEM_ERR_TIMEOUT)
    e.step(5)
    assert np.isfinite(e.download()["position"]).all()
    e.close()

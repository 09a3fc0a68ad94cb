"""Insertion boundaries (CubeInsertionBoundary, Kernel/Boundaries/
InsertionBoundary.cc:184-296) on the engine against the reference build.

* CPU: the oracle's own restatement of the insertion and of the chute fill
  against the reference build (placements bit for bit, then the run).
* CPU: the engine's restatements of the reference's generators -- RNG
  (Kernel/Math/RNG.cc, lagged Fibonacci 607/273 seeded by the linear
  congruential generator) and PSD::drawSample (Kernel/Math/PSD.cc:114-128)
  after PSD::setDistributionUniform -- give bit-identical sequences to the
  reference's own classes (dem_rng_draws / dem_psd_draws run the kernel's
  code on the host).
* GPU: a box whose bed fills its bottom, with a CubeInsertionBoundary over
  the bed's top, run on the engine and on the reference Kernel from the same
  inputs: the same particles are placed (count, volume, rows, radii, masses
  bit for bit) and the run continues like the law tests (positions 1e-12 of
  a diameter, velocities and forces 1e-9 of their largest magnitude). Walled
  and periodic sides, the three PSD forms, a volume flow rate that stops the
  insertion between steps (the drawn particle waits for the next step), and
  a run out of free rows (DEM_ERR_CAPACITY).
"""
import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import _abi
from mercurydpm_fork_b200.engine import DemError, insertion_boundary, psd_draws, rng_draws
from mercurydpm_fork_b200.host import psd_uniform

needs_ref = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")


@needs_ref
@pytest.mark.parametrize("seed", [0, 1, 12345, 2 ** 31 + 7])
def test_rng_matches_reference(seed):
    ours = rng_draws(seed, 5000)
    ref = H.reference_rng_draws(seed, 5000)
    np.testing.assert_array_equal(ours, ref)
    assert 0.0 <= ours.min() and ours.max() < 1.0


@needs_ref
@pytest.mark.parametrize("rmin,rmax,bins,seed", [(0.4e-3, 0.6e-3, 2, 0), (0.5e-3, 0.5e-3, 50, 0),
                                                 (0.45e-3, 0.55e-3, 8, 3), (1.0, 3.0, 64, 17)])
def test_psd_draws_match_reference(rmin, rmax, bins, seed):
    b = insertion_boundary((0, 0, 0), (1, 1, 1), 1.0, psd=psd_uniform(rmin, rmax, bins), psd_seed=seed)
    ours = psd_draws(b, 3000)
    ref = H.reference_psd_draws(rmin, rmax, bins, seed, 3000)
    np.testing.assert_array_equal(ours, ref)


@needs_ref
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("psd", ["range", "single", "bins"])
def test_oracle_insertion_matches_reference(periodic, psd):
    """The oracle's own restatement of the insertion (oracle/dem_oracle.cpp:
    the reference's generators kept as the reference stores them, every
    candidate tested against every particle) places the reference's particles,
    on the CPU."""
    sc, bnd = cases.insertion_box(periodic=periodic, psd=psd, psd_seed=5)
    o = H.run_oracle(sc, 400, insertions=bnd, seed=3)
    r = H.run_reference(sc, 400, insertions=bnd, seed=3)
    np.testing.assert_array_equal(o["inserted"], r["inserted"])
    np.testing.assert_array_equal(o["inserted_volume"], r["inserted_volume"])
    _compare(o, r)


@needs_ref
@pytest.mark.parametrize("seed", range(8))
def test_oracle_insertion_seeds_match_reference(seed):
    """More seeds, walled and periodic in turn, all three PSD forms: the
    reference's HGrid also files a particle one cell off when the step's
    drift carried it over an ordinary cell boundary, which the restatements
    (oracle and engine) leave out; it changes no placement here."""
    sc, bnd = cases.insertion_box(periodic=bool(seed % 2), psd=("range", "single", "bins")[seed % 3],
                                  seed=30 + seed, psd_seed=seed)
    o = H.run_oracle(sc, 400, insertions=bnd, seed=seed)
    r = H.run_reference(sc, 400, insertions=bnd, seed=seed)
    np.testing.assert_array_equal(o["inserted"], r["inserted"])
    _compare(o, r)


@needs_ref
def test_oracle_insertion_with_deletion_matches_reference():
    """Particles placed above z = 10 d are removed by a DeletionBoundary at
    the next step and placed again: some 2,000 of 2,500 placements are
    deleted, and the survivors keep the rows their placement gave them."""
    sc, bnd = cases.insertion_box(psd="range", n_free=4000)
    dels = [((0, 0, 1), 10e-3)]
    o = H.run_oracle(sc, 200, insertions=bnd, seed=6, deletions=dels)
    r = H.run_reference(sc, 200, insertions=bnd, seed=6, deletions=dels)
    np.testing.assert_array_equal(o["inserted"], r["inserted"])
    assert r["inserted"][0] - ((r["instance"] >= 0).sum() - 300) > 1000
    _compare(o, r)


@needs_ref
def test_oracle_chute_insertion_and_fill_match_reference():
    """The oracle's ChuteInsertionBoundary and Chute::addFlowParticlesCompactly
    against the reference, on the CPU."""
    for periodic in (False, True):
        sc, bnd = cases.insertion_box(periodic=periodic, psd="bins", psd_seed=2, chute=True)
        o = H.run_oracle(sc, 300, insertions=bnd, seed=4)
        r = H.run_reference(sc, 300, insertions=bnd, seed=4)
        np.testing.assert_array_equal(o["inserted"], r["inserted"])
        _compare(o, r)
    sc, f = cases.chute_fill_case()
    o = H.run_oracle(sc, 30, chute_fill=f, seed=7)
    r = H.run_reference_chute_fill(sc, f, 7, 30)
    assert o["inflow_height"] == r["inflow_height"] > f.inflow_height
    _compare(o, r)


def _compare(a, r):
    live = r["instance"] >= 0
    np.testing.assert_array_equal(a["instance"] >= 0, live)
    np.testing.assert_array_equal(a["radius"][live], r["radius"][live])
    np.testing.assert_array_equal(a["inv_mass"][live], r["inv_mass"][live])
    np.testing.assert_array_equal(a["inv_inertia"][live], r["inv_inertia"][live])
    assert H.pair_set(a["contacts"]) == H.pair_set(r["contacts"])
    assert H.rel_err(a["position"][live], r["position"][live], 1e-3) < 1e-12
    for k in ("velocity", "force"):
        assert H.rel_err(a[k][live], r[k][live]) < 1e-9, k


def _run_both(sc, bnd, steps, seed=0):
    a = H.run_gpu(sc, steps, insertions=bnd, seed=seed)
    r = H.run_reference(sc, steps, insertions=bnd, seed=seed)
    return a, r


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("psd", ["range", "single", "bins"])
def test_insertion_matches_reference(gpu, periodic, psd):
    sc, bnd = cases.insertion_box(periodic=periodic, psd=psd, psd_seed=5)
    a, r = _run_both(sc, bnd, 400, seed=3)
    np.testing.assert_array_equal(a["inserted"], r["inserted"])
    np.testing.assert_array_equal(a["inserted_volume"], r["inserted_volume"])
    n_live0 = int(np.count_nonzero(sc.radius))
    assert r["inserted"][0] > 100  # the first step fills much of the region
    assert int((r["instance"] >= 0).sum()) == n_live0 + int(r["inserted"][0])
    _compare(a, r)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("periodic", [False, True])
def test_chute_insertion_matches_reference(gpu, periodic):
    """ChuteInsertionBoundary (ChuteInsertionBoundary.cc:163-190): particles fed
    into one plane of x, over a y range one radius wider than the boundary on
    each side (with periodic y, candidates beyond the period meet the images)."""
    sc, bnd = cases.insertion_box(periodic=periodic, psd="bins", psd_seed=2, chute=True)
    a, r = _run_both(sc, bnd, 300, seed=4)
    np.testing.assert_array_equal(a["inserted"], r["inserted"])
    np.testing.assert_array_equal(a["inserted_volume"], r["inserted_volume"])
    assert r["inserted"][0] > 20
    _compare(a, r)


@pytest.mark.gpu
@needs_ref
def test_insertion_with_deletion_matches_reference(gpu):
    """Placements above z = 10 d deleted at the next step and made again
    (most of some 2,500): the placements, the deletions and the rows kept."""
    sc, bnd = cases.insertion_box(psd="range", n_free=4000)
    dels = [((0, 0, 1), 10e-3)]
    a = H.run_gpu(sc, 200, insertions=bnd, seed=6, deletions=dels)
    r = H.run_reference(sc, 200, insertions=bnd, seed=6, deletions=dels)
    np.testing.assert_array_equal(a["inserted"], r["inserted"])
    _compare(a, r)


@pytest.mark.gpu
@needs_ref
def test_insertion_flow_rate_limits_between_steps(gpu):
    """A volume flow rate of about half a particle per time step: most steps
    place one particle or none, and the particle drawn last waits (its radius
    already drawn) for the step whose volume allows it."""
    d = 1e-3
    vp = 4.0 / 3.0 * np.pi * (0.5 * d) ** 3
    sc, bnd = cases.insertion_box(rate=0.5 * vp / 2e-6, psd="range")
    a, r = _run_both(sc, bnd, 80, seed=9)
    np.testing.assert_array_equal(a["inserted"], r["inserted"])
    assert 20 <= r["inserted"][0] <= 60
    _compare(a, r)


@pytest.mark.gpu
def test_insertion_without_free_rows_reports_capacity(gpu):
    sc, bnd = cases.insertion_box(n_free=5)
    e = sc.engine(insertions=bnd, insertion_seeds=[0])
    with pytest.raises(DemError) as err:
        e.step(2)
    assert err.value.code == _abi.DEM_ERR_CAPACITY
    e.close()


def test_insertion_boundary_validation():
    """Bad PSDs and ranges are refused before anything reaches a device."""
    with pytest.raises(ValueError):
        insertion_boundary((0, 0, 0), (1, 1, 1), 1.0)  # neither radius nor PSD
    b = insertion_boundary((0, 0, 0), (1, 1, 1), 1.0, psd=([1.0, 2.0], [0.0, 1.0]))
    out = psd_draws(b, 100)
    assert np.all((out >= 1.0 - 1e-12) & (out <= 2.0 + 1e-12))


@pytest.mark.gpu
@needs_ref
def test_chute_fill_matches_reference(gpu):
    """Chute::addFlowParticlesCompactly (Chute.cc:1083-1115) on a periodic
    chute over a rough base: the same particles, in the same places (bit for
    bit, before any step), the same final inflow height after some 70,000
    rejected candidates; then 30 steps like the other runs."""
    sc, f = cases.chute_fill_case()
    a0 = H.run_gpu(sc, 0, chute_fill=f, seed=7)
    r0 = H.run_reference_chute_fill(sc, f, 7, 0)
    live = r0["instance"] >= 0
    np.testing.assert_array_equal(a0["instance"] >= 0, live)
    assert a0["filled"] == int(live.sum()) - int(np.count_nonzero(sc.radius)) > 400
    assert a0["inflow_height"] == r0["inflow_height"] > f.inflow_height
    for k in ("position", "radius", "inv_mass", "inv_inertia"):
        np.testing.assert_array_equal(a0[k][live], r0[k][live], err_msg=k)
    a = H.run_gpu(sc, 30, chute_fill=f, seed=7)
    r = H.run_reference_chute_fill(sc, f, 7, 30)
    _compare(a, r)


@pytest.mark.gpu
@needs_ref
def test_insertion_in_batch_members(gpu):
    """Two instances of one handle, each with its own insertion boundary and
    generator seed (the k_insert blocks of one launch run side by side):
    each member places what the reference places when run alone."""
    from mercurydpm_fork_b200 import scenarios
    s0, (b0,) = cases.insertion_box(seed=11, n_free=600)
    s1, (b1,) = cases.insertion_box(periodic=True, seed=12, psd="bins", psd_seed=1, n_free=600)
    bt = scenarios.batch([s0, s1])
    b1.instance = 1
    e = bt.engine(insertions=[b0, b1], insertion_seeds=[3, 5])
    e.step(200)
    g = e.download()
    g["force"], g["torque"] = e.forces()
    c = e.contacts()
    cnt, vol = e.insertion_counts()
    e.close()
    for k, (sc, b, seed) in enumerate(((s0, b0, 3), (s1, b1, 5))):
        b.instance = 0  # the reference runs the member alone
        r = H.run_reference(sc, 200, insertions=[b], seed=seed)
        assert cnt[k] == r["inserted"][0] and vol[k] == r["inserted_volume"][0]
        sl = bt.member_slice(k)
        a = {key: g[key][sl] for key in ("position", "velocity", "force", "radius", "inv_mass", "inv_inertia")}
        a["instance"] = np.where(g["instance"][sl] == k, 0, -1)
        a["contacts"] = _member_contacts(bt, c, k)
        _compare(a, r)


def _member_contacts(b, c, k):
    lo, hi = b.offsets[k], b.offsets[k + 1]
    wall_off = sum(len(m.walls) for m in b.members[:k])
    sel = (c["id_p"] >= lo) & (c["id_p"] < hi)
    out = {key: v[sel].copy() for key, v in c.items()}
    out["id_p"] -= lo
    w = out["is_wall"] != 0
    out["id_i"] = np.where(w, out["id_i"] - wall_off, out["id_i"] - lo)
    return H.sort_contacts(out)

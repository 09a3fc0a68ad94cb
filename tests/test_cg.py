"""Gaussian coarse-graining: the reference's CG (driven through its own API in
oracle/_ref) pinned to its known answers, and the engine's dem_cg_eval
against it.

Tolerance: every field within 1e-10 of the largest magnitude of that field
over the grid (exp/erf come from different math libraries and the sums run
in another order, so results agree to rounding, not bit for bit). The
engine's own evaluations are bit-for-bit reproducible: every point gathers in
a fixed order, whatever order the contact records were written in.
"""
import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import _abi

needs_ref = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build (oracle/_ref) absent")


def _close(a, b, tol=1e-10):
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    err = (np.abs(a - b) / scale).max()
    assert err < tol, err


@needs_ref
def test_reference_cg_packing_known_answer():
    """CG3DPackingUnitTest.cpp:86-99: density n^3/V, contact stress n^3 0.99/V (1e-10)."""
    sc, info = cases.cubic_packing()
    L = info["n"] * info["distance"]
    out = H.reference_cg(sc, 10, H.cg_grid(_abi.DEM_CG_O, (1, 1, 1), (0, 0, 0), (L, L, L), 1.0))
    V = info["volume"]
    assert abs(out[0, 1] - info["n"] ** 3 / V) <= 1e-10 * out[0, 1]
    for k in (11, 15, 19):
        assert abs(out[0, k] - info["n"] ** 3 * 0.99 / V) <= 1e-10 * out[0, k]


@pytest.mark.gpu
def test_cg_packing_known_answer(gpu):
    sc, info = cases.cubic_packing()
    L = info["n"] * info["distance"]
    e = sc.engine()
    e.step(10)
    out = e.cg(_abi.DEM_CG_O, (1, 1, 1), (0, 0, 0), (L, L, L), 1.0)
    e.close()
    V = info["volume"]
    assert abs(out[0, 1] - info["n"] ** 3 / V) <= 1e-10 * out[0, 1]
    for k in (11, 15, 19):
        assert abs(out[0, k] - info["n"] ** 3 * 0.99 / V) <= 1e-10 * out[0, k]
    if H.reference_available("serial"):
        ref = H.reference_cg(sc, 10, H.cg_grid(_abi.DEM_CG_O, (1, 1, 1), (0, 0, 0), (L, L, L), 1.0))
        _close(out, ref)


@pytest.mark.gpu
@needs_ref
@pytest.mark.parametrize("nsteps", [0, 5])
def test_cg_chute_xz_matches_reference(gpu, nsteps):
    """CG<XZ> on the periodic bidisperse chute (rough base: contacts with fixed
    particles use the contact-point integrals)."""
    sc = cases.small_chute()
    args = (_abi.DEM_CG_XZ, (20, 1, 10), (0.0, 0.0, 0.0), (0.02, 0.01, 0.02), 1e-3)
    e = sc.engine()
    e.step(nsteps)
    out = e.cg(*args)
    e.close()
    ref = H.reference_cg(sc, nsteps, H.cg_grid(*args))
    assert np.abs(ref[:, 11]).max() > 0
    _close(out, ref)


@pytest.mark.gpu
@needs_ref
def test_cg_box_xyz_matches_reference(gpu):
    """CG<XYZ> with wall contacts (contact to P integrals) in the settling box."""
    sc = cases.compressed_box()
    args = (_abi.DEM_CG_XYZ, (5, 5, 10), (0.0, 0.0, 0.0), (0.01, 0.01, 0.02), 1e-3)
    e = sc.engine()
    e.step(300)
    out = e.cg(*args)
    e.close()
    ref = H.reference_cg(sc, 300, H.cg_grid(*args))
    _close(out, ref, tol=1e-8)  # 300 steps of chaotic divergence at the 1e-12 level


@pytest.mark.gpu
@needs_ref
def test_cg_time_average_matches_reference(gpu):
    """TimeAveragedCG<XZ> on the chute: evaluations after 5, 10 and 15 steps
    averaged, against the mean of the reference's CG at the same states (the
    reference's time average sums the raw fields and divides by the volume
    and the number of evaluations, TimeAveragedCG.hcc:80-107)."""
    sc = cases.small_chute()
    args = (_abi.DEM_CG_XZ, (20, 1, 10), (0.0, 0.0, 0.0), (0.02, 0.01, 0.02), 1e-3)
    e = sc.engine()
    e.step(5)
    out = e.cg_time_average(*args, steps_between=5, evaluations=3)
    e.close()
    ref = sum(H.reference_cg(sc, k, H.cg_grid(*args)) for k in (5, 10, 15)) / 3.0
    assert np.abs(ref[:, 11]).max() > 0
    _close(out, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("coord", ["XZ", "XYZ", "O"])
def test_cg_is_reproducible_bit_for_bit(gpu, coord):
    """Two evaluations of one state, and the same run made again in a second
    engine (its contact records written in another order), give identical
    fields."""
    sc = cases.small_chute()
    args = {"XZ": (_abi.DEM_CG_XZ, (20, 1, 10), (0.0, 0.0, 0.0), (0.02, 0.01, 0.02), 1e-3),
            "XYZ": (_abi.DEM_CG_XYZ, (10, 5, 10), (0.0, 0.0, 0.0), (0.02, 0.01, 0.02), 1e-3),
            "O": (_abi.DEM_CG_O, (1, 1, 1), (0.0, 0.0, 0.0), (0.02, 0.01, 0.02), 1e-3)}[coord]
    runs = []
    for _ in range(2):
        e = sc.engine()
        e.step(40)
        runs.append(e.cg(*args))
        runs.append(e.cg(*args))
        e.close()
    assert np.abs(runs[0][:, 11]).max() > 0
    for r in runs[1:]:
        np.testing.assert_array_equal(r, runs[0])

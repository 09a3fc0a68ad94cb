"""The reference's text outputs (.ene, .fstat, .data) written from the engine.

CPU: the .data writer, given the reference's own state after 20 steps of the
small periodic chute, reproduces the reference's .data text character for
character (DPMBase::outputXBallsData through the reference build), and the
.ene header matches the reference's.

GPU: the three files written from the CUDA path's state match the files the
reference writes for the same run: the same header lines, the same set of
.fstat records, numbers within the tolerances below (the state agrees to
about 1e-13 of a diameter; files carry 10 significant digits, positions 15).
"""
import os

import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import output

STEPS = 20


def _numbers(line):
    return [float(x) for x in line.split()]


def _ref_files(tmp_path, sc, steps=STEPS):
    prefix = str(tmp_path / "ref")
    H.reference_outputs(sc, steps, prefix)
    return {ext: open(prefix + "." + ext).read() for ext in ("ene", "fstat", "data")}


needs_reference = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")


@needs_reference
def test_data_writer_reproduces_reference_text(tmp_path):
    sc = cases.small_chute(n_flow=600)
    ref = _ref_files(tmp_path, sc)
    r = H.run_reference(sc, STEPS)
    state = dict(position=r["position"], velocity=r["velocity"], angular_velocity=r["angular_velocity"],
                 orientation=r["orientation"], radius=sc.radius, species=sc.species_index, instance=r["instance"])
    t = output.time_after(STEPS, sc.time_step)
    ours = output.data_text(t, sc.instance.domain_min, sc.instance.domain_max, state)
    assert ours == ref["data"]
    assert ref["ene"].splitlines()[0] + "\n" == output.ene_header()


@pytest.mark.gpu
@needs_reference
def test_outputs_match_reference_files(gpu, tmp_path):
    sc = cases.small_chute(n_flow=600)
    ref = _ref_files(tmp_path, sc)
    e = sc.engine()
    e.step(STEPS)
    prefix = str(tmp_path / "gpu")
    output.write_outputs(e, prefix, STEPS, sc.time_step, sc.instance.domain_min, sc.instance.domain_max,
                         sc.instance.gravity)
    e.close()
    ours = {ext: open(prefix + "." + ext).read() for ext in ("ene", "fstat", "data")}

    # .ene: header identical; time, energies, centre of mass and the number of interactions
    re_, oe = ref["ene"].splitlines(), ours["ene"].splitlines()
    assert re_[0] == oe[0]
    a, b = _numbers(re_[1]), _numbers(oe[1])
    assert a[0] == b[0] and a[-1] == b[-1]
    np.testing.assert_allclose(b[1:-1], a[1:-1], rtol=1e-8, atol=0)

    # .data: header line identical; per particle positions to 1e-12 m, the rest to 1e-8 relative
    rd, od = ref["data"].splitlines(), ours["data"].splitlines()
    assert rd[0] == od[0] and len(rd) == len(od)
    A = np.array([_numbers(x) for x in rd[1:]])
    B = np.array([_numbers(x) for x in od[1:]])
    np.testing.assert_allclose(B[:, :3], A[:, :3], rtol=0, atol=1e-12)
    np.testing.assert_allclose(B[:, 3:], A[:, 3:], rtol=1e-8, atol=1e-14)

    # .fstat: three header lines identical; the same records (per (i, j) line)
    rf, of = ref["fstat"].splitlines(), ours["fstat"].splitlines()
    assert rf[:3] == of[:3]
    assert len(rf) == len(of)

    def records(lines):
        out = {}
        for x in lines[3:]:
            v = _numbers(x)
            out[(int(v[1]), int(v[2]))] = np.array(v)
        return out

    R, O = records(rf), records(of)
    assert set(R) == set(O)
    assert len(R) > 200
    # columns: time, i, j, contact point (3), overlap, tangential overlap, normal force,
    # tangential force, normal (3), tangential direction (3)
    for k in R:
        a, b = R[k], O[k]
        np.testing.assert_allclose(b[:9], a[:9], rtol=1e-7, atol=1e-12, err_msg=str(k))
        assert abs(b[9] - a[9]) <= 1e-7 * abs(a[9]) + 1e-9 * abs(a[8]) + 1e-15, (k, a[9], b[9])
        np.testing.assert_allclose(b[10:13], a[10:13], rtol=1e-7, atol=1e-9, err_msg=str(k))
        if a[9] > 1e-6 * abs(a[8]):  # the tangential direction is defined
            np.testing.assert_allclose(b[13:16], a[13:16], rtol=0, atol=1e-6, err_msg=str(k))

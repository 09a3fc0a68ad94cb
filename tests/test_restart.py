"""Restart files (mercurydpm_fork_b200/restart.py) against the reference's own.

Reading: the reference writes a restart file after 30 steps (DPMBase::write,
15 significant digits); the file is parsed into the engine's inputs and the
run continues. The reference, restarted from the same file by its own reader
(DPMBase::readRestartFile, then initialiseSolve without
setupInitialConditions), continues too. Both re-evaluate the forces with the
stored springs first. Compared at that evaluation and 20 steps later: the same
contact pairs, and positions, forces and springs within the tolerances below
(1e-12 relative; the rotated intersection wall rebuilds its face normals from
the file's 15-digit quaternions, which moves its forces by ~1e-13).

Writing: the engine writes its state after 30 steps; the reference reads that
file and continues, next to the reference reading the file it wrote itself
after the same 30 steps. Particle and interaction lines of the two files
agree under the reference's fpdiff rule (0.1 %), and the two continued runs
agree like the read test (the states differ by the rounding of the 30 steps
before writing: 1e-9 relative).
"""
import os

import numpy as np
import pytest

import cases
import harness as H
from mercurydpm_fork_b200 import restart

needs_reference = pytest.mark.skipif(not H.reference_available("serial"), reason="reference build absent")

CASES = {
    "periodic_chute": cases.small_chute,
    "rotating_drum": cases.small_drum,
    "settling_box": cases.compressed_box,
    "rotated_intersection_wall": lambda: cases.wall_probe("box_corner"),
}
STEPS_BEFORE = 30


def _compare(a, b, tol):
    assert H.pair_set(a["contacts"]) == H.pair_set(b["contacts"])
    assert H.rel_err(a["position"], b["position"], 1e-3) < tol
    assert H.rel_err(a["force"], b["force"]) < tol
    if len(b["contacts"]["id_p"]):
        assert H.rel_err(a["contacts"]["springs"], b["contacts"]["springs"]) < tol


def _reference_file(sc, tmp_path, name):
    path = str(tmp_path / f"{name}.restart")
    return path, H.reference_restart(sc, STEPS_BEFORE, path)


@needs_reference
@pytest.mark.parametrize("name", sorted(CASES))
def test_reader_continues_like_the_reference(name, tmp_path):
    """CPU: the oracle (the FP64 restatement) continued from the parsed file."""
    sc = CASES[name]()
    path, text = _reference_file(sc, tmp_path, name)
    st = restart.read(text)
    assert st.n_steps == STEPS_BEFORE and len(st.interactions["id_p"]) > 0
    sc2, contacts = st.scenario()
    for steps in (0, 20):
        _compare(H.run_oracle(sc2, steps, contacts=contacts), H.reference_restart_run(path, steps, sc.n), 1e-12)


def test_reader_rejects_what_the_engine_does_not_have():
    text = ("MercuryDPM 1.0 name x revision 0 repository 0\nxMin 0 xMax 1 yMin 0 yMax 1 zMin 0 zMax 1\n"
            "timeStep 1e-05 time 0 ntimeSteps 0 timeMax 1\nsystemDimensions 3 particleDimensions 3 gravity 0 0 -1 "
            "backgroundDrag 0\nSpecies 1\nLinearViscoelasticReversibleAdhesiveSpecies id 0 density 1 stiffness 1 "
            "dissipation 0\n")
    with pytest.raises(ValueError, match="no such contact law"):
        restart.read(text)


@pytest.mark.gpu
@needs_reference
@pytest.mark.parametrize("name", sorted(CASES) + ["triangle_mesh"])
def test_engine_restarts_from_reference_file(gpu, name, tmp_path):
    sc = cases.triangle_mesh() if name == "triangle_mesh" else CASES[name]()
    path, text = _reference_file(sc, tmp_path, name)
    sc2, contacts = restart.read(text).scenario()
    for steps in (0, 20):
        _compare(H.run_gpu(sc2, steps, contacts=contacts), H.reference_restart_run(path, steps, sc.n), 1e-12)


def _sections(text, title):
    lines = text.splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.startswith(title + " "))
    n = int(lines[k].split()[1])
    return lines[k + 1:k + 1 + n]


def _without(line, key, count):
    t = line.split()
    if key in t:
        i = t.index(key)
        del t[i:i + 1 + count]
    return " ".join(t)


@pytest.mark.gpu
@needs_reference
@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_restart_file_is_read_by_the_reference(gpu, name, tmp_path):
    sc = CASES[name]()
    theirs, their_text = _reference_file(sc, tmp_path, name + "_ref")
    e = sc.engine()
    try:
        e.step(STEPS_BEFORE)
        ours_text = restart.write(e, sc, STEPS_BEFORE, name=name)
    finally:
        e.close()
    ours = str(tmp_path / f"{name}_engine.restart")
    open(ours, "w").write(ours_text)
    # the particle lines; the interaction lines without their torque (the
    # engine writes none) in a common order
    assert not H.fpdiff("\n".join(_sections(ours_text, "Particles")), "\n".join(_sections(their_text, "Particles")))
    key = lambda ln: (ln.split()[1], int(ln.split()[2]), int(ln.split()[3]))
    a = sorted((_without(ln, "torque", 3) for ln in _sections(ours_text, "Interactions")), key=key)
    b = sorted((_without(ln, "torque", 3) for ln in _sections(their_text, "Interactions")), key=key)
    assert not H.fpdiff("\n".join(a), "\n".join(b))
    for steps in (0, 20):
        _compare(H.reference_restart_run(ours, steps, sc.n), H.reference_restart_run(theirs, steps, sc.n), 1e-9)

"""Regenerates the golden fixtures in this directory from the reference
checkout (run in a container that has it; the fixtures are committed so the
tests never read the reference at run time).

* tangential_spring.json: the known answers that
  Drivers/UnitTests/TangentialSpringUnitTest.cpp asserts (final position,
  velocity and angular velocity of the rolling sphere, tolerance 1e-7), plus
  the set-up numbers of that test.
* settling_box_ene.json: the .ene file the reference writes (its own
  DPMBase::solve and writeEneTimeStep, a line every 500 steps) for the
  5,000-sphere settling box over 20,000 steps (scenarios.settling_box), from
  its serial build and from its OpenMP build on 8 threads. The two builds
  differ only in the order of floating-point sums; their difference is the
  chaos envelope the GPU run is held to. Needs the reference build
  (oracle/_ref, `make -f oracle/ref.mk`).

* selftest/*.gz: the gold files of the reference's own self tests that cover
  the time step (Drivers/SelfTests/Interactions/SelfTestData/
  ForceSelfTest{0..9}.{data,ene}, FreeFallSelfTest.{ene,restart}), copied
  byte for byte and gzipped; the tests compare them with the reference's
  fpdiff rule (0.1 % relative, 1e-14 numerical zero).

Usage: python tests/golden/make_golden.py [REFERENCE_CHECKOUT] [fixture ...]
(the checkout defaults to $MERCURYDPM_REF).
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = sys.argv[1] if len(sys.argv) > 1 and os.path.isdir(sys.argv[1]) else os.environ.get("MERCURYDPM_REF", "")


def vec(s):
    return [float(x) for x in s.split(",")]


def tangential_spring():
    path = os.path.join(REF, "Drivers", "UnitTests", "TangentialSpringUnitTest.cpp")
    src = open(path).read()
    checks = re.findall(r"get(Position|Velocity|AngularVelocity)\(\)\.isEqualTo\(Vec3D\(([^)]*)\),\s*([0-9.e-]+)\)",
                        src)
    # the second particle's checks are the last three
    p1 = checks[-3:]
    out = {
        "source": "Drivers/UnitTests/TangentialSpringUnitTest.cpp",
        "time_step": float(re.search(r"setTimeStep\(([^)]*)\)", src).group(1)),
        "time_max": float(re.search(r"setTimeMax\(([^)]*)\)", src).group(1)),
        "collision_time_restitution_mass": vec(
            re.search(r"setCollisionTimeAndRestitutionCoefficient\(([^)]*)\)", src).group(1).replace("1. / 8", "0.125")),
        "gravity": vec(re.search(r"setGravity\(Vec3D\(([^)]*)\)\)", src).group(1)),
        "expected": {k: {"value": vec(v), "tol": float(t)} for k, v, t in p1},
    }
    return out


ENE_STEPS = 20_000
ENE_SAVE = 500


def settling_box_ene():
    import tempfile
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.dirname(HERE))
    import harness as H
    from mercurydpm_fork_b200 import scenarios
    sc = scenarios.settling_box()
    with tempfile.TemporaryDirectory() as tmp:
        serial = H.reference_ene(sc, ENE_STEPS, ENE_SAVE, os.path.join(tmp, "serial"), "serial")
        omp = H.reference_ene(sc, ENE_STEPS, ENE_SAVE, os.path.join(tmp, "omp"), "omp", threads=8)
    return {"scenario": "scenarios.settling_box() (5,000 spheres, 20 x 20 x 40 d box, dt = tc/50 = 2e-6 s)",
            "steps": ENE_STEPS, "save_count": ENE_SAVE,
            "columns": ["time", "gravitational", "kinetic", "rotational", "elastic", "com_x", "com_y", "com_z",
                        "interactions"],
            "serial": serial.tolist(), "omp8": omp.tolist()}


def selftest():
    import gzip
    src = os.path.join(REF, "Drivers", "SelfTests", "Interactions", "SelfTestData")
    names = [f"ForceSelfTest{k}.{ext}" for k in range(10) for ext in ("data", "ene")]
    names += ["FreeFallSelfTest.ene", "FreeFallSelfTest.restart"]
    out = os.path.join(HERE, "selftest")
    os.makedirs(out, exist_ok=True)
    for n in names:
        with open(os.path.join(src, n), "rb") as f:
            data = f.read()
        with gzip.GzipFile(os.path.join(out, n + ".gz"), "wb", mtime=0) as g:
            g.write(data)
    return {"source": "Drivers/SelfTests/Interactions/SelfTestData", "files": names}


FIXTURES = {"tangential_spring": tangential_spring, "settling_box_ene": settling_box_ene, "selftest": selftest}

if __name__ == "__main__":
    if not REF:
        sys.exit("give the reference checkout as the first argument or in $MERCURYDPM_REF")
    names = [a for a in sys.argv[1:] if a in FIXTURES] or list(FIXTURES)
    for name in names:
        data = FIXTURES[name]()
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(data, f, indent=1)
        print(name, "written")

"""Regenerates the golden fixtures in this directory from the reference
checkout (run in a container that has it; the fixtures are committed so the
tests never read the reference at run time).

* tangential_spring.json: the known answers that
  Drivers/UnitTests/TangentialSpringUnitTest.cpp asserts (final position,
  velocity and angular velocity of the rolling sphere, tolerance 1e-7), plus
  the set-up numbers of that test.
"""
from __future__ import annotations

import json
import os
import re
import sys

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
HERE = os.path.dirname(os.path.abspath(__file__))


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


if __name__ == "__main__":
    data = tangential_spring()
    with open(os.path.join(HERE, "tangential_spring.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps(data, indent=1))

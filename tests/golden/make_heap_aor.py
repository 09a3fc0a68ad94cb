"""Writes tests/golden/heap_aor.json: the angle of repose of three cased heaps
(calibration.cased_heap_scenario, 2,000 spheres each) from the procedure of
Drivers/Calibration/CalibrationHeap.cpp run on the reference Kernel
(mdpm_ref_heap_procedure in oracle/ref_drivers/mdpm_ref_driver.cpp), serial
and with 4 OpenMP threads: the two runs differ only in the order of the force
sums, so their spread is the chaos envelope of the measurement.

Run from the repository root after building oracle/_ref:
    python tests/golden/make_heap_aor.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import harness as H  # noqa: E402
from mercurydpm_fork_b200 import calibration as cal  # noqa: E402

HEAPS = [dict(n=2000, sigma=0.1, mu=0.5, mu_r=0.1, restitution=0.5, seed=7),
         dict(n=2000, sigma=0.0, mu=0.3, mu_r=0.05, restitution=0.7, seed=11),
         dict(n=2000, sigma=0.2, mu=0.8, mu_r=0.2, restitution=0.4, seed=13)]


def main():
    rows = []
    for hp in HEAPS:
        sc, R = cal.cased_heap_scenario(cal.HeapParams(**hp))
        ser = H.reference_heap_procedure(sc, R, variant="serial")
        omp = H.reference_heap_procedure(sc, R, variant="omp", threads=4)
        rows.append(dict(params=hp, base_radius=R, time_step=sc.time_step,
                         serial={k: float(v) for k, v in ser.items()}, omp4={k: float(v) for k, v in omp.items()}))
        print(rows[-1], flush=True)
    with open(os.path.join(ROOT, "tests", "golden", "heap_aor.json"), "w") as f:
        json.dump(dict(procedure="Drivers/Calibration/CalibrationHeap.cpp:119-160 on the reference Kernel",
                       scenario="calibration.cased_heap_scenario(HeapParams(**params)) defaults", heaps=rows),
                  f, indent=1)


if __name__ == "__main__":
    main()

"""The reference's own self-test gold files for the time step
(Drivers/SelfTests/Interactions/SelfTestData: ForceSelfTest{0..9}.{data,ene},
ten oblique particle-particle and particle-wall collisions with every law
variant of LinearViscoelasticSlidingFriction; FreeFallSelfTest.{ene,restart},
an elastic sphere bouncing on a wall for 1,000,000 steps), compared with the
reference's fpdiff rule: 0.1 % relative per field, 1e-14 numerical zero (the
gold .ene files predate the interaction-count column the reference's writer
now appends; their eight columns are compared).

* CPU: the self tests compiled from the reference's sources as they are
  (oracle/_ref/selftest_*_reference) reproduce the gold files: the checker
  build is the reference.
* GPU: the same sources with their base class swapped for the engine's
  drop-in base class (oracle/_ref/selftest_*_gpu: DPMBase -> GpuDPMBase,
  Mercury2D -> GpuMercury2D), every time step on the GPU, reproduce the gold
  files; their .data and .restart files come from the reference's own writers
  on the state the binding copies back, their .ene files from the engine's
  balances.
"""
import os

import pytest

import harness as H


def _check(name: str, variant: str, tmp_path):
    exe = H.selftest_executable(name, variant)
    if not os.path.exists(exe):
        pytest.skip(f"{exe} not built (make -f oracle/ref.mk gpu)")
    r = H.run_selftest(name, variant, str(tmp_path))
    assert r["returncode"] == 0, r["log"]
    for f, text in r["files"].items():
        assert text is not None, f"{f} not written"
        # the gold .ene files predate the interaction-count column that the
        # reference's writeEneTimeStep now appends (DPMBase.cc:2121): their
        # eight columns are compared
        bad = H.fpdiff(text, H.selftest_gold(f), skip_first_line=f.endswith(".restart"),
                       fields_of_b=f.endswith(".ene"))
        assert not bad, (f, bad[:5], len(bad))


@pytest.mark.parametrize("name", sorted(H.SELFTESTS))
def test_reference_build_reproduces_gold_files(name, tmp_path):
    _check(name, "reference", tmp_path)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(H.SELFTESTS))
def test_gold_files_through_gpu_base_class(gpu, name, tmp_path):
    _check(name, "gpu", tmp_path)

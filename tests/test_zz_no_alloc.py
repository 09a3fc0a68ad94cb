"""dem_reduce_noalloc: the global balances without any device allocation.

Some callers cannot allocate GPU memory when they ask for the balances (a
coupled solver that reserved the whole device memory budget up front, a
monitoring hook in a host application that forbids allocation between time
steps). For them the entry point keeps its partial sums in a static device
array instead of the temporary buffer dem_reduce allocates.

Checked here, through the C ABI:
* two calls in a row (on a changed state) give exactly dem_reduce's numbers:
  the same partial sums added in the same order;
* a call right after the upload, before any time step, agrees with
  dem_reduce too (no force evaluation yet: no contacts, zero elastic energy);
* the calls allocate nothing: free device memory (cudaMemGetInfo) is the same
  before and after them, and the high-water mark of the device's default
  stream-ordered memory pool, reset before them, does not rise above the
  pool's use when they start;
* a handle of more than 2,097,152 particles is refused with DEM_ERR_CAPACITY
  and a message naming the limit.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test. It passes both alone in a
fresh process and after the other tests (the static array keeps the previous
call's contents, which the entry point never reads before overwriting).
"""
import ctypes as C

import numpy as np
import pytest

import cases
from mercurydpm_fork_b200 import _abi, lib, scenarios

pytestmark = pytest.mark.gpu

FIELDS = ("kinetic_energy", "rotational_energy", "gravitational_energy", "elastic_energy", "mass",
          "time", "n_steps", "n_contacts", "n_wall_contacts")
VECTORS = ("momentum", "angular_momentum", "centre_of_mass")


def _globals(engine, noalloc: bool) -> _abi.Globals:
    g = _abi.Globals()
    fn = lib().dem_reduce_noalloc if noalloc else lib().dem_reduce
    rc = fn(engine._h, 0, C.byref(g))
    assert rc == 0, lib().dem_last_error(engine._h)
    return g


def _assert_identical(a: _abi.Globals, b: _abi.Globals):
    for f in FIELDS:
        assert getattr(a, f) == getattr(b, f), (f, getattr(a, f), getattr(b, f))
    for f in VECTORS:
        assert list(getattr(a, f)) == list(getattr(b, f)), f


class _DeviceMemory:
    """Free device memory and the default memory pool's use, read through the
    CUDA runtime (cuda-python)."""

    def __init__(self, device: int = 0):
        from cuda.bindings import driver, runtime as rt
        self.rt = rt
        self.u64 = driver.cuuint64_t
        err, = rt.cudaSetDevice(device)
        assert err == rt.cudaError_t.cudaSuccess
        err, self.pool = rt.cudaDeviceGetDefaultMemPool(device)
        assert err == rt.cudaError_t.cudaSuccess

    def _attr(self, a):
        err, v = self.rt.cudaMemPoolGetAttribute(self.pool, a)
        assert err == self.rt.cudaError_t.cudaSuccess
        return int(v)

    def reset_high_water(self):
        rt = self.rt
        err, = rt.cudaMemPoolSetAttribute(self.pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                                          self.u64(0))
        assert err == rt.cudaError_t.cudaSuccess

    def used(self) -> int:
        return self._attr(self.rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)

    def used_high(self) -> int:
        return self._attr(self.rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)

    def free(self) -> int:
        err, free, _total = self.rt.cudaMemGetInfo()
        assert err == self.rt.cudaError_t.cudaSuccess
        return int(free)


def test_noalloc_reduce_matches_reduce_twice(gpu):
    sc = cases.compressed_box()
    e = sc.engine()
    try:
        e.step(10)
        first = _globals(e, True)
        _assert_identical(first, _globals(e, False))
        e.step(15)  # a second call in a row, on a changed state
        second = _globals(e, True)
        _assert_identical(second, _globals(e, False))
        assert second.kinetic_energy != first.kinetic_energy
        assert second.n_contacts > 0
    finally:
        e.close()


def test_noalloc_reduce_before_first_step(gpu):
    sc = cases.compressed_box(n=300)
    e = sc.engine()
    try:
        g = _globals(e, True)
        _assert_identical(g, _globals(e, False))
        assert g.n_contacts == 0 and g.elastic_energy == 0.0 and g.kinetic_energy > 0.0
    finally:
        e.close()


def test_noalloc_reduce_allocates_nothing(gpu):
    sc = cases.compressed_box()
    e = sc.engine()
    try:
        e.step(5)
        _globals(e, True)  # first call on this device: looks up the array's address
        mem = _DeviceMemory(0)
        free_before = mem.free()
        used_before = mem.used()
        mem.reset_high_water()
        results = [_globals(e, True) for _ in range(3)]
        assert mem.used_high() <= used_before
        assert mem.free() == free_before
        for r in results[1:]:
            _assert_identical(r, results[0])
    finally:
        e.close()


def test_noalloc_reduce_refuses_more_than_its_array_holds(gpu):
    """2,097,153 spheres on a sparse lattice (no contacts): the handle is
    uploaded, and the no-alloc reduction refuses it before launching
    anything; the handle stays usable for dem_reduce."""
    n = 2_097_153
    sc = scenarios.settling_box(n=n, seed=1, box=(150, 150, 150), spacing=1.1, jitter=0.0, vstd=0.0)
    e = sc.engine()
    try:
        g = _abi.Globals()
        rc = lib().dem_reduce_noalloc(e._h, 0, C.byref(g))
        assert rc == _abi.DEM_ERR_CAPACITY
        assert b"2,097,152" in lib().dem_last_error(e._h)
        ref = e.reduce()
        assert ref["mass"] > 0.0 and np.isfinite(ref["kinetic_energy"])
    finally:
        e.close()

"""dem_reduce_noalloc: the global balances without any device allocation.

Some callers cannot allocate GPU memory when they ask for the balances (a
coupled solver that reserved the whole device memory budget up front, a
monitoring hook in a host application that forbids allocation between time
steps). For them the entry point keeps its partial sums in a static device
array instead of the temporary buffer dem_reduce allocates.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test. It passes both alone in a
fresh process and after the other tests (the static array keeps the previous
call's contents, which the entry point never reads before overwriting).
"""
import ctypes as C

import pytest

import cases
from mercurydpm_fork_b200 import _abi, lib

pytestmark = pytest.mark.gpu

FIELDS = ("kinetic_energy", "rotational_energy", "gravitational_energy", "elastic_energy", "mass")


def _globals(engine, noalloc: bool) -> _abi.Globals:
    g = _abi.Globals()
    fn = lib().dem_reduce_noalloc if noalloc else lib().dem_reduce
    rc = fn(engine._h, 0, C.byref(g))
    assert rc == 0, lib().dem_last_error(engine._h)
    return g


def _compare(a: _abi.Globals, b: _abi.Globals):
    for f in FIELDS:
        x, y = getattr(a, f), getattr(b, f)
        assert abs(x - y) <= 1e-12 * max(abs(y), 1e-300), (f, x, y)
    for k in range(3):
        for f in ("momentum", "angular_momentum", "centre_of_mass"):
            x, y = getattr(a, f)[k], getattr(b, f)[k]
            assert abs(x - y) <= 1e-12 * max(abs(y), 1e-30), (f, k, x, y)
    assert a.n_contacts == b.n_contacts
    assert a.n_wall_contacts == b.n_wall_contacts


def test_noalloc_reduce_matches_reduce_twice(gpu):
    sc = cases.compressed_box()
    e = sc.engine()
    try:
        e.step(10)
        first = _globals(e, True)
        _compare(first, _globals(e, False))
        e.step(15)  # a second call in a row, on a changed state
        second = _globals(e, True)
        _compare(second, _globals(e, False))
        assert second.kinetic_energy != first.kinetic_energy
    finally:
        e.close()

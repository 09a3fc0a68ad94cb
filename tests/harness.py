"""Test harness: runs one Scenario through the CPU oracle (oracle/), the
reference build (oracle/_ref) and the GPU engine, returning comparable dicts.

Only tests import this module; the oracle and the reference are checkers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from mercurydpm_fork_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "libdem_oracle.so")
REF_LIBS = {v: os.path.join(ROOT, "oracle", "_ref", f"libmdpm_ref_{v}.so") for v in ("serial", "omp")}

_pd = C.POINTER(C.c_double)
_pi = C.POINTER(C.c_int32)
_oracle = None
_ref = {}


def _dp(a):
    return None if a is None else a.ctypes.data_as(_pd)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_pi)


def oracle_lib():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_LIB):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True, capture_output=True)
        lib = C.CDLL(ORACLE_LIB)
        lib.oracle_run.restype = C.c_int
        lib.oracle_run.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair),
                                   C.c_int, C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA),
                                   C.POINTER(_abi.ContactsSoA), C.c_int, C.POINTER(_abi.ParticlesSoA), _pd, _pd,
                                   C.POINTER(_abi.ContactsSoA), C.c_int64, C.POINTER(C.c_int64)]
        lib.oracle_set_contact_report.restype = None
        lib.oracle_set_contact_report.argtypes = [C.c_int]
        lib.oracle_set_deletion.restype = None
        lib.oracle_set_deletion.argtypes = [C.POINTER(_abi.DeletionBoundary), C.c_int]
        lib.oracle_set_insertion.restype = None
        lib.oracle_set_insertion.argtypes = [C.POINTER(_abi.InsertionBoundary), C.c_int, C.c_ulonglong]
        lib.oracle_set_chute_fill.restype = None
        lib.oracle_set_chute_fill.argtypes = [C.POINTER(_abi.ChuteFill), C.c_int, C.c_ulonglong]
        lib.oracle_chute_fill_height.restype = C.c_double
        lib.oracle_chute_fill_height.argtypes = []
        lib.oracle_insertion_counts.restype = C.c_int
        lib.oracle_insertion_counts.argtypes = [C.POINTER(C.c_longlong), _pd, C.c_int]
        _oracle = lib
    return _oracle


def reference_available(variant="serial") -> bool:
    return os.path.exists(REF_LIBS[variant])


def ref_lib(variant="serial"):
    if variant not in _ref:
        lib = C.CDLL(REF_LIBS[variant])
        common = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                  C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA)]
        lib.mdpm_ref_run.restype = C.c_int
        lib.mdpm_ref_run.argtypes = common + [C.c_int, C.POINTER(_abi.ParticlesSoA), _pd, _pd,
                                              C.POINTER(_abi.ContactsSoA), C.c_int64, C.POINTER(C.c_int64), _pd]
        lib.mdpm_ref_time.restype = C.c_int
        lib.mdpm_ref_time.argtypes = common + [C.c_int, C.c_int, C.c_int, _pd]
        lib.mdpm_ref_set_deletion.restype = None
        lib.mdpm_ref_set_deletion.argtypes = [C.POINTER(_abi.DeletionBoundary), C.c_int]
        lib.mdpm_ref_set_event.restype = None
        lib.mdpm_ref_set_event.argtypes = [C.c_longlong, C.c_int, C.POINTER(_abi.DeletionBoundary), C.c_int]
        lib.mdpm_ref_set_insertion.restype = None
        lib.mdpm_ref_set_insertion.argtypes = [C.POINTER(_abi.InsertionBoundary), C.c_int, C.c_ulonglong]
        lib.mdpm_ref_insertion_counts.restype = C.c_int
        lib.mdpm_ref_insertion_counts.argtypes = [C.POINTER(C.c_longlong), _pd, C.c_int]
        lib.mdpm_ref_rng_draws.restype = None
        lib.mdpm_ref_rng_draws.argtypes = [C.c_ulonglong, C.c_int, _pd]
        lib.mdpm_ref_run_chute_fill.restype = C.c_int
        lib.mdpm_ref_run_chute_fill.argtypes = common + [C.POINTER(_abi.ChuteFill), C.c_ulonglong, C.c_int,
                                                        C.POINTER(_abi.ParticlesSoA), _pd, _pd,
                                                        C.POINTER(_abi.ContactsSoA), C.c_int64, C.POINTER(C.c_int64),
                                                        _pd]
        lib.mdpm_ref_psd_draws.restype = None
        lib.mdpm_ref_psd_draws.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, _pd]
        _ref[variant] = lib
    return _ref[variant]


class _Inputs:
    """Keeps the ctypes views of a Scenario alive."""

    def __init__(self, sc, contacts=None):
        n = sc.n
        self.pos = np.ascontiguousarray(sc.position, np.float64)
        self.vel = np.ascontiguousarray(sc.velocity, np.float64)
        self.rad = np.ascontiguousarray(sc.radius, np.float64)
        self.im = np.ascontiguousarray(sc.inv_mass, np.float64)
        self.ii = np.ascontiguousarray(sc.inv_inertia, np.float64)
        self.sp = np.ascontiguousarray(sc.species_index, np.int32)
        self.ids = np.ascontiguousarray(sc.ids, np.int32)
        w = getattr(sc, "angular_velocity", None)
        q = getattr(sc, "orientation", None)
        self.ang = None if w is None else np.ascontiguousarray(w, np.float64)
        self.ori = None if q is None else np.ascontiguousarray(q, np.float64)
        self.soa = _abi.ParticlesSoA(n, _dp(self.pos), _dp(self.vel), _dp(self.ang), _dp(self.ori), _dp(self.rad),
                                     _dp(self.im), _dp(self.ii), _ip(self.sp), _ip(self.ids), None)
        self.cfg = sc.config()
        self.inst = sc.instance.to_c()
        self.species = (_abi.SpeciesPair * len(sc.species))(*sc.species)
        self.walls = (_abi.Wall * max(1, len(sc.walls)))(*sc.walls)
        self.nwalls = len(sc.walls)
        self.density = np.ascontiguousarray(sc.density, np.float64)
        self.contacts_in = None
        if contacts is not None:
            m = len(contacts["id_p"])
            self._c = {k: np.ascontiguousarray(v) for k, v in contacts.items()}
            self.contacts_in = _abi.ContactsSoA(m, _ip(self._c["id_p"].astype(np.int32)), None, None, None, None,
                                                None, None)
            self._cid = [self._c["id_p"].astype(np.int32), self._c["id_i"].astype(np.int32),
                         self._c.get("is_wall", np.zeros(m)).astype(np.int32),
                         self._c.get("periodic", np.zeros(m)).astype(np.int32),
                         np.ascontiguousarray(self._c["springs"], np.float64)]
            self.contacts_in = _abi.ContactsSoA(m, _ip(self._cid[0]), _ip(self._cid[1]), _ip(self._cid[2]),
                                                _ip(self._cid[3]), _dp(self._cid[4]), None, None)


def _deletions(planes):
    """ctypes array of DeletionBoundary from [(normal, distance), ...]."""
    from mercurydpm_fork_b200.engine import deletion_boundary
    planes = planes or []
    arr = (_abi.DeletionBoundary * max(1, len(planes)))(*[deletion_boundary(nn, dd) for nn, dd in planes])
    return arr, len(planes)


def _outputs(n, cap):
    o = dict(position=np.zeros((n, 3)), velocity=np.zeros((n, 3)), angular_velocity=np.zeros((n, 3)),
             orientation=np.zeros((n, 4)), radius=np.zeros(n), inv_mass=np.zeros(n), inv_inertia=np.zeros(n),
             force=np.zeros((n, 3)), torque=np.zeros((n, 3)), instance=np.zeros(n, np.int32))
    c = dict(id_p=np.zeros(cap, np.int32), id_i=np.zeros(cap, np.int32), is_wall=np.zeros(cap, np.int32),
             periodic=np.zeros(cap, np.int32), springs=np.zeros((cap, 9)), force=np.zeros((cap, 3)),
             overlap=np.zeros(cap))
    soa = _abi.ParticlesSoA(n, _dp(o["position"]), _dp(o["velocity"]), _dp(o["angular_velocity"]),
                            _dp(o["orientation"]), _dp(o["radius"]), _dp(o["inv_mass"]), _dp(o["inv_inertia"]), None, None,
                            _ip(o["instance"]))
    csoa = _abi.ContactsSoA(cap, _ip(c["id_p"]), _ip(c["id_i"]), _ip(c["is_wall"]), _ip(c["periodic"]),
                            _dp(c["springs"]), _dp(c["force"]), _dp(c["overlap"]))
    return o, c, soa, csoa


def _trim(c, m):
    assert m <= len(c["id_p"]), f"{m} contacts exceed the {len(c['id_p'])} rows allocated"
    return {k: v[:m] for k, v in c.items()}


def _contact_rows(n: int) -> int:
    """Contact rows allocated for a run of n particles: 16 per particle for
    small cases (dense packings of several sizes), 4 per particle above
    100,000 (the large workloads have under 2 contacts per particle)."""
    return 16 * n + 64 if n <= 100_000 else 4 * n + 4096


def sort_contacts(c):
    order = np.lexsort((c["id_i"], c["id_p"], c["is_wall"]))
    return {k: v[order] for k, v in c.items()}


def run_oracle(sc, nsteps: int, contacts=None, report: str = "evaluated", deletions=None, insertions=None,
               seed: int = 0, chute_fill=None) -> dict:
    """report="evaluated": contacts of the last force evaluation (what the
    engine records); "handler": every interaction the reference still holds.
    deletions: DeletionBoundary planes [(normal, distance), ...]; the output
    "instance" is -1 for deleted particles."""
    oracle_lib().oracle_set_contact_report(1 if report == "handler" else 0)
    darr, nd = _deletions(deletions)
    oracle_lib().oracle_set_deletion(darr, nd)
    iarr, ni = _insertions(insertions)
    oracle_lib().oracle_set_insertion(iarr, ni, seed)
    oracle_lib().oracle_set_chute_fill(C.byref(chute_fill) if chute_fill is not None else None,
                                       1 if chute_fill is not None else 0, seed)
    inp = _Inputs(sc, contacts)
    cap = _contact_rows(sc.n)
    o, c, soa, csoa = _outputs(sc.n, cap)
    cnt = C.c_int64(0)
    rc = oracle_lib().oracle_run(C.byref(inp.cfg), C.byref(inp.inst), inp.species, len(sc.species), inp.walls,
                                 inp.nwalls, C.byref(inp.soa), C.byref(inp.contacts_in) if inp.contacts_in else None,
                                 nsteps, C.byref(soa), _dp(o["force"]), _dp(o["torque"]), C.byref(csoa), cap,
                                 C.byref(cnt))
    oracle_lib().oracle_set_insertion(iarr, 0, 0)
    oracle_lib().oracle_set_chute_fill(None, 0, 0)
    assert rc == 0
    if chute_fill is not None:
        o["inflow_height"] = float(oracle_lib().oracle_chute_fill_height())
    o["contacts"] = sort_contacts(_trim(c, cnt.value))
    if ni:
        k = np.zeros(ni, np.int64)
        v = np.zeros(ni)
        m = oracle_lib().oracle_insertion_counts(k.ctypes.data_as(C.POINTER(C.c_longlong)), _dp(v), ni)
        assert m == ni
        o["inserted"], o["inserted_volume"] = k, v
    return o


def _insertions(insertions):
    ins = list(insertions or [])
    return (_abi.InsertionBoundary * max(1, len(ins)))(*ins), len(ins)


def run_reference(sc, nsteps: int, variant: str = "serial", deletions=None, event=None, insertions=None,
                  seed: int = 0) -> dict:
    """event = (step, wall, planes): after time step `step` the reference's
    driver removes wall `wall` (handler index, -1: none) and adds the
    DeletionBoundary planes [(normal, distance), ...]. insertions:
    dem_insertion_boundary structures made CubeInsertionBoundary objects, with
    DPMBase::random seeded by `seed`; rows of radius 0 are left out (the
    engine's free rows) and the output "inserted" / "inserted_volume" are the
    boundaries' counters."""
    darr, nd = _deletions(deletions)
    ref_lib(variant).mdpm_ref_set_deletion(darr, nd)
    iarr, ni = _insertions(insertions)
    ref_lib(variant).mdpm_ref_set_insertion(iarr, ni, seed)
    step, wall, planes = event if event is not None else (-1, -1, [])
    earr, ne = _deletions(planes)
    ref_lib(variant).mdpm_ref_set_event(step, wall, earr, ne)
    inp = _Inputs(sc)
    cap = _contact_rows(sc.n)
    o, c, soa, csoa = _outputs(sc.n, cap)
    cnt = C.c_int64(0)
    ene = np.zeros(4)
    rc = ref_lib(variant).mdpm_ref_run(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls,
                                       inp.nwalls, C.byref(inp.soa), nsteps, C.byref(soa), _dp(o["force"]),
                                       _dp(o["torque"]), C.byref(csoa), cap, C.byref(cnt), _dp(ene))
    ref_lib(variant).mdpm_ref_set_insertion(iarr, 0, 0)
    assert rc == 0
    o["contacts"] = sort_contacts(_trim(c, cnt.value))
    o["energies"] = dict(kinetic=ene[0], rotational=ene[1], gravitational=ene[2], elastic=ene[3])
    if ni:
        k = np.zeros(ni, np.int64)
        v = np.zeros(ni)
        m = ref_lib(variant).mdpm_ref_insertion_counts(k.ctypes.data_as(C.POINTER(C.c_longlong)), _dp(v), ni)
        assert m == ni
        o["inserted"], o["inserted_volume"] = k, v
    return o


def run_reference_chute_fill(sc, fill, seed: int, nsteps: int, variant: str = "serial") -> dict:
    """The scenario on a reference Chute whose set-up ends with
    Chute::addFlowParticlesCompactly (`fill`, DPMBase::random seeded with
    `seed`); rows of radius 0 receive the placed particles in id order.
    Adds "inflow_height", the height the fill ended with."""
    inp = _Inputs(sc)
    cap = _contact_rows(sc.n)
    o, c, soa, csoa = _outputs(sc.n, cap)
    cnt = C.c_int64(0)
    hgt = np.zeros(1)
    with quiet_stdout():
        rc = ref_lib(variant).mdpm_ref_run_chute_fill(
            C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
            C.byref(inp.soa), C.byref(fill), seed, nsteps, C.byref(soa), _dp(o["force"]), _dp(o["torque"]),
            C.byref(csoa), cap, C.byref(cnt), _dp(hgt))
    assert rc == 0
    o["contacts"] = sort_contacts(_trim(c, cnt.value))
    o["inflow_height"] = float(hgt[0])
    return o


def reference_rng_draws(seed: int, n: int, variant: str = "serial") -> np.ndarray:
    """RNG::getRandomNumber(0, 1) after RNG::setRandomSeed(seed), from the reference build."""
    out = np.zeros(n)
    ref_lib(variant).mdpm_ref_rng_draws(seed, n, _dp(out))
    return out


def reference_psd_draws(rmin: float, rmax: float, bins: int, seed: int, n: int, variant: str = "serial"):
    """PSD::drawSample after setDistributionUniform(rmin, rmax, bins) and setFixedSeed(seed)."""
    out = np.zeros(n)
    ref_lib(variant).mdpm_ref_psd_draws(rmin, rmax, bins, seed, n, _dp(out))
    return out


def reference_heap_procedure(sc, base_radius: float, casing: int = 1, check_every: int = 1000,
                             max_steps: int = 400_000, variant: str = "serial", threads: int = 1) -> dict:
    """Drivers/Calibration/CalibrationHeap.cpp's procedure on the reference
    Kernel (oracle/ref_drivers/mdpm_ref_driver.cpp, mdpm_ref_heap_procedure)
    for the heap set up by `sc` (casing = the casing's wall index)."""
    darr, nd = _deletions(None)
    lib = ref_lib(variant)
    lib.mdpm_ref_set_deletion(darr, nd)
    lib.mdpm_ref_set_event(-1, -1, darr, 0)
    fn = lib.mdpm_ref_heap_procedure
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                   C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int, C.c_double, C.c_int,
                   C.c_longlong, C.c_int, _pd]
    inp = _Inputs(sc)
    out = np.zeros(6)
    rc = fn(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
            C.byref(inp.soa), casing, base_radius, check_every, max_steps, threads, _dp(out))
    assert rc == 0
    return dict(aor=out[0], removal_time=out[1], end_time=out[2], steps=int(out[3]), n_remaining=int(out[4]),
                com_z=out[5])


def reference_outputs(sc, nsteps: int, prefix: str, variant: str = "serial"):
    """The reference writes its own prefix.ene / .fstat / .data after nsteps."""
    darr, nd = _deletions(None)
    lib = ref_lib(variant)
    lib.mdpm_ref_set_deletion(darr, nd)
    inp = _Inputs(sc)
    fn = lib.mdpm_ref_write_outputs
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                   C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int, C.c_char_p]
    rc = fn(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
            C.byref(inp.soa), nsteps, prefix.encode())
    assert rc == 0


def cg_grid(coordinates: int, n, lo, hi, width: float, cutoff_factor: float = 3.0) -> _abi.CGGrid:
    g = _abi.CGGrid()
    g.coordinates = coordinates
    g.n[:] = list(map(int, n))
    g.min[:] = list(map(float, lo))
    g.max[:] = list(map(float, hi))
    g.width = width
    g.cutoff_factor = cutoff_factor
    return g


def reference_cg(sc, nsteps: int, grid: _abi.CGGrid, variant: str = "serial") -> np.ndarray:
    """The reference's CG<Coordinates, Gauss, StandardFields> after nsteps steps (29 fields per point)."""
    darr, nd = _deletions(None)
    ref_lib(variant).mdpm_ref_set_deletion(darr, nd)
    inp = _Inputs(sc)
    npts = 1
    for k, res in enumerate((grid.coordinates != _abi.DEM_CG_O, grid.coordinates == _abi.DEM_CG_XYZ,
                             grid.coordinates != _abi.DEM_CG_O)):
        npts *= grid.n[k] if res else 1
    out = np.zeros((npts, _abi.DEM_CG_NFIELDS))
    lib = ref_lib(variant)
    fn = lib.mdpm_ref_cg
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                   C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int, C.POINTER(_abi.CGGrid), _pd]
    rc = fn(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
            C.byref(inp.soa), nsteps, C.byref(grid), _dp(out))
    assert rc == 0
    return out


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null while the reference runs (its
    logger prints thread and time-step lines to stdout)."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def reference_ene(sc, nsteps: int, save_count: int, prefix: str, variant: str = "serial", threads: int = 1):
    """The reference's DPMBase::solve() over nsteps time steps with its own
    .ene writer (a line every save_count steps and one at the end); returns
    the parsed rows (time, gravitational, kinetic, rotational, elastic
    energy, centre of mass x y z, interactions), one per distinct time."""
    darr, nd = _deletions(None)
    lib = ref_lib(variant)
    lib.mdpm_ref_set_deletion(darr, nd)
    fn = lib.mdpm_ref_solve_ene
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                   C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int, C.c_int, C.c_int, C.c_char_p]
    inp = _Inputs(sc)
    with quiet_stdout():
        rc = fn(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
                C.byref(inp.soa), nsteps, save_count, threads, prefix.encode())
    assert rc == 0
    return parse_ene(open(prefix + ".ene").read())


def parse_ene(text: str) -> np.ndarray:
    """Rows of a .ene file (header lines skipped, repeated times dropped)."""
    rows, seen = [], set()
    for ln in text.splitlines():
        parts = ln.split()
        try:
            vals = [float(x) for x in parts]
        except ValueError:
            continue
        if len(vals) != 9 or vals[0] in seen:
            continue
        seen.add(vals[0])
        rows.append(vals)
    return np.array(rows)


def time_reference(sc, warmup: int, nsteps: int, threads: int, variant: str = "omp") -> float:
    return time_reference_window(sc, warmup, nsteps, threads, variant)["seconds"]


def time_reference_window(sc, warmup: int, nsteps: int, threads: int, variant: str = "omp") -> dict:
    """The reference's wall time of time steps warmup+1 .. warmup+nsteps
    (std::chrono around computeOneTimeStep, set-up excluded) and the number
    of interactions its handler holds at the start and end of that window."""
    darr, nd = _deletions(None)
    lib = ref_lib(variant)
    lib.mdpm_ref_set_deletion(darr, nd)
    fn = lib.mdpm_ref_time_window
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                   C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int, C.c_int, C.c_int, _pd,
                   C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    inp = _Inputs(sc)
    sec = C.c_double(0)
    a, b = C.c_int64(0), C.c_int64(0)
    with quiet_stdout():
        rc = fn(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
                C.byref(inp.soa), warmup, nsteps, threads, C.byref(sec), C.byref(a), C.byref(b))
    assert rc == 0
    return dict(seconds=sec.value, interactions_start=a.value, interactions_end=b.value)


def run_gpu(sc, nsteps: int, contacts=None, deletions=None, event=None, insertions=None, seed: int = 0,
            chute_fill=None, **kw) -> dict:
    """event: as in run_reference, made between two dem_step calls.
    insertions / seed: as in run_reference (the engine fills the rows of radius 0)."""
    from mercurydpm_fork_b200.engine import deletion_boundary
    if deletions:
        kw["deletions"] = [deletion_boundary(nn, dd) for nn, dd in deletions]
    if insertions:
        kw["insertions"] = list(insertions)
    if insertions or chute_fill is not None:
        kw["insertion_seeds"] = [seed]
    if chute_fill is not None:
        kw["chute_fills"] = [chute_fill]
    e = sc.engine(**kw)
    if contacts is not None:
        e.upload_contacts(contacts["id_p"], contacts["id_i"], contacts["springs"], contacts.get("is_wall"),
                          contacts.get("periodic"))
    if event is not None and 0 <= event[0] < nsteps:
        step, wall, planes = event
        e.step(step)
        if wall >= 0:
            e.remove_wall(wall)
        e.set_deletion_boundaries([deletion_boundary(nn, dd) for nn, dd in list(deletions or []) + list(planes)])
        e.step(nsteps - step)
    else:
        e.step(nsteps)
    out = e.download()
    out["force"], out["torque"] = e.forces()
    out["contacts"] = sort_contacts(e.contacts())
    out["globals"] = e.reduce()
    out["stats"] = e.stats()
    if insertions:
        out["inserted"], out["inserted_volume"] = e.insertion_counts()
    if chute_fill is not None:
        hh, kk = e.chute_fill_results()
        out["inflow_height"], out["filled"] = float(hh[0]), int(kk[0])
    e.close()
    return out


def pair_set(c) -> set:
    return {(int(a), int(b), int(w)) for a, b, w in zip(c["id_p"], c["id_i"], c["is_wall"])}


def rel_err(a, b, scale=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.size == 0 and b.size == 0:
        return 0.0
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def engine_ene(sc, steps: int, save: int, **engine_kw) -> np.ndarray:
    """The .ene lines of the engine's run driven from Python (output.ene_line
    from dem_reduce after dem_step(0) and every `save` further steps, 10
    significant digits like the reference's file), parsed back."""
    from mercurydpm_fork_b200 import output
    e = sc.engine(**engine_kw)
    try:
        text = output.ene_header()
        e.step(0)
        for k in range(steps // save + 1):
            if k:
                e.step(save)
            g = e.reduce()
            text += output.ene_line(output.time_after(k * save, sc.time_step), sc.instance.gravity, g,
                                    g["n_contacts"] + g["n_wall_contacts"])
    finally:
        e.close()
    return parse_ene(text)


def check_ene_against_golden(ours: np.ndarray, gold: dict):
    """The settling box's .ene rows against the reference's (the fixture
    tests/golden/settling_box_ene.json): while the reference's serial and
    OpenMP builds still write identical lines, 1e-8 relative per column and
    the exact interaction count; over the whole run, at most 3x the largest
    difference between the reference's two builds in that column plus 1e-9 of
    the column's magnitude."""
    serial, omp = np.array(gold["serial"]), np.array(gold["omp8"])
    assert ours.shape == serial.shape
    np.testing.assert_array_equal(ours[:, 0], serial[:, 0])
    agree = np.all(serial == omp, axis=1)
    n_same = int(np.argmin(agree)) if not agree.all() else len(agree)
    assert n_same >= 10
    for col in range(1, 8):
        scale = np.abs(serial[:n_same, col]).max()
        err = np.abs(ours[:n_same, col] - serial[:n_same, col]).max()
        assert err <= 1e-8 * max(scale, 1e-300), (gold["columns"][col], err, scale)
    np.testing.assert_array_equal(ours[:n_same, 8], serial[:n_same, 8])
    for col in range(1, 9):
        mag = np.abs(serial[:, col]).max()
        envelope = np.abs(serial[:, col] - omp[:, col]).max()
        err = np.abs(ours[:, col] - serial[:, col]).max()
        assert err <= 3.0 * envelope + 1e-9 * mag, (gold["columns"][col], err, envelope)


GPU_BINDING_LIB = os.path.join(ROOT, "oracle", "_ref", "libmdpm_gpu_binding.so")
GPU_UNIT_TEST = os.path.join(ROOT, "oracle", "_ref", "gpu_tangential_spring_unit_test")


def gpu_binding_available() -> bool:
    return os.path.exists(GPU_BINDING_LIB) and os.path.exists(GPU_UNIT_TEST)


def _gpu_binding():
    lib = C.CDLL(GPU_BINDING_LIB)
    common = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
              C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int]
    lib.mdpm_gpu_solve_ene.restype = C.c_int
    lib.mdpm_gpu_solve_ene.argtypes = common + [C.c_int, C.c_int, C.c_int, C.c_char_p]
    lib.mdpm_gpu_solve_state.restype = C.c_int
    lib.mdpm_gpu_solve_state.argtypes = common + [C.c_int, C.c_int, C.POINTER(_abi.ParticlesSoA), _pd]
    return lib


def gpu_binding_ene(sc, nsteps: int, save_count: int, prefix: str, device: int = 0, sync_interval: int = 1):
    """DPMBase::solve() of the checker's Mercury3D driver on the engine's
    drop-in base class (GpuMercury3D), with the reference's .ene writer."""
    inp = _Inputs(sc)
    with quiet_stdout():
        rc = _gpu_binding().mdpm_gpu_solve_ene(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density),
                                               inp.walls, inp.nwalls, C.byref(inp.soa), nsteps, save_count, device,
                                               sync_interval, prefix.encode())
    assert rc == 0
    return parse_ene(open(prefix + ".ene").read())


def gpu_binding_state(sc, nsteps: int, device: int = 0, sync_interval: int = 1, event=None) -> dict:
    """The host's particle state after DPMBase::solve() on GpuMercury3D
    (instance -1: the particle left the handler). event: as in
    run_reference, made by the driver's actionsAfterTimeStep."""
    inp = _Inputs(sc)
    n = sc.n
    o = dict(position=np.zeros((n, 3)), velocity=np.zeros((n, 3)), angular_velocity=np.zeros((n, 3)),
             instance=np.zeros(n, np.int32))
    soa = _abi.ParticlesSoA(n, _dp(o["position"]), _dp(o["velocity"]), _dp(o["angular_velocity"]), None, None,
                            None, None, None, None, o["instance"].ctypes.data_as(C.POINTER(C.c_int32)))
    step, wall, planes = event if event is not None else (-1, -1, [])
    earr, ne = _deletions(planes)
    lib = _gpu_binding()
    lib.mdpm_gpu_set_event.restype = None
    lib.mdpm_gpu_set_event.argtypes = [C.c_longlong, C.c_int, C.POINTER(_abi.DeletionBoundary), C.c_int]
    lib.mdpm_gpu_set_event(step, wall, earr, ne)
    host = np.zeros(2)
    with quiet_stdout():
        rc = _gpu_binding().mdpm_gpu_solve_state(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density),
                                                 inp.walls, inp.nwalls, C.byref(inp.soa), nsteps, device,
                                                 sync_interval, C.byref(soa), _dp(host))
    assert rc == 0
    o["host_elastic_energy"], o["host_interactions"] = float(host[0]), int(host[1])
    return o


def fpdiff(text_a: str, text_b: str, relative_error: float = 0.1, small: float = 1e-14,
           skip_first_line: bool = False, fields_of_b: bool = False) -> list:
    """The self-test comparison rule of the reference's Configuration/fpdiff.py,
    restated: the files must have the same lines and fields; identical fields
    pass; otherwise both must be numbers, and pass if both magnitudes are at
    most `small` or their difference is at most `relative_error` PERCENT of the
    larger magnitude (.restart files: the first line, name and revision, is
    not compared). fields_of_b: a line of text_a may carry more fields than
    the line of text_b, and only text_b's are compared. Returns the mismatches
    (line, field, a, b); empty = pass."""
    import re
    number = re.compile(r"(^[+-]?[0-9]*[.]?[0-9]+$)|(^[+-]?[0-9]+[.]?[0-9]*$)|(^[+-]?[0-9]?[.]?[0-9]+[EeDd][+-][0-9]+$)")
    la, lb = text_a.splitlines(), text_b.splitlines()
    if skip_first_line:
        la, lb = la[1:], lb[1:]
    bad = []
    if len(la) != len(lb):
        return [("lines", len(la), len(lb), None)]
    for i, (a, b) in enumerate(zip(la, lb)):
        fa, fb = a.split(), b.split()
        if fields_of_b and len(fa) > len(fb):
            fa = fa[:len(fb)]
        if len(fa) != len(fb):
            bad.append((i, "fields", len(fa), len(fb)))
            continue
        for j, (x, y) in enumerate(zip(fa, fb)):
            if x == y:
                continue
            if not (number.match(x) and number.match(y)):
                bad.append((i, j, x, y))
                continue
            u, v = float(x.lower().replace("d", "e")), float(y.lower().replace("d", "e"))
            if abs(u) <= small and abs(v) <= small:
                continue
            if 100.0 * abs(u - v) / max(abs(u), abs(v)) > relative_error:
                bad.append((i, j, x, y))
    return bad


SELFTEST_GOLD = os.path.join(ROOT, "tests", "golden", "selftest")
# self test -> the output files its gold data covers
SELFTESTS = {
    "ForceSelfTest": [f"ForceSelfTest{k}.{ext}" for k in range(10) for ext in ("data", "ene")],
    "FreeFallSelfTest": ["FreeFallSelfTest.ene", "FreeFallSelfTest.restart"],
}


def selftest_executable(name: str, variant: str) -> str:
    """oracle/_ref/selftest_<name>_<variant>: variant "reference" is the
    reference's self-test source as it is, "gpu" the same source on the
    engine's drop-in base class."""
    return os.path.join(ROOT, "oracle", "_ref", f"selftest_{name}_{variant}")


def run_selftest(name: str, variant: str, workdir: str, timeout: float = 1800) -> dict:
    """Runs a self-test executable in workdir; returns its output files'
    texts (the ones the gold data covers) and its exit status."""
    r = subprocess.run([selftest_executable(name, variant)], cwd=workdir, capture_output=True, text=True,
                       timeout=timeout)
    files = {}
    for f in SELFTESTS[name]:
        p = os.path.join(workdir, f)
        files[f] = open(p).read() if os.path.exists(p) else None
    return dict(returncode=r.returncode, log=r.stdout[-3000:] + r.stderr[-3000:], files=files)


def selftest_gold(filename: str) -> str:
    import gzip
    with gzip.open(os.path.join(SELFTEST_GOLD, filename + ".gz"), "rt") as f:
        return f.read()


def reference_restart(sc, nsteps: int, path: str) -> str:
    """The reference's restart file (DPMBase::write, 15 digits) after nsteps
    time steps of the scenario; returns its text."""
    darr, nd = _deletions(None)
    lib = ref_lib("serial")
    lib.mdpm_ref_set_deletion(darr, nd)
    fn = lib.mdpm_ref_write_restart
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_abi.Config), C.POINTER(_abi.InstanceDesc), C.POINTER(_abi.SpeciesPair), _pd,
                   C.POINTER(_abi.Wall), C.c_int, C.POINTER(_abi.ParticlesSoA), C.c_int, C.c_char_p]
    inp = _Inputs(sc)
    with quiet_stdout():
        rc = fn(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls, inp.nwalls,
                C.byref(inp.soa), nsteps, path.encode())
    assert rc == 0
    return open(path).read()


def reference_restart_run(path: str, nsteps: int, n: int) -> dict:
    """The reference restarted from `path` (its own reader) and advanced
    nsteps time steps: state, forces and the last evaluation's contacts."""
    lib = ref_lib("serial")
    fn = lib.mdpm_ref_restart_run
    fn.restype = C.c_int
    fn.argtypes = [C.c_char_p, C.c_int, C.c_int64, C.POINTER(_abi.ParticlesSoA), _pd, _pd,
                   C.POINTER(_abi.ContactsSoA), C.c_int64, C.POINTER(C.c_int64)]
    cap = _contact_rows(n)
    o, c, soa, csoa = _outputs(n, cap)
    cnt = C.c_int64(0)
    with quiet_stdout():
        rc = fn(path.encode(), nsteps, n, C.byref(soa), _dp(o["force"]), _dp(o["torque"]), C.byref(csoa), cap,
                C.byref(cnt))
    assert rc == 0
    o["contacts"] = sort_contacts(_trim(c, cnt.value))
    return o

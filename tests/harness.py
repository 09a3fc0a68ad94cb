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
        self.soa = _abi.ParticlesSoA(n, _dp(self.pos), _dp(self.vel), None, None, _dp(self.rad), _dp(self.im),
                                     _dp(self.ii), _ip(self.sp), _ip(self.ids), None)
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
             orientation=np.zeros((n, 4)), inv_mass=np.zeros(n), inv_inertia=np.zeros(n),
             force=np.zeros((n, 3)), torque=np.zeros((n, 3)), instance=np.zeros(n, np.int32))
    c = dict(id_p=np.zeros(cap, np.int32), id_i=np.zeros(cap, np.int32), is_wall=np.zeros(cap, np.int32),
             periodic=np.zeros(cap, np.int32), springs=np.zeros((cap, 9)), force=np.zeros((cap, 3)),
             overlap=np.zeros(cap))
    soa = _abi.ParticlesSoA(n, _dp(o["position"]), _dp(o["velocity"]), _dp(o["angular_velocity"]),
                            _dp(o["orientation"]), None, _dp(o["inv_mass"]), _dp(o["inv_inertia"]), None, None,
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


def run_oracle(sc, nsteps: int, contacts=None, report: str = "evaluated", deletions=None) -> dict:
    """report="evaluated": contacts of the last force evaluation (what the
    engine records); "handler": every interaction the reference still holds.
    deletions: DeletionBoundary planes [(normal, distance), ...]; the output
    "instance" is -1 for deleted particles."""
    oracle_lib().oracle_set_contact_report(1 if report == "handler" else 0)
    darr, nd = _deletions(deletions)
    oracle_lib().oracle_set_deletion(darr, nd)
    inp = _Inputs(sc, contacts)
    cap = _contact_rows(sc.n)
    o, c, soa, csoa = _outputs(sc.n, cap)
    cnt = C.c_int64(0)
    rc = oracle_lib().oracle_run(C.byref(inp.cfg), C.byref(inp.inst), inp.species, len(sc.species), inp.walls,
                                 inp.nwalls, C.byref(inp.soa), C.byref(inp.contacts_in) if inp.contacts_in else None,
                                 nsteps, C.byref(soa), _dp(o["force"]), _dp(o["torque"]), C.byref(csoa), cap,
                                 C.byref(cnt))
    assert rc == 0
    o["contacts"] = sort_contacts(_trim(c, cnt.value))
    return o


def run_reference(sc, nsteps: int, variant: str = "serial", deletions=None) -> dict:
    darr, nd = _deletions(deletions)
    ref_lib(variant).mdpm_ref_set_deletion(darr, nd)
    inp = _Inputs(sc)
    cap = _contact_rows(sc.n)
    o, c, soa, csoa = _outputs(sc.n, cap)
    cnt = C.c_int64(0)
    ene = np.zeros(4)
    rc = ref_lib(variant).mdpm_ref_run(C.byref(inp.cfg), C.byref(inp.inst), inp.species, _dp(inp.density), inp.walls,
                                       inp.nwalls, C.byref(inp.soa), nsteps, C.byref(soa), _dp(o["force"]),
                                       _dp(o["torque"]), C.byref(csoa), cap, C.byref(cnt), _dp(ene))
    assert rc == 0
    o["contacts"] = sort_contacts(_trim(c, cnt.value))
    o["energies"] = dict(kinetic=ene[0], rotational=ene[1], gravitational=ene[2], elastic=ene[3])
    return o


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


def run_gpu(sc, nsteps: int, contacts=None, deletions=None, **kw) -> dict:
    if deletions:
        from mercurydpm_fork_b200.engine import deletion_boundary
        kw["deletions"] = [deletion_boundary(nn, dd) for nn, dd in deletions]
    e = sc.engine(**kw)
    if contacts is not None:
        e.upload_contacts(contacts["id_p"], contacts["id_i"], contacts["springs"], contacts.get("is_wall"),
                          contacts.get("periodic"))
    e.step(nsteps)
    out = e.download()
    out["force"], out["torque"] = e.forces()
    out["contacts"] = sort_contacts(e.contacts())
    out["globals"] = e.reduce()
    out["stats"] = e.stats()
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

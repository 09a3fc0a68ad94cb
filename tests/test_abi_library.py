"""CPU checks of the drop-in boundary: the shared library loads without a GPU
and exports every entry point include/dem_b200.h declares, and the ctypes
mirror of the ABI structures has the C layout."""
import ctypes as C
import os
import re
import subprocess

import pytest

from harness import ROOT
from mercurydpm_fork_b200 import _abi

HEADER = os.path.join(ROOT, "include", "dem_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dem_[a-z_0-9]+)\s*\(", src)))


def test_header_declarations_match_bindings():
    assert set(declared_functions()) == set(_abi.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_abi.LIB_PATH)
    for name in declared_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (dem_[a-z_0-9]+)$", out, flags=re.M))
    assert set(declared_functions()) <= exported


def test_struct_layouts_match_c():
    """Compiles a tiny C program against the header and compares sizeof/offsetof."""
    src = r"""
    #include <stddef.h>
    #include <stdio.h>
    #include "dem_b200.h"
    int main(void){
      printf("%zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(dem_species_pair), sizeof(dem_wall),
             sizeof(dem_particles_soa), sizeof(dem_contacts_soa), sizeof(dem_instance_desc), sizeof(dem_config),
             sizeof(dem_globals), sizeof(dem_cg_grid));
      printf("%zu %zu %zu %zu\n", offsetof(dem_wall, faces), offsetof(dem_instance_desc, periodic_min),
             offsetof(dem_cg_grid, width), offsetof(dem_species_pair, interaction_distance));
      printf("%zu %zu %zu %zu\n", sizeof(dem_insertion_boundary), offsetof(dem_insertion_boundary, density),
             offsetof(dem_insertion_boundary, psd_probability), offsetof(dem_insertion_boundary, psd_seed));
      return 0; }
    """
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        lines = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sizes = list(map(int, lines[0].split()))
    offs = list(map(int, lines[1].split()))
    assert sizes == [C.sizeof(t) for t in (_abi.SpeciesPair, _abi.Wall, _abi.ParticlesSoA, _abi.ContactsSoA,
                                           _abi.InstanceDesc, _abi.Config, _abi.Globals, _abi.CGGrid)]
    assert offs == [_abi.Wall.faces.offset, _abi.InstanceDesc.periodic_min.offset, _abi.CGGrid.width.offset,
                    _abi.SpeciesPair.interaction_distance.offset]
    ins = list(map(int, lines[2].split()))
    B = _abi.InsertionBoundary
    assert ins == [C.sizeof(B), B.density.offset, B.psd_probability.offset, B.psd_seed.offset]


def test_create_without_gpu_reports_error():
    """Without a device, dem_create returns a status instead of falling back."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    from mercurydpm_fork_b200 import DemEngine, DemError, Instance, species_pair
    with pytest.raises(DemError):
        DemEngine(1e-5, [Instance((0, 0, 0), (1, 1, 1))], [species_pair(stiffness=1.0)])

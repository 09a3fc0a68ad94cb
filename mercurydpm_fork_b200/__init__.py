"""B200 DEM time-step engine: a device-resident replacement for the force /
broad-phase / integration loop of MercuryDPM's DPMBase::computeOneTimeStep.

The compute path is the CUDA shared library ``libdem_b200.so`` (C ABI in
``include/dem_b200.h``). There is no CPU fallback: importing this package
fails if the library is missing.
"""
from . import _abi
from .engine import DemEngine, DemError, Instance, infinite_wall, lib, species_pair

__all__ = ["DemEngine", "DemError", "Instance", "infinite_wall", "species_pair", "lib", "_abi"]

lib()  # load eagerly: a missing or broken library is an import error

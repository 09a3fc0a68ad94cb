"""B200 DEM time-step engine: a device-resident replacement for the force /
broad-phase / integration loop of MercuryDPM's DPMBase::computeOneTimeStep.

The compute path is the CUDA shared library ``libdem_b200.so`` (C ABI in
``include/dem_b200.h``). There is no CPU fallback: the library is loaded the
first time an engine is created (or ``lib()`` is called), and a missing or
broken library raises ImportError there. Importing the package itself maps
no shared library, so the ABI structures and the seeded scenario generators
can be used by processes that never run the engine (the reference's timing
arm of ``bench.py``).
"""
from . import _abi
from .engine import DemEngine, DemError, Instance, infinite_wall, lib, species_pair

__all__ = ["DemEngine", "DemError", "Instance", "infinite_wall", "species_pair", "lib", "_abi"]

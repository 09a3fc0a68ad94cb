// tangential_spring_unit_test.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's own unit test Drivers/UnitTests/TangentialSpringUnitTest.cpp,
// compiled from its source file unmodified, with one change made by the
// preprocessor: its driver class derives from GpuDPMBase (the engine's drop-in
// base class, mercurydpm_fork_b200/mercury/GpuTimeStep.h) instead of DPMBase.
// Its main() sets up the species, runs DPMBase::solve() and asserts the
// golden position, velocity and angular velocity to 1e-7 with
// logger.assert_always, which ends the process with a non-zero status on a
// mismatch. Every header the test includes is included first, so the macro
// renames only the base class in the test's own text.
#include <iostream>

#include "DPMBase.h"
#include "Logger.h"
#include "Species/LinearViscoelasticSlidingFrictionSpecies.h"

#include "GpuTimeStep.h"

#define DPMBase GpuDPMBase
#include "Drivers/UnitTests/TangentialSpringUnitTest.cpp"
#undef DPMBase

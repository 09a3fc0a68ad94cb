// force_self_test.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's self test Drivers/SelfTests/Interactions/ForceSelfTest.cpp
// (ten oblique particle-particle and particle-wall collisions, random seed 5,
// .data and .ene written every step), compiled from its source unmodified
// except that its driver class derives from GpuDPMBase
// (mercurydpm_fork_b200/mercury/GpuTimeStep.h) instead of DPMBase. Every header
// the test includes is included first, so the macro renames only the base
// class in the test's own text.
#include "DPMBase.h"
#include "Species/LinearViscoelasticSlidingFrictionSpecies.h"
#include "Species/Species.h"
#include "Walls/InfiniteWall.h"

#include "GpuTimeStep.h"

#define DPMBase GpuDPMBase
#include "Drivers/SelfTests/Interactions/ForceSelfTest.cpp"
#undef DPMBase

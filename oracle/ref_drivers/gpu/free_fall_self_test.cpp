// free_fall_self_test.cpp -- TEST INFRASTRUCTURE ONLY.
//
// The reference's self test Drivers/SelfTests/Interactions/FreeFallSelfTest.cpp
// (one elastic sphere bouncing on an InfiniteWall for 1,000,000 steps, .ene and
// .restart written every 500 steps), compiled from its source unmodified
// except that its driver class derives from GpuMercury2D
// (mercurydpm_fork_b200/mercury/GpuTimeStep.h) instead of Mercury2D.
#include "Mercury2D.h"
#include "Species/LinearViscoelasticSpecies.h"
#include "Walls/InfiniteWall.h"

#include "GpuTimeStep.h"

#define Mercury2D GpuMercury2D
#include "Drivers/SelfTests/Interactions/FreeFallSelfTest.cpp"
#undef Mercury2D

// Stand-in for the reference's CMake-generated src/building_config.h (from building_config.in):
// the GPU build with the default random engine.
#pragma once
#define KMC_GPU_MODE
#define RAND_MT

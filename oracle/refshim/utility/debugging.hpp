// Stand-in for the reference's utility/debugging.hpp (test infrastructure):
// the assert macros without OptiX.
#ifndef DEBUGGING_HPP
#define DEBUGGING_HPP
#include <cstdio>
#include "cuda_runtime.h"
#define CUDA_ASSERT(ans) { (void)(ans); }
#define OPTIX_ASSERT(ans) { (void)(ans); }
#endif

// Stand-in for the reference's utility/debugging.hpp (test infrastructure):
// the assert macros without OptiX.
#ifndef DEBUGGING_HPP
#define DEBUGGING_HPP
#include <cstdio>
#include "cuda_runtime.h"
#define CUDA_ASSERT(ans) { (void)(ans); }
#define OPTIX_ASSERT(ans) { (void)(ans); }
#include <glm/glm.hpp>
namespace rt {
// The LOD colour of the VISUALIZE_LODS debug mode, which nothing here renders.
inline glm::vec3 mapLODs(float) { return glm::vec3(0.f); }
}  // namespace rt
#endif

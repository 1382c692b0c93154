// Stand-in for the reference's CDeviceScene (scene/device_scene_impl.hpp) on
// the host (test infrastructure).  The OptiX trace and closest-hit programs
// are replaced by r2ref::scene_intersect, which ref_kat.cpp implements over
// the oracle's BVH: the closest FILTER-visible triangle along the ray, its
// interpolated and object-transformed shading normal, texture coordinates 0,
// the material's ior and the material itself (shaders.optix.cu:28-130).
#ifndef R2_REFSHIM_DEVICE_SCENE_IMPL_HPP
#define R2_REFSHIM_DEVICE_SCENE_IMPL_HPP
#include <glm/glm.hpp>
#include <optix_types.h>

#include "intersect/ray.hpp"
#include "scene/interaction.hpp"
#include "scene/sceneobject_mask.hpp"

namespace rt {
class CDeviceScene;
}
namespace r2ref {
void scene_intersect(const rt::CRay& ray, rt::SInteraction* si, unsigned int mask);
}
namespace rt {
class CDeviceScene {
 public:
  void intersect(const CRay& ray, SInteraction* si, OptixVisibilityMask mask) const {
    r2ref::scene_intersect(ray, si, mask);
    if (si->hitInformation.hit) ray.m_t_max = si->hitInformation.t;
  }
};
}  // namespace rt
#endif

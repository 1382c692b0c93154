// Stand-in for the reference's CDeviceScene (scene/device_scene_impl.hpp) on
// the host (test infrastructure).  The OptiX trace and closest-hit programs
// are replaced by r2ref::scene_intersect, which ref_kat.cpp implements over
// the oracle's BVH with __closesthit__ch's normal rule
// (shaders.optix.cu:28-130); the environment queries by the oracle's
// environment map; intersectTr follows device_scene_impl.hpp:93-114 for
// scenes without media (the walk ends at the first hit).  A medium instance
// stand-in completes the types the integrator names for media, which these
// scenes do not have.
#ifndef R2_REFSHIM_DEVICE_SCENE_IMPL_HPP
#define R2_REFSHIM_DEVICE_SCENE_IMPL_HPP
#include <glm/glm.hpp>
#include <optix_types.h>

#include "intersect/ray.hpp"
#include "medium/phase_function_impl.hpp"
#include "scene/interaction.hpp"
#include "scene/sceneobject_mask.hpp"

namespace rt {
class CSampler;
// Stand-in: media are not part of the scenes driven through this header.
class CMediumInstance {
 public:
  template <typename... A> glm::vec3 sample(A&&...) const { return glm::vec3(1.f); }
  template <typename... A> glm::vec3 tr(A&&...) const { return glm::vec3(1.f); }
  CRay moveToVoxelBorder(const CRay& r) const { return r; }
  const CPhaseFunction& phase() const { return *m_phase; }
  float voxelSizeFiltering() const { return 0.f; }
  const CPhaseFunction* m_phase = nullptr;
};
}  // namespace rt

namespace r2ref {
void scene_intersect(const rt::CRay& ray, rt::SInteraction* si, unsigned int mask);
glm::vec3 scene_sample_light(float u0, float u1, glm::vec3* dir, float* pdf);
glm::vec3 scene_le(const glm::vec3& dir, float* pdf);
}  // namespace r2ref

inline uint3 optixGetLaunchIndex() { return make_uint3(0, 0, 0); }

namespace rt {
class CDeviceScene {
 public:
  void intersect(const CRay& ray, SInteraction* si, OptixVisibilityMask mask = 255) const {
    r2ref::scene_intersect(ray, si, mask);
    if (si->hitInformation.hit) ray.m_t_max = si->hitInformation.t;
  }
  // CEnvironmentMap::sample draws the marginal's uniform, then the row's.
  glm::vec3 sampleLightSources(CSampler& sampler, glm::vec3* direction, float* pdf) const;
  glm::vec3 le(const glm::vec3& direction, float* pdf) const { return r2ref::scene_le(direction, pdf); }
  SInteraction intersectTr(const CRay& ray, CSampler& sampler, glm::vec3* Tr, bool useBrickGrid,
                           size_t* numLookups) const {
    *Tr = glm::vec3(1.f);
    const glm::vec3 p1 = ray.m_origin + ray.m_t_max * ray.m_direction;
    CRay r = CRay::spawnRay(ray.m_origin, p1, ray.m_medium);
    SInteraction interaction;
    intersect(r, &interaction);
    return interaction;
  }
};
}  // namespace rt
#endif

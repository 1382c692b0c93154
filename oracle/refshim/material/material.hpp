// Stand-in for the reference's CMaterial (material/material.hpp) on the host
// (test infrastructure): the three accessors CMeshFilter::run reads, with the
// untextured values of CMaterial (material.cu:80-148): Kd, Ks and the GGX
// roughness alpha.
#ifndef R2_REFSHIM_MATERIAL_HPP
#define R2_REFSHIM_MATERIAL_HPP
#include <glm/glm.hpp>
namespace rt {
class CMaterial {
 public:
  glm::vec3 kd{0.f}, ks{0.f};
  float alpha = 0.f;
  float specularRoughness() const { return alpha; }
  glm::vec3 diffuse(const glm::vec2&) const { return kd; }
  glm::vec3 glossy(const glm::vec2&) const { return ks; }
};
}  // namespace rt
#endif

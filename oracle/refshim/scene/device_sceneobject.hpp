// Stand-in for the reference's CDeviceSceneobject (test infrastructure): only
// the accessors that CMeshFilter::debug names, which nothing here calls.
#ifndef R2_REFSHIM_DEVICE_SCENEOBJECT_HPP
#define R2_REFSHIM_DEVICE_SCENEOBJECT_HPP
#include <cstddef>
namespace rt {
struct R2StubMedium {
  template <typename... A> void sample(A&&...) const {}
};
class CDeviceSceneobject {
 public:
  const void* mesh() const { return nullptr; }
  const R2StubMedium* medium() const { return nullptr; }
};
}  // namespace rt
#endif

// Host declaration of CUDA's texture fetch template (test infrastructure):
// the reference's CTexture::operator() calls tex2D<float4>, which CUDA's
// headers declare for device code only.  Untextured materials never call it.
#ifndef R2_REFSHIM_HOST_TEXFETCH_H
#define R2_REFSHIM_HOST_TEXFETCH_H
#include <cuda_runtime.h>
template <class T>
inline T tex2D(cudaTextureObject_t, float, float) {
  return T{};
}
#endif

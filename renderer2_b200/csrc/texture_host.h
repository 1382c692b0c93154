// Host side of the texture maps of OBJ materials: loading (PNG), the texel
// conversions of the reference's CTexture load paths, the material rules of
// CMaterial(aiMaterial*) (raytracer/src/material/material.cu:110-143) and the
// upload as one texel array with per-texture offsets (texture.h).
#pragma once
#include <string>
#include <vector>

#include "runtime.h"
#include "texture.h"

namespace r2 {

class TextureSet {
 public:
  // Index of the texture of file `path` converted as `kind` (loaded once).
  int add(const std::string& path, int kind);
  // Texture indices {albedo, glossy, normal, opacity} (-1: none) of a material
  // with the maps `maps` (nullable): glossy from the albedo's luma when a
  // specular channel is at most 0.02, else the specular map; opacity from
  // map_d, else from the albedo's alpha channel when it has one.
  void material_maps(const r2_material& mat, const r2_material_maps* maps, int tex[4]);
  bool empty() const { return list_.empty(); }
  // Uploads every texture; returns false when there is none.
  bool upload(DBuf<float4>* texels, DBuf<TexInfo>* info, cudaStream_t s) const;

 private:
  struct Tex {
    std::string path;
    int kind = 0, W = 0, H = 0, channels = 0;
    std::vector<float4> texels;
  };
  std::vector<Tex> list_;
};

}  // namespace r2

// Host readers and writers of the pipeline's asset files.
//
// OBJ + MTL meshes: replaces CAssetManager::loadWithAssimp
// (raytracer/src/backend/asset_manager.cu:25-84) with the import flags the
// reference passes (triangulate, flat normals where a face has none, join
// identical vertices) and CMaterial(aiMaterial*) (raytracer/src/material/material.cu:80-143):
// Kd -> diffuse, Ks -> glossy, Oren-Nayar roughness 0, alpha = (2/(Ns+2))^0.5,
// eta_i = 1, eta_t = Ni (1.5 when Ni == 1).  Texture maps are not read.
//
// Radiance RGBE (.hdr) environment maps: the loader path of CTexture
// (raytracer/src/texture/texture.cu:64-79, stbi_loadf with 3 channels): flat
// and new-style run-length scanlines, "-Y H +X W" orientation, texel =
// mantissa * 2^(e - 136).
//
// PNG: 8-bit RGB with stored (uncompressed) deflate blocks, optionally flipped
// vertically like the reference's writer (visualisation/src/image_writer.cpp:7-24);
// JPEG: see jpeg_writer.cpp.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/r2.h"

namespace r2 {

struct ObjSubmesh {
  std::string materialName;
  std::vector<float> positions;  // 3 per vertex
  std::vector<float> normals;    // 3 per vertex
  std::vector<float> uvs;        // 2 per vertex, empty when no face has texture coordinates
  std::vector<uint32_t> indices; // 3 per triangle
  r2_material material;
  // texture maps of the material (paths joined to the OBJ's directory, empty: none):
  // map_Kd (albedo), map_Ks (specular), map_Bump / bump (normal map), map_d (opacity)
  std::string texAlbedo, texSpecular, texNormal, texAlpha;
};

// Submeshes of <directory>/<filename> in order of first use of their material
// (vertices joined on identical position, texture coordinate and normal).
std::vector<ObjSubmesh> load_obj(const std::string& directory, const std::string& filename);

struct RgbImage {
  uint32_t width = 0, height = 0;
  std::vector<float> rgb;  // row 0 = top
};
RgbImage read_hdr(const std::string& path);

// 8-bit RGBA texels (row 0 = top) and the source's channel count (1-4).
struct RgbaImage8 {
  uint32_t width = 0, height = 0;
  int channels = 0;
  std::vector<uint8_t> rgba;
};
RgbaImage8 read_png(const std::string& path);  // png_reader.cpp
void write_hdr(const std::string& path, const float* rgb, uint32_t width, uint32_t height);

void write_png(const std::string& path, const uint8_t* rgb, uint32_t width, uint32_t height, bool flipVertical);
// Baseline JPEG, 4:4:4, quality 1..100 (the reference writes quality 100); jpeg_writer.cpp.
void write_jpg(const std::string& path, const uint8_t* rgb, uint32_t width, uint32_t height, bool flipVertical,
               int quality);

}  // namespace r2

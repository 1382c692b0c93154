// TextureSet (texture_host.h).
#include "texture_host.h"

#include <ctype.h>

#include "asset_io.h"

namespace r2 {

int TextureSet::add(const std::string& path, int kind) {
  for (size_t i = 0; i < list_.size(); ++i)
    if (list_[i].path == path && list_[i].kind == kind) return (int)i;
  const size_t dot = path.find_last_of('.');
  std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
  for (char& c : ext) c = (char)tolower(c);
  R2_REQUIRE(ext == "png", R2_ERR_UNSUPPORTED, "texture maps are read from PNG files: " + path);
  const RgbaImage8 img = read_png(path);
  Tex t;
  t.path = path;
  t.kind = kind;
  t.W = (int)img.width;
  t.H = (int)img.height;
  t.channels = img.channels;
  t.texels.resize((size_t)t.W * t.H);
  for (size_t i = 0; i < t.texels.size(); ++i) {
    const uint8_t* p = &img.rgba[4 * i];
    const float r = (float)p[0] / 255.0f, g = (float)p[1] / 255.0f, b = (float)p[2] / 255.0f;
    if (kind == kTexAlphaChannel) {  // CTexture::loadAlpha (texture.cu:249-270): the alpha channel in rgb
      const float a = (float)p[3] / 255.0f;
      t.texels[i] = make_float4(a, a, a, 1.0f);
    } else if (kind == kTexLuma) {  // CAssetManager::specularFromDiffuse (asset_manager.cu:165-184), luma.hpp:4-6
      float l = 0.2126f * r;
      l += 0.7152f * g;
      l += 0.0722f * b;
      t.texels[i] = make_float4(l, l, l, 1.0f);
    } else {  // stbi_load with 3 channels / 255 (texture.cu:82-95)
      t.texels[i] = make_float4(r, g, b, 1.0f);
    }
  }
  list_.push_back(std::move(t));
  return (int)list_.size() - 1;
}

void TextureSet::material_maps(const r2_material& mat, const r2_material_maps* maps, int tex[4]) {
  for (int k = 0; k < 4; ++k) tex[k] = -1;
  if (!maps) return;
  const bool hasAlbedo = maps->albedo && maps->albedo[0];
  if (hasAlbedo) tex[0] = add(maps->albedo, kTexColor);
  if (hasAlbedo && (mat.specular[0] <= 0.02f || mat.specular[1] <= 0.02f || mat.specular[2] <= 0.02f))
    tex[1] = add(maps->albedo, kTexLuma);
  else if (maps->specular && maps->specular[0])
    tex[1] = add(maps->specular, kTexColor);
  if (maps->normal && maps->normal[0]) tex[2] = add(maps->normal, kTexColor);
  if (maps->alpha && maps->alpha[0]) tex[3] = add(maps->alpha, kTexColor);
  else if (hasAlbedo && list_[tex[0]].channels == 4) tex[3] = add(maps->albedo, kTexAlphaChannel);
}

bool TextureSet::upload(DBuf<float4>* texels, DBuf<TexInfo>* info, cudaStream_t s) const {
  if (list_.empty()) return false;
  std::vector<TexInfo> ti;
  std::vector<float4> all;
  for (const Tex& t : list_) {
    TexInfo x;
    x.offset = (uint32_t)all.size();
    x.W = t.W;
    x.H = t.H;
    x.pad = 0;
    ti.push_back(x);
    all.insert(all.end(), t.texels.begin(), t.texels.end());
  }
  R2_REQUIRE(all.size() < (1ull << 32), R2_ERR_UNSUPPORTED, "texture maps larger than 2^32 texels");
  texels->upload(all.data(), all.size(), s);
  info->upload(ti.data(), ti.size(), s);
  return true;
}

}  // namespace r2

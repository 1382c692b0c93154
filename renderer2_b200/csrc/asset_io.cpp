// Host readers and writers of the pipeline's asset files (see asset_io.h).
#include "asset_io.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <sstream>
#include <tuple>

#include "json.h"
#include "runtime.h"

namespace r2 {

// ---------------------------------------------------------------- OBJ / MTL
namespace {

struct MtlEntry {
  float kd[3] = {0.6f, 0.6f, 0.6f};  // the OBJ importer's defaults
  float ks[3] = {0.0f, 0.0f, 0.0f};
  float ns = 0.0f;
  float ni = 1.0f;
  std::string mapKd, mapKs, mapBump, mapD;
};

// The file name of a map_* statement: its last token (options such as -bm come first).
std::string map_file(std::istringstream& ls) {
  std::string tok, last;
  while (ls >> tok) last = tok;
  return last;
}

r2_material material_from_mtl(const MtlEntry& m) {
  r2_material r;
  memset(&r, 0, sizeof(r));
  for (int k = 0; k < 3; ++k) {
    r.diffuse[k] = m.kd[k];
    r.specular[k] = m.ks[k];
  }
  r.diffuse_roughness = 0.0f;
  const float a = powf(2.0f / (m.ns + 2.0f), 0.5f);  // CMaterial::roughnessFromExponent
  r.alpha_x = a;
  r.alpha_y = a;
  r.eta_i = 1.0f;
  r.eta_t = m.ni == 1.0f ? 1.5f : m.ni;
  return r;
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

void parse_mtl(const std::string& path, std::map<std::string, MtlEntry>* out) {
  std::istringstream in(read_text_file(path));
  std::string line, cur;
  while (std::getline(in, line)) {
    line = trim(line);
    if (line.empty() || line[0] == '#') continue;
    std::istringstream ls(line);
    std::string key;
    ls >> key;
    if (key == "newmtl") {
      std::string rest;
      std::getline(ls, rest);
      cur = trim(rest);
      (*out)[cur] = MtlEntry();
    } else if (!cur.empty()) {
      MtlEntry& m = (*out)[cur];
      if (key == "Kd") ls >> m.kd[0] >> m.kd[1] >> m.kd[2];
      else if (key == "Ks") ls >> m.ks[0] >> m.ks[1] >> m.ks[2];
      else if (key == "Ns") ls >> m.ns;
      else if (key == "Ni") ls >> m.ni;
      else if (key == "map_Kd") m.mapKd = map_file(ls);
      else if (key == "map_Ks") m.mapKs = map_file(ls);
      else if (key == "map_Bump" || key == "map_bump" || key == "bump") m.mapBump = map_file(ls);
      else if (key == "map_d") m.mapD = map_file(ls);
    }
  }
}

// one corner of a face: 0-based position / texture coordinate / normal index (-1: none)
struct Corner {
  int64_t v, vt, vn;
};

int64_t resolve(long long i, size_t count, const std::string& path) {
  const long long r = i > 0 ? i - 1 : (long long)count + i;
  R2_REQUIRE(i != 0 && r >= 0 && r < (long long)count, R2_ERR_IO, "OBJ index out of range in " + path);
  return (int64_t)r;
}

}  // namespace

std::vector<ObjSubmesh> load_obj(const std::string& directory, const std::string& filename) {
  const std::string path = directory + "/" + filename;
  std::istringstream in(read_text_file(path));
  std::vector<float> v, vn, vt;
  std::map<std::string, MtlEntry> mtl;
  std::vector<ObjSubmesh> subs;
  std::map<std::string, size_t> subIndex;
  std::vector<std::map<std::tuple<int64_t, int64_t, int64_t>, uint32_t>> dedup;
  std::vector<bool> anyUv;
  size_t cur = (size_t)-1;
  auto select = [&](const std::string& name) {
    auto it = subIndex.find(name);
    if (it == subIndex.end()) {
      ObjSubmesh s;
      s.materialName = name;
      subIndex[name] = subs.size();
      subs.push_back(s);
      dedup.emplace_back();
      anyUv.push_back(false);
      cur = subs.size() - 1;
    } else {
      cur = it->second;
    }
  };
  std::string line;
  while (std::getline(in, line)) {
    const std::string t = trim(line);
    if (t.empty() || t[0] == '#') continue;
    std::istringstream ls(t);
    std::string key;
    ls >> key;
    if (key == "v") {
      float x = 0, y = 0, z = 0;
      ls >> x >> y >> z;
      v.push_back(x); v.push_back(y); v.push_back(z);
    } else if (key == "vn") {
      float x = 0, y = 0, z = 0;
      ls >> x >> y >> z;
      vn.push_back(x); vn.push_back(y); vn.push_back(z);
    } else if (key == "vt") {
      float x = 0, y = 0;
      ls >> x >> y;
      vt.push_back(x); vt.push_back(y);
    } else if (key == "mtllib") {
      std::string rest;
      std::getline(ls, rest);
      parse_mtl(directory + "/" + trim(rest), &mtl);
    } else if (key == "usemtl") {
      std::string rest;
      std::getline(ls, rest);
      select(trim(rest));
    } else if (key == "f") {
      if (cur == (size_t)-1) select("");
      std::vector<Corner> face;
      std::string tok;
      while (ls >> tok) {
        long long iv = 0, it = 0, in2 = 0;
        int n = 0;
        Corner c = {-1, -1, -1};
        bool hasT = false;
        if (sscanf(tok.c_str(), "%lld/%lld/%lld", &iv, &it, &in2) == 3) n = 3, hasT = true;
        else if (sscanf(tok.c_str(), "%lld//%lld", &iv, &in2) == 2) n = 2;
        else if (sscanf(tok.c_str(), "%lld/%lld", &iv, &it) == 2) n = 1, hasT = true;
        else if (sscanf(tok.c_str(), "%lld", &iv) == 1) n = 1;
        R2_REQUIRE(n > 0, R2_ERR_IO, "bad OBJ face corner '" + tok + "' in " + path);
        c.v = resolve(iv, v.size() / 3, path);
        if (n >= 2) c.vn = resolve(in2, vn.size() / 3, path);
        if (hasT && !vt.empty()) c.vt = resolve(it, vt.size() / 2, path);  // without vt lines the index is ignored
        face.push_back(c);
      }
      R2_REQUIRE(face.size() >= 3, R2_ERR_IO, "OBJ face with fewer than 3 corners in " + path);
      ObjSubmesh& s = subs[cur];
      bool hasN = true;
      for (const Corner& c : face) hasN = hasN && c.vn >= 0;
      for (const Corner& c : face) anyUv[cur] = anyUv[cur] || c.vt >= 0;
      // texture coordinates of every vertex so far (0 where a corner has none)
      auto push_uv = [&](const Corner& c) {
        s.uvs.push_back(c.vt >= 0 ? vt[2 * c.vt] : 0.0f);
        s.uvs.push_back(c.vt >= 0 ? vt[2 * c.vt + 1] : 0.0f);
      };
      for (size_t k = 1; k + 1 < face.size(); ++k) {  // fan triangulation
        const Corner tri[3] = {face[0], face[k], face[k + 1]};
        if (hasN) {
          for (const Corner& c : tri) {
            auto key = std::make_tuple(c.v, c.vt, c.vn);
            auto it2 = dedup[cur].find(key);
            if (it2 == dedup[cur].end()) {
              const uint32_t id = (uint32_t)(s.positions.size() / 3);
              for (int a = 0; a < 3; ++a) s.positions.push_back(v[3 * c.v + a]);
              for (int a = 0; a < 3; ++a) s.normals.push_back(vn[3 * c.vn + a]);
              push_uv(c);
              dedup[cur][key] = id;
              s.indices.push_back(id);
            } else {
              s.indices.push_back(it2->second);
            }
          }
        } else {
          // flat normal of the face (generated normals): normalize((p1-p0) x (p2-p0))
          float p[3][3];
          for (int i = 0; i < 3; ++i)
            for (int a = 0; a < 3; ++a) p[i][a] = v[3 * tri[i].v + a];
          const float e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
          const float e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
          float nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
          const float l = sqrtf(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
          for (int a = 0; a < 3; ++a) nn[a] = l > 0.0f ? nn[a] / l : 0.0f;
          for (int i = 0; i < 3; ++i) {
            const uint32_t id = (uint32_t)(s.positions.size() / 3);
            for (int a = 0; a < 3; ++a) s.positions.push_back(p[i][a]);
            for (int a = 0; a < 3; ++a) s.normals.push_back(nn[a]);
            push_uv(tri[i]);
            s.indices.push_back(id);
          }
        }
      }
    }
  }
  std::vector<ObjSubmesh> out;
  for (size_t k = 0; k < subs.size(); ++k) {
    ObjSubmesh& s = subs[k];
    if (s.indices.empty()) continue;
    if (!anyUv[k]) s.uvs.clear();
    auto it = mtl.find(s.materialName);
    const MtlEntry m = it == mtl.end() ? MtlEntry() : it->second;
    s.material = material_from_mtl(m);
    auto joined = [&](const std::string& f) { return f.empty() ? f : directory + "/" + f; };
    s.texAlbedo = joined(m.mapKd);
    s.texSpecular = joined(m.mapKs);
    s.texNormal = joined(m.mapBump);
    s.texAlpha = joined(m.mapD);
    out.push_back(std::move(s));
  }
  R2_REQUIRE(!out.empty(), R2_ERR_IO, "no triangles in " + path);
  return out;
}

// ---------------------------------------------------------------- Radiance RGBE
RgbImage read_hdr(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path);
  std::vector<uint8_t> buf;
  {
    uint8_t tmp[1 << 16];
    size_t n;
    while ((n = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    fclose(f);
  }
  size_t pos = 0;
  auto getline = [&](std::string* s) {
    s->clear();
    while (pos < buf.size() && buf[pos] != '\n') s->push_back((char)buf[pos++]);
    R2_REQUIRE(pos < buf.size(), R2_ERR_IO, "truncated header in " + path);
    ++pos;
  };
  std::string line;
  getline(&line);
  R2_REQUIRE(line == "#?RADIANCE" || line == "#?RGBE", R2_ERR_IO, "not a Radiance HDR file: " + path);
  bool format = false;
  for (;;) {
    getline(&line);
    if (line.empty()) break;
    if (line == "FORMAT=32-bit_rle_rgbe") format = true;
  }
  R2_REQUIRE(format, R2_ERR_UNSUPPORTED, "unsupported HDR format in " + path);
  getline(&line);
  int h = 0, w = 0;
  R2_REQUIRE(sscanf(line.c_str(), "-Y %d +X %d", &h, &w) == 2 && h > 0 && w > 0 && h <= (1 << 16) && w <= (1 << 16),
             R2_ERR_UNSUPPORTED, "unsupported HDR orientation/size in " + path);
  RgbImage img;
  img.width = (uint32_t)w;
  img.height = (uint32_t)h;
  img.rgb.resize((size_t)w * h * 3);
  std::vector<uint8_t> scan((size_t)w * 4);
  auto need = [&](size_t n) { R2_REQUIRE(pos + n <= buf.size(), R2_ERR_IO, "truncated pixel data in " + path); };
  for (int y = 0; y < h; ++y) {
    bool rle = false;
    if (w >= 8 && w < 32768) {
      need(4);
      rle = buf[pos] == 2 && buf[pos + 1] == 2 && !(buf[pos + 2] & 0x80);
      if (rle) {
        R2_REQUIRE(((int)buf[pos + 2] << 8 | buf[pos + 3]) == w, R2_ERR_IO, "bad scanline width in " + path);
        pos += 4;
      }
    }
    if (rle) {
      for (int c = 0; c < 4; ++c) {
        int x = 0;
        while (x < w) {
          need(1);
          int count = buf[pos++];
          if (count > 128) {
            count -= 128;
            R2_REQUIRE(x + count <= w, R2_ERR_IO, "bad run in " + path);
            need(1);
            const uint8_t val = buf[pos++];
            for (int i = 0; i < count; ++i) scan[4 * (x++) + c] = val;
          } else {
            R2_REQUIRE(count > 0 && x + count <= w, R2_ERR_IO, "bad run in " + path);
            need((size_t)count);
            for (int i = 0; i < count; ++i) scan[4 * (x++) + c] = buf[pos++];
          }
        }
      }
    } else {
      need((size_t)w * 4);
      memcpy(scan.data(), &buf[pos], (size_t)w * 4);
      pos += (size_t)w * 4;
    }
    for (int x = 0; x < w; ++x) {
      const uint8_t* p = &scan[4 * x];
      float* o = &img.rgb[3 * ((size_t)y * w + x)];
      if (p[3] == 0) {
        o[0] = o[1] = o[2] = 0.0f;
      } else {
        const float f = ldexpf(1.0f, (int)p[3] - (128 + 8));
        o[0] = p[0] * f;
        o[1] = p[1] * f;
        o[2] = p[2] * f;
      }
    }
  }
  return img;
}

void write_hdr(const std::string& path, const float* rgb, uint32_t width, uint32_t height) {
  FILE* f = fopen(path.c_str(), "wb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path + " for writing");
  fprintf(f, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y %u +X %u\n", height, width);
  std::vector<uint8_t> row((size_t)width * 4);
  bool ok = true;
  for (uint32_t y = 0; y < height && ok; ++y) {
    for (uint32_t x = 0; x < width; ++x) {
      const float* p = &rgb[3 * ((size_t)y * width + x)];
      const float m = fmaxf(p[0], fmaxf(p[1], p[2]));
      uint8_t* o = &row[4 * x];
      if (!(m >= 1e-32f)) {
        o[0] = o[1] = o[2] = o[3] = 0;
      } else {
        int e;
        const float s = frexpf(m, &e) * 256.0f / m;  // mantissa scaled to [128, 256)
        o[0] = (uint8_t)(p[0] * s);
        o[1] = (uint8_t)(p[1] * s);
        o[2] = (uint8_t)(p[2] * s);
        o[3] = (uint8_t)(e + 128);
      }
    }
    ok = fwrite(row.data(), 1, row.size(), f) == row.size();
  }
  ok = (fclose(f) == 0) && ok;
  R2_REQUIRE(ok, R2_ERR_IO, "short write to " + path);
}

// ---------------------------------------------------------------- PNG
namespace {

uint32_t crc32_update(uint32_t crc, const uint8_t* d, size_t n) {
  static uint32_t table[256];
  static bool init = false;
  if (!init) {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t c = i;
      for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
      table[i] = c;
    }
    init = true;
  }
  for (size_t i = 0; i < n; ++i) crc = table[(crc ^ d[i]) & 0xFF] ^ (crc >> 8);
  return crc;
}

void put32(std::vector<uint8_t>& o, uint32_t v) {
  o.push_back((uint8_t)(v >> 24));
  o.push_back((uint8_t)(v >> 16));
  o.push_back((uint8_t)(v >> 8));
  o.push_back((uint8_t)v);
}

void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
  put32(out, (uint32_t)data.size());
  const size_t start = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data.begin(), data.end());
  const uint32_t crc = crc32_update(0xFFFFFFFFu, &out[start], out.size() - start) ^ 0xFFFFFFFFu;
  put32(out, crc);
}

}  // namespace

void write_png(const std::string& path, const uint8_t* rgb, uint32_t width, uint32_t height, bool flipVertical) {
  R2_REQUIRE(rgb && width > 0 && height > 0, R2_ERR_INVALID_ARGUMENT, "empty image");
  std::vector<uint8_t> raw;
  raw.reserve((size_t)height * (1 + 3 * (size_t)width));
  for (uint32_t r = 0; r < height; ++r) {
    const uint32_t y = flipVertical ? height - 1 - r : r;
    raw.push_back(0);  // filter: none
    raw.insert(raw.end(), rgb + 3 * (size_t)y * width, rgb + 3 * ((size_t)y + 1) * width);
  }
  // zlib stream of stored deflate blocks
  std::vector<uint8_t> z = {0x78, 0x01};
  for (size_t off = 0; off < raw.size() || off == 0; off += 65535) {
    const size_t n = std::min<size_t>(65535, raw.size() - off);
    const bool last = off + n >= raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back((uint8_t)(n & 0xFF));
    z.push_back((uint8_t)(n >> 8));
    z.push_back((uint8_t)(~n & 0xFF));
    z.push_back((uint8_t)((~n >> 8) & 0xFF));
    z.insert(z.end(), raw.begin() + (ptrdiff_t)off, raw.begin() + (ptrdiff_t)(off + n));
    if (last) break;
  }
  uint32_t a = 1, b = 0;  // Adler-32
  for (uint8_t c : raw) {
    a = (a + c) % 65521u;
    b = (b + a) % 65521u;
  }
  put32(z, (b << 16) | a);
  std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
  std::vector<uint8_t> ihdr;
  put32(ihdr, width);
  put32(ihdr, height);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit RGB, deflate, no interlace
  chunk(out, "IHDR", ihdr);
  chunk(out, "IDAT", z);
  chunk(out, "IEND", {});
  FILE* f = fopen(path.c_str(), "wb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path + " for writing");
  bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
  ok = (fclose(f) == 0) && ok;
  R2_REQUIRE(ok, R2_ERR_IO, "short write to " + path);
}

}  // namespace r2

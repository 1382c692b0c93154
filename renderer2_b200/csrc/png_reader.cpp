// PNG reader for texture maps of OBJ materials (the reference loads them with
// stb_image, raytracer/src/texture/texture.cu:64-97).  Non-interlaced PNG of
// every colour type (grey, RGB, palette, grey + alpha, RGBA) at 8 bits per
// sample, palette/grey also at 1, 2 and 4 bits, 16-bit samples reduced to
// their high byte; a zlib inflater (stored, fixed and dynamic Huffman
// blocks, RFC 1950/1951) and the five scanline filters of the PNG standard.
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "asset_io.h"
#include "runtime.h"

namespace r2 {
namespace {

struct BitReader {
  const uint8_t* p;
  size_t n, pos = 0;  // bit position
  uint32_t bits(int k) {
    uint32_t v = 0;
    for (int i = 0; i < k; ++i) {
      R2_REQUIRE((pos >> 3) < n, R2_ERR_IO, "truncated deflate stream");
      v |= (uint32_t)((p[pos >> 3] >> (pos & 7)) & 1u) << i;
      ++pos;
    }
    return v;
  }
  void align() { pos = (pos + 7) & ~(size_t)7; }
};

// Canonical Huffman decoding table: counts per length and symbols by code order.
struct Huffman {
  uint16_t count[16] = {};
  std::vector<uint16_t> symbol;
  void build(const uint8_t* lengths, int n) {
    memset(count, 0, sizeof(count));
    for (int i = 0; i < n; ++i) count[lengths[i]]++;
    count[0] = 0;
    uint16_t offs[16];
    offs[1] = 0;
    for (int l = 1; l < 15; ++l) offs[l + 1] = offs[l] + count[l];
    symbol.assign(n, 0);
    for (int i = 0; i < n; ++i)
      if (lengths[i]) symbol[offs[lengths[i]]++] = (uint16_t)i;
  }
  int decode(BitReader& br) const {
    int code = 0, first = 0, index = 0;
    for (int l = 1; l < 16; ++l) {
      code |= (int)br.bits(1);
      const int c = count[l];
      if (code - c < first) return symbol[index + (code - first)];
      index += c;
      first += c;
      first <<= 1;
      code <<= 1;
    }
    throw Error{R2_ERR_IO, "bad Huffman code in deflate stream"};
  }
};

const uint16_t kLenBase[29] = {3, 4, 5, 6, 7, 8, 9, 10, 11, 13, 15, 17, 19, 23, 27, 31,
                               35, 43, 51, 59, 67, 83, 99, 115, 131, 163, 195, 227, 258};
const uint8_t kLenExtra[29] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3, 4, 4, 4, 4, 5, 5, 5, 5, 0};
const uint16_t kDistBase[30] = {1,   2,   3,   4,   5,   7,    9,    13,   17,   25,   33,   49,   65,    97,    129,
                                193, 257, 385, 513, 769, 1025, 1537, 2049, 3073, 4097, 6145, 8193, 12289, 16385, 24577};
const uint8_t kDistExtra[30] = {0, 0, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13};

void inflate_block(BitReader& br, const Huffman& lit, const Huffman& dist, std::vector<uint8_t>& out) {
  for (;;) {
    const int sym = lit.decode(br);
    if (sym < 256) {
      out.push_back((uint8_t)sym);
    } else if (sym == 256) {
      return;
    } else {
      const int li = sym - 257;
      R2_REQUIRE(li < 29, R2_ERR_IO, "bad length code in deflate stream");
      const size_t len = kLenBase[li] + br.bits(kLenExtra[li]);
      const int di = dist.decode(br);
      R2_REQUIRE(di < 30, R2_ERR_IO, "bad distance code in deflate stream");
      const size_t d = kDistBase[di] + br.bits(kDistExtra[di]);
      R2_REQUIRE(d <= out.size(), R2_ERR_IO, "distance beyond the start of the deflate stream");
      const size_t from = out.size() - d;
      for (size_t i = 0; i < len; ++i) out.push_back(out[from + i]);
    }
  }
}

std::vector<uint8_t> zlib_inflate(const std::vector<uint8_t>& z, size_t expected) {
  R2_REQUIRE(z.size() >= 2 && (z[0] & 0x0F) == 8 && ((z[0] << 8) | z[1]) % 31 == 0 && !(z[1] & 0x20), R2_ERR_IO,
             "bad zlib header in PNG");
  BitReader br{z.data() + 2, z.size() - 2};
  std::vector<uint8_t> out;
  out.reserve(expected);
  bool last = false;
  while (!last) {
    last = br.bits(1) != 0;
    const uint32_t type = br.bits(2);
    if (type == 0) {
      br.align();
      const size_t at = br.pos >> 3;
      R2_REQUIRE(at + 4 <= br.n, R2_ERR_IO, "truncated stored block");
      const uint32_t len = br.p[at] | (br.p[at + 1] << 8), nlen = br.p[at + 2] | (br.p[at + 3] << 8);
      R2_REQUIRE((len ^ 0xFFFFu) == nlen, R2_ERR_IO, "bad stored block length");
      R2_REQUIRE(at + 4 + len <= br.n, R2_ERR_IO, "truncated stored block");
      out.insert(out.end(), br.p + at + 4, br.p + at + 4 + len);
      br.pos = (at + 4 + len) * 8;
    } else if (type == 1) {
      static Huffman fl, fd;
      static bool init = false;
      if (!init) {
        uint8_t l[288], d[30];
        for (int i = 0; i < 144; ++i) l[i] = 8;
        for (int i = 144; i < 256; ++i) l[i] = 9;
        for (int i = 256; i < 280; ++i) l[i] = 7;
        for (int i = 280; i < 288; ++i) l[i] = 8;
        for (int i = 0; i < 30; ++i) d[i] = 5;
        fl.build(l, 288);
        fd.build(d, 30);
        init = true;
      }
      inflate_block(br, fl, fd, out);
    } else if (type == 2) {
      const int hlit = (int)br.bits(5) + 257, hdist = (int)br.bits(5) + 1, hclen = (int)br.bits(4) + 4;
      static const uint8_t order[19] = {16, 17, 18, 0, 8, 7, 9, 6, 10, 5, 11, 4, 12, 3, 13, 2, 14, 1, 15};
      uint8_t cl[19] = {};
      for (int i = 0; i < hclen; ++i) cl[order[i]] = (uint8_t)br.bits(3);
      Huffman ch;
      ch.build(cl, 19);
      uint8_t lens[320] = {};
      int k = 0;
      while (k < hlit + hdist) {
        const int sym = ch.decode(br);
        if (sym < 16) {
          lens[k++] = (uint8_t)sym;
        } else {
          int rep = 0;
          uint8_t val = 0;
          if (sym == 16) {
            R2_REQUIRE(k > 0, R2_ERR_IO, "repeat without a previous length");
            val = lens[k - 1];
            rep = 3 + (int)br.bits(2);
          } else if (sym == 17) {
            rep = 3 + (int)br.bits(3);
          } else {
            rep = 11 + (int)br.bits(7);
          }
          R2_REQUIRE(k + rep <= hlit + hdist, R2_ERR_IO, "code lengths overflow");
          while (rep--) lens[k++] = val;
        }
      }
      Huffman lit, dist;
      lit.build(lens, hlit);
      dist.build(lens + hlit, hdist);
      inflate_block(br, lit, dist, out);
    } else {
      throw Error{R2_ERR_IO, "bad deflate block type"};
    }
  }
  return out;
}

uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }

int paeth(int a, int b, int c) {
  const int p = a + b - c, pa = p > a ? p - a : a - p, pb = p > b ? p - b : b - p, pc = p > c ? p - c : c - p;
  return (pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c);
}

}  // namespace

RgbaImage8 read_png(const std::string& path) {
  FILE* f = fopen(path.c_str(), "rb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path);
  std::vector<uint8_t> buf;
  uint8_t tmp[1 << 16];
  size_t got;
  while ((got = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + got);
  fclose(f);
  static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
  R2_REQUIRE(buf.size() >= 8 && memcmp(buf.data(), sig, 8) == 0, R2_ERR_IO, path + " is not a PNG file");
  uint32_t W = 0, H = 0;
  int depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat, plte, trns;
  size_t pos = 8;
  while (pos + 12 <= buf.size()) {
    const uint32_t len = be32(&buf[pos]);
    R2_REQUIRE(pos + 12 + (size_t)len <= buf.size(), R2_ERR_IO, "truncated chunk in " + path);
    const std::string type((const char*)&buf[pos + 4], 4);
    const uint8_t* d = &buf[pos + 8];
    if (type == "IHDR") {
      R2_REQUIRE(len == 13, R2_ERR_IO, "bad IHDR in " + path);
      W = be32(d);
      H = be32(d + 4);
      depth = d[8];
      ctype = d[9];
      interlace = d[12];
    } else if (type == "PLTE") {
      plte.assign(d, d + len);
    } else if (type == "tRNS") {
      trns.assign(d, d + len);
    } else if (type == "IDAT") {
      idat.insert(idat.end(), d, d + len);
    } else if (type == "IEND") {
      break;
    }
    pos += 12 + len;
  }
  R2_REQUIRE(W > 0 && H > 0 && W < (1u << 16) && H < (1u << 16), R2_ERR_IO, "bad PNG size in " + path);
  R2_REQUIRE(interlace == 0, R2_ERR_UNSUPPORTED, "interlaced PNG not supported: " + path);
  const int samples = ctype == 0 ? 1 : ctype == 2 ? 3 : ctype == 3 ? 1 : ctype == 4 ? 2 : ctype == 6 ? 4 : 0;
  R2_REQUIRE(samples > 0, R2_ERR_IO, "bad PNG colour type in " + path);
  R2_REQUIRE(depth == 8 || depth == 16 || ((ctype == 0 || ctype == 3) && (depth == 1 || depth == 2 || depth == 4)),
             R2_ERR_UNSUPPORTED, "unsupported PNG bit depth in " + path);
  R2_REQUIRE(ctype != 3 || !plte.empty(), R2_ERR_IO, "palette PNG without PLTE: " + path);
  const size_t bitsPerPixel = (size_t)samples * depth;
  const size_t stride = (W * bitsPerPixel + 7) / 8, bpp = (bitsPerPixel + 7) / 8;
  std::vector<uint8_t> raw = zlib_inflate(idat, (stride + 1) * H);
  R2_REQUIRE(raw.size() >= (stride + 1) * H, R2_ERR_IO, "short image data in " + path);
  std::vector<uint8_t> cur(stride), prev(stride, 0);
  RgbaImage8 img;
  img.width = W;
  img.height = H;
  img.channels = (ctype == 3) ? (trns.empty() ? 3 : 4) : samples;  // colour-key tRNS of grey/RGB is ignored
  img.rgba.resize((size_t)W * H * 4);
  for (uint32_t y = 0; y < H; ++y) {
    const uint8_t* row = &raw[(size_t)y * (stride + 1)];
    const int filter = row[0];
    for (size_t i = 0; i < stride; ++i) {
      const int a = i >= bpp ? cur[i - bpp] : 0, b = prev[i], c = i >= bpp ? prev[i - bpp] : 0;
      int v = row[1 + i];
      switch (filter) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) >> 1; break;
        case 4: v += paeth(a, b, c); break;
        default: throw Error{R2_ERR_IO, "bad PNG filter in " + path};
      }
      cur[i] = (uint8_t)v;
    }
    for (uint32_t x = 0; x < W; ++x) {
      uint8_t* o = &img.rgba[((size_t)y * W + x) * 4];
      auto sample = [&](int s) -> int {  // sample s of pixel x at the image's depth, as 8 bits
        if (depth == 8) return cur[x * samples + s];
        if (depth == 16) return cur[(x * samples + s) * 2];
        const size_t bit = (size_t)x * depth;
        const int v = (cur[bit >> 3] >> (8 - depth - (int)(bit & 7))) & ((1 << depth) - 1);
        return ctype == 3 ? v : v * 255 / ((1 << depth) - 1);
      };
      if (ctype == 3) {
        const int k = sample(0);
        R2_REQUIRE((size_t)k * 3 + 2 < plte.size(), R2_ERR_IO, "palette index out of range in " + path);
        o[0] = plte[3 * k];
        o[1] = plte[3 * k + 1];
        o[2] = plte[3 * k + 2];
        o[3] = (size_t)k < trns.size() ? trns[k] : 255;
      } else if (ctype == 0 || ctype == 4) {
        o[0] = o[1] = o[2] = (uint8_t)sample(0);
        o[3] = ctype == 4 ? (uint8_t)sample(1) : 255;
      } else {
        o[0] = (uint8_t)sample(0);
        o[1] = (uint8_t)sample(1);
        o[2] = (uint8_t)sample(2);
        o[3] = ctype == 6 ? (uint8_t)sample(3) : 255;
      }
    }
    std::swap(cur, prev);
  }
  return img;
}

}  // namespace r2

// Baseline JPEG writer (ITU-T T.81 sequential DCT, Huffman, 8-bit, JFIF), the
// second output file of the reference's pipeline: output.jpg written by
// CImageWriter::writeToFile with quality 100 and the vertical flip
// (visualisation/src/image_writer.cpp:7-24, raytracer/pipeline.cu:72,84).
//
// Every component is sampled 1x1 (4:4:4), the quantisation tables are the
// standard Annex K.1 tables scaled by the IJG quality rule (quality 100 gives
// all-ones tables), and the Huffman tables are the typical tables of Annex K.3.
// The forward DCT is the exact separable cosine transform in double precision.
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <string>
#include <vector>

#include "asset_io.h"
#include "runtime.h"

namespace r2 {
namespace {

// natural (row-major) index of zigzag position k
const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                             12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                             35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                             58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

const uint8_t kLumaQ[64] = {16, 11, 10, 16, 24,  40,  51,  61,  12, 12, 14, 19, 26,  58,  60,  55,
                            14, 13, 16, 24, 40,  57,  69,  56,  14, 17, 22, 29, 51,  87,  80,  62,
                            18, 22, 37, 56, 68,  109, 103, 77,  24, 35, 55, 64, 81,  104, 113, 92,
                            49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99};
const uint8_t kChromaQ[64] = {17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99,
                              24, 26, 56, 99, 99, 99, 99, 99, 47, 66, 99, 99, 99, 99, 99, 99,
                              99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99,
                              99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99};

// Huffman table specifications: code counts per length 1..16, then symbols.
const uint8_t kDcLumaBits[16] = {0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0};
const uint8_t kDcChromaBits[16] = {0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0};
const uint8_t kDcVals[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
const uint8_t kAcLumaBits[16] = {0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d};
const uint8_t kAcLumaVals[162] = {
    0x01, 0x02, 0x03, 0x00, 0x04, 0x11, 0x05, 0x12, 0x21, 0x31, 0x41, 0x06, 0x13, 0x51, 0x61, 0x07, 0x22, 0x71,
    0x14, 0x32, 0x81, 0x91, 0xa1, 0x08, 0x23, 0x42, 0xb1, 0xc1, 0x15, 0x52, 0xd1, 0xf0, 0x24, 0x33, 0x62, 0x72,
    0x82, 0x09, 0x0a, 0x16, 0x17, 0x18, 0x19, 0x1a, 0x25, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x34, 0x35, 0x36, 0x37,
    0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59,
    0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x83,
    0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3,
    0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3,
    0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe1, 0xe2,
    0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};
const uint8_t kAcChromaBits[16] = {0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77};
const uint8_t kAcChromaVals[162] = {
    0x00, 0x01, 0x02, 0x03, 0x11, 0x04, 0x05, 0x21, 0x31, 0x06, 0x12, 0x41, 0x51, 0x07, 0x61, 0x71, 0x13, 0x22,
    0x32, 0x81, 0x08, 0x14, 0x42, 0x91, 0xa1, 0xb1, 0xc1, 0x09, 0x23, 0x33, 0x52, 0xf0, 0x15, 0x62, 0x72, 0xd1,
    0x0a, 0x16, 0x24, 0x34, 0xe1, 0x25, 0xf1, 0x17, 0x18, 0x19, 0x1a, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x35, 0x36,
    0x37, 0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58,
    0x59, 0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a,
    0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a,
    0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba,
    0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda,
    0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};

// Canonical codes of a table specification (T.81 Annex C): code and length per symbol.
struct HuffTable {
  uint16_t code[256];
  uint8_t len[256];
};
HuffTable make_table(const uint8_t* bits, const uint8_t* vals) {
  HuffTable t = {};
  uint16_t code = 0;
  int k = 0;
  for (int l = 1; l <= 16; ++l) {
    for (int i = 0; i < bits[l - 1]; ++i, ++k) {
      t.code[vals[k]] = code++;
      t.len[vals[k]] = (uint8_t)l;
    }
    code <<= 1;
  }
  return t;
}

struct BitWriter {
  std::vector<uint8_t>& out;
  uint32_t acc = 0;
  int n = 0;
  explicit BitWriter(std::vector<uint8_t>& o) : out(o) {}
  void put(uint32_t bits, int len) {
    for (int i = len - 1; i >= 0; --i) {
      acc = (acc << 1) | ((bits >> i) & 1u);
      if (++n == 8) {
        out.push_back((uint8_t)acc);
        if (acc == 0xFF) out.push_back(0x00);  // byte stuffing
        acc = 0;
        n = 0;
      }
    }
  }
  void flush() {
    while (n != 0) put(1, 1);  // pad with one bits
  }
};

// Magnitude category and the value's low bits (T.81 F.1.2.1).
void magnitude(int v, int* cat, uint32_t* bits) {
  int a = v < 0 ? -v : v, c = 0;
  while (a) {
    ++c;
    a >>= 1;
  }
  *cat = c;
  *bits = (uint32_t)(v < 0 ? v + (1 << c) - 1 : v) & ((1u << c) - 1u);
}

void encode_block(BitWriter& bw, const int* zz, int* prevDc, const HuffTable& dc, const HuffTable& ac) {
  int cat;
  uint32_t bits;
  magnitude(zz[0] - *prevDc, &cat, &bits);
  *prevDc = zz[0];
  bw.put(dc.code[cat], dc.len[cat]);
  bw.put(bits, cat);
  int run = 0;
  for (int k = 1; k < 64; ++k) {
    if (zz[k] == 0) {
      ++run;
      continue;
    }
    while (run > 15) {
      bw.put(ac.code[0xF0], ac.len[0xF0]);  // ZRL
      run -= 16;
    }
    magnitude(zz[k], &cat, &bits);
    const int sym = (run << 4) | cat;
    bw.put(ac.code[sym], ac.len[sym]);
    bw.put(bits, cat);
    run = 0;
  }
  if (run > 0) bw.put(ac.code[0x00], ac.len[0x00]);  // EOB
}

void put16(std::vector<uint8_t>& o, int v) {
  o.push_back((uint8_t)(v >> 8));
  o.push_back((uint8_t)(v & 0xFF));
}

}  // namespace

void write_jpg(const std::string& path, const uint8_t* rgb, uint32_t width, uint32_t height, bool flipVertical,
               int quality) {
  R2_REQUIRE(rgb && width > 0 && height > 0, R2_ERR_INVALID_ARGUMENT, "empty image");
  R2_REQUIRE(width < 65536 && height < 65536, R2_ERR_UNSUPPORTED, "JPEG images are at most 65535 pixels wide and high");
  quality = quality < 1 ? 1 : (quality > 100 ? 100 : quality);
  const int scale = quality < 50 ? 5000 / quality : 200 - 2 * quality;  // IJG quality rule
  int q[2][64];
  for (int i = 0; i < 64; ++i) {
    const int a = (kLumaQ[i] * scale + 50) / 100, b = (kChromaQ[i] * scale + 50) / 100;
    q[0][i] = a < 1 ? 1 : (a > 255 ? 255 : a);
    q[1][i] = b < 1 ? 1 : (b > 255 ? 255 : b);
  }
  std::vector<uint8_t> out = {0xFF, 0xD8};  // SOI
  // APP0 JFIF 1.01, aspect 1:1
  out.insert(out.end(), {0xFF, 0xE0, 0x00, 0x10, 'J', 'F', 'I', 'F', 0x00, 0x01, 0x01, 0x00, 0x00, 0x01, 0x00, 0x01,
                         0x00, 0x00});
  for (int t = 0; t < 2; ++t) {  // DQT, zigzag order
    out.insert(out.end(), {0xFF, 0xDB, 0x00, 0x43, (uint8_t)t});
    for (int k = 0; k < 64; ++k) out.push_back((uint8_t)q[t][kZigzag[k]]);
  }
  // SOF0: 8-bit, H x W, three components sampled 1x1 (Y uses table 0, Cb/Cr table 1)
  out.insert(out.end(), {0xFF, 0xC0, 0x00, 0x11, 0x08});
  put16(out, (int)height);
  put16(out, (int)width);
  out.insert(out.end(), {0x03, 0x01, 0x11, 0x00, 0x02, 0x11, 0x01, 0x03, 0x11, 0x01});
  auto dht = [&](int cls, int id, const uint8_t* bits, const uint8_t* vals) {
    int nv = 0;
    for (int i = 0; i < 16; ++i) nv += bits[i];
    out.insert(out.end(), {0xFF, 0xC4});
    put16(out, 2 + 1 + 16 + nv);
    out.push_back((uint8_t)((cls << 4) | id));
    out.insert(out.end(), bits, bits + 16);
    out.insert(out.end(), vals, vals + nv);
  };
  dht(0, 0, kDcLumaBits, kDcVals);
  dht(1, 0, kAcLumaBits, kAcLumaVals);
  dht(0, 1, kDcChromaBits, kDcVals);
  dht(1, 1, kAcChromaBits, kAcChromaVals);
  // SOS: components 1..3 with tables (0,0), (1,1), (1,1); full spectral range
  out.insert(out.end(), {0xFF, 0xDA, 0x00, 0x0C, 0x03, 0x01, 0x00, 0x02, 0x11, 0x03, 0x11, 0x00, 0x3F, 0x00});
  const HuffTable dcL = make_table(kDcLumaBits, kDcVals), acL = make_table(kAcLumaBits, kAcLumaVals);
  const HuffTable dcC = make_table(kDcChromaBits, kDcVals), acC = make_table(kAcChromaBits, kAcChromaVals);
  double cosT[8][8];  // C(u)/2 cos((2x + 1) u pi / 16)
  for (int u = 0; u < 8; ++u)
    for (int x = 0; x < 8; ++x)
      cosT[u][x] = (u == 0 ? sqrt(0.5) : 1.0) * 0.5 * cos((2.0 * x + 1.0) * u * 3.14159265358979323846 / 16.0);
  BitWriter bw(out);
  int prev[3] = {0, 0, 0};
  const uint32_t bw8 = (width + 7) / 8, bh8 = (height + 7) / 8;
  for (uint32_t by = 0; by < bh8; ++by) {
    for (uint32_t bx = 0; bx < bw8; ++bx) {
      double blk[3][64];
      for (int y = 0; y < 8; ++y) {
        const uint32_t ry = std::min(by * 8 + (uint32_t)y, height - 1);  // edge pixels repeat
        const uint32_t sy = flipVertical ? height - 1 - ry : ry;
        for (int x = 0; x < 8; ++x) {
          const uint32_t sx = std::min(bx * 8 + (uint32_t)x, width - 1);
          const uint8_t* p = rgb + 3 * ((size_t)sy * width + sx);
          const double r = p[0], g = p[1], b = p[2];
          blk[0][8 * y + x] = 0.299 * r + 0.587 * g + 0.114 * b - 128.0;
          blk[1][8 * y + x] = -0.168735892 * r - 0.331264108 * g + 0.5 * b;
          blk[2][8 * y + x] = 0.5 * r - 0.418687589 * g - 0.081312411 * b;
        }
      }
      for (int c = 0; c < 3; ++c) {
        double tmp[64], F[64];
        for (int y = 0; y < 8; ++y)  // rows
          for (int u = 0; u < 8; ++u) {
            double s = 0.0;
            for (int x = 0; x < 8; ++x) s += cosT[u][x] * blk[c][8 * y + x];
            tmp[8 * y + u] = s;
          }
        for (int u = 0; u < 8; ++u)  // columns
          for (int v = 0; v < 8; ++v) {
            double s = 0.0;
            for (int y = 0; y < 8; ++y) s += cosT[v][y] * tmp[8 * y + u];
            F[8 * v + u] = s;
          }
        int zz[64];
        const int* qt = q[c == 0 ? 0 : 1];
        for (int k = 0; k < 64; ++k) {
          const int i = kZigzag[k];
          zz[k] = (int)lround(F[i] / qt[i]);
        }
        encode_block(bw, zz, &prev[c], c == 0 ? dcL : dcC, c == 0 ? acL : acC);
      }
    }
  }
  bw.flush();
  out.insert(out.end(), {0xFF, 0xD9});  // EOI
  FILE* f = fopen(path.c_str(), "wb");
  R2_REQUIRE(f, R2_ERR_IO, "cannot open " + path + " for writing");
  bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
  ok = (fclose(f) == 0) && ok;
  R2_REQUIRE(ok, R2_ERR_IO, "short write to " + path);
}

}  // namespace r2

// rdb_palette_png.cpp -- rdither's palette image files (--palette-export and
// --palette-from with an image path), in the PNG form.
//
// Writer: src/rd_im.cpp:1047-1118 (ImWritePalette, image branch): a 1 x N strip,
// one pixel per palette entry, written through ImageMagick's PNG8 coder, so an
// 8-bit indexed PNG whose pixel i is entry i with each channel narrowed by
// ImageMagick's ScaleQuantumToChar (q <= 0 -> 0, q / 257 >= 255 -> 255, else
// q / 257 + 0.5 truncated, in double).  This writer emits that strip as a
// colour-type-3 PNG (PLTE = the N narrowed colours, pixel i = index i, one
// IDAT, zlib's default compression).  ImageMagick also writes ancillary chunks
// (gAMA, cHRM, tIME, text); none of them affects the colours a reader gets.
//
// Reader: src/rd_im.cpp:1362-1388 (ImReadPalette, image branch) and
// :731-888 (ImAdoptPaletteFromColormap): an image with a colormap (an indexed
// PNG: its PLTE, alpha from tRNS) gives its colormap entries in order; any
// other image gives its distinct RGB values in scan order, opaque.  Channel
// values are Q16: 8-bit samples scale by 257, 16-bit samples are taken as
// they are.  `expect_colors` > 0 must equal the number of colours the image
// holds.  Exact duplicates are dropped, and the tree is built from a swatch
// image -- each colour an 8 x 8 square, ceil(sqrt(n)) squares per row -- with
// as many colours as entries, no alpha association, greyscale when every
// entry is grey; the tree's colormap is the palette.  (ImageMagick may attach
// a 2^depth-entry grey colormap to a greyscale PNG; this reader takes such an
// image's distinct grey values instead.)
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rdb.h"
#include "rdb_numeric.h"
#include "rdb_runtime.h"

namespace rdb {
namespace {

constexpr unsigned char kSignature[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};

void Put32(std::vector<unsigned char>* v, uint32_t x) {
  v->push_back(static_cast<unsigned char>(x >> 24));
  v->push_back(static_cast<unsigned char>(x >> 16));
  v->push_back(static_cast<unsigned char>(x >> 8));
  v->push_back(static_cast<unsigned char>(x));
}

uint32_t Get32(const unsigned char* p) {
  return (static_cast<uint32_t>(p[0]) << 24) | (static_cast<uint32_t>(p[1]) << 16) |
         (static_cast<uint32_t>(p[2]) << 8) | static_cast<uint32_t>(p[3]);
}

void Chunk(std::vector<unsigned char>* out, const char* type, const std::vector<unsigned char>& data) {
  Put32(out, static_cast<uint32_t>(data.size()));
  const std::size_t at = out->size();
  out->insert(out->end(), type, type + 4);
  out->insert(out->end(), data.begin(), data.end());
  const uLong crc = crc32(0L, out->data() + at, static_cast<uInt>(4 + data.size()));
  Put32(out, static_cast<uint32_t>(crc));
}

// ImageMagick's ScaleQuantumToChar for a Q16 HDRI quantum (a float).
unsigned char QuantumToChar(double v) {
  const double q = static_cast<double>(static_cast<float>(v));
  if (!(q > 0.0)) return 0;
  if (q / 257.0 >= 255.0) return 255;
  return static_cast<unsigned char>(q / 257.0 + 0.5);
}

int Paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  if (pb <= pc) return b;
  return c;
}

// Reverses the row filters of one (sub-)image in place: `rows` rows of
// `row_bytes` bytes, each preceded by its filter byte, `bpp` bytes per
// complete pixel (at least 1).
bool Unfilter(unsigned char* data, std::size_t rows, std::size_t row_bytes, std::size_t bpp,
              std::vector<unsigned char>* out) {
  out->assign(rows * row_bytes, 0);
  for (std::size_t y = 0; y < rows; ++y) {
    const unsigned char* src = data + y * (row_bytes + 1);
    const int filter = src[0];
    ++src;
    unsigned char* cur = out->data() + y * row_bytes;
    const unsigned char* prev = y ? cur - row_bytes : nullptr;
    for (std::size_t x = 0; x < row_bytes; ++x) {
      const int a = x >= bpp ? cur[x - bpp] : 0;
      const int b = prev ? prev[x] : 0;
      const int c = (prev && x >= bpp) ? prev[x - bpp] : 0;
      int v = src[x];
      switch (filter) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += b; break;
        case 3: v += (a + b) >> 1; break;
        case 4: v += Paeth(a, b, c); break;
        default: return false;
      }
      cur[x] = static_cast<unsigned char>(v);
    }
  }
  return true;
}

struct Png {
  uint32_t width = 0, height = 0;
  int depth = 0, color = 0, interlace = 0;
  std::vector<unsigned char> plte, trns;
  std::vector<uint16_t> samples;  // width * height * channels, at the file's depth
  int channels = 0;
};

int Decode(const std::string& path, Png* png) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return Fail(RDB_E_INVALID, "cannot open " + path + " for reading");
  std::vector<unsigned char> file;
  unsigned char buf[1 << 16];
  std::size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) file.insert(file.end(), buf, buf + got);
  std::fclose(f);
  if (file.size() < 8 || std::memcmp(file.data(), kSignature, 8) != 0) {
    return Fail(RDB_E_UNSUPPORTED, path + " is not a PNG file (the image form of a palette is read "
                                          "as PNG here)");
  }
  std::vector<unsigned char> idat;
  bool have_header = false, ended = false;
  for (std::size_t at = 8; at + 12 <= file.size() && !ended;) {
    const uint32_t len = Get32(file.data() + at);
    if (len > file.size() - at - 12) return Fail(RDB_E_INVALID, path + ": truncated PNG chunk");
    const unsigned char* type = file.data() + at + 4;
    const unsigned char* data = type + 4;
    const uLong crc = crc32(0L, type, len + 4);
    if (crc != Get32(data + len)) return Fail(RDB_E_INVALID, path + ": PNG chunk CRC mismatch");
    if (!std::memcmp(type, "IHDR", 4) && len == 13) {
      png->width = Get32(data);
      png->height = Get32(data + 4);
      png->depth = data[8];
      png->color = data[9];
      png->interlace = data[12];
      have_header = true;
    } else if (!std::memcmp(type, "PLTE", 4)) {
      png->plte.assign(data, data + len);
    } else if (!std::memcmp(type, "tRNS", 4)) {
      png->trns.assign(data, data + len);
    } else if (!std::memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), data, data + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      ended = true;
    }
    at += 12 + len;
  }
  if (!have_header || png->width == 0 || png->height == 0) return Fail(RDB_E_INVALID, path + ": no PNG header");
  static const int kChannels[7] = {1, 0, 3, 1, 2, 0, 4};
  if (png->color > 6 || kChannels[png->color] == 0 || png->interlace > 1) {
    return Fail(RDB_E_INVALID, path + ": unknown PNG colour type or interlace method");
  }
  png->channels = kChannels[png->color];
  const int d = png->depth;
  const bool depth_ok = (d == 8 || d == 16) || (png->color == 0 && (d == 1 || d == 2 || d == 4)) ||
                        (png->color == 3 && (d == 1 || d == 2 || d == 4));
  if (!depth_ok || (png->color == 3 && d == 16)) return Fail(RDB_E_INVALID, path + ": bad PNG bit depth");
  if (png->color == 3 && (png->plte.empty() || png->plte.size() % 3)) {
    return Fail(RDB_E_INVALID, path + ": indexed PNG without a palette");
  }
  if (static_cast<uint64_t>(png->width) * png->height > (uint64_t{1} << 28)) {
    return Fail(RDB_E_UNSUPPORTED, path + ": image too large for a palette");
  }
  // Inflate.
  std::vector<unsigned char> raw;
  z_stream zs{};
  if (inflateInit(&zs) != Z_OK) return Fail(RDB_E_INVALID, "zlib inflateInit failed");
  zs.next_in = idat.data();
  zs.avail_in = static_cast<uInt>(idat.size());
  int zr = Z_OK;
  while (zr == Z_OK) {
    zs.next_out = buf;
    zs.avail_out = sizeof buf;
    zr = inflate(&zs, Z_NO_FLUSH);
    raw.insert(raw.end(), buf, buf + (sizeof buf - zs.avail_out));
    if (zr == Z_BUF_ERROR && zs.avail_in == 0) break;
  }
  inflateEnd(&zs);
  if (zr != Z_STREAM_END) return Fail(RDB_E_INVALID, path + ": corrupt PNG image data");
  const std::size_t bits_px = static_cast<std::size_t>(png->channels) * d;
  const std::size_t bpp = std::max<std::size_t>(1, bits_px / 8);
  const std::size_t W = png->width, H = png->height;
  png->samples.assign(W * H * png->channels, 0);
  // Passes: the whole image, or Adam7's seven (start x, start y, step x, step y).
  static const int kAdam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                   {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
  const int passes = png->interlace ? 7 : 1;
  std::size_t at = 0;
  std::vector<unsigned char> rows;
  for (int p = 0; p < passes; ++p) {
    const std::size_t x0 = png->interlace ? kAdam7[p][0] : 0, y0 = png->interlace ? kAdam7[p][1] : 0;
    const std::size_t sx = png->interlace ? kAdam7[p][2] : 1, sy = png->interlace ? kAdam7[p][3] : 1;
    if (x0 >= W || y0 >= H) continue;
    const std::size_t pw = (W - x0 + sx - 1) / sx, ph = (H - y0 + sy - 1) / sy;
    const std::size_t row_bytes = (pw * bits_px + 7) / 8;
    if (raw.size() - at < ph * (row_bytes + 1)) return Fail(RDB_E_INVALID, path + ": short PNG image data");
    if (!Unfilter(raw.data() + at, ph, row_bytes, bpp, &rows)) {
      return Fail(RDB_E_INVALID, path + ": bad PNG row filter");
    }
    at += ph * (row_bytes + 1);
    for (std::size_t y = 0; y < ph; ++y) {
      const unsigned char* r = rows.data() + y * row_bytes;
      for (std::size_t x = 0; x < pw; ++x) {
        uint16_t* dst = png->samples.data() + ((y0 + y * sy) * W + (x0 + x * sx)) * png->channels;
        for (int c = 0; c < png->channels; ++c) {
          const std::size_t bit = (x * png->channels + c) * d;
          uint16_t v;
          if (d == 16) {
            v = static_cast<uint16_t>((r[bit / 8] << 8) | r[bit / 8 + 1]);
          } else if (d == 8) {
            v = r[bit / 8];
          } else {
            v = static_cast<uint16_t>((r[bit / 8] >> (8 - d - bit % 8)) & ((1 << d) - 1));
          }
          dst[c] = v;
        }
      }
    }
  }
  return RDB_OK;
}

struct Entry {
  double r, g, b, a;
};

}  // namespace

int WritePalettePng(const double* colors, int count, const std::string& path) {
  if (count <= 0) return Fail(RDB_E_INVALID, "palette is empty");
  if (count > 256) return Fail(RDB_E_UNSUPPORTED, "an indexed PNG holds at most 256 colours");
  std::vector<unsigned char> out(kSignature, kSignature + 8);
  std::vector<unsigned char> ihdr;
  Put32(&ihdr, static_cast<uint32_t>(count));
  Put32(&ihdr, 1u);
  ihdr.insert(ihdr.end(), {8, 3, 0, 0, 0});  // depth 8, indexed, deflate, no filter, no interlace
  Chunk(&out, "IHDR", ihdr);
  std::vector<unsigned char> plte;
  for (int i = 0; i < count; ++i) {
    const double* e = colors + 4 * static_cast<std::size_t>(i);
    plte.push_back(QuantumToChar(e[0]));
    plte.push_back(QuantumToChar(e[1]));
    plte.push_back(QuantumToChar(e[2]));
  }
  Chunk(&out, "PLTE", plte);
  std::vector<unsigned char> row(static_cast<std::size_t>(count) + 1);
  row[0] = 0;  // filter: none
  for (int i = 0; i < count; ++i) row[static_cast<std::size_t>(i) + 1] = static_cast<unsigned char>(i);
  uLongf zlen = compressBound(static_cast<uLong>(row.size()));
  std::vector<unsigned char> z(zlen);
  if (compress(z.data(), &zlen, row.data(), static_cast<uLong>(row.size())) != Z_OK) {
    return Fail(RDB_E_INVALID, "zlib compress failed");
  }
  z.resize(zlen);
  Chunk(&out, "IDAT", z);
  Chunk(&out, "IEND", {});
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return Fail(RDB_E_INVALID, "cannot open " + path + " for writing");
  const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  return (std::fclose(f) == 0 && ok) ? RDB_OK : Fail(RDB_E_INVALID, "cannot write " + path);
}

int ReadPalettePng(const std::string& path, int expect_colors, std::vector<float>* swatch,
                   std::size_t* width, std::size_t* height, int* count, bool* grayscale) {
  Png png;
  if (int rc = Decode(path, &png)) return rc;
  std::vector<Entry> pal;
  int held = 0;
  const auto q16 = [&](uint16_t v) {
    if (png.depth == 16) return static_cast<double>(v);
    if (png.depth == 8) return static_cast<double>(v) * 257.0;
    // 1, 2 and 4-bit grey widen to 8 bits by the PNG rule (v * 255 / max).
    const int maxv = (1 << png.depth) - 1;
    return static_cast<double>(v * 255 / maxv) * 257.0;
  };
  if (png.color == 3) {
    // The colormap: every PLTE entry in order, alpha from tRNS.
    const int n = static_cast<int>(png.plte.size() / 3);
    held = n;
    const int keep = expect_colors > 0 ? std::min(n, expect_colors) : n;
    for (int i = 0; i < keep; ++i) {
      const double a = static_cast<std::size_t>(i) < png.trns.size() ? png.trns[static_cast<std::size_t>(i)] * 257.0
                                                                      : kQuantumRange;
      pal.push_back(Entry{png.plte[3 * i] * 257.0, png.plte[3 * i + 1] * 257.0,
                          png.plte[3 * i + 2] * 257.0, a});
    }
  } else {
    // Distinct RGB values in scan order, opaque, up to the cap.
    const int limit = expect_colors > 0 ? expect_colors : 65536;
    const std::size_t n_px = static_cast<std::size_t>(png.width) * png.height;
    bool capped = false;
    for (std::size_t i = 0; i < n_px; ++i) {
      const uint16_t* s = png.samples.data() + i * png.channels;
      const bool grey = png.color == 0 || png.color == 4;
      const Entry e{q16(s[0]), q16(grey ? s[0] : s[1]), q16(grey ? s[0] : s[2]), kQuantumRange};
      bool dup = false;
      for (const Entry& k : pal) {
        if (k.r == e.r && k.g == e.g && k.b == e.b) {
          dup = true;
          break;
        }
      }
      if (dup) continue;
      if (static_cast<int>(pal.size()) == limit) {
        capped = true;
        break;
      }
      pal.push_back(e);
    }
    held = capped ? -1 : static_cast<int>(pal.size());
  }
  if (pal.empty()) return Fail(RDB_E_INVALID, path + ": the image has no colours");
  if (expect_colors > 0 && held != expect_colors) {
    return Fail(RDB_E_INVALID,
                path + (held < 0 ? ": the palette image holds more than " + std::to_string(expect_colors)
                                 : ": the palette image holds " + std::to_string(held)) +
                    " colours, not " + std::to_string(expect_colors));
  }
  // Exact duplicates dropped, first occurrence kept.
  std::vector<Entry> uniq;
  for (const Entry& e : pal) {
    bool dup = false;
    for (const Entry& k : uniq) {
      if (k.r == e.r && k.g == e.g && k.b == e.b) {
        dup = true;
        break;
      }
    }
    if (!dup) uniq.push_back(e);
  }
  const int n = static_cast<int>(uniq.size());
  const int block = std::max(1, static_cast<int>(std::ceil(std::sqrt(static_cast<double>(n)))));
  const int rows = (n + block - 1) / block;
  const std::size_t W = static_cast<std::size_t>(block) * 8, H = static_cast<std::size_t>(rows) * 8;
  swatch->assign(W * H * 4, 0.0f);
  bool gray = true;
  for (int i = 0; i < n; ++i) {
    const Entry& e = uniq[static_cast<std::size_t>(i)];
    if (e.r != e.g || e.g != e.b) gray = false;
    const std::size_t gx = static_cast<std::size_t>(i % block) * 8, gy = static_cast<std::size_t>(i / block) * 8;
    for (std::size_t y = 0; y < 8; ++y) {
      for (std::size_t x = 0; x < 8; ++x) {
        float* px = swatch->data() + ((gy + y) * W + gx + x) * 4;
        px[0] = static_cast<float>(e.r);
        px[1] = static_cast<float>(e.g);
        px[2] = static_cast<float>(e.b);
        px[3] = static_cast<float>(e.a);
      }
    }
  }
  *width = W;
  *height = H;
  *count = n;
  *grayscale = gray;
  return RDB_OK;
}

}  // namespace rdb

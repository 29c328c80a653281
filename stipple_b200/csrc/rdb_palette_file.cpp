// rdb_palette_file.cpp -- rdither's palette text files (--palette-export and
// --palette-from with a .txt or .text path).
//
// Writer: src/rd_im.cpp:994-1030 (ImWritePalette, text branch): two comment
// lines, then one tab-separated row per colour: index, r, g, b, a as Q16
// doubles with six decimals, and the 8-bit hex of r, g, b rounded as
// v / 257 + 0.5.
//
// Reader: src/rd_im.cpp:1175-1350 (ImReadPalette, text branch): every line
// that is not blank or a comment is "index r g b [a] [hex]"; the alpha column
// is read only when the hex column follows it; indices must be contiguous from
// 0; r, g, b are rounded through float; the colours are sorted by (r, g, b, a);
// the tree is then built from a one-row strip of them with as many colours as
// rows, no alpha association, greyscale when every row is grey, and must keep
// every colour.  The palette's alpha association is "some alpha is not opaque".
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/rdb.h"
#include "rdb_numeric.h"
#include "rdb_runtime.h"

namespace rdb {

bool PaletteTextPath(const std::string& path) {
  const auto ends = [&](const char* suffix) {
    const std::size_t n = std::char_traits<char>::length(suffix);
    return path.size() >= n && path.compare(path.size() - n, n, suffix) == 0;
  };
  return ends(".txt") || ends(".text");
}

int WritePaletteText(const double* colors, int count, const std::string& path) {
  if (count <= 0) return Fail(RDB_E_INVALID, "palette is empty");
  if (!PaletteTextPath(path)) {
    return Fail(RDB_E_UNSUPPORTED,
                "the text palette form takes .txt / .text paths; write the image form with "
                "rdb_palette_write_png");
  }
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return Fail(RDB_E_INVALID, "cannot open " + path + " for writing");
  std::fprintf(f, "# rdither palette, %d colours, Q16 (0..65535) and 8-bit hex\n", count);
  std::fprintf(f, "# count\tr\tg\tb\ta\thex\n");
  for (int i = 0; i < count; ++i) {
    const double* e = colors + 4 * static_cast<std::size_t>(i);
    const auto hex8 = [](double v) { return static_cast<unsigned>(v / 257.0 + 0.5); };
    std::fprintf(f, "%d\t%.6f\t%.6f\t%.6f\t%.6f\t%02X%02X%02X\n", i, e[0], e[1], e[2], e[3],
                 hex8(e[0]), hex8(e[1]), hex8(e[2]));
  }
  const bool ok = std::fclose(f) == 0;
  return ok ? RDB_OK : Fail(RDB_E_INVALID, "cannot write " + path);
}

int ReadPaletteText(const std::string& path, int expect_colors, std::vector<float>* strip,
                    int* count, bool* associate_alpha, bool* grayscale) {
  if (!PaletteTextPath(path)) {
    return Fail(RDB_E_UNSUPPORTED,
                "the text palette form takes .txt / .text paths; read the image form with "
                "rdb_palette_read_png");
  }
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return Fail(RDB_E_INVALID, "cannot open " + path + " for reading");
  struct Row {
    double r, g, b, a;
  };
  std::vector<Row> rows;
  std::vector<bool> seen;
  bool transparent = false;
  char line[512];
  int lineno = 0;
  while (std::fgets(line, sizeof line, f)) {
    ++lineno;
    if (line[0] == '#' || line[0] == '\n' || line[0] == '\r') continue;
    int index = 0;
    double r = 0.0, g = 0.0, b = 0.0;
    char fifth[32] = {0}, sixth[32] = {0};
    const int got = std::sscanf(line, "%d %lf %lf %lf %31s %31s", &index, &r, &g, &b, fifth, sixth);
    const std::string where = path + ": line " + std::to_string(lineno);
    if (got < 4) {
      std::fclose(f);
      return Fail(RDB_E_INVALID, where + " is not a palette row (want: index r g b [a] [hex])");
    }
    double alpha = kQuantumRange;
    if (got >= 6) {
      char* end = nullptr;
      const double v = std::strtod(fifth, &end);
      if (end == fifth || *end != '\0' || !(v >= 0.0 && v <= kQuantumRange)) {
        std::fclose(f);
        return Fail(RDB_E_INVALID, where + " alpha '" + fifth + "' is not a number in 0..65535");
      }
      alpha = v;
    }
    if (index < 0 || index >= 65536) {
      std::fclose(f);
      return Fail(RDB_E_INVALID, where + " index " + std::to_string(index) + " is out of range");
    }
    const std::size_t at = static_cast<std::size_t>(index);
    if (at >= rows.size()) {
      rows.resize(at + 1, Row{0.0, 0.0, 0.0, kQuantumRange});
      seen.resize(at + 1, false);
    }
    rows[at] = Row{r, g, b, alpha};
    seen[at] = true;
    if (alpha != kQuantumRange) transparent = true;
  }
  std::fclose(f);
  if (rows.empty()) return Fail(RDB_E_INVALID, path + " contains no palette rows");
  for (std::size_t i = 0; i < rows.size(); ++i) {
    if (!seen[i]) {
      return Fail(RDB_E_INVALID, path + ": no row declares index " + std::to_string(i) +
                                     " below the highest index " + std::to_string(rows.size() - 1));
    }
  }
  const int n = static_cast<int>(rows.size());
  if (expect_colors > 0 && n != expect_colors) {
    return Fail(RDB_E_INVALID, path + " holds " + std::to_string(n) + " colours, not " +
                                   std::to_string(expect_colors));
  }
  for (Row& e : rows) {
    e.r = static_cast<double>(static_cast<float>(e.r));
    e.g = static_cast<double>(static_cast<float>(e.g));
    e.b = static_cast<double>(static_cast<float>(e.b));
  }
  std::sort(rows.begin(), rows.end(), [](const Row& x, const Row& y) {
    if (x.r != y.r) return x.r < y.r;
    if (x.g != y.g) return x.g < y.g;
    if (x.b != y.b) return x.b < y.b;
    return x.a < y.a;
  });
  strip->assign(4 * rows.size(), 0.0f);
  bool gray = true;
  for (std::size_t i = 0; i < rows.size(); ++i) {
    (*strip)[4 * i + 0] = static_cast<float>(rows[i].r);
    (*strip)[4 * i + 1] = static_cast<float>(rows[i].g);
    (*strip)[4 * i + 2] = static_cast<float>(rows[i].b);
    (*strip)[4 * i + 3] = static_cast<float>(rows[i].a);
    if (rows[i].r != rows[i].g || rows[i].g != rows[i].b) gray = false;
  }
  *count = n;
  *associate_alpha = transparent;
  *grayscale = gray;
  return RDB_OK;
}

}  // namespace rdb

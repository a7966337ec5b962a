// Image I/O and hologram preprocessing for the command-line driver.
#include "rihvr_image.h"

#include "rihvr.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>

namespace rihvr_io {

namespace {

bool read_file(const std::string& path, std::vector<uint8_t>& buf) {
  std::ifstream f(path, std::ios::binary);
  if (!f) return false;
  buf.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

// cvtColor(BGR2GRAY) of 8-bit samples: 0.299 R + 0.587 G + 0.114 B in 15-bit
// fixed point, rounded (the OpenCV 4 coefficients; equal to cv2 4.13 on all
// 2^24 colours)
int gray8(int r, int g, int b) { return (r * 9798 + g * 19235 + b * 3735 + (1 << 14)) >> 15; }

struct Tiff {
  const std::vector<uint8_t>& d;
  bool le = true;
  explicit Tiff(const std::vector<uint8_t>& b) : d(b) {}
  bool ok(size_t off, size_t n) const { return off + n <= d.size(); }
  uint16_t u16(size_t o) const {
    return le ? (uint16_t)(d[o] | (d[o + 1] << 8)) : (uint16_t)((d[o] << 8) | d[o + 1]);
  }
  uint32_t u32(size_t o) const {
    return le ? (uint32_t)d[o] | ((uint32_t)d[o + 1] << 8) | ((uint32_t)d[o + 2] << 16) | ((uint32_t)d[o + 3] << 24)
              : ((uint32_t)d[o] << 24) | ((uint32_t)d[o + 1] << 16) | ((uint32_t)d[o + 2] << 8) | (uint32_t)d[o + 3];
  }
};

struct Entry {
  uint16_t tag, type;
  uint32_t count;
  size_t pos;  // position of the value field
};

bool entry_values(const Tiff& t, const Entry& e, std::vector<uint32_t>& v) {
  const size_t sz = e.type == 3 ? 2 : (e.type == 4 ? 4 : (e.type == 1 ? 1 : 0));
  if (!sz) return false;
  size_t off = e.pos;
  if (sz * e.count > 4) off = t.u32(e.pos);
  if (!t.ok(off, sz * e.count)) return false;
  v.resize(e.count);
  for (uint32_t i = 0; i < e.count; ++i)
    v[i] = sz == 2 ? t.u16(off + 2 * i) : (sz == 4 ? t.u32(off + 4 * i) : t.d[off + i]);
  return true;
}

bool unpack_bits(const uint8_t* s, size_t n, std::vector<uint8_t>& out) {
  size_t i = 0;
  while (i < n) {
    const int8_t c = (int8_t)s[i++];
    if (c >= 0) {
      const size_t k = (size_t)c + 1;
      if (i + k > n) return false;
      out.insert(out.end(), s + i, s + i + k);
      i += k;
    } else if (c != -128) {
      if (i >= n) return false;
      out.insert(out.end(), (size_t)(1 - c), s[i++]);
    }
  }
  return true;
}

// TIFF LZW: MSB-first codes of 9..12 bits, 256 = clear, 257 = end, the code
// width grows one code early (as libtiff writes it).
bool unlzw(const uint8_t* s, size_t n, std::vector<uint8_t>& out) {
  std::vector<std::vector<uint8_t>> table;
  auto reset = [&]() {
    table.assign(258, {});
    for (int i = 0; i < 256; ++i) table[i] = {(uint8_t)i};
  };
  reset();
  size_t bitpos = 0;
  int width = 9;
  int prev = -1;
  auto read = [&](int w) -> int {
    if ((bitpos + w + 7) / 8 > n) return 257;
    int v = 0;
    for (int k = 0; k < w; ++k, ++bitpos) v = (v << 1) | ((s[bitpos >> 3] >> (7 - (bitpos & 7))) & 1);
    return v;
  };
  for (;;) {
    const int code = read(width);
    if (code == 257) break;
    if (code == 256) {
      reset();
      width = 9;
      prev = -1;
      continue;
    }
    std::vector<uint8_t> entry;
    if (code < (int)table.size()) {
      entry = table[code];
      if (prev >= 0) {
        std::vector<uint8_t> add = table[prev];
        add.push_back(entry[0]);
        table.push_back(std::move(add));
      }
    } else if (code == (int)table.size() && prev >= 0) {
      entry = table[prev];
      entry.push_back(table[prev][0]);
      table.push_back(entry);
    } else {
      return false;
    }
    out.insert(out.end(), entry.begin(), entry.end());
    prev = code;
    if ((int)table.size() >= (1 << width) - 1 && width < 12) ++width;
  }
  return true;
}

bool read_tiff(const std::vector<uint8_t>& buf, Image& img, std::string& err) {
  Tiff t(buf);
  if (buf.size() < 8) return err = "file too short", false;
  if (buf[0] == 'I' && buf[1] == 'I') t.le = true;
  else if (buf[0] == 'M' && buf[1] == 'M') t.le = false;
  else return err = "not a TIFF file", false;
  if (t.u16(2) != 42) return err = "not a classic TIFF file", false;
  const size_t ifd = t.u32(4);
  if (!t.ok(ifd, 2)) return err = "bad IFD offset", false;
  const int n = t.u16(ifd);
  if (!t.ok(ifd + 2, 12 * (size_t)n)) return err = "truncated IFD", false;
  uint32_t W = 0, H = 0, bps = 8, comp = 1, photo = 1, spp = 1, rps = 0, pred = 1, planar = 1, fmt = 1;
  std::vector<uint32_t> offs, counts, v;
  for (int i = 0; i < n; ++i) {
    const size_t p = ifd + 2 + 12 * (size_t)i;
    Entry e{t.u16(p), t.u16(p + 2), t.u32(p + 4), p + 8};
    if (!entry_values(t, e, v) || v.empty()) continue;
    switch (e.tag) {
      case 256: W = v[0]; break;
      case 257: H = v[0]; break;
      case 258: bps = v[0]; break;
      case 259: comp = v[0]; break;
      case 262: photo = v[0]; break;
      case 273: offs = v; break;
      case 277: spp = v[0]; break;
      case 278: rps = v[0]; break;
      case 279: counts = v; break;
      case 284: planar = v[0]; break;
      case 317: pred = v[0]; break;
      case 339: fmt = v[0]; break;
      default: break;
    }
  }
  if (!W || !H) return err = "missing image size", false;
  if (bps != 8 && bps != 16) return err = "unsupported bits per sample " + std::to_string(bps), false;
  if (fmt != 1) return err = "only unsigned integer samples are supported", false;
  if (spp != 1 && spp != 3) return err = "unsupported samples per pixel " + std::to_string(spp), false;
  if (planar != 1 && spp > 1) return err = "planar RGB is not supported", false;
  if (comp != 1 && comp != 5 && comp != 32773) return err = "unsupported compression " + std::to_string(comp), false;
  if (offs.empty() || offs.size() != counts.size()) return err = "missing strip table", false;
  if (!rps || rps > H) rps = H;
  const size_t bytes_pp = (size_t)spp * (bps / 8);
  const size_t row_bytes = (size_t)W * bytes_pp;
  std::vector<uint8_t> raw;
  raw.reserve(row_bytes * H);
  for (size_t s = 0; s < offs.size(); ++s) {
    if (!t.ok(offs[s], counts[s])) return err = "strip outside the file", false;
    const uint8_t* src = buf.data() + offs[s];
    std::vector<uint8_t> strip;
    bool good = true;
    if (comp == 1) strip.assign(src, src + counts[s]);
    else if (comp == 32773) good = unpack_bits(src, counts[s], strip);
    else good = unlzw(src, counts[s], strip);
    if (!good) return err = "corrupt compressed strip", false;
    const size_t rows = std::min<size_t>(rps, H - s * rps);
    if (strip.size() < rows * row_bytes) return err = "short strip", false;
    strip.resize(rows * row_bytes);
    if (pred == 2) {  // horizontal differencing, per sample
      for (size_t r = 0; r < rows; ++r) {
        uint8_t* row = strip.data() + r * row_bytes;
        if (bps == 8) {
          for (size_t i = spp; i < row_bytes; ++i) row[i] = (uint8_t)(row[i] + row[i - spp]);
        } else {
          for (size_t i = spp; i < (size_t)W * spp; ++i) {
            auto rd = [&](size_t k) { return t.le ? (uint16_t)(row[2 * k] | (row[2 * k + 1] << 8))
                                                  : (uint16_t)((row[2 * k] << 8) | row[2 * k + 1]); };
            const uint16_t val = (uint16_t)(rd(i) + rd(i - spp));
            if (t.le) { row[2 * i] = val & 0xff; row[2 * i + 1] = val >> 8; }
            else { row[2 * i] = val >> 8; row[2 * i + 1] = val & 0xff; }
          }
        }
      }
    }
    raw.insert(raw.end(), strip.begin(), strip.end());
  }
  img.width = (int)W;
  img.height = (int)H;
  img.bits = (int)bps;
  img.pixels.assign((size_t)W * H, 0.f);
  const double maxv = bps == 8 ? 255.0 : 65535.0;
  for (size_t i = 0; i < (size_t)W * H; ++i) {
    double s[3] = {0, 0, 0};
    for (uint32_t c = 0; c < spp; ++c) {
      const size_t k = i * spp + c;
      s[c] = bps == 8 ? raw[k] : (t.le ? (raw[2 * k] | (raw[2 * k + 1] << 8)) : ((raw[2 * k] << 8) | raw[2 * k + 1]));
    }
    double g = s[0];
    if (spp == 3) {  // imread gives BGR; cvtColor(BGR2GRAY) weights R, G, B
      g = bps == 8 ? (double)gray8((int)s[0], (int)s[1], (int)s[2])
                   : std::nearbyint(0.299 * s[0] + 0.587 * s[1] + 0.114 * s[2]);
    }
    if (photo == 0) g = maxv - g;
    img.pixels[i] = (float)g;
  }
  return true;
}

bool read_pnm(const std::vector<uint8_t>& buf, Image& img, std::string& err) {
  size_t p = 2;
  auto next_int = [&](long& v) -> bool {
    while (p < buf.size()) {
      if (buf[p] == '#') { while (p < buf.size() && buf[p] != '\n') ++p; }
      else if (std::isspace(buf[p])) ++p;
      else break;
    }
    if (p >= buf.size() || !std::isdigit(buf[p])) return false;
    v = 0;
    while (p < buf.size() && std::isdigit(buf[p])) v = v * 10 + (buf[p++] - '0');
    return true;
  };
  long W, H, M;
  if (!next_int(W) || !next_int(H) || !next_int(M)) return err = "bad PGM header", false;
  ++p;
  const int bpp = M > 255 ? 2 : 1;
  if (p + (size_t)W * H * bpp > buf.size()) return err = "short PGM", false;
  img.width = (int)W;
  img.height = (int)H;
  img.bits = bpp == 1 ? 8 : 16;
  img.pixels.resize((size_t)W * H);
  for (size_t i = 0; i < (size_t)W * H; ++i)
    img.pixels[i] = bpp == 1 ? buf[p + i] : (float)((buf[p + 2 * i] << 8) | buf[p + 2 * i + 1]);
  return true;
}

uint32_t be32(const uint8_t* p) { return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3]; }

// PNG (ISO/IEC 15948): non-interlaced 8/16-bit grayscale or 8-bit RGB, as
// Hologram::read accepts after imread (hologram.cu:146-183: CV_8U, CV_16U,
// and CV_8UC3 converted to gray).
bool read_png(const std::vector<uint8_t>& buf, Image& img, std::string& err) {
  size_t p = 8;
  uint32_t W = 0, H = 0;
  int depth = 0, color = -1, interlace = 0;
  std::vector<uint8_t> z;
  bool end = false;
  while (!end) {
    if (p + 12 > buf.size()) return err = "truncated PNG", false;
    const uint32_t len = be32(&buf[p]);
    const uint8_t* type = &buf[p + 4];
    const uint8_t* data = &buf[p + 8];
    if (len > buf.size() - p - 12) return err = "truncated PNG chunk", false;
    if (crc32(crc32(0L, Z_NULL, 0), type, len + 4) != be32(data + len)) return err = "PNG chunk CRC mismatch", false;
    if (!std::memcmp(type, "IHDR", 4)) {
      if (len != 13) return err = "bad PNG header", false;
      W = be32(data);
      H = be32(data + 4);
      depth = data[8];
      color = data[9];
      interlace = data[12];
    } else if (!std::memcmp(type, "IDAT", 4)) {
      z.insert(z.end(), data, data + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      end = true;
    }
    p += 12 + (size_t)len;
  }
  if (!W || !H) return err = "missing PNG header", false;
  if (interlace) return err = "interlaced PNG is not supported", false;
  int ch;
  if (color == 0 && (depth == 8 || depth == 16)) ch = 1;
  else if (color == 2 && depth == 8) ch = 3;
  else return err = "unsupported PNG type (color " + std::to_string(color) + ", depth " + std::to_string(depth) +
                    "): 8/16-bit grayscale or 8-bit RGB", false;
  const size_t bpp = (size_t)ch * (depth / 8), row = (size_t)W * bpp;
  std::vector<uint8_t> raw((row + 1) * H);
  uLongf got = (uLongf)raw.size();
  if (uncompress(raw.data(), &got, z.data(), (uLong)z.size()) != Z_OK || got != raw.size())
    return err = "corrupt PNG image data", false;
  // undo the per-row filters in place (filter byte, then the row)
  std::vector<uint8_t> px(row * H);
  for (size_t y = 0; y < H; ++y) {
    const int f = raw[y * (row + 1)];
    const uint8_t* s = &raw[y * (row + 1) + 1];
    uint8_t* o = &px[y * row];
    const uint8_t* up = y ? &px[(y - 1) * row] : nullptr;
    for (size_t i = 0; i < row; ++i) {
      const int a = i >= bpp ? o[i - bpp] : 0, b = up ? up[i] : 0, c = (up && i >= bpp) ? up[i - bpp] : 0;
      int v;
      switch (f) {
        case 0: v = s[i]; break;
        case 1: v = s[i] + a; break;
        case 2: v = s[i] + b; break;
        case 3: v = s[i] + ((a + b) >> 1); break;
        case 4: {
          const int q = a + b - c, pa = std::abs(q - a), pb = std::abs(q - b), pc = std::abs(q - c);
          v = s[i] + ((pa <= pb && pa <= pc) ? a : (pb <= pc ? b : c));
          break;
        }
        default: return err = "bad PNG filter type", false;
      }
      o[i] = (uint8_t)v;
    }
  }
  img.width = (int)W;
  img.height = (int)H;
  img.bits = depth;
  img.pixels.resize((size_t)W * H);
  for (size_t i = 0; i < (size_t)W * H; ++i) {
    if (ch == 3) {  // R, G, B in the file
      const uint8_t* q = &px[3 * i];
      img.pixels[i] = (float)gray8(q[0], q[1], q[2]);
    } else {
      img.pixels[i] = depth == 8 ? px[i] : (float)((px[2 * i] << 8) | px[2 * i + 1]);
    }
  }
  return true;
}

void put_be32(std::vector<uint8_t>& b, uint32_t v) {
  for (int k = 3; k >= 0; --k) b.push_back((v >> (8 * k)) & 0xff);
}

void put16(std::vector<uint8_t>& b, uint16_t v) {
  b.push_back(v & 0xff);
  b.push_back(v >> 8);
}
void put32(std::vector<uint8_t>& b, uint32_t v) {
  for (int k = 0; k < 4; ++k) b.push_back((v >> (8 * k)) & 0xff);
}

}  // namespace

bool read_image(const std::string& path, Image& out, std::string& err) {
  std::vector<uint8_t> buf;
  if (!read_file(path, buf)) return err = "cannot read " + path, false;
  if (buf.size() >= 2 && buf[0] == 'P' && buf[1] == '5') return read_pnm(buf, out, err);
  static const uint8_t kPng[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  if (buf.size() >= 8 && !std::memcmp(buf.data(), kPng, 8)) return read_png(buf, out, err);
  return read_tiff(buf, out, err);
}

bool write_png8(const std::string& path, const uint8_t* pixels, int width, int height, std::string& err) {
  const size_t row = (size_t)width;
  std::vector<uint8_t> raw((row + 1) * height);
  for (int y = 0; y < height; ++y) {
    raw[y * (row + 1)] = 0;  // no filter
    std::memcpy(&raw[y * (row + 1) + 1], pixels + (size_t)y * row, row);
  }
  uLongf zn = compressBound((uLong)raw.size());
  std::vector<uint8_t> z(zn);
  if (compress2(z.data(), &zn, raw.data(), (uLong)raw.size(), 1) != Z_OK) return err = "PNG compression failed", false;
  z.resize(zn);
  std::vector<uint8_t> b = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  auto chunk = [&](const char* type, const std::vector<uint8_t>& data) {
    put_be32(b, (uint32_t)data.size());
    const size_t t0 = b.size();
    b.insert(b.end(), type, type + 4);
    b.insert(b.end(), data.begin(), data.end());
    put_be32(b, (uint32_t)crc32(crc32(0L, Z_NULL, 0), &b[t0], (uInt)(data.size() + 4)));
  };
  std::vector<uint8_t> ihdr;
  put_be32(ihdr, (uint32_t)width);
  put_be32(ihdr, (uint32_t)height);
  ihdr.insert(ihdr.end(), {8, 0, 0, 0, 0});  // 8-bit grayscale, deflate, no interlace
  chunk("IHDR", ihdr);
  chunk("IDAT", z);
  chunk("IEND", {});
  std::ofstream f(path, std::ios::binary);
  if (!f) return err = "cannot open " + path, false;
  f.write(reinterpret_cast<const char*>(b.data()), (std::streamsize)b.size());
  return (bool)f || (err = "write failed: " + path, false);
}

bool write_tiff8(const std::string& path, const uint8_t* pixels, int width, int height, std::string& err) {
  std::vector<uint8_t> b;
  const uint32_t data_off = 8;
  const uint32_t nbytes = (uint32_t)width * height;
  b.insert(b.end(), {'I', 'I', 42, 0});
  const uint32_t ifd_off = data_off + nbytes + (nbytes & 1);
  put32(b, ifd_off);
  b.insert(b.end(), pixels, pixels + nbytes);
  if (nbytes & 1) b.push_back(0);
  const struct { uint16_t tag, type; uint32_t count, value; } e[] = {
      {256, 4, 1, (uint32_t)width}, {257, 4, 1, (uint32_t)height}, {258, 3, 1, 8}, {259, 3, 1, 1},
      {262, 3, 1, 1},               {273, 4, 1, data_off},         {277, 3, 1, 1}, {278, 4, 1, (uint32_t)height},
      {279, 4, 1, nbytes},          {284, 3, 1, 1}};
  put16(b, (uint16_t)(sizeof(e) / sizeof(e[0])));
  for (const auto& x : e) {
    put16(b, x.tag);
    put16(b, x.type);
    put32(b, x.count);
    if (x.type == 3) {
      put16(b, (uint16_t)x.value);
      put16(b, 0);
    } else {
      put32(b, x.value);
    }
  }
  put32(b, 0);
  std::ofstream f(path, std::ios::binary);
  if (!f) return err = "cannot write " + path, false;
  f.write(reinterpret_cast<const char*>(b.data()), (std::streamsize)b.size());
  return (bool)f || (err = "write failed: " + path, false);
}

bool exact_unit_mean(const float* v, size_t n, double* mean) {
  unsigned __int128 acc = 0;
  for (size_t i = 0; i < n; ++i) {
    const float x = v[i];
    if (!(x >= 0.f && x <= 65535.f && x == std::floor(x))) return false;
    const float q = x / 255.0f;
    acc += (unsigned long long)(q * 2147483648.0f);  // q * 2^31, an integer below 2^40
  }
  *mean = unit_mean_from_sum((unsigned long long)acc, (unsigned long long)(acc >> 64), n);
  return true;
}

double unit_mean_from_sum(unsigned long long lo, unsigned long long hi, size_t n) {
  const unsigned __int128 s = ((unsigned __int128)hi << 64) | lo;
  // one rounding to double, exact scaling by 2^-31, one rounding of the quotient
  return std::ldexp((double)s, -31) / (double)n;
}

uint8_t to_u8(double v) {
  if (!(v > 0)) return 0;  // NaN and negatives
  if (v >= 255) return 255;
  return (uint8_t)std::nearbyint(v);  // default rounding mode: half to even
}

bool preprocess(const Image& holo, const Image* bg, const Preprocess& pp, std::vector<float>& b, int& width,
                int& height, std::string& err) {
  const int W0 = holo.width, H0 = holo.height;
  const size_t n0 = (size_t)W0 * H0;
  // float32 arithmetic throughout (OpenCV's CV_32F matrices); the mean in
  // double as cv::mean gives it
  std::vector<float> f(n0);
  for (size_t i = 0; i < n0; ++i) f[i] = holo.pixels[i] / 255.0f;  // rescale (hologram.cu:401-439), 16-bit too
  if (pp.remove_background) {
    if (!bg || bg->width != W0 || bg->height != H0) return err = "background must match the hologram size", false;
    // (I - B) / max(sqrt(B), 0.1)  (hologram.cu:1365-1432)
    for (size_t i = 0; i < n0; ++i) {
      const float B = bg->pixels[i] / 255.0f;
      float sb = std::sqrt(B);
      if (sb < 0.1f) sb = 0.1f;
      f[i] = (f[i] - B) / sb;
    }
  } else {
    // I / mean - 1  (hologram.cu:332-358).  cv::mean sums in double; here the
    // sum is exact (then rounded once) for camera samples, so that the device
    // path gives the same mean; other float inputs are summed in order.
    double m = 0;
    if (!exact_unit_mean(holo.pixels.data(), n0, &m)) {
      for (size_t i = 0; i < n0; ++i) m += f[i];
      m /= (double)n0;
    }
    if (!(m != 0)) return err = "hologram mean is zero", false;
    const float mf = (float)m;
    for (size_t i = 0; i < n0; ++i) f[i] = f[i] / mf - 1.0f;
  }
  const CropRect cr = crop_rect(pp, W0, H0);
  const int rx = cr.x, ry = cr.y, rw = cr.w, rh = cr.h;
  const int p = pp.zero_padding;
  width = rw + 2 * p;
  height = rh + 2 * p;
  b.assign((size_t)width * height, 0.f);
  for (int y = 0; y < rh; ++y)
    for (int x = 0; x < rw; ++x) {
      const int sx = rx + x, sy = ry + y;
      if (sx < 0 || sy < 0 || sx >= W0 || sy >= H0) continue;
      b[(size_t)(y + p) * width + (x + p)] = f[(size_t)sy * W0 + sx];
    }
  return true;
}

}  // namespace rihvr_io

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
namespace {
thread_local std::string g_io_error;
}

extern "C" {

int rihvr_read_image(const char* path, float* pixels, int* width, int* height, int* bits) {
  if (!path || !width || !height) return RIHVR_ERR_INVALID_ARGUMENT;
  rihvr_io::Image img;
  if (!rihvr_io::read_image(path, img, g_io_error)) return RIHVR_ERR_BAD_FILENAME;
  const bool fits = pixels && *width == img.width && *height == img.height;
  *width = img.width;
  *height = img.height;
  if (bits) *bits = img.bits;
  if (!pixels) return RIHVR_OK;
  if (!fits) return RIHVR_ERR_INVALID_ARGUMENT;
  std::memcpy(pixels, img.pixels.data(), sizeof(float) * img.pixels.size());
  return RIHVR_OK;
}

int rihvr_write_tiff8(const char* path, const unsigned char* pixels, int width, int height) {
  if (!path || !pixels || width <= 0 || height <= 0) return RIHVR_ERR_INVALID_ARGUMENT;
  return rihvr_io::write_tiff8(path, pixels, width, height, g_io_error) ? RIHVR_OK : RIHVR_ERR_BAD_FILENAME;
}

int rihvr_write_png8(const char* path, const unsigned char* pixels, int width, int height) {
  if (!path || !pixels || width <= 0 || height <= 0) return RIHVR_ERR_INVALID_ARGUMENT;
  return rihvr_io::write_png8(path, pixels, width, height, g_io_error) ? RIHVR_OK : RIHVR_ERR_BAD_FILENAME;
}

int rihvr_preprocess(const float* holo, int width, int height, const float* background,
                     const rihvr_file_params* files, int zero_padding, float* out, int* out_width, int* out_height) {
  if (!holo || width <= 0 || height <= 0 || !out_width || !out_height) return RIHVR_ERR_INVALID_ARGUMENT;
  rihvr_io::Image h, b;
  h.width = b.width = width;
  h.height = b.height = height;
  h.pixels.assign(holo, holo + (size_t)width * height);
  if (background) b.pixels.assign(background, background + (size_t)width * height);
  rihvr_io::Preprocess pp;
  if (files) {
    pp.remove_background = files->remove_background != 0;
    pp.roi_x = files->roi_x;
    pp.roi_y = files->roi_y;
    pp.roi_size = files->roi_size;
    pp.roi_rect_x = files->roi_rect_x;
    pp.roi_rect_y = files->roi_rect_y;
    pp.roi_rect_w = files->roi_rect_w;
    pp.roi_rect_h = files->roi_rect_h;
  }
  if (pp.remove_background && !background) return RIHVR_ERR_MISSING_DATA;
  pp.zero_padding = zero_padding;
  std::vector<float> res;
  int W, Hh;
  if (!rihvr_io::preprocess(h, background ? &b : nullptr, pp, res, W, Hh, g_io_error)) return RIHVR_ERR_INVALID_DATA;
  const bool fits = out && *out_width == W && *out_height == Hh;
  *out_width = W;
  *out_height = Hh;
  if (!out) return RIHVR_OK;
  if (!fits) return RIHVR_ERR_INVALID_ARGUMENT;
  std::memcpy(out, res.data(), sizeof(float) * res.size());
  return RIHVR_OK;
}

const char* rihvr_io_error(void) { return g_io_error.c_str(); }

}  // extern "C"

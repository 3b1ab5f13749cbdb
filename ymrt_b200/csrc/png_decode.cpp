// PNG decoding for image texture nodes: chunk parsing, inflate (zlib),
// scanline unfiltering (None, Sub, Up, Average, Paeth), Adam7
// de-interlacing, palette and colour-key expansion, vertical flip.
#include "png_decode.h"

#include <zlib.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace ym {

namespace {

uint32_t be32(const uint8_t* p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

bool fail(std::string* error, const std::string& msg) {
  if (error) *error = msg;
  return false;
}

int paeth(int a, int b, int c) {
  const int p = a + b - c;
  const int pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  if (pb <= pc) return b;
  return c;
}

// Reverses the filter of one scanline in place (bpp: bytes per complete
// pixel, at least 1; prev: the previous unfiltered line or null).
bool unfilter(uint8_t type, uint8_t* line, const uint8_t* prev, size_t n, size_t bpp) {
  switch (type) {
    case 0: return true;
    case 1:
      for (size_t i = bpp; i < n; ++i) line[i] = (uint8_t)(line[i] + line[i - bpp]);
      return true;
    case 2:
      if (prev)
        for (size_t i = 0; i < n; ++i) line[i] = (uint8_t)(line[i] + prev[i]);
      return true;
    case 3:
      for (size_t i = 0; i < n; ++i) {
        const int a = i >= bpp ? line[i - bpp] : 0, b = prev ? prev[i] : 0;
        line[i] = (uint8_t)(line[i] + ((a + b) >> 1));
      }
      return true;
    case 4:
      for (size_t i = 0; i < n; ++i) {
        const int a = i >= bpp ? line[i - bpp] : 0, b = prev ? prev[i] : 0;
        const int c = (prev && i >= bpp) ? prev[i - bpp] : 0;
        line[i] = (uint8_t)(line[i] + paeth(a, b, c));
      }
      return true;
    default:
      return false;
  }
}

// Sample k of an unfiltered scanline at the given bit depth.
uint16_t sample_at(const uint8_t* line, size_t k, int depth) {
  switch (depth) {
    case 16: return (uint16_t)(line[2 * k] << 8 | line[2 * k + 1]);
    case 8: return line[k];
    default: {
      const size_t bit = k * depth;
      const int shift = 8 - depth - (int)(bit & 7);
      return (uint16_t)((line[bit >> 3] >> shift) & ((1 << depth) - 1));
    }
  }
}

}  // namespace

bool decode_png(const uint8_t* d, size_t size, PngImage* out, std::string* error) {
  static const uint8_t kSig[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (size < 8 || std::memcmp(d, kSig, 8) != 0) return fail(error, "not a PNG file");
  uint32_t w = 0, h = 0;
  int depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat, palette, trns;
  bool have_trns = false, end = false;
  for (size_t at = 8; !end;) {
    if (at + 12 > size) return fail(error, "truncated PNG chunk");
    const uint32_t len = be32(d + at);
    const uint8_t* type = d + at + 4;
    if (len > size - at - 12) return fail(error, "truncated PNG chunk");
    const uint8_t* body = d + at + 8;
    if (!std::memcmp(type, "IHDR", 4)) {
      if (len != 13) return fail(error, "bad IHDR");
      w = be32(body);
      h = be32(body + 4);
      depth = body[8];
      ctype = body[9];
      interlace = body[12];
      if (body[10] != 0 || body[11] != 0 || interlace > 1) return fail(error, "unsupported PNG compression, filter or interlace method");
    } else if (!std::memcmp(type, "PLTE", 4)) {
      palette.assign(body, body + len);
    } else if (!std::memcmp(type, "tRNS", 4)) {
      trns.assign(body, body + len);
      have_trns = true;
    } else if (!std::memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), body, body + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      end = true;
    } else if (!(type[0] & 0x20)) {
      return fail(error, "unknown critical PNG chunk");
    }
    at += 12 + (size_t)len;
  }
  if (ctype < 0) return fail(error, "missing IHDR");
  if (w == 0 || h == 0 || w > (1u << 24) || h > (1u << 24) || (uint64_t)w * h > (1ull << 28))
    return fail(error, "bad PNG size");
  int file_n;
  switch (ctype) {
    case 0: file_n = 1; break;
    case 2: file_n = 3; break;
    case 3: file_n = 1; break;
    case 4: file_n = 2; break;
    case 6: file_n = 4; break;
    default: return fail(error, "bad PNG colour type");
  }
  const bool depth_ok = (ctype == 0 && (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)) ||
                        (ctype == 3 && (depth == 1 || depth == 2 || depth == 4 || depth == 8)) ||
                        ((ctype == 2 || ctype == 4 || ctype == 6) && (depth == 8 || depth == 16));
  if (!depth_ok) return fail(error, "bad PNG bit depth");
  if (ctype == 3 && (palette.empty() || palette.size() % 3 != 0)) return fail(error, "missing PNG palette");
  if (have_trns && (ctype == 4 || ctype == 6)) return fail(error, "PNG tRNS chunk on an image with alpha");
  if (have_trns && ctype == 3 && trns.size() > palette.size() / 3) return fail(error, "PNG tRNS chunk longer than the palette");

  // passes: x0, y0, dx, dy (Adam7, or one pass)
  static const int kAdam7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4},
                                   {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
  static const int kSingle[1][4] = {{0, 0, 1, 1}};
  const int (*passes)[4] = interlace ? kAdam7 : kSingle;
  const int n_passes = interlace ? 7 : 1;
  const size_t bits_pp = (size_t)file_n * depth;
  const size_t bpp = std::max<size_t>(1, bits_pp / 8);
  size_t expect = 0;
  for (int p = 0; p < n_passes; ++p) {
    const size_t pw = (w - passes[p][0] + passes[p][2] - 1) / passes[p][2];
    const size_t ph = (h - passes[p][1] + passes[p][3] - 1) / passes[p][3];
    if (passes[p][0] >= (int)w || passes[p][1] >= (int)h || pw == 0 || ph == 0) continue;
    expect += ph * (1 + (pw * bits_pp + 7) / 8);
  }
  std::vector<uint8_t> raw(expect);
  {
    z_stream zs;
    std::memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) return fail(error, "inflate failed");
    zs.next_in = idat.data();
    zs.avail_in = (uInt)idat.size();
    zs.next_out = raw.data();
    zs.avail_out = (uInt)raw.size();
    const int rc = inflate(&zs, Z_FINISH);
    const size_t got = raw.size() - zs.avail_out;
    inflateEnd(&zs);
    if ((rc != Z_STREAM_END && rc != Z_BUF_ERROR && rc != Z_OK) || got < expect)
      return fail(error, "PNG image data is corrupt or short");
  }

  // samples per pixel as the file holds them, top row first
  std::vector<uint16_t> file(static_cast<size_t>(w) * h * file_n);
  const uint8_t* src = raw.data();
  for (int p = 0; p < n_passes; ++p) {
    const int x0 = passes[p][0], y0 = passes[p][1], dx = passes[p][2], dy = passes[p][3];
    if (x0 >= (int)w || y0 >= (int)h) continue;
    const size_t pw = (w - x0 + dx - 1) / dx, ph = (h - y0 + dy - 1) / dy;
    const size_t row = (pw * bits_pp + 7) / 8;
    std::vector<uint8_t> prev_line, line(row);
    for (size_t r = 0; r < ph; ++r) {
      const uint8_t ft = *src++;
      std::memcpy(line.data(), src, row);
      src += row;
      if (!unfilter(ft, line.data(), prev_line.empty() ? nullptr : prev_line.data(), row, bpp))
        return fail(error, "bad PNG filter type");
      const size_t y = y0 + r * dy;
      for (size_t c = 0; c < pw; ++c) {
        const size_t x = x0 + c * dx;
        for (int k = 0; k < file_n; ++k)
          file[(y * w + x) * file_n + k] = sample_at(line.data(), c * file_n + k, depth);
      }
      prev_line = line;
    }
  }

  // output channels and values (palette, colour key, low-depth grey scale)
  const bool key = have_trns && ctype != 3;
  int out_n = file_n;
  if (ctype == 3) out_n = have_trns ? 4 : 3;
  else if (key) out_n = file_n + 1;
  if (key && ((ctype == 0 && trns.size() < 2) || (ctype == 2 && trns.size() < 6)))
    return fail(error, "bad PNG tRNS chunk");
  static const int kScale[17] = {0, 0xff, 0x55, 0, 0x11, 0, 0, 0, 0x01};
  const int scale = depth <= 8 ? kScale[depth] : 1;
  uint16_t keyv[3] = {0, 0, 0};
  if (key)
    for (int k = 0; k < (ctype == 0 ? 1 : 3); ++k) {
      const uint16_t v = (uint16_t)(trns[2 * k] << 8 | trns[2 * k + 1]);
      keyv[k] = depth == 16 ? v : (uint16_t)((v & 255) * scale);
    }
  out->width = (int)w;
  out->height = (int)h;
  out->channels = out_n;
  out->sixteen = depth == 16;
  out->samples.assign(static_cast<size_t>(w) * h * out_n, 0);
  const uint16_t opaque = depth == 16 ? 65535 : 255;
  const size_t n_pal = palette.size() / 3;
  for (size_t y = 0; y < h; ++y) {
    const size_t oy = h - 1 - y;  // bottom row first
    for (size_t x = 0; x < w; ++x) {
      const uint16_t* s = &file[(y * w + x) * file_n];
      uint16_t* o = &out->samples[(oy * w + x) * out_n];
      if (ctype == 3) {
        const size_t i = s[0];
        if (i >= n_pal) return fail(error, "PNG palette index out of range");
        o[0] = palette[3 * i];
        o[1] = palette[3 * i + 1];
        o[2] = palette[3 * i + 2];
        if (out_n == 4) o[3] = i < trns.size() ? trns[i] : 255;
        continue;
      }
      for (int k = 0; k < file_n; ++k) o[k] = (ctype == 0 && depth < 8) ? (uint16_t)(s[k] * scale) : s[k];
      if (key) {
        bool match = true;
        for (int k = 0; k < file_n; ++k) match = match && o[k] == keyv[k];
        o[file_n] = match ? 0 : opaque;
      }
    }
  }
  return true;
}

bool decode_png_file(const std::string& path, PngImage* out, std::string* error) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return fail(error, "cannot open " + path);
  std::vector<uint8_t> data;
  uint8_t buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof(buf), f)) > 0) data.insert(data.end(), buf, buf + n);
  std::fclose(f);
  return decode_png(data.data(), data.size(), out, error);
}

}  // namespace ym

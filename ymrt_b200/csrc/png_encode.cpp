// PNG writing of rendered images (this project's encoder, written from the
// PNG specification; deflate by the system zlib).
//
// ymrt_save_png keeps the reference's SavePngImage (src/FileIO.cpp:167-194)
// as a caller sees it: the same argument checks, the path's extension
// replaced by .png, missing parent directories created, 8-bit RGBA with each
// channel stored as (uint8)(clamp(v, 0, 1) * 255 + 0.5), and the first row
// in memory written as the bottom row of the file (the reference flips on
// write; render output holds the bottom row first). The file's bytes differ
// from the reference's image library's (its own deflate and row filters);
// the decoded pixels are the same.
#include <zlib.h>

#include <cstdint>
#include <cstdio>
#include <filesystem>
#include <string>
#include <system_error>
#include <vector>

#include "ymrt.h"

namespace {

void put32(std::vector<uint8_t>& out, uint32_t v) {
  out.push_back((uint8_t)(v >> 24));
  out.push_back((uint8_t)(v >> 16));
  out.push_back((uint8_t)(v >> 8));
  out.push_back((uint8_t)v);
}

// One chunk: length, type, body, CRC-32 of type and body.
void put_chunk(std::vector<uint8_t>& out, const char type[4], const uint8_t* body, size_t n) {
  put32(out, (uint32_t)n);
  const size_t at = out.size();
  out.insert(out.end(), type, type + 4);
  if (n) out.insert(out.end(), body, body + n);
  uLong crc = crc32(0L, Z_NULL, 0);
  crc = crc32(crc, out.data() + at, (uInt)(4 + n));
  put32(out, (uint32_t)crc);
}

uint8_t quantise(float v) {
  // (unsigned char)(glm::clamp(v, 0.0f, 1.0f) * 255.0f + 0.5f), float arithmetic
  const float c = v < 0.0f ? 0.0f : (v > 1.0f ? 1.0f : v);
  return (uint8_t)(c * 255.0f + 0.5f);
}

}  // namespace

extern "C" int ymrt_save_png(const char* path, const float* rgba, int width, int height) {
  if (!path || !*path || !rgba || width <= 0 || height <= 0) return YMRT_ERR_INVALID;
  const size_t row = (size_t)width * 4;
  if ((size_t)height > ((size_t)1 << 31) / (row + 1)) return YMRT_ERR_INVALID;
  std::filesystem::path file(path);
  file.replace_extension(".png");
  std::error_code ec;
  if (file.has_parent_path()) std::filesystem::create_directories(file.parent_path(), ec);
  // scanlines, top row of the image first (the last row in memory), each
  // with filter type 0
  std::vector<uint8_t> raw((row + 1) * (size_t)height);
  for (int y = 0; y < height; ++y) {
    uint8_t* line = raw.data() + (row + 1) * (size_t)y;
    line[0] = 0;
    const float* src = rgba + (size_t)(height - 1 - y) * row;
    for (size_t k = 0; k < row; ++k) line[1 + k] = quantise(src[k]);
  }
  uLongf packed_size = compressBound((uLong)raw.size());
  std::vector<uint8_t> packed(packed_size);
  if (compress2(packed.data(), &packed_size, raw.data(), (uLong)raw.size(), 6) != Z_OK) return YMRT_ERR_INVALID;
  std::vector<uint8_t> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
  uint8_t ihdr[13];
  for (int k = 0; k < 4; ++k) {
    ihdr[k] = (uint8_t)((uint32_t)width >> (24 - 8 * k));
    ihdr[4 + k] = (uint8_t)((uint32_t)height >> (24 - 8 * k));
  }
  ihdr[8] = 8;   // bit depth
  ihdr[9] = 6;   // colour type: RGBA
  ihdr[10] = 0;  // deflate
  ihdr[11] = 0;  // adaptive filtering
  ihdr[12] = 0;  // not interlaced
  put_chunk(out, "IHDR", ihdr, sizeof(ihdr));
  put_chunk(out, "IDAT", packed.data(), packed_size);
  put_chunk(out, "IEND", nullptr, 0);
  FILE* f = std::fopen(file.string().c_str(), "wb");
  if (!f) return YMRT_ERR_IO;
  const bool ok = std::fwrite(out.data(), 1, out.size(), f) == out.size();
  const bool closed = std::fclose(f) == 0;
  return ok && closed ? YMRT_OK : YMRT_ERR_IO;
}

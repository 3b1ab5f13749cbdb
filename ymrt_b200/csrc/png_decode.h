// PNG decoding for image texture nodes (this project's decoder, written from
// the PNG specification; inflate by the system zlib).
//
// The output is what the reference's loader takes from its image library
// (src/FileIO.cpp:17-75, LoadPng8 / LoadPng16): samples per pixel as the file
// holds them (grey 1, grey+alpha 2, RGB 3, RGBA 4; a palette image expands to
// RGB, or RGBA when it has a tRNS chunk; a tRNS colour key on a grey or RGB
// image adds an alpha channel), rows bottom-up (the reference flips images
// vertically on load), 8-bit samples for bit depths up to 8 (grey depths
// 1, 2 and 4 scaled to 0..255) and 16-bit samples for 16-bit files.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ym {

struct PngImage {
  int width = 0, height = 0, channels = 0;
  bool sixteen = false;            // samples are 16-bit (else 8-bit)
  std::vector<uint16_t> samples;   // width * height * channels, bottom row first
};

// Decodes a PNG file. Returns false with a message when the file cannot be
// read or is not a valid PNG.
bool decode_png_file(const std::string& path, PngImage* out, std::string* error);
bool decode_png(const uint8_t* data, size_t size, PngImage* out, std::string* error);

}  // namespace ym

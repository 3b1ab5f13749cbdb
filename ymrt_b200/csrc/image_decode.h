// Decoders for the image formats other than PNG that image texture nodes
// read (this project's code, written from the formats' specifications):
// baseline JPEG (ITU-T T.81), Radiance RGBE (.hdr), BMP and TGA.
//
// The output is what the reference's loader takes from its image library
// through stbi_load (src/FileIO.cpp:17-45, LoadPng8): 8-bit samples, rows
// bottom-up (the reference flips images vertically on load), and as many
// channels as the library reports for the file (JPEG: 1 grey or 3 colour;
// HDR: 3, tone-mapped to 8 bits with gamma 1/2.2 as the library does for an
// 8-bit request; BMP: 3, or 4 with an alpha mask; TGA: 1, 3 or 4). Where the
// library's arithmetic defines the samples (the JPEG inverse DCT, chroma
// upsampling and colour conversion; the HDR tone map) the decoders compute
// them in the same integer and float steps, so the samples are equal bit
// for bit.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace ym {

struct Image8 {
  int width = 0, height = 0, channels = 0;
  std::vector<uint8_t> samples;  // width * height * channels, bottom row first
};

enum class ImageFormat { kUnknown, kPng, kJpeg, kHdr, kBmp, kTga };

// The format of a file's first bytes (TGA, which has no signature, by the
// plausibility of its header, as the library tests it last).
ImageFormat sniff_image(const uint8_t* data, size_t size);

// Each returns false with a message when the data cannot be decoded (a
// progressive or arithmetic-coded JPEG is reported as unsupported through
// *unsupported).
bool decode_jpeg(const uint8_t* data, size_t size, Image8* out, std::string* error, bool* unsupported);
bool decode_hdr(const uint8_t* data, size_t size, Image8* out, std::string* error);
bool decode_bmp(const uint8_t* data, size_t size, Image8* out, std::string* error, bool* unsupported);
bool decode_tga(const uint8_t* data, size_t size, Image8* out, std::string* error, bool* unsupported);

}  // namespace ym

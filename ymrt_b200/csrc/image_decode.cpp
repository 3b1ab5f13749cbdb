// Decoders for JPEG, Radiance HDR, BMP and TGA image textures (see
// image_decode.h for what they produce and why).
#include "image_decode.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace ym {

namespace {

// Rows top-down -> bottom-up, in place.
void flip_rows(Image8* im) {
  const size_t row = (size_t)im->width * im->channels;
  std::vector<uint8_t> tmp(row);
  for (int y = 0; y < im->height / 2; ++y) {
    uint8_t* a = im->samples.data() + (size_t)y * row;
    uint8_t* b = im->samples.data() + (size_t)(im->height - 1 - y) * row;
    std::memcpy(tmp.data(), a, row);
    std::memcpy(a, b, row);
    std::memcpy(b, tmp.data(), row);
  }
}

constexpr int kMaxDimension = 1 << 24;  // the library's STBI_MAX_DIMENSIONS

// ------------------------------------------------------------------ JPEG ---
// Baseline sequential Huffman JPEG (ITU-T T.81, processes SOF0 / SOF1):
// markers, Huffman tables, DC prediction, restart intervals, dequantisation
// and the zig-zag order are the specification's. The inverse DCT is the
// Loeffler-Ligtenberg-Moschytz factorisation in fixed point with 12-bit
// constants and the rounding of the IJG "islow" method; chroma is upsampled
// with the JFIF-centred triangle filter (3/4, 1/4 weights, horizontally,
// vertically or both), and YCbCr is converted to RGB in 20-bit fixed point
// -- the integer steps the reference's image library takes, so the samples
// are the library's.

constexpr uint8_t kZigzag[64 + 15] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
    41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
    30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63,
    // a corrupt run past the end lands on the last coefficient
    63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63, 63};

struct Huffman {
  // canonical code: for each length 1..16 the first code, the count, and
  // the index of its first symbol
  int mincode[17], maxcode[18], valptr[17];
  uint8_t symbols[256];
  bool present = false;
};

bool build_huffman(Huffman* h, const uint8_t counts[16], const uint8_t* syms, int n) {
  std::memcpy(h->symbols, syms, (size_t)n);
  int code = 0, k = 0;
  for (int len = 1; len <= 16; ++len) {
    h->valptr[len] = k;
    h->mincode[len] = code;
    code += counts[len - 1];
    k += counts[len - 1];
    if (counts[len - 1] && code - 1 >= (1 << len)) return false;  // over-subscribed
    h->maxcode[len] = counts[len - 1] ? code - 1 : -1;
    code <<= 1;
  }
  h->maxcode[17] = 0x7fffffff;
  h->present = true;
  return true;
}

struct Component {
  int id = 0, h = 1, v = 1, tq = 0;
  int td = 0, ta = 0;         // Huffman tables of the current scan
  int dc_pred = 0;
  int x = 0, y = 0;           // samples of this component
  int w2 = 0, h2 = 0;         // plane size (whole MCUs)
  std::vector<uint8_t> plane;
};

struct JpegState {
  const uint8_t* p;
  const uint8_t* end;
  uint32_t bits = 0;  // bit buffer, most significant bits first
  int nbits = 0;
  int marker = -1;    // a marker met inside entropy-coded data
  uint16_t quant[4][64];
  Huffman dc[4], ac[4];
  Component comp[4];
  int n_comp = 0;
  int width = 0, height = 0;
  int hmax = 1, vmax = 1;
  int restart_interval = 0;
  bool jfif = false;
  int app14_transform = -1;
  bool rgb_ids = false;

  int byte() { return p < end ? *p++ : 0; }
  int u16() {
    const int a = byte();
    return (a << 8) | byte();
  }
  void fill() {
    while (nbits <= 24) {
      int c = 0;
      if (marker < 0 && p < end) {
        c = *p++;
        if (c == 0xFF) {
          int c2 = p < end ? *p : 0;
          while (c2 == 0xFF && p + 1 < end) {
            ++p;
            c2 = *p;
          }
          if (c2 == 0) {
            ++p;  // a stuffed zero byte
          } else {
            marker = c2;  // a marker: feed zeros from here on
            ++p;
            c = 0;
          }
        }
      }
      bits |= (uint32_t)c << (24 - nbits);
      nbits += 8;
    }
  }
  int bit() {
    if (nbits < 1) fill();
    const int b = (int)(bits >> 31);
    bits <<= 1;
    --nbits;
    return b;
  }
  int receive(int n) {  // n raw bits, most significant first
    int v = 0;
    for (int k = 0; k < n; ++k) v = (v << 1) | bit();
    return v;
  }
  int extend(int v, int n) { return n == 0 ? 0 : (v < (1 << (n - 1)) ? v - (1 << n) + 1 : v); }
  int decode(const Huffman& h) {
    int code = 0;
    for (int len = 1; len <= 16; ++len) {
      code = (code << 1) | bit();
      if (h.maxcode[len] >= 0 && code <= h.maxcode[len]) return h.symbols[h.valptr[len] + code - h.mincode[len]];
    }
    return -1;  // a code the table does not hold
  }
  void reset_bits() {
    bits = 0;
    nbits = 0;
    marker = -1;
  }
};

inline uint8_t clamp_byte(int x) { return (uint8_t)(x < 0 ? 0 : (x > 255 ? 255 : x)); }

// 12-bit fixed-point constants of the factorisation (single-precision
// values, scaled and rounded in double).
constexpr int fix12(float x) { return (int)((double)x * 4096 + 0.5); }

// One 1-D pass: even part from s0, s2, s4, s6; odd part from s1, s3, s5, s7.
// On return x0..x3 hold the even sums and t0..t3 the odd terms, so that the
// eight outputs are x0 +- t3, x1 +- t2, x2 +- t1, x3 +- t0.
struct Idct1D {
  int x0, x1, x2, x3, t0, t1, t2, t3;
  Idct1D(int s0, int s1, int s2, int s3, int s4, int s5, int s6, int s7) {
    // even part: rotation of (s2, s6) by 3 pi / 8
    const int r = (s2 + s6) * fix12(0.5411961f);
    const int e2 = r + s6 * fix12(-1.847759065f);
    const int e3 = r + s2 * fix12(0.765366865f);
    const int e0 = (s0 + s4) * 4096, e1 = (s0 - s4) * 4096;
    x0 = e0 + e3;
    x3 = e0 - e3;
    x1 = e1 + e2;
    x2 = e1 - e2;
    // odd part
    int a0 = s7, a1 = s5, a2 = s3, a3 = s1;
    int q3 = a0 + a2, q4 = a1 + a3, q1 = a0 + a3, q2 = a1 + a2;
    const int q5 = (q3 + q4) * fix12(1.175875602f);
    a0 *= fix12(0.298631336f);
    a1 *= fix12(2.053119869f);
    a2 *= fix12(3.072711026f);
    a3 *= fix12(1.501321110f);
    q1 = q5 + q1 * fix12(-0.899976223f);
    q2 = q5 + q2 * fix12(-2.562915447f);
    q3 *= fix12(-1.961570560f);
    q4 *= fix12(-0.390180644f);
    t3 = a3 + q1 + q4;
    t2 = a2 + q2 + q3;
    t1 = a1 + q2 + q4;
    t0 = a0 + q1 + q3;
  }
};

// Inverse DCT of one dequantised block (natural order) into 8x8 samples.
void idct_block(const short in[64], uint8_t* out, int stride) {
  int col[64];
  for (int i = 0; i < 8; ++i) {  // columns: keep 2 extra bits
    const short* d = in + i;
    const Idct1D c(d[0], d[8], d[16], d[24], d[32], d[40], d[48], d[56]);
    const int x0 = c.x0 + 512, x1 = c.x1 + 512, x2 = c.x2 + 512, x3 = c.x3 + 512;
    col[i] = (x0 + c.t3) >> 10;
    col[56 + i] = (x0 - c.t3) >> 10;
    col[8 + i] = (x1 + c.t2) >> 10;
    col[48 + i] = (x1 - c.t2) >> 10;
    col[16 + i] = (x2 + c.t1) >> 10;
    col[40 + i] = (x2 - c.t1) >> 10;
    col[24 + i] = (x3 + c.t0) >> 10;
    col[32 + i] = (x3 - c.t0) >> 10;
  }
  for (int r = 0; r < 8; ++r) {  // rows: remove 2^17, round, shift by 128
    const int* v = col + 8 * r;
    const Idct1D c(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]);
    const int bias = 65536 + (128 << 17);
    const int x0 = c.x0 + bias, x1 = c.x1 + bias, x2 = c.x2 + bias, x3 = c.x3 + bias;
    uint8_t* o = out + (size_t)r * stride;
    o[0] = clamp_byte((x0 + c.t3) >> 17);
    o[7] = clamp_byte((x0 - c.t3) >> 17);
    o[1] = clamp_byte((x1 + c.t2) >> 17);
    o[6] = clamp_byte((x1 - c.t2) >> 17);
    o[2] = clamp_byte((x2 + c.t1) >> 17);
    o[5] = clamp_byte((x2 - c.t1) >> 17);
    o[3] = clamp_byte((x3 + c.t0) >> 17);
    o[4] = clamp_byte((x3 - c.t0) >> 17);
  }
}

bool decode_block(JpegState& s, Component& c, short blk[64]) {
  std::memset(blk, 0, 64 * sizeof(short));
  const Huffman& hd = s.dc[c.td];
  const Huffman& ha = s.ac[c.ta];
  const int t = s.decode(hd);
  if (t < 0 || t > 16) return false;
  const int diff = s.extend(s.receive(t), t);
  const int dc = c.dc_pred + diff;
  c.dc_pred = dc;
  const uint16_t* q = s.quant[c.tq];
  blk[0] = (short)(dc * q[0]);
  for (int k = 1; k < 64;) {
    const int rs = s.decode(ha);
    if (rs < 0) return false;
    const int run = rs >> 4, size = rs & 15;
    if (size == 0) {
      if (run != 15) break;  // end of block
      k += 16;
      continue;
    }
    k += run;
    const int zz = kZigzag[k < 64 ? k : 64];
    blk[zz] = (short)(s.extend(s.receive(size), size) * q[k < 64 ? k : 63]);
    ++k;
  }
  return true;
}

// One scan of entropy-coded data: the components `scomp` (indices into
// s.comp), interleaved when there are several.
bool decode_scan(JpegState& s, const int* scomp, int ns, std::string* error) {
  short blk[64];
  s.reset_bits();
  for (int i = 0; i < ns; ++i) s.comp[scomp[i]].dc_pred = 0;
  int todo = s.restart_interval ? s.restart_interval : 0x7fffffff;
  auto restart = [&]() -> bool {
    // the entropy-coded segment ends at a marker; RSTn restarts prediction
    if (--todo > 0) return true;
    if (s.marker < 0) {
      // find the marker after the padding bits
      while (s.p < s.end) {
        if (*s.p == 0xFF && s.p + 1 < s.end && s.p[1] != 0 && s.p[1] != 0xFF) {
          s.marker = s.p[1];
          s.p += 2;
          break;
        }
        ++s.p;
      }
    }
    if (s.marker < 0xD0 || s.marker > 0xD7) return false;  // not a restart: the scan is over
    todo = s.restart_interval;
    s.reset_bits();
    for (int i = 0; i < ns; ++i) s.comp[scomp[i]].dc_pred = 0;
    return true;
  };
  if (ns == 1) {
    Component& c = s.comp[scomp[0]];
    const int bw = (c.x + 7) >> 3, bh = (c.y + 7) >> 3;
    for (int by = 0; by < bh; ++by)
      for (int bx = 0; bx < bw; ++bx) {
        if (!decode_block(s, c, blk)) {
          if (error) *error = "corrupt JPEG data";
          return false;
        }
        idct_block(blk, c.plane.data() + (size_t)by * 8 * c.w2 + (size_t)bx * 8, c.w2);
        if (!restart()) return true;
      }
    return true;
  }
  const int mx = (s.width + 8 * s.hmax - 1) / (8 * s.hmax), my = (s.height + 8 * s.vmax - 1) / (8 * s.vmax);
  for (int j = 0; j < my; ++j)
    for (int i = 0; i < mx; ++i) {
      for (int k = 0; k < ns; ++k) {
        Component& c = s.comp[scomp[k]];
        for (int y = 0; y < c.v; ++y)
          for (int x = 0; x < c.h; ++x) {
            if (!decode_block(s, c, blk)) {
              if (error) *error = "corrupt JPEG data";
              return false;
            }
            const int px = (i * c.h + x) * 8, py = (j * c.v + y) * 8;
            idct_block(blk, c.plane.data() + (size_t)py * c.w2 + px, c.w2);
          }
      }
      if (!restart()) return true;
    }
  return true;
}

inline uint8_t div4(int x) { return (uint8_t)(x >> 2); }
inline uint8_t div16(int x) { return (uint8_t)(x >> 4); }

// One output row of a subsampled component from its nearer and farther
// source rows (w source samples, hs output samples per source sample).
const uint8_t* upsample_row(uint8_t* out, const uint8_t* near_row, const uint8_t* far_row, int w, int hs, int vs) {
  if (hs == 1 && vs == 1) return near_row;
  if (hs == 1 && vs == 2) {
    for (int i = 0; i < w; ++i) out[i] = div4(3 * near_row[i] + far_row[i] + 2);
    return out;
  }
  if (hs == 2 && vs == 1) {
    if (w == 1) {
      out[0] = out[1] = near_row[0];
      return out;
    }
    out[0] = near_row[0];
    out[1] = div4(near_row[0] * 3 + near_row[1] + 2);
    int i = 1;
    for (; i < w - 1; ++i) {
      const int n = 3 * near_row[i] + 2;
      out[2 * i] = div4(n + near_row[i - 1]);
      out[2 * i + 1] = div4(n + near_row[i + 1]);
    }
    out[2 * i] = div4(near_row[w - 2] * 3 + near_row[w - 1] + 2);
    out[2 * i + 1] = near_row[w - 1];
    return out;
  }
  if (hs == 2 && vs == 2) {
    if (w == 1) {
      out[0] = out[1] = div4(3 * near_row[0] + far_row[0] + 2);
      return out;
    }
    int t1 = 3 * near_row[0] + far_row[0];
    out[0] = div4(t1 + 2);
    for (int i = 1; i < w; ++i) {
      const int t0 = t1;
      t1 = 3 * near_row[i] + far_row[i];
      out[2 * i - 1] = div16(3 * t0 + t1 + 8);
      out[2 * i] = div16(3 * t1 + t0 + 8);
    }
    out[2 * w - 1] = div4(t1 + 2);
    return out;
  }
  for (int i = 0; i < w; ++i)  // other factors: nearest neighbour
    for (int j = 0; j < hs; ++j) out[i * hs + j] = near_row[i];
  return out;
}

// JFIF YCbCr -> RGB in 20-bit fixed point (constants to 12 bits, the
// green term's Cb product truncated to 16 fractional bits).
inline int fix20(float x) { return ((int)(x * 4096.0f + 0.5f)) << 8; }
void ycbcr_row(uint8_t* out, const uint8_t* y, const uint8_t* cb, const uint8_t* cr, int count) {
  for (int i = 0; i < count; ++i) {
    const int yf = (y[i] << 20) + (1 << 19);
    const int vr = cr[i] - 128, vb = cb[i] - 128;
    int r = yf + vr * fix20(1.40200f);
    int g = yf + (vr * -fix20(0.71414f)) + ((vb * -fix20(0.34414f)) & (int)0xffff0000);
    int b = yf + vb * fix20(1.77200f);
    out[3 * i] = clamp_byte(r >> 20);
    out[3 * i + 1] = clamp_byte(g >> 20);
    out[3 * i + 2] = clamp_byte(b >> 20);
  }
}

}  // namespace

bool decode_jpeg(const uint8_t* data, size_t size, Image8* out, std::string* error, bool* unsupported) {
  if (unsupported) *unsupported = false;
  auto fail = [&](const char* msg) {
    if (error) *error = msg;
    return false;
  };
  auto unsup = [&](const char* msg) {
    if (unsupported) *unsupported = true;
    return fail(msg);
  };
  if (size < 4 || data[0] != 0xFF || data[1] != 0xD8) return fail("not a JPEG file");
  JpegState s;
  s.p = data + 2;
  s.end = data + size;
  std::memset(s.quant, 0, sizeof(s.quant));
  bool have_frame = false, any_scan = false;
  for (;;) {
    // next marker
    while (s.p < s.end && *s.p != 0xFF) ++s.p;
    while (s.p < s.end && *s.p == 0xFF) ++s.p;
    if (s.p >= s.end) break;
    const int m = *s.p++;
    if (m == 0xD9) break;  // EOI
    if (m == 0x00 || m == 0xD8 || (m >= 0xD0 && m <= 0xD7) || m == 0x01) continue;
    const int len = s.u16();
    if (len < 2 || s.p + (len - 2) > s.end) return fail("truncated JPEG segment");
    const uint8_t* seg_end = s.p + (len - 2);
    if (m == 0xDB) {  // DQT
      while (s.p < seg_end) {
        const int pq_tq = s.byte();
        const int pq = pq_tq >> 4, tq = pq_tq & 15;
        if (tq > 3 || pq > 1) return fail("bad quantisation table");
        for (int k = 0; k < 64; ++k) s.quant[tq][k] = (uint16_t)(pq ? s.u16() : s.byte());
      }
    } else if (m == 0xC4) {  // DHT
      while (s.p < seg_end) {
        const int tc_th = s.byte();
        const int tc = tc_th >> 4, th = tc_th & 15;
        if (tc > 1 || th > 3) return fail("bad Huffman table");
        uint8_t counts[16];
        int n = 0;
        for (int k = 0; k < 16; ++k) {
          counts[k] = (uint8_t)s.byte();
          n += counts[k];
        }
        if (n > 256 || s.p + n > seg_end) return fail("bad Huffman table");
        if (!build_huffman(tc ? &s.ac[th] : &s.dc[th], counts, s.p, n)) return fail("bad Huffman table");
        s.p += n;
      }
    } else if (m == 0xC0 || m == 0xC1) {  // baseline / extended sequential, Huffman
      if (s.byte() != 8) return unsup("JPEG sample precision other than 8 bits");
      s.height = s.u16();
      s.width = s.u16();
      s.n_comp = s.byte();
      if (s.width <= 0 || s.height <= 0) return unsup("JPEG with a DNL height");
      if (s.width > kMaxDimension || s.height > kMaxDimension) return fail("JPEG too large");
      if (s.n_comp != 1 && s.n_comp != 3) return unsup("JPEG with other than 1 or 3 components");
      for (int k = 0; k < s.n_comp; ++k) {
        Component& c = s.comp[k];
        c.id = s.byte();
        const int hv = s.byte();
        c.h = hv >> 4;
        c.v = hv & 15;
        c.tq = s.byte();
        if (c.h < 1 || c.h > 4 || c.v < 1 || c.v > 4 || c.tq > 3) return fail("bad JPEG frame header");
        s.hmax = std::max(s.hmax, c.h);
        s.vmax = std::max(s.vmax, c.v);
      }
      if (s.n_comp == 3 && s.comp[0].id == 'R' && s.comp[1].id == 'G' && s.comp[2].id == 'B') s.rgb_ids = true;
      const int mx = (s.width + 8 * s.hmax - 1) / (8 * s.hmax), my = (s.height + 8 * s.vmax - 1) / (8 * s.vmax);
      for (int k = 0; k < s.n_comp; ++k) {
        Component& c = s.comp[k];
        c.x = (s.width * c.h + s.hmax - 1) / s.hmax;
        c.y = (s.height * c.v + s.vmax - 1) / s.vmax;
        c.w2 = mx * c.h * 8;
        c.h2 = my * c.v * 8;
        c.plane.assign((size_t)c.w2 * c.h2, 0);
      }
      have_frame = true;
    } else if (m >= 0xC2 && m <= 0xCF && m != 0xC4 && m != 0xC8 && m != 0xCC) {
      return unsup("progressive, lossless or arithmetic-coded JPEG");
    } else if (m == 0xDD) {  // DRI
      s.restart_interval = s.u16();
    } else if (m == 0xDA) {  // SOS
      if (!have_frame) return fail("JPEG scan before the frame header");
      const int ns = s.byte();
      if (ns < 1 || ns > s.n_comp) return fail("bad JPEG scan header");
      int scomp[4];
      for (int k = 0; k < ns; ++k) {
        const int id = s.byte(), tables = s.byte();
        int which = -1;
        for (int q = 0; q < s.n_comp; ++q)
          if (s.comp[q].id == id) which = q;
        if (which < 0) return fail("bad JPEG scan component");
        s.comp[which].td = tables >> 4;
        s.comp[which].ta = tables & 15;
        if (s.comp[which].td > 3 || s.comp[which].ta > 3 || !s.dc[s.comp[which].td].present ||
            !s.ac[s.comp[which].ta].present)
          return fail("JPEG scan without its Huffman tables");
        scomp[k] = which;
      }
      const int ss = s.byte(), se = s.byte();
      s.byte();  // Ah / Al
      if (ss != 0 || se != 63) return unsup("spectral selection in a sequential JPEG");
      s.p = seg_end;
      if (!decode_scan(s, scomp, ns, error)) return false;
      any_scan = true;
      // resume marker parsing where the entropy-coded data stopped
      if (s.marker >= 0) {
        s.p -= 2;  // back onto the marker (FF xx)
        if (s.p < data) s.p = data;
        s.marker = -1;
      }
      continue;
    } else if (m == 0xE0) {  // APP0: JFIF
      if (len >= 7 && std::memcmp(s.p, "JFIF\0", 5) == 0) s.jfif = true;
    } else if (m == 0xEE) {  // APP14: Adobe colour transform
      if (len >= 14 && std::memcmp(s.p, "Adobe", 5) == 0) s.app14_transform = s.p[11];
    }
    s.p = seg_end;
  }
  if (!have_frame || !any_scan) return fail("JPEG without image data");
  // upsample and convert, top row first
  const int n = s.n_comp >= 3 ? 3 : 1;
  const bool is_rgb = s.n_comp == 3 && (s.rgb_ids || (s.app14_transform == 0 && !s.jfif));
  out->width = s.width;
  out->height = s.height;
  out->channels = n;
  out->samples.assign((size_t)s.width * s.height * n, 0);
  struct Resample {
    int hs, vs, ystep, ypos, w_lores;
    const uint8_t *line0, *line1;
    std::vector<uint8_t> buf;
  } rs[3];
  for (int k = 0; k < s.n_comp; ++k) {
    Resample& r = rs[k];
    r.hs = s.hmax / s.comp[k].h;
    r.vs = s.vmax / s.comp[k].v;
    r.ystep = r.vs >> 1;
    r.w_lores = (s.width + r.hs - 1) / r.hs;
    r.ypos = 0;
    r.line0 = r.line1 = s.comp[k].plane.data();
    r.buf.assign((size_t)s.width + 3, 0);
  }
  const uint8_t* row[3] = {nullptr, nullptr, nullptr};
  for (int j = 0; j < s.height; ++j) {
    uint8_t* o = out->samples.data() + (size_t)j * s.width * n;
    for (int k = 0; k < s.n_comp; ++k) {
      Resample& r = rs[k];
      const bool y_bot = r.ystep >= (r.vs >> 1);
      row[k] = upsample_row(r.buf.data(), y_bot ? r.line1 : r.line0, y_bot ? r.line0 : r.line1, r.w_lores, r.hs, r.vs);
      if (++r.ystep >= r.vs) {
        r.ystep = 0;
        r.line0 = r.line1;
        if (++r.ypos < s.comp[k].y) r.line1 += s.comp[k].w2;
      }
    }
    if (n == 3) {
      if (is_rgb) {
        for (int i = 0; i < s.width; ++i) {
          o[3 * i] = row[0][i];
          o[3 * i + 1] = row[1][i];
          o[3 * i + 2] = row[2][i];
        }
      } else {
        ycbcr_row(o, row[0], row[1], row[2], s.width);
      }
    } else {
      std::memcpy(o, row[0], (size_t)s.width);
    }
  }
  flip_rows(out);
  return true;
}

// ------------------------------------------------------------ Radiance ---
// RGBE pixels (Ward, "Real Pixels", Graphics Gems II), flat or with the
// per-channel run-length scanlines of the Radiance format; converted to
// float by the shared exponent and, as the library does for an 8-bit
// request, to 8 bits by x^(1/2.2) * 255 + 0.5, clamped and truncated.

namespace {

void rgbe_to_float(const uint8_t* e, float* out) {
  if (e[3] != 0) {
    const float f = (float)std::ldexp(1.0f, e[3] - (int)(128 + 8));
    out[0] = e[0] * f;
    out[1] = e[1] * f;
    out[2] = e[2] * f;
  } else {
    out[0] = out[1] = out[2] = 0.0f;
  }
}

bool hdr_line(const uint8_t*& p, const uint8_t* end, std::string* line) {
  line->clear();
  while (p < end && *p != '\n') line->push_back((char)*p++);
  if (p >= end) return false;
  ++p;
  return true;
}

}  // namespace

bool decode_hdr(const uint8_t* data, size_t size, Image8* out, std::string* error) {
  auto fail = [&](const char* msg) {
    if (error) *error = msg;
    return false;
  };
  const uint8_t* p = data;
  const uint8_t* end = data + size;
  std::string line;
  if (!hdr_line(p, end, &line) || (line != "#?RADIANCE" && line != "#?RGBE")) return fail("not a Radiance HDR file");
  bool valid = false;
  for (;;) {
    if (!hdr_line(p, end, &line)) return fail("truncated HDR header");
    if (line.empty()) break;
    if (line == "FORMAT=32-bit_rle_rgbe") valid = true;
  }
  if (!valid) return fail("HDR format other than 32-bit_rle_rgbe");
  if (!hdr_line(p, end, &line) || line.compare(0, 3, "-Y ") != 0) return fail("HDR data layout other than -Y +X");
  const char* t = line.c_str() + 3;
  char* rest = nullptr;
  const long h = std::strtol(t, &rest, 10);
  while (*rest == ' ') ++rest;
  if (std::strncmp(rest, "+X ", 3) != 0) return fail("HDR data layout other than -Y +X");
  const long w = std::strtol(rest + 3, nullptr, 10);
  if (w <= 0 || h <= 0 || w > kMaxDimension || h > kMaxDimension) return fail("bad HDR size");
  const int width = (int)w, height = (int)h;
  std::vector<float> px((size_t)width * height * 3);
  auto get = [&]() -> int { return p < end ? *p++ : 0; };
  std::vector<uint8_t> scan((size_t)width * 4);
  bool flat = width < 8 || width >= 32768;
  int j0 = 0;
  if (!flat) {
    for (int j = 0; j < height; ++j) {
      const int c1 = get(), c2 = get();
      int len = get();
      if (c1 != 2 || c2 != 2 || (len & 0x80)) {
        // not run-length encoded: these four bytes are the first pixel of
        // flat data for the whole image
        const uint8_t e[4] = {(uint8_t)c1, (uint8_t)c2, (uint8_t)len, (uint8_t)get()};
        rgbe_to_float(e, px.data());
        flat = true;
        j0 = -1;
        break;
      }
      len = (len << 8) | get();
      if (len != width) return fail("corrupt HDR scanline");
      for (int k = 0; k < 4; ++k) {
        int i = 0;
        while (width - i > 0) {
          int count = get();
          if (count > 128) {
            const int v = get();
            count -= 128;
            if (count == 0 || count > width - i) return fail("corrupt HDR run");
            for (int z = 0; z < count; ++z) scan[(size_t)(i++) * 4 + k] = (uint8_t)v;
          } else {
            if (count == 0 || count > width - i) return fail("corrupt HDR run");
            for (int z = 0; z < count; ++z) scan[(size_t)(i++) * 4 + k] = (uint8_t)get();
          }
        }
      }
      for (int i = 0; i < width; ++i) rgbe_to_float(&scan[(size_t)i * 4], &px[((size_t)j * width + i) * 3]);
    }
  }
  if (flat) {
    // j0 == -1: the first pixel is already converted
    size_t first = j0 < 0 ? 1 : 0;
    for (size_t q = first; q < (size_t)width * height; ++q) {
      const uint8_t e[4] = {(uint8_t)get(), (uint8_t)get(), (uint8_t)get(), (uint8_t)get()};
      rgbe_to_float(e, &px[q * 3]);
    }
  }
  out->width = width;
  out->height = height;
  out->channels = 3;
  out->samples.resize(px.size());
  const float gamma = 1.0f / 2.2f;
  for (size_t q = 0; q < px.size(); ++q) {
    float z = (float)std::pow(px[q] * 1.0f, gamma) * 255 + 0.5f;
    if (z < 0) z = 0;
    if (z > 255) z = 255;
    out->samples[q] = (uint8_t)(int)z;
  }
  flip_rows(out);
  return true;
}

// ------------------------------------------------------------------ BMP ---
// Windows bitmaps (BITMAPCOREHEADER, BITMAPINFOHEADER and the V3/V4/V5
// headers): 1-, 4- and 8-bit palettes, 24-bit BGR, and 16- and 32-bit pixels
// through channel masks (the defaults 5-5-5 and 8-8-8(-8), or BI_BITFIELDS),
// a masked channel of n bits widened to 8 by repeating its bits; RLE and
// embedded JPEG/PNG are not decoded. As the library reports them: three
// channels, or four when there is an alpha mask (not for 24-bit pixels); an
// alpha channel that is zero everywhere reads as opaque.

namespace {

struct Reader {
  const uint8_t* p;
  const uint8_t* end;
  int u8() { return p < end ? *p++ : 0; }
  int u16() {
    const int a = u8();
    return a | (u8() << 8);
  }
  uint32_t u32() {
    const uint32_t a = (uint32_t)u16();
    return a | ((uint32_t)u16() << 16);
  }
  // as the library skips: a negative count moves to the end of the data
  void skip(long n) { p = n < 0 ? end : (n <= end - p ? p + n : end); }
};

int high_bit(uint32_t z) {
  int n = -1;
  while (z) {
    ++n;
    z >>= 1;
  }
  return n;
}
int bit_count(uint32_t z) {
  int n = 0;
  for (; z; z &= z - 1) ++n;
  return n;
}
// The masked value v (its highest set bit moved to bit 7 by `shift`) of
// `bits` significant bits, widened to 8 bits by repeating its bit pattern.
int widen(uint32_t v, int shift, int bits) {
  v = shift < 0 ? v << -shift : v >> shift;
  v >>= (8 - bits);
  if (bits <= 0) return 0;
  int out = 0;
  for (int s = 8 - bits; s > -bits; s -= bits) out |= s >= 0 ? (int)(v << s) : (int)(v >> -s);
  return out & 255;
}

}  // namespace

bool decode_bmp(const uint8_t* data, size_t size, Image8* out, std::string* error, bool* unsupported) {
  if (unsupported) *unsupported = false;
  auto fail = [&](const char* msg) {
    if (error) *error = msg;
    return false;
  };
  auto unsup = [&](const char* msg) {
    if (unsupported) *unsupported = true;
    return fail(msg);
  };
  Reader r{data, data + size};
  if (r.u8() != 'B' || r.u8() != 'M') return fail("not a BMP file");
  r.u32();
  r.u16();
  r.u16();
  const long offset = (long)(int32_t)r.u32();
  const int hsz = (int)r.u32();
  int extra_read = 14;
  if (offset < 0) return fail("bad BMP");
  if (hsz != 12 && hsz != 40 && hsz != 56 && hsz != 108 && hsz != 124) return unsup("BMP header type");
  long w, h;
  if (hsz == 12) {
    w = r.u16();
    h = r.u16();
  } else {
    w = (int32_t)r.u32();
    h = (int32_t)r.u32();
  }
  if (r.u16() != 1) return fail("bad BMP");
  const int bpp = r.u16();
  uint32_t mr = 0, mg = 0, mb = 0, ma = 0;
  uint32_t all_a = 255;  // set to 0 where an alpha mask is assumed: an alpha that stays 0 reads as opaque
  if (hsz != 12) {
    const int compress = (int)r.u32();
    if (compress == 1 || compress == 2) return unsup("RLE-compressed BMP");
    if (compress >= 4) return unsup("BMP with embedded JPEG or PNG");
    if (compress == 3 && bpp != 16 && bpp != 32) return fail("bad BMP");
    for (int k = 0; k < 5; ++k) r.u32();
    auto defaults = [&]() {
      if (bpp == 16) {
        mr = 31u << 10;
        mg = 31u << 5;
        mb = 31u;
      } else if (bpp == 32) {
        mr = 0xffu << 16;
        mg = 0xffu << 8;
        mb = 0xffu;
        ma = 0xffu << 24;
        all_a = 0;
      } else {
        mr = mg = mb = ma = 0;
      }
    };
    if (hsz == 40 || hsz == 56) {
      if (hsz == 56)
        for (int k = 0; k < 4; ++k) r.u32();
      if (bpp == 16 || bpp == 32) {
        if (compress == 0) {
          defaults();
        } else if (compress == 3) {
          mr = r.u32();
          mg = r.u32();
          mb = r.u32();
          extra_read += 12;
          if (mr == mg && mg == mb) return fail("bad BMP masks");
        } else {
          return fail("bad BMP");
        }
      }
    } else {
      mr = r.u32();
      mg = r.u32();
      mb = r.u32();
      ma = r.u32();
      if (compress == 0) defaults();
      for (int k = 0; k < 13; ++k) r.u32();
      if (hsz == 124)
        for (int k = 0; k < 4; ++k) r.u32();
    }
  }
  const bool bottom_up = h > 0;
  if (h < 0) h = -h;
  if (w <= 0 || h <= 0 || w > kMaxDimension || h > kMaxDimension) return fail("bad BMP size");
  int psize = 0;
  if (hsz == 12) {
    if (bpp < 24) psize = (int)((offset - extra_read - 24) / 3);
  } else {
    if (bpp < 16) psize = (int)((offset - extra_read - hsz) >> 2);
  }
  if (psize == 0) {
    const long so_far = (long)(r.p - data);
    if (so_far <= 0 || so_far > 1024 || offset < so_far || offset - so_far > 256 * 4) return fail("corrupt BMP");
    r.skip(offset - so_far);
  }
  const int n = (bpp == 24 && ma == 0xff000000u) ? 3 : (ma ? 4 : 3);
  const int W = (int)w, H = (int)h;
  std::vector<uint8_t> img((size_t)W * H * n);
  size_t z = 0;
  if (bpp < 16) {
    if (psize == 0 || psize > 256) return fail("corrupt BMP palette");
    uint8_t pal[256][3] = {};
    for (int i = 0; i < psize; ++i) {
      pal[i][2] = (uint8_t)r.u8();
      pal[i][1] = (uint8_t)r.u8();
      pal[i][0] = (uint8_t)r.u8();
      if (hsz != 12) r.u8();
    }
    r.skip(offset - extra_read - hsz - psize * (hsz == 12 ? 3 : 4));
    int width;
    if (bpp == 1) width = (W + 7) >> 3;
    else if (bpp == 4) width = (W + 1) >> 1;
    else if (bpp == 8) width = W;
    else return fail("bad BMP bit count");
    const int pad = (-width) & 3;
    auto put = [&](int v) {
      img[z++] = pal[v][0];
      img[z++] = pal[v][1];
      img[z++] = pal[v][2];
      if (n == 4) img[z++] = 255;
    };
    for (int j = 0; j < H; ++j) {
      if (bpp == 1) {
        int bit = 7, v = r.u8();
        for (int i = 0; i < W; ++i) {
          put((v >> bit) & 1);
          if (i + 1 == W) break;
          if (--bit < 0) {
            bit = 7;
            v = r.u8();
          }
        }
      } else {
        for (int i = 0; i < W; i += 2) {
          int v = r.u8(), v2 = 0;
          if (bpp == 4) {
            v2 = v & 15;
            v >>= 4;
          }
          put(v);
          if (i + 1 == W) break;
          put(bpp == 8 ? r.u8() : v2);
        }
      }
      r.skip(pad);
    }
  } else {
    r.skip(offset - extra_read - hsz);
    const int width = bpp == 24 ? 3 * W : (bpp == 16 ? 2 * W : 0);
    const int pad = (-width) & 3;
    int easy = 0;
    if (bpp == 24) easy = 1;
    else if (bpp == 32 && mb == 0xffu && mg == 0xff00u && mr == 0x00ff0000u && ma == 0xff000000u) easy = 2;
    int rs = 0, gs = 0, bs = 0, as = 0, rc = 0, gc = 0, bc = 0, ac = 0;
    if (!easy) {
      if (!mr || !mg || !mb) return fail("bad BMP masks");
      rs = high_bit(mr) - 7;
      rc = bit_count(mr);
      gs = high_bit(mg) - 7;
      gc = bit_count(mg);
      bs = high_bit(mb) - 7;
      bc = bit_count(mb);
      as = high_bit(ma) - 7;
      ac = bit_count(ma);
      if (rc > 8 || gc > 8 || bc > 8 || ac > 8) return fail("bad BMP masks");
    }
    for (int j = 0; j < H; ++j) {
      for (int i = 0; i < W; ++i) {
        if (easy) {
          img[z + 2] = (uint8_t)r.u8();
          img[z + 1] = (uint8_t)r.u8();
          img[z + 0] = (uint8_t)r.u8();
          z += 3;
          const int a = easy == 2 ? r.u8() : 255;
          all_a |= (uint32_t)a;
          if (n == 4) img[z++] = (uint8_t)a;
        } else {
          const uint32_t v = bpp == 16 ? (uint32_t)r.u16() : r.u32();
          img[z++] = (uint8_t)widen(v & mr, rs, rc);
          img[z++] = (uint8_t)widen(v & mg, gs, gc);
          img[z++] = (uint8_t)widen(v & mb, bs, bc);
          const uint32_t a = ma ? (uint32_t)widen(v & ma, as, ac) : 255u;
          all_a |= a;
          if (n == 4) img[z++] = (uint8_t)a;
        }
      }
      r.skip(pad);
    }
  }
  if (n == 4 && all_a == 0)
    for (size_t q = 3; q < img.size(); q += 4) img[q] = 255;
  out->width = W;
  out->height = H;
  out->channels = n;
  out->samples.swap(img);
  if (!bottom_up) flip_rows(out);  // rows as stored are top-down: make them bottom-up
  return true;
}

// ------------------------------------------------------------------ TGA ---
// Truevision TGA: colour-mapped (type 1), true-colour (2) and grey (3)
// images, uncompressed or run-length encoded (9, 10, 11); 8-bit grey, 16-bit
// grey + alpha, 15/16-bit RGB (five bits per channel scaled to 0..255, no
// alpha), 24-bit RGB and 32-bit RGBA, and palettes of those; rows in either
// vertical order.

bool decode_tga(const uint8_t* data, size_t size, Image8* out, std::string* error, bool* unsupported) {
  if (unsupported) *unsupported = false;
  auto fail = [&](const char* msg) {
    if (error) *error = msg;
    return false;
  };
  Reader r{data, data + size};
  const int id_len = r.u8();
  const int indexed = r.u8();
  int type = r.u8();
  const int pal_start = r.u16(), pal_len = r.u16(), pal_bits = r.u8();
  r.u16();
  r.u16();
  const int W = r.u16(), H = r.u16(), bpp = r.u8();
  const int desc = r.u8();
  bool rle = false;
  if (type >= 8) {
    type -= 8;
    rle = true;
  }
  const bool top_down = ((desc >> 5) & 1) != 0;
  auto comp_of = [](int bits, bool grey, bool* rgb16) {
    *rgb16 = false;
    switch (bits) {
      case 8: return 1;
      case 16:
        if (grey) return 2;
        *rgb16 = true;
        return 3;
      case 15: *rgb16 = true; return 3;
      case 24:
      case 32: return bits / 8;
      default: return 0;
    }
  };
  bool rgb16 = false;
  const int comp = indexed ? comp_of(pal_bits, false, &rgb16) : comp_of(bpp, type == 3, &rgb16);
  if (!comp) return fail("bad TGA pixel format");
  if (W <= 0 || H <= 0) return fail("bad TGA size");
  std::vector<uint8_t> img((size_t)W * H * comp);
  r.skip(id_len);
  auto rgb16_px = [&](uint8_t* o) {
    const int px = r.u16();
    o[0] = (uint8_t)((((px >> 10) & 31) * 255) / 31);
    o[1] = (uint8_t)((((px >> 5) & 31) * 255) / 31);
    o[2] = (uint8_t)(((px & 31) * 255) / 31);
  };
  std::vector<uint8_t> pal;
  if (indexed) {
    if (pal_len == 0) return fail("bad TGA palette");
    r.skip(pal_start);
    pal.resize((size_t)pal_len * comp);
    if (!rgb16 && (size_t)(r.end - r.p) < pal.size()) return fail("truncated TGA palette");
    for (int i = 0; i < pal_len; ++i) {
      if (rgb16) rgb16_px(&pal[(size_t)i * comp]);
      else
        for (int k = 0; k < comp; ++k) pal[(size_t)i * comp + k] = (uint8_t)r.u8();
    }
  }
  // pixels in file order (bottom row first unless top_down)
  uint8_t raw[4] = {0, 0, 0, 0};
  int run = 0;
  bool repeating = false, read_next = true;
  for (size_t i = 0; i < (size_t)W * H; ++i) {
    if (rle) {
      if (run == 0) {
        const int cmd = r.u8();
        run = 1 + (cmd & 127);
        repeating = (cmd >> 7) != 0;
        read_next = true;
      } else if (!repeating) {
        read_next = true;
      }
    } else {
      read_next = true;
    }
    if (read_next) {
      if (indexed) {
        int idx = bpp == 8 ? r.u8() : r.u16();
        if (idx >= pal_len) idx = 0;
        for (int k = 0; k < comp; ++k) raw[k] = pal[(size_t)idx * comp + k];
      } else if (rgb16) {
        rgb16_px(raw);
      } else {
        for (int k = 0; k < comp; ++k) raw[k] = (uint8_t)r.u8();
      }
      read_next = false;
    }
    for (int k = 0; k < comp; ++k) img[i * comp + k] = raw[k];
    --run;
  }
  if (comp >= 3 && !rgb16)  // BGR(A) -> RGB(A)
    for (size_t i = 0; i < (size_t)W * H; ++i) std::swap(img[i * comp], img[i * comp + 2]);
  out->width = W;
  out->height = H;
  out->channels = comp;
  out->samples.swap(img);
  if (top_down) flip_rows(out);
  return true;
}

// ------------------------------------------------------------ sniffing ---

ImageFormat sniff_image(const uint8_t* d, size_t n) {
  static const uint8_t kPng[8] = {137, 80, 78, 71, 13, 10, 26, 10};
  if (n >= 8 && std::memcmp(d, kPng, 8) == 0) return ImageFormat::kPng;
  if (n >= 3 && d[0] == 0xFF && d[1] == 0xD8 && d[2] == 0xFF) return ImageFormat::kJpeg;
  if (n >= 2 && d[0] == 'B' && d[1] == 'M') return ImageFormat::kBmp;
  if ((n >= 11 && std::memcmp(d, "#?RADIANCE\n", 11) == 0) || (n >= 7 && std::memcmp(d, "#?RGBE\n", 7) == 0))
    return ImageFormat::kHdr;
  // TGA: colour-map type 0 or 1, a supported image type, a plausible
  // colour map and pixel size (the library's tga test)
  if (n >= 18) {
    const int cmap = d[1], type = d[2];
    if (cmap <= 1) {
      const bool ok_type = cmap == 1 ? (type == 1 || type == 9) : (type == 2 || type == 3 || type == 10 || type == 11);
      if (ok_type) {
        const int w = d[12] | (d[13] << 8), h = d[14] | (d[15] << 8), bpp = d[16];
        const int cmap_bpp = d[7];
        const bool cmap_ok = cmap == 0 || cmap_bpp == 8 || cmap_bpp == 15 || cmap_bpp == 16 || cmap_bpp == 24 ||
                             cmap_bpp == 32;
        const bool bpp_ok = cmap == 1 ? (bpp == 8 || bpp == 16) : (bpp == 8 || bpp == 15 || bpp == 16 || bpp == 24 || bpp == 32);
        if (w >= 1 && h >= 1 && cmap_ok && bpp_ok) return ImageFormat::kTga;
      }
    }
  }
  return ImageFormat::kUnknown;
}

}  // namespace ym

// Texture nodes on the device: Perlin noise, the solid (procedural) nodes,
// density grids, and the evaluation of a node graph at a surface or medium
// point.
//
// Follows src/TextureEval.cuh (PerlinNoiseEval :55-132, PerlinNoiseFBM
// :134-145, PerlinNoiseTurbulence :146-160, the node evaluators :240-418,
// TextureEval :419-481) and src/Texture.h (GetUpperBound :1181-1251), in the
// reference's operand order (the kernels are built with -fmad=false, so
// every product and sum rounds as written).
#pragma once

#include <cuda_fp16.h>

#include "dev_bound.cuh"
#include "ymrt_scene.h"

namespace ym {

// Lattice permutation of the reference's Perlin noise (src/TextureEval.cuh:19);
// kept identical so that procedural densities match the reference's value for
// value. Indexed modulo 256 (the reference stores it twice in a row).
static __constant__ uint8_t c_perlin_perm[256] = {
    172, 142, 240, 182, 179, 214,  29, 111, 156,   3, 131, 161, 164, 194, 243, 124,
    127, 236,  88, 166,  83, 134,  71, 183, 227, 235, 106, 226, 216,  99, 149, 241,
    206,  63,  48,  31,  20, 171,  46, 185,   6, 125, 184, 133, 199, 201,  58,  81,
    177, 174,  92,  78,  32, 190,  89, 229,  14, 159, 196,  69, 242, 222,  13,  54,
    200,  50,  26, 218,   5, 101,  18,  72, 203, 191, 104, 141, 252,  65, 139, 210,
     22, 180, 113, 253,  27, 102,  25, 169,  56, 110, 178, 105, 254,  80,  73,   4,
     90, 155,  91, 120, 181,   9, 123, 198, 193, 118, 146,  44, 247, 162, 231, 143,
    153, 160,  57, 112, 238,  77,  95,  34, 168, 195, 126, 224, 213, 187,  41,  42,
    152, 219, 220,  39,  53, 138, 239, 157,  12,  38,  24, 188,  76,   7, 103,   1,
     33, 130,  74, 189,  79, 232,  96,  86, 135,  35, 234, 205, 150, 165,  30, 109,
    212,  66,   0, 228, 129,  23,  97,   8, 107, 209, 192, 175,  11,  52,  16, 248,
     55,  28, 173, 115,  51, 163, 197,   2, 208,  64, 148,  37,  19, 167,  84,  61,
    176, 211,  17,  93, 108, 121, 116,  87,  43, 249, 147, 122,  21, 117, 136, 233,
    145,  15, 245,  59,  75, 137, 151, 255, 154, 204, 244,  98,  40,  70,  10,  85,
    225, 223, 251, 158, 132,  45, 119, 114,  60,  67, 140, 144, 207, 215,  47, 246,
    230, 186, 250, 100,  36, 221, 217,  68, 128,  49,  62, 237,  82,  94, 170, 202,
};

__device__ __forceinline__ int perlin_hash(int x, int y, int z) {
  return c_perlin_perm[(c_perlin_perm[(c_perlin_perm[x] + y) & 255] + z) & 255];
}

// Gradient dot products of the 16 lattice directions (PerlinNoiseEval).
__device__ __forceinline__ float perlin_grad(int h, float x, float y, float z) {
  switch (h & 15) {
    case 0: return x + y;
    case 1: return -x + y;
    case 2: return x - y;
    case 3: return -x - y;
    case 4: return x + z;
    case 5: return -x + z;
    case 6: return x - z;
    case 7: return -x - z;
    case 8: return y + z;
    case 9: return -y + z;
    case 10: return y - z;
    case 11: return -y - z;
    case 12: return y + x;
    case 13: return -x + y;
    case 14: return -y + z;
    default: return -y - z;
  }
}

__device__ __forceinline__ float perlin_fade(float t) { return t * t * t * (t * (t * 6.0f - 15.0f) + 10.0f); }

// PerlinNoiseEval (src/TextureEval.cuh:55-132). Out of line: the solid
// nodes, fBm and turbulence call it from a dozen sites, and one shared copy
// keeps the texture-enabled media shading kernel, which is bound by
// instruction fetch, within its instruction cache (the 1280x720 32-spp
// textured frame 889 -> 745 ms; the fBm media frame 892 -> 882 ms; fBm
// itself out of line as well gained nothing more).
static __device__ __noinline__ float perlin_noise(vec3 p) {
  int x0 = (int)floorf(p.x), y0 = (int)floorf(p.y), z0 = (int)floorf(p.z);
  const float tx = p.x - (float)x0, ty = p.y - (float)y0, tz = p.z - (float)z0;
  const int x1 = (x0 + 1) & 255, y1 = (y0 + 1) & 255, z1 = (z0 + 1) & 255;
  x0 &= 255;
  y0 &= 255;
  z0 &= 255;
  const float v000 = perlin_grad(perlin_hash(x0, y0, z0), tx, ty, tz);
  const float v100 = perlin_grad(perlin_hash(x1, y0, z0), tx - 1, ty, tz);
  const float v010 = perlin_grad(perlin_hash(x0, y1, z0), tx, ty - 1, tz);
  const float v001 = perlin_grad(perlin_hash(x0, y0, z1), tx, ty, tz - 1);
  const float v110 = perlin_grad(perlin_hash(x1, y1, z0), tx - 1, ty - 1, tz);
  const float v011 = perlin_grad(perlin_hash(x0, y1, z1), tx, ty - 1, tz - 1);
  const float v101 = perlin_grad(perlin_hash(x1, y0, z1), tx - 1, ty, tz - 1);
  const float v111 = perlin_grad(perlin_hash(x1, y1, z1), tx - 1, ty - 1, tz - 1);
  const float ix = perlin_fade(tx), iy = perlin_fade(ty), iz = perlin_fade(tz);
  const float v00 = v000 + ix * (v100 - v000);
  const float v01 = v001 + ix * (v101 - v001);
  const float v10 = v010 + ix * (v110 - v010);
  const float v11 = v011 + ix * (v111 - v011);
  const float v0 = v00 + iy * (v10 - v00);
  const float v1 = v01 + iy * (v11 - v01);
  return v0 + iz * (v1 - v0);
}

// PerlinNoiseFBM (src/TextureEval.cuh:134-145): layers of noise, each at
// `lacunarity` times the previous frequency and `gain` times its amplitude
// and offset.
__device__ __forceinline__ float perlin_fbm(vec3 p, float lacunarity, float gain, int layers, float amplitude,
                                            float offset) {
  float r = 0.0f, freq = 1.0f;
  for (int i = 0; i < layers; ++i) {
    r += amplitude * perlin_noise(freq * p) + offset;
    amplitude *= gain;
    offset *= gain;
    freq *= lacunarity;
  }
  return r;
}

// PerlinNoiseTurbulence (src/TextureEval.cuh:146-160): fBm of |noise|.
__device__ __forceinline__ float perlin_turbulence(vec3 p, float lacunarity, float gain, int layers, float amplitude,
                                                   float offset) {
  float r = 0.0f, freq = 1.0f;
  for (int i = 0; i < layers; ++i) {
    r += amplitude * fabsf(perlin_noise(freq * p)) + offset;
    amplitude *= gain;
    offset *= gain;
    freq *= lacunarity;
  }
  return r;
}

// ---- density grids (kTexGrid) ----

// The lattice cell of an object-space point along one axis: lower and upper
// sample index and the upper sample's weight, clamped to the edge samples
// outside [0.5/n, 1 - 0.5/n] (and for a NaN coordinate).
__device__ __forceinline__ void grid_axis(float p, int n, int* i0, int* i1, float* w) {
  const float g = (p + 0.5f) * (float)n - 0.5f;
  if (!(g > 0.0f)) {
    *i0 = *i1 = 0;
    *w = 0.0f;
  } else if (!(g < (float)(n - 1))) {
    *i0 = *i1 = n - 1;
    *w = 0.0f;
  } else {
    const float fl = floorf(g);
    *i0 = (int)fl;
    *i1 = *i0 + 1;
    *w = g - fl;
  }
}

__device__ __forceinline__ float grid_at(const Texture& t, int x, int y, int z) {
  const size_t k = ((size_t)z * (size_t)t.grid_n[1] + (size_t)y) * (size_t)t.grid_n[0] + (size_t)x;
  if (t.grid_half) return __half2float(__ushort_as_half(__ldg(static_cast<const unsigned short*>(t.grid) + k)));
  return __ldg(static_cast<const float*>(t.grid) + k);
}

__device__ __forceinline__ float lerp1(float a, float b, float w) { return a + w * (b - a); }

// Trilinear read of a grid node at an object-space point. A constant grid
// reads back its value exactly (a + w * 0 == a). Out of line, so that the
// procedural nodes' tracking loops do not carry its registers.
static __device__ __noinline__ float grid_eval(const Texture& t, vec3 p) {
  int x0, x1, y0, y1, z0, z1;
  float wx, wy, wz;
  grid_axis(p.x, t.grid_n[0], &x0, &x1, &wx);
  grid_axis(p.y, t.grid_n[1], &y0, &y1, &wy);
  grid_axis(p.z, t.grid_n[2], &z0, &z1, &wz);
  const float c00 = lerp1(grid_at(t, x0, y0, z0), grid_at(t, x1, y0, z0), wx);
  const float c10 = lerp1(grid_at(t, x0, y1, z0), grid_at(t, x1, y1, z0), wx);
  const float c01 = lerp1(grid_at(t, x0, y0, z1), grid_at(t, x1, y0, z1), wx);
  const float c11 = lerp1(grid_at(t, x0, y1, z1), grid_at(t, x1, y1, z1), wx);
  return lerp1(lerp1(c00, c10, wy), lerp1(c01, c11, wy), wz);
}

// Where a texture is read (TextureCoordinate, src/Texture.h:61-81, reduced
// to what the supported nodes read): surface texture coordinates (s, t) and
// the object-space position. A medium point has s = t = 0.
struct TexCoord {
  float s, t;
  vec3 p;
};

__device__ __forceinline__ vec3 blend(vec3 black, vec3 white, float v) { return black + v * (white - black); }

// fract(x) * 114 of the polka-dot node's cell-centre jitter.
__device__ __forceinline__ float polka_hash(float x, float m) {
  const float y = x * m;
  return (y - floorf(y)) * 114.f;
}

// The solid nodes (EvalTexCheckerBoard .. EvalTexPerlinNoiseWave,
// src/TextureEval.cuh:246-391), given their inputs' results.
static __device__ __noinline__ vec3 solid_node(const Texture& t, vec3 black, vec3 white, const TexCoord& tc) {
  switch (t.type) {
    case kTexChecker: {
      const float x = sinf(tc.p.x * t.frequency), y = sinf(tc.p.y * t.frequency), z = sinf(tc.p.z * t.frequency);
      return x * y * z < 0.0f ? white : black;
    }
    case kTexNoise: {
      float v = perlin_noise(tc.p * t.frequency);
      if (t.flags & kTexNormalized) v = v * 0.5f + 0.5f;
      return blend(black, white, v);
    }
    case kTexTurbulence:
      return blend(black, white,
                   perlin_turbulence(t.frequency * tc.p, t.lacunarity, t.gain, t.layer_count, t.amplitude, t.offset));
    case kTexMarble: {
      const float fbm = perlin_fbm(t.frequency * tc.p, t.lacunarity, t.gain, t.layer_count, 1.0f, 0.0f);
      float phase = 0.0f;
      phase += (t.flags & kTexTurbX) ? tc.p.x : 0.0f;
      phase += (t.flags & kTexTurbY) ? tc.p.y : 0.0f;
      phase += (t.flags & kTexTurbZ) ? tc.p.z : 0.0f;
      return blend(black, white, sinf(phase + t.variation * fbm) * 0.5f + 0.5f);
    }
    case kTexWood: {
      float w = perlin_noise(tc.p * t.frequency) * t.variation;
      w = w - floorf(w);
      return blend(black, white, w);
    }
    case kTexPolkaDot: {
      const float s = tc.s * t.frequency, u = tc.t * t.frequency;
      const float cs = floorf(s), cu = floorf(u);
      if (!(perlin_noise(vec3(cs + 0.5f, cu + 0.5f, 0.0f)) > 0.0f)) return black;
      const float max_offset = 0.5f - t.radius;
      const float ds = s - cs, du = u - cu;
      const float sc = 0.5f + max_offset * perlin_noise(vec3(polka_hash(s, 1145.14f), polka_hash(u, 9807.26f), 0.0f));
      const float uc = 0.5f + max_offset * perlin_noise(vec3(polka_hash(s, 4444.44f), polka_hash(u, 2333.33f), 0.0f));
      return sqr(ds - sc) + sqr(du - uc) < t.radius * t.radius ? white : black;
    }
    case kTexWave: {
      const float f0 = perlin_fbm(tc.p * t.frequency, t.lacunarity, t.gain, t.layer_count, 1.0f, 0.0f);
      const float f1 = perlin_fbm(tc.p * t.frequency1, t.lacunarity1, t.gain1, t.layer_count1, 1.0f, 0.0f);
      return blend(black, white, fabsf(f0) * f1);
    }
    default:
      return vec3(0.0f);
  }
}

// EvalTexImage (src/TextureEval.cuh:162-237): the image's texture
// coordinates (scaled, offset, negative ones moved up by whole periods),
// bilinear between the four texels around them (texel centres at
// half-integers), each fetched with the node's wrap mode; one channel reads
// as grey, more give their first three.
static __device__ __noinline__ vec3 image_node(const Texture& t, const TexCoord& tc) {
  if (!t.image) return vec3(0.0f);
  float u = tc.s * t.scale_u + t.offset_u;
  if (u < 0.0f) u = gmax(0.0f, u + fabsf(floorf(u)));
  float v = tc.t * t.scale_v + t.offset_v;
  if (v < 0.0f) v = gmax(0.0f, v + fabsf(floorf(v)));
  const float px = u * (float)t.width - 0.5f, py = v * (float)t.height - 0.5f;
  const int x0 = (int)floorf(px), y0 = (int)floorf(py);
  const float fx = px - (float)x0, fy = py - (float)y0;
  const int w = t.width, h = t.height, n = t.channels;
  auto texel = [&](int x, int y) {
    if (t.wrap == kWrapClamp) {
      x = x < 0 ? 0 : (x > w - 1 ? w - 1 : x);
      y = y < 0 ? 0 : (y > h - 1 ? h - 1 : y);
    } else {
      x = ((x % w) + w) % w;
      y = ((y % h) + h) % h;
    }
    const float* p = t.image + ((size_t)y * (size_t)w + (size_t)x) * (size_t)n;
    if (n == 1) return vec3(__ldg(p));
    vec3 r(0.0f);
    for (int c = 0; c < 3 && c < n; ++c) r[c] = __ldg(p + c);
    return r;
  };
  return (1.0f - fx) * (1.0f - fy) * texel(x0, y0) + fx * (1.0f - fy) * texel(x0 + 1, y0) +
         (1.0f - fx) * fy * texel(x0, y0 + 1) + fx * fy * texel(x0 + 1, y0 + 1);
}

// The inputs a node reads: two for the solid nodes, none for constants,
// grids and unknown types.
__device__ __forceinline__ int texture_inputs(uint32_t type) {
  return (type >= kTexChecker && type <= kTexWave) ? 2 : 0;
}

// TextureEval (src/TextureEval.cuh:419-481): a post-order walk of the node
// graph with an explicit stack of kTextureStack nodes, as the reference; an
// absent input reads as black. A deeper graph (the loader rejects those)
// sets bit 1 (kDevErrStack) in *errors and reads as black. kF selects the node types compiled in:
// constants and fBm always, grids with kFeatGrids, the other solid nodes
// with kFeatTextures.
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ vec3 texture_eval(const Texture* __restrict__ tex, uint32_t root, const TexCoord& tc,
                                             uint32_t* errors) {
  struct Frame {
    uint32_t idx;
    int parent, slot, next;
    vec3 in[2];
  };
  Frame st[kTextureStack];
  int top = 0;
  st[0].idx = root;
  st[0].parent = -1;
  st[0].slot = -1;
  st[0].next = 0;
  // at most 3 steps per node of the graph unfolded into a tree (2^kTextureStack - 1 nodes)
  for (int guard = 0; guard < (3 << kTextureStack); ++guard) {
    Frame& f = st[top];
    const Texture& t = tex[f.idx];
    const int n_in = (kF & kFeatTextures) ? texture_inputs(t.type) : (t.type == kTexFbm ? 2 : 0);
    if (f.next < n_in) {
      const uint32_t c = t.child[f.next];
      if (c == kEmpty) {
        f.in[f.next] = vec3(0.0f);
        ++f.next;
        continue;
      }
      if (top + 1 >= kTextureStack) {
        atomicOr(errors, 1u);
        return vec3(0.0f);
      }
      Frame& g = st[++top];
      g.idx = c;
      g.parent = top - 1;
      g.slot = f.next;
      g.next = 0;
      continue;
    }
    vec3 r(0.0f);
    if (t.type == kTexConstFloat) {
      r = vec3(t.value);
    } else if (t.type == kTexConstRgb) {
      r = t.color;
    } else if (t.type == kTexFbm) {
      r = blend(f.in[0], f.in[1],
                perlin_fbm(t.frequency * tc.p, t.lacunarity, t.gain, t.layer_count, t.amplitude, t.offset));
    } else if ((kF & kFeatGrids) && t.type == kTexGrid) {
      r = vec3(grid_eval(t, tc.p));
    } else if ((kF & kFeatTextures) && n_in == 2) {
      r = solid_node(t, f.in[0], f.in[1], tc);
    } else if ((kF & kFeatTextures) && t.type == kTexImage) {
      r = image_node(t, tc);
    }
    if (f.parent < 0) return r;
    Frame& par = st[f.parent];
    par.in[f.slot] = r;
    ++par.next;
    --top;
  }
  atomicOr(errors, 4u);
  note_bound(kBoundTextureWalk, 3u << kTextureStack, tc.p, vec3(0.0f), 0.0f, kEmpty, root, nullptr);
  return vec3(0.0f);
}

// A medium's density node at an object-space point (s = t = 0).
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ vec3 texture_eval(const Texture* __restrict__ tex, uint32_t root, vec3 p_object,
                                             uint32_t* errors) {
  const TexCoord tc{0.0f, 0.0f, p_object};
  return texture_eval<kF>(tex, root, tc, errors);
}

// Texture::GetUpperBound (src/Texture.h:1181-1251): the majorant a medium
// with this density node tracks against.
__device__ __forceinline__ float texture_upper_bound(const Texture& t) {
  switch (t.type) {
    case kTexConstFloat:
    case kTexGrid:
      return t.value;
    case kTexConstRgb:
      return gmax(t.color.x, gmax(t.color.y, t.color.z));
    case kTexFbm:
    case kTexTurbulence: {
      float r = 0.0f, a = t.amplitude, o = t.offset;
      for (int i = 0; i < t.layer_count; ++i) {
        r += a + o;
        a *= t.gain;
        o *= t.gain;
      }
      return r;
    }
    case kTexChecker:
    case kTexNoise:
    case kTexMarble:
    case kTexWood:
    case kTexPolkaDot:
      return 1.0f;
    case kTexWave:
      return safe_rcp(1.0f - t.gain) * safe_rcp(1.0f - t.gain1);
    default:
      return 0.0f;
  }
}

}  // namespace ym

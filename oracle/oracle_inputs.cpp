/*
 * ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of the inputs the cloud march samples: the three noise
 * bakes, the blue-noise tile, layer synthesis, the weather map, the wind
 * field and the headless-render camera.  Floating-point work is done in
 * IEEE binary32 with the operation order written out explicitly and no FMA
 * contraction (the Makefile passes -ffp-contract=off), so that the CUDA
 * bake kernels can be held to byte equality with it.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "oracle_common.h"

using namespace oracle;

namespace {

/* -------------------------------------------------------------------------
 * Noise bakes.  shaders/clouds/noise_base.comp.wgsl:25-139,
 * noise_detail.comp.wgsl:13-72, noise_curl.comp.wgsl:13-74.
 * WGSL vector built-ins are spelled out: length(v) = sqrt((x*x + y*y) + z*z),
 * normalize(v) = v / length(v), mix(a, b, t) = a*(1-t) + b*t (the WGSL
 * specification's formula), dot((a,b,c),(d,e,f)) = (a*d + b*e) + c*f.
 * ---------------------------------------------------------------------- */

inline uint32_t hash3(uint32_t x, uint32_t y, uint32_t z) {  // noise_base:25-30
  uint32_t h = x * 0x27d4eb2du + y * 0x165667b1u + z * 0x9e3779b9u;
  h = (h ^ (h >> 15)) * 0x2c1b3c6du;
  h = (h ^ (h >> 12)) * 0x297a2d39u;
  return h ^ (h >> 15);
}

inline float u16_unit(uint32_t h) { return (float)(h & 0xffffu) / 65535.0f; }

struct F3 {
  float x, y, z;
};

inline F3 rand3(uint32_t x, uint32_t y, uint32_t z) {  // noise_base:32-41
  F3 r;
  r.x = u16_unit(hash3(x, y, z));
  r.y = u16_unit(hash3(x + 1u, y, z));
  r.z = u16_unit(hash3(x, y + 1u, z));
  return r;
}

inline float len3(float x, float y, float z) {
  const float xx = x * x;
  const float yy = y * y;
  const float zz = z * z;
  return std::sqrt((xx + yy) + zz);
}

inline uint32_t wrapi(int32_t c, int32_t f) {
  return (uint32_t)(((c % f) + f) % f);
}

/* Tileable Worley noise (noise_base:45-70).  `off` is the hash offset the
 * detail bake adds (noise_detail.comp.wgsl:49). */
float worley_tile(F3 p, uint32_t freq, uint32_t off) {
  const float fq = (float)freq;
  const float sx = p.x * fq, sy = p.y * fq, sz = p.z * fq;
  const float flx = std::floor(sx), fly = std::floor(sy), flz = std::floor(sz);
  const int32_t cx = (int32_t)flx, cy = (int32_t)fly, cz = (int32_t)flz;
  const float fx = sx - flx, fy = sy - fly, fz = sz - flz;
  float min_d = 1.0f;
  const int32_t f = (int32_t)freq;
  for (int32_t dz = -1; dz <= 1; ++dz) {
    for (int32_t dy = -1; dy <= 1; ++dy) {
      for (int32_t dx = -1; dx <= 1; ++dx) {
        const uint32_t wx = wrapi(cx + dx, f), wy = wrapi(cy + dy, f),
                       wz = wrapi(cz + dz, f);
        const F3 j = off ? rand3(wx + 73u, wy + 19u, wz + 41u) : rand3(wx, wy, wz);
        const float ccx = (float)dx + j.x, ccy = (float)dy + j.y,
                    ccz = (float)dz + j.z;
        const float d = len3(ccx - fx, ccy - fy, ccz - fz);
        min_d = std::fmin(min_d, d);
      }
    }
  }
  return clampv(1.0f - min_d, 0.0f, 1.0f);
}

float worley_fbm(F3 p, uint32_t freq, uint32_t off) {  // noise_base:72-77
  const float f1 = worley_tile(p, freq, off);
  const float f2 = worley_tile(p, freq * 2u, off);
  const float f3 = worley_tile(p, freq * 4u, off);
  return (f1 * 0.625f + f2 * 0.25f) + f3 * 0.125f;
}

inline float fade(float t) {  // noise_base:79-81
  return ((t * t) * t) * (t * (t * 6.0f - 15.0f) + 10.0f);
}

inline float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }

F3 perlin_grad3(int32_t cx, int32_t cy, int32_t cz, uint32_t freq) {  // :83-90
  const int32_t f = (int32_t)freq;
  const F3 r = rand3(wrapi(cx, f), wrapi(cy, f), wrapi(cz, f));
  const float vx = r.x * 2.0f - 1.0f, vy = r.y * 2.0f - 1.0f,
              vz = r.z * 2.0f - 1.0f;
  const float l = len3(vx, vy, vz);
  return F3{vx / l, vy / l, vz / l};
}

float perlin_tile(F3 p, uint32_t freq) {  // noise_base:92-115
  const float fq = (float)freq;
  const float sx = p.x * fq, sy = p.y * fq, sz = p.z * fq;
  const float flx = std::floor(sx), fly = std::floor(sy), flz = std::floor(sz);
  const int32_t cx = (int32_t)flx, cy = (int32_t)fly, cz = (int32_t)flz;
  const float fx = sx - flx, fy = sy - fly, fz = sz - flz;
  const float ux = fade(fx), uy = fade(fy), uz = fade(fz);
  float dots[8];
  for (int iz = 0; iz < 2; ++iz) {
    for (int iy = 0; iy < 2; ++iy) {
      for (int ix = 0; ix < 2; ++ix) {
        const F3 g = perlin_grad3(cx + ix, cy + iy, cz + iz, freq);
        const float dx = fx - (float)ix, dy = fy - (float)iy, dz = fz - (float)iz;
        dots[ix + iy * 2 + iz * 4] = (g.x * dx + g.y * dy) + g.z * dz;
      }
    }
  }
  const float x00 = mixf(dots[0], dots[1], ux);
  const float x10 = mixf(dots[2], dots[3], ux);
  const float x01 = mixf(dots[4], dots[5], ux);
  const float x11 = mixf(dots[6], dots[7], ux);
  const float y0 = mixf(x00, x10, uy);
  const float y1 = mixf(x01, x11, uy);
  return mixf(y0, y1, uz) * 0.5f + 0.5f;
}

float perlin_fbm(F3 p, uint32_t f) {  // noise_base:117-122
  const float p1 = perlin_tile(p, f);
  const float p2 = perlin_tile(p, f * 2u);
  const float p3 = perlin_tile(p, f * 4u);
  return (p1 * 0.5f + p2 * 0.25f) + p3 * 0.125f;
}

inline float remapf(float v, float a, float b, float c, float d) {  // math.wgsl:7
  return c + ((v - a) * (d - c)) / std::fmax(b - a, 1e-5f);
}

/* textureStore into a unorm8 target: round-to-nearest of clamp(v)*255. */
inline uint8_t unorm8(float v) {
  return (uint8_t)std::nearbyint(clampv(v, 0.0f, 1.0f) * 255.0f);
}

inline F3 voxel_centre(uint32_t x, uint32_t y, uint32_t z, float size) {
  return F3{((float)x + 0.5f) / size, ((float)y + 0.5f) / size,
            ((float)z + 0.5f) / size};
}

/* curl (noise_curl.comp.wgsl) */
inline uint32_t hash2u(uint32_t x, uint32_t y) {  // :13-18
  uint32_t h = x * 0x27d4eb2du + y * 0x165667b1u;
  h = (h ^ (h >> 15)) * 0x2c1b3c6du;
  h = (h ^ (h >> 12)) * 0x297a2d39u;
  return h ^ (h >> 15);
}

float perlin2(float px, float py, uint32_t freq) {  // :36-56
  const float fq = (float)freq;
  const float sx = px * fq, sy = py * fq;
  const float flx = std::floor(sx), fly = std::floor(sy);
  const int32_t cx = (int32_t)flx, cy = (int32_t)fly;
  const float fx = sx - flx, fy = sy - fly;
  const float ux = fade(fx), uy = fade(fy);
  const int32_t f = (int32_t)freq;
  float g[4][2];
  const int offs[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
  for (int k = 0; k < 4; ++k) {
    const uint32_t wx = wrapi(cx + offs[k][0], f), wy = wrapi(cy + offs[k][1], f);
    const float rx = (float)(hash2u(wx, wy) & 0xffffu) / 65535.0f * 2.0f - 1.0f;
    const float ry = (float)(hash2u(wx + 1u, wy) & 0xffffu) / 65535.0f * 2.0f - 1.0f;
    const float l = std::sqrt(rx * rx + ry * ry);
    g[k][0] = rx / l;
    g[k][1] = ry / l;
  }
  const float d00 = g[0][0] * (fx - 0.0f) + g[0][1] * (fy - 0.0f);
  const float d10 = g[1][0] * (fx - 1.0f) + g[1][1] * (fy - 0.0f);
  const float d01 = g[2][0] * (fx - 0.0f) + g[2][1] * (fy - 1.0f);
  const float d11 = g[3][0] * (fx - 1.0f) + g[3][1] * (fy - 1.0f);
  const float x0 = mixf(d00, d10, ux);
  const float x1 = mixf(d01, d11, ux);
  return mixf(x0, x1, uy);
}

inline float potential(float x, float y) {  // noise_curl:58-60
  return perlin2(x, y, 4u) + 0.5f * perlin2(x, y, 8u);
}

}  // namespace

extern "C" {

uint16_t oracle_f32_to_f16(float f) { return f32_to_f16(f); }
float oracle_f16_to_f32(uint16_t h) { return f16_to_f32(h); }

int oracle_bake_noise_base(uint8_t* out) {  // noise_base.comp.wgsl:124-139
  if (!out) return -1;
  const uint32_t N = 128;
#pragma omp parallel for schedule(dynamic)
  for (int z = 0; z < (int)N; ++z) {
    for (uint32_t y = 0; y < N; ++y) {
      for (uint32_t x = 0; x < N; ++x) {
        const F3 p = voxel_centre(x, y, (uint32_t)z, 128.0f);
        const float perlin = perlin_fbm(p, 4u);
        const float worley_low = worley_fbm(p, 4u, 0);
        const float pw = clampv(remapf(perlin, worley_low - 1.0f, 1.0f, 0.0f, 1.0f),
                                0.0f, 1.0f);
        const float g = worley_fbm(p, 2u, 0);
        const float b = worley_fbm(p, 8u, 0);
        const float a = worley_fbm(p, 14u, 0);
        uint8_t* t = out + (((size_t)z * N + y) * N + x) * 4;
        t[0] = unorm8(pw);
        t[1] = unorm8(g);
        t[2] = unorm8(b);
        t[3] = unorm8(a);
      }
    }
  }
  return 0;
}

int oracle_bake_noise_detail(uint8_t* out) {  // noise_detail.comp.wgsl:62-72
  if (!out) return -1;
  const uint32_t N = 32;
#pragma omp parallel for schedule(dynamic)
  for (int z = 0; z < (int)N; ++z) {
    for (uint32_t y = 0; y < N; ++y) {
      for (uint32_t x = 0; x < N; ++x) {
        const F3 p = voxel_centre(x, y, (uint32_t)z, 32.0f);
        uint8_t* t = out + (((size_t)z * N + y) * N + x) * 4;
        t[0] = unorm8(worley_fbm(p, 2u, 1));
        t[1] = unorm8(worley_fbm(p, 8u, 1));
        t[2] = unorm8(worley_fbm(p, 16u, 1));
        t[3] = 0;
      }
    }
  }
  return 0;
}

int oracle_bake_noise_curl(uint8_t* out) {  // noise_curl.comp.wgsl:62-74
  if (!out) return -1;
  const uint32_t N = 128;
  const float eps = 1.0f / 128.0f;
  for (uint32_t y = 0; y < N; ++y) {
    for (uint32_t x = 0; x < N; ++x) {
      const float px = ((float)x + 0.5f) / 128.0f, py = ((float)y + 0.5f) / 128.0f;
      const float dpdx = (potential(px + eps, py + 0.0f) - potential(px - eps, py - 0.0f)) /
                         (2.0f * eps);
      const float dpdy = (potential(px + 0.0f, py + eps) - potential(px - 0.0f, py - eps)) /
                         (2.0f * eps);
      const float cx = dpdy, cy = -dpdx;
      out[(y * N + x) * 2 + 0] = unorm8(clampv(cx * 0.5f + 0.5f, 0.0f, 1.0f));
      out[(y * N + x) * 2 + 1] = unorm8(clampv(cy * 0.5f + 0.5f, 0.0f, 1.0f));
    }
  }
  return 0;
}

/* Void-and-cluster blue noise, crates/ps-clouds/src/noise.rs:646-704. */
int oracle_blue_noise(uint8_t* out) {
  if (!out) return -1;
  const int size = 64;
  const int n = size * size;
  std::vector<char> taken(n, 0);
  std::vector<uint32_t> ranks(n, 0);
  std::vector<float> energy(n, 0.0f);
  const float sigma = 1.9f;
  const int radius = 6;
  const float inv_two_sigma2 = 1.0f / ((2.0f * sigma) * sigma);
  auto idx = [&](int x, int y) {
    int mx = ((x % size) + size) % size;
    int my = ((y % size) + size) % size;
    return my * size + mx;
  };
  for (int placement = 0; placement < n; ++placement) {
    int best = 0;
    float best_e = INFINITY;
    for (int i = 0; i < n; ++i) {
      if (!taken[i] && energy[i] < best_e) {
        best_e = energy[i];
        best = i;
      }
    }
    taken[best] = 1;
    ranks[best] = (uint32_t)placement;
    const int cx = best % size, cy = best / size;
    for (int dy = -radius; dy <= radius; ++dy) {
      for (int dx = -radius; dx <= radius; ++dx) {
        const float r2 = (float)(dx * dx + dy * dy);
        const float w = std::exp(-r2 * inv_two_sigma2) * 1.0f;
        energy[idx(cx + dx, cy + dy)] += w;
      }
    }
  }
  const float max_rank = (float)(n - 1);
  for (int i = 0; i < n; ++i) {
    float v = std::round(((float)ranks[i] / max_rank) * 255.0f);
    v = clampv(v, 0.0f, 255.0f);
    out[i] = (uint8_t)v;
  }
  return 0;
}

/* crates/ps-synthesis/src/cloud_layers.rs:106-126 */
float oracle_remap_coverage(float scene_coverage) {
  const float VISIBLE_LOW = 0.40f, VISIBLE_HIGH = 0.60f, KNEE_END = 0.10f;
  const float t = clampv(scene_coverage, 0.0f, 1.0f);
  if (t <= 0.0f) return 0.0f;
  if (t < KNEE_END) {
    const float s = t / KNEE_END;
    const float smoothed = s * s * (3.0f - 2.0f * s);
    return smoothed * VISIBLE_LOW;
  }
  const float band_t = clampv((t - KNEE_END) / (1.0f - KNEE_END), 0.0f, 1.0f);
  return VISIBLE_LOW + band_t * (VISIBLE_HIGH - VISIBLE_LOW);
}

/* synthesise_cloud_layers + check_non_overlap, cloud_layers.rs:44-74,136-150;
 * per-type defaults from crates/ps-core/src/scene.rs:293-352. */
int oracle_synthesise_layers(const PscCloudLayerDesc* in, uint32_t n,
                             PscCloudLayerGpu* out) {
  static const float density_default[8] = {1.0f, 1.0f, 1.0f, 0.85f,
                                           0.7f, 0.55f, 0.4f, 1.4f};
  static const float droplet_default[8] = {20.0f, 16.0f, 16.0f, 14.0f,
                                           30.0f, 50.0f, 50.0f, 20.0f};
  if ((!in && n) || !out) return -1;
  for (uint32_t i = 0; i < n; ++i) {
    const PscCloudLayerDesc& l = in[i];
    if (l.cloud_type > 7) return -1;
    PscCloudLayerGpu g;
    std::memset(&g, 0, sizeof(g));
    g.base_m = l.base_m;
    g.top_m = l.top_m;
    g.coverage = oracle_remap_coverage(l.coverage);
    g.density_scale = l.density_scale >= 0.0f ? l.density_scale
                                              : density_default[l.cloud_type];
    g.cloud_type = l.cloud_type;
    g.shape_bias = l.shape_octave_bias;
    g.detail_bias = l.detail_octave_bias;
    g.anvil_bias = l.anvil_bias >= 0.0f ? l.anvil_bias
                                        : (l.cloud_type == 7 ? 1.0f : 0.0f);
    g.droplet_diameter_um = l.droplet_diameter_um >= 0.0f
                                ? l.droplet_diameter_um
                                : droplet_default[l.cloud_type];
    out[i] = g;
  }
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = i + 1; j < n; ++j)
      if (out[i].base_m < out[j].top_m && out[j].base_m < out[i].top_m) return -3;
  return 0;
}

/* weather_map.rs:160-183 */
static float weather_hash2(int32_t x, int32_t y) {
  uint32_t h = (uint32_t)x * 2654435761u;
  h ^= (uint32_t)y * 2246822519u;
  h ^= h >> 16;
  h = h * 2654435761u;
  h ^= h >> 13;
  return clampv((float)h / 4294967296.0f, 0.0f, 1.0f);
}

float oracle_value_noise_2d(float x, float y) {  // weather_map.rs:160-176
  const float xi = std::floor(x), yi = std::floor(y);
  const float xf = x - xi, yf = y - yi;
  const int32_t ix = (int32_t)xi, iy = (int32_t)yi;
  const float h00 = weather_hash2(ix, iy);
  const float h10 = weather_hash2(ix + 1, iy);
  const float h01 = weather_hash2(ix, iy + 1);
  const float h11 = weather_hash2(ix + 1, iy + 1);
  const float sx = xf * xf * (3.0f - 2.0f * xf);
  const float sy = yf * yf * (3.0f - 2.0f * yf);
  const float bottom = h00 + (h10 - h00) * sx;
  const float top = h01 + (h11 - h01) * sx;
  return bottom + (top - bottom) * sy;
}

/* coverage_grid.rs:34-60 */
static float grid_sample_world(const float* d, uint32_t w, uint32_t h,
                               float extent, float x, float z) {
  const float half = extent * 0.5f;
  const float u = clampv((x + half) / extent, 0.0f, 1.0f);
  const float v = clampv((z + half) / extent, 0.0f, 1.0f);
  const float fx = u * ((float)w - 1.0f);
  const float fy = v * ((float)h - 1.0f);
  const uint32_t x0 = (uint32_t)std::floor(fx), y0 = (uint32_t)std::floor(fy);
  const uint32_t x1 = std::min(x0 + 1, w - 1), y1 = std::min(y0 + 1, h - 1);
  const float tx = fx - (float)x0, ty = fy - (float)y0;
  const float v00 = d[y0 * w + x0], v10 = d[y0 * w + x1];
  const float v01 = d[y1 * w + x0], v11 = d[y1 * w + x1];
  const float bottom = v00 + (v10 - v00) * tx;
  const float top = v01 + (v11 - v01) * tx;
  return clampv(bottom + (top - bottom) * ty, 0.0f, 1.0f);
}

/* WeatherMap::synthesise, weather_map.rs:46-101. */
int oracle_weather_map(uint32_t n_layers, float precip, float wetness,
                       const float* grid, uint32_t gw, uint32_t gh,
                       float extent, uint16_t* out) {
  if (!out) return -1;
  const uint32_t S = 128;
  const float EXTENT = 32000.0f;
  const float gate = n_layers > 0 ? 1.0f : 0.0f;
  const float precip_alpha = clampv(precip / 50.0f, 0.0f, 1.0f);
  const float wet_alpha = clampv(wetness, 0.0f, 1.0f);
  const float alpha = std::fmax(precip_alpha, wet_alpha);
  for (uint32_t y = 0; y < S; ++y) {
    for (uint32_t x = 0; x < S; ++x) {
      const float half = EXTENT * 0.5f;
      const float fx = ((float)x + 0.5f) / (float)S;
      const float fy = ((float)y + 0.5f) / (float)S;
      const float gx = fx * EXTENT - half, gy = fy * EXTENT - half;
      const float cov = grid ? grid_sample_world(grid, gw, gh, extent, gx, gy) : gate;
      const float bias = oracle_value_noise_2d((float)x * 0.05f, (float)y * 0.05f) * 2.0f - 1.0f;
      uint16_t* t = out + (y * S + x) * 4;
      t[0] = f32_to_f16(cov);
      t[1] = f32_to_f16(0.0f);
      t[2] = f32_to_f16(bias);
      t[3] = f32_to_f16(alpha);
    }
  }
  return 0;
}

/* WindField::synthesise, procedural branch (wind_field.rs:71-116,150-170).
 * Only the u/v channels feed the march (cloud_density_common.wgsl:154-161);
 * w and turbulence are written as 0. */
int oracle_wind_field(float speed, float dir_deg, uint16_t* out) {
  if (!out) return -1;
  const float PI_F = 3.14159265358979323846f;
  const float rads_per_deg = PI_F / 180.0f;
  const float dir_to_rad = (dir_deg + 180.0f) * rads_per_deg;
  const float ekman = 30.0f * PI_F / 180.0f;
  const uint32_t SX = 32, SY = 16, SZ = 32;
  for (uint32_t z = 0; z < SZ; ++z) {
    for (uint32_t y = 0; y < SY; ++y) {
      for (uint32_t x = 0; x < SX; ++x) {
        const float alt = ((float)y + 0.5f) / (float)SY * 12000.0f;
        const float sp = speed * std::pow(std::fmax(alt, 10.0f) / 10.0f, 0.143f);
        const float veer = std::pow(clampv(alt / 12000.0f, 0.0f, 1.0f), 0.7f);
        const float vr = dir_to_rad + veer * ekman;
        const float u = sp * std::sin(vr);
        const float v = sp * -std::cos(vr);
        uint16_t* t = out + ((z * SY * SX + y * SX + x) * 4);
        t[0] = f32_to_f16(u);
        t[1] = f32_to_f16(v);
        t[2] = 0;
        t[3] = 0;
      }
    }
  }
  return 0;
}

/* FlyCamera view/projection (crates/ps-core/src/camera.rs:44-70; glam's
 * look_to_rh / perspective_infinite_reverse_rh), FrameUniforms::set_matrices
 * and set_sun (frame_uniforms.rs:80-118) as the headless harness fills them
 * (crates/ps-app/src/test_harness.rs:353-387), and altaz_to_world
 * (crates/ps-core/src/world.rs:110-114).  Computed in double, stored f32. */
int oracle_frame_from_camera(const PscFlyCamera* cam, uint32_t width,
                             uint32_t height, float sun_alt, float sun_az,
                             float sun_ang, float lux, PscFrameUniformsGpu* o) {
  if (!cam || !o || !width || !height) return -1;
  std::memset(o, 0, sizeof(*o));
  typedef double M4[4][4];  // [col][row]
  const double sy = std::sin((double)cam->yaw_rad), cy = std::cos((double)cam->yaw_rad);
  const double sp = std::sin((double)cam->pitch_rad), cp = std::cos((double)cam->pitch_rad);
  double f[3] = {cp * sy, sp, -cp * cy};
  double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (double& v : f) v /= fl;
  // s = f x up(0,1,0) = (-f.z, 0, f.x)
  double s[3] = {-f[2], 0.0, f[0]};
  double sl = std::sqrt(s[0] * s[0] + s[2] * s[2]);
  for (double& v : s) v /= sl;
  double u[3] = {s[1] * f[2] - s[2] * f[1], s[2] * f[0] - s[0] * f[2],
                 s[0] * f[1] - s[1] * f[0]};
  const double e[3] = {cam->position[0], cam->position[1], cam->position[2]};
  M4 view = {{s[0], u[0], -f[0], 0}, {s[1], u[1], -f[1], 0}, {s[2], u[2], -f[2], 0},
             {-(e[0] * s[0] + e[1] * s[1] + e[2] * s[2]),
              -(e[0] * u[0] + e[1] * u[1] + e[2] * u[2]),
              (e[0] * f[0] + e[1] * f[1] + e[2] * f[2]), 1}};
  if (cam->roll_rad != 0.0f) {
    const double c = std::cos((double)cam->roll_rad), sn = std::sin((double)cam->roll_rad);
    M4 rz = {{c, sn, 0, 0}, {-sn, c, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
    M4 r;
    for (int col = 0; col < 4; ++col)
      for (int row = 0; row < 4; ++row) {
        double acc = 0;
        for (int k = 0; k < 4; ++k) acc += rz[k][row] * view[col][k];
        r[col][row] = acc;
      }
    std::memcpy(view, r, sizeof(M4));
  }
  const double aspect = (double)width / (double)height;
  const double fy = 1.0 / std::tan(0.5 * (double)cam->fov_y_rad);
  M4 proj = {{fy / aspect, 0, 0, 0}, {0, fy, 0, 0}, {0, 0, 0, -1}, {0, 0, cam->near_m, 0}};
  M4 vp;
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      double acc = 0;
      for (int k = 0; k < 4; ++k) acc += proj[k][row] * view[col][k];
      vp[col][row] = acc;
    }
  // inverse by Gauss-Jordan on the row-major copy
  double a[4][8];
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      a[r][c] = vp[c][r];
      a[r][c + 4] = (r == c) ? 1.0 : 0.0;
    }
  for (int c = 0; c < 4; ++c) {
    int piv = c;
    for (int r = c + 1; r < 4; ++r)
      if (std::fabs(a[r][c]) > std::fabs(a[piv][c])) piv = r;
    if (a[piv][c] == 0.0) return -1;
    if (piv != c)
      for (int k = 0; k < 8; ++k) std::swap(a[c][k], a[piv][k]);
    const double d = a[c][c];
    for (int k = 0; k < 8; ++k) a[c][k] /= d;
    for (int r = 0; r < 4; ++r)
      if (r != c) {
        const double m = a[r][c];
        for (int k = 0; k < 8; ++k) a[r][k] -= m * a[c][k];
      }
  }
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      o->view[col][row] = (float)view[col][row];
      o->proj[col][row] = (float)proj[col][row];
      o->view_proj[col][row] = (float)vp[col][row];
      o->prev_view_proj[col][row] = (float)vp[col][row];
      o->inv_view_proj[col][row] = (float)a[row][col + 4];
    }
  o->camera_position_world[0] = cam->position[0];
  o->camera_position_world[1] = std::fmax(cam->position[1], 0.1f);
  o->camera_position_world[2] = cam->position[2];
  o->viewport_size[0] = (float)width;
  o->viewport_size[1] = (float)height;
  o->viewport_size[2] = 1.0f / (float)width;
  o->viewport_size[3] = 1.0f / (float)height;
  const double sa = std::sin((double)sun_alt), ca = std::cos((double)sun_alt);
  const double sz = std::sin((double)sun_az), cz = std::cos((double)sun_az);
  o->sun_direction[0] = (float)(ca * sz);
  o->sun_direction[1] = (float)sa;
  o->sun_direction[2] = (float)(-ca * cz);
  o->sun_direction[3] = sun_ang;
  for (int i = 0; i < 4; ++i) o->sun_illuminance[i] = lux;
  return 0;
}

/* CloudParamsGpu::default() (crates/ps-clouds/src/params.rs:142-212), field
 * by field in declaration order. */
int oracle_params_default(PscCloudParamsGpu* o) {
  if (!o) return -1;
  std::memset(o, 0, sizeof(*o));
  const float sig_s[3] = {0.030f, 0.040f, 0.060f};
  for (int k = 0; k < 3; ++k) o->sigma_s[k] = sig_s[k];
  o->droplet_diameter_bias = 1.0f;
  o->cone_light_sampling = 0u;
  o->forward_bias = 0.0f;
  o->detail_strength = 0.05f;
  o->curl_strength = 0.1f;
  o->powder_strength = 1.0f;
  o->multi_scatter_a = 0.5f;
  o->multi_scatter_b = 0.5f;
  o->multi_scatter_c = 0.5f;
  o->ambient_strength = 1.0f;
  o->base_scale_m = 4500.0f;
  o->detail_scale_m = 800.0f;
  o->weather_scale_m = 32000.0f;
  o->light_steps = 6u;
  o->cloud_steps = 192u;
  o->multi_scatter_octaves = 4u;
  o->cloud_layer_count = 0u;
  o->temporal_jitter = 0u;
  o->wind_drift_strength = 1.0f;
  o->wind_skew_strength = 0.5f;
  o->diurnal_strength = 1.0f;
  return 0;
}

/* AtmosphereParams::default() (crates/ps-core/src/weather.rs:60-84). */
int oracle_world_default(PscWorldUniformsGpu* o) {
  if (!o) return -1;
  std::memset(o, 0, sizeof(*o));
  o->planet_radius_m = 6360000.0f;
  o->atmosphere_top_m = 6460000.0f;
  o->rayleigh_scale_height_m = 8000.0f;
  o->mie_scale_height_m = 1200.0f;
  const float rayleigh[4] = {5.802e-6f, 13.558e-6f, 33.100e-6f, 0.0f};
  const float ozone[4] = {0.650e-6f, 1.881e-6f, 0.085e-6f, 0.0f};
  for (int k = 0; k < 4; ++k) {
    const float rgb = k < 3 ? 1.0f : 0.0f;  // w components are 0
    o->rayleigh_scattering[k] = rayleigh[k];
    o->mie_scattering[k] = 3.996e-6f * rgb;
    o->mie_absorption[k] = 4.4e-6f * rgb;
    o->ozone_absorption[k] = ozone[k];
    o->ground_albedo[k] = 0.18f * rgb;
    o->haze_extinction_per_m[k] = 0.0f;
  }
  o->mie_g = 0.8f;
  o->ozone_center_m = 25000.0f;
  o->ozone_thickness_m = 30000.0f;
  return 0;
}

}  // extern "C"

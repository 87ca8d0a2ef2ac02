// Gradient of the procedural march's image loss with respect to one cloud
// layer's parameters: coverage, shape_bias, detail_bias, density_scale,
// base_m and top_m.
//
// The first four enter the march only through sample_density
// (cloud_march.wgsl:432-530; march_plain.cuh:density_at): the coverage gate
// and remap (eff = clamp(weather.r * coverage, 0, 1)), the low-frequency
// erosion (lf = clamp(fbm + shape_bias * diurnal / 2, 0, 1)), the detail
// erosion (clamp(detail_strength + detail_bias * diurnal, 0, 1)) and the
// final scale.  The layer's base and top enter geometrically: the ray's
// entry and exit distances are its intersections with the spheres at planet
// radius + base and + top, the primary samples are spread over that
// interval, the normalised height h = (alt - base) / (top - base) drives the
// profile, the height-scaled skew (skew_thickness = (top - base) * skew
// strength) and the detail polarity, the wind offset is the wind field at the
// layer's mid-altitude, the light path runs to the top, and the ambient
// gradient uses h.  Every quantity of the per-ray march is carried here as a
// value with its six derivatives (forward mode), one thread per ray, in the
// PLAIN march's FP32 arithmetic and order with exact (FP32-weight)
// filtering: sample positions and altitudes, the weather, base, curl and
// detail taps (their filter weights' derivatives with respect to the
// position), the density, the light march's optical depth, Beer-powder and
// the multi-scatter octaves, the sun transmittance and sky-view lookups, the
// in-scattered step integral, the transmittance, the luminance-weighted
// cloud distance and the aerial-perspective blend it selects.  The branch
// decisions (the 1e-3 density threshold, the 0.01 coverage gate, the early
// exits, the layer hits and their order) are taken on the values and are
// constant under the derivative, as for any tangent of the march.  With the
// Kahan option the values are summed plainly.
//
// The loss is the adjoint's: sum((I - target)^2) / (3 * viewport pixels),
// I = L + background * T per pixel and channel, over the view's rectangle;
// each ray adds its 2 (I - target) / N . dI to the six results.
#include <cuda_runtime.h>
#include <stdint.h>

#include "march_common.cuh"
#include "march_plain.cuh"
#include "march_ray.cuh"
#include "psc_internal.h"

namespace psc {
namespace {

constexpr int kTileW = 16;
constexpr int kTileH = 8;
constexpr int kThreads = 128;
// derivative slots: coverage, shape_bias, detail_bias, density_scale, base_m, top_m
constexpr int kP = 6;
constexpr int kBase = 4, kTop = 5;

struct DV {
  float v;
  float d[kP];
};
__device__ __forceinline__ DV dc(float v) {
  DV r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = 0.0f;
  return r;
}
// a value with slope k along another value's derivatives
__device__ __forceinline__ DV along(float v, float k, const DV& x) {
  DV r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = k * x.d[i];
  return r;
}
__device__ __forceinline__ DV operator+(const DV& x, const DV& y) {
  DV r;
  r.v = x.v + y.v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] + y.d[i];
  return r;
}
__device__ __forceinline__ DV operator-(const DV& x, const DV& y) {
  DV r;
  r.v = x.v - y.v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] - y.d[i];
  return r;
}
__device__ __forceinline__ DV operator+(const DV& x, float s) {
  DV r = x;
  r.v = x.v + s;
  return r;
}
__device__ __forceinline__ DV operator+(float s, const DV& x) { return x + s; }
__device__ __forceinline__ DV operator-(const DV& x, float s) {
  DV r = x;
  r.v = x.v - s;
  return r;
}
__device__ __forceinline__ DV operator-(float s, const DV& x) {
  DV r;
  r.v = s - x.v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = -x.d[i];
  return r;
}
__device__ __forceinline__ DV operator-(const DV& x) { return 0.0f - x; }
__device__ __forceinline__ DV operator*(const DV& x, float s) {
  DV r;
  r.v = x.v * s;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] * s;
  return r;
}
__device__ __forceinline__ DV operator*(float s, const DV& x) {
  DV r;
  r.v = s * x.v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] * s;
  return r;
}
__device__ __forceinline__ DV operator*(const DV& x, const DV& y) {
  DV r;
  r.v = x.v * y.v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = fmaf(x.d[i], y.v, x.v * y.d[i]);
  return r;
}
__device__ __forceinline__ DV operator/(const DV& x, const DV& y) {
  const float q = x.v / y.v, iy = 1.0f / y.v;
  DV r;
  r.v = q;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = (x.d[i] - q * y.d[i]) * iy;
  return r;
}
__device__ __forceinline__ DV operator/(const DV& x, float s) {
  const float is = 1.0f / s;
  DV r;
  r.v = x.v / s;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] * is;
  return r;
}
__device__ __forceinline__ DV dexp(const DV& x) {
  const float e = expf(x.v);
  return along(e, e, x);
}
__device__ __forceinline__ DV dlog(const DV& x) { return along(logf(x.v), 1.0f / x.v, x); }
__device__ __forceinline__ DV dsqrt(const DV& x) {
  const float r = sqrtf(fmaxf(x.v, 0.0f));
  return along(r, r > 0.0f ? 0.5f / r : 0.0f, x);
}
__device__ __forceinline__ DV dmax(const DV& x, float m) { return x.v > m ? x : dc(fmaxf(x.v, m)); }
__device__ __forceinline__ DV dmin(const DV& x, float m) { return x.v < m ? x : dc(fminf(x.v, m)); }
__device__ __forceinline__ DV dclamp(const DV& x, float lo, float hi) {
  return (x.v > lo && x.v < hi) ? x : dc(clampf(x.v, lo, hi));
}
__device__ __forceinline__ DV dclamp01(const DV& x) { return dclamp(x, 0.0f, 1.0f); }
// mixf(a, b, t) = a (1 - t) + b t
__device__ __forceinline__ DV dmix(const DV& a, const DV& b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ DV dmix(const DV& a, const DV& b, const DV& t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ DV dmix(float a, float b, const DV& t) { return along(mixf(a, b, t.v), b - a, t); }
// remapf(v, a, 1, 0, 1) = 0 + ((v - a) * 1) / max(1 - a, 1e-5)
__device__ __forceinline__ DV dremap01(const DV& v, const DV& a) { return (v - a) * 1.0f / dmax(1.0f - a, 1e-5f); }
// smoothstepf(e0, e1, x), reversed ramps included
__device__ __forceinline__ DV dsmooth(float e0, float e1, const DV& x) {
  const float t = clamp01((x.v - e0) / (e1 - e0));
  const float k = (t > 0.0f && t < 1.0f) ? 6.0f * t * (1.0f - t) / (e1 - e0) : 0.0f;
  return along(t * t * (3.0f - 2.0f * t), k, x);
}
// atan2(y, x): d = (x dy - y dx) / (x^2 + y^2)
__device__ __forceinline__ DV datan2(const DV& y, const DV& x) {
  const float n = fmaf(x.v, x.v, y.v * y.v), k = n > 0.0f ? 1.0f / n : 0.0f;
  DV r;
  r.v = atan2f(y.v, x.v);
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) * k;
  return r;
}
__device__ __forceinline__ DV dasin(const DV& x) {
  const float q = fmaf(-x.v, x.v, 1.0f);
  return along(asinf(x.v), q > 0.0f ? rsqrtf(q) : 0.0f, x);
}
struct DV3 {
  DV x, y, z;
};
struct DV4 {
  DV x, y, z, w;
};
// value v + gradient g along coordinates (a, b, c): v + g . d(a, b, c)
__device__ __forceinline__ DV chain3(float v, float ga, float gb, float gc, const DV& a, const DV& b, const DV& c) {
  DV r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = fmaf(ga, a.d[i], fmaf(gb, b.d[i], gc * c.d[i]));
  return r;
}

// ------------------------------------------------ filters with gradients
// trilinear_repeat (march_common.cuh) and its gradient with respect to the
// normalised coordinates (texel weights w = u N - 0.5 - floor: dw/du = N).
template <int ST, int N>
__device__ __forceinline__ DV4 trilinear_d(const void* vol, const DV& u, const DV& v, const DV& w, float vscale) {
  const float x = u.v * (float)N - 0.5f, y = v.v * (float)N - 0.5f, z = w.v * (float)N - 0.5f;
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  const float wx = x - fx, wy = y - fy, wz = z - fz;
  const uint32_t x0 = (uint32_t)ix & (N - 1), x1 = (uint32_t)(ix + 1) & (N - 1);
  const uint32_t y0 = (uint32_t)iy & (N - 1), y1 = (uint32_t)(iy + 1) & (N - 1);
  const uint32_t z0 = (uint32_t)iz & (N - 1), z1 = (uint32_t)(iz + 1) & (N - 1);
  const uint32_t r00 = (z0 * N + y0) * N, r10 = (z0 * N + y1) * N;
  const uint32_t r01 = (z1 * N + y0) * N, r11 = (z1 * N + y1) * N;
  const float4 c[8] = {load_texel<ST>(vol, r00 + x0), load_texel<ST>(vol, r00 + x1),
                       load_texel<ST>(vol, r10 + x0), load_texel<ST>(vol, r10 + x1),
                       load_texel<ST>(vol, r01 + x0), load_texel<ST>(vol, r01 + x1),
                       load_texel<ST>(vol, r11 + x0), load_texel<ST>(vol, r11 + x1)};
  const float s = storage_scale<ST>(vscale);
  float val[4], gx[4], gy[4], gz[4];
#pragma unroll
  for (int ch = 0; ch < 4; ++ch) {
    auto C = [&](int k) {
      const float4 t = c[k];
      return ch == 0 ? t.x : (ch == 1 ? t.y : (ch == 2 ? t.z : t.w));
    };
    // the value exactly as trilinear_repeat forms it
    const float a = lerpf(lerpf(C(0), C(1), wx), lerpf(C(2), C(3), wx), wy);
    const float b = lerpf(lerpf(C(4), C(5), wx), lerpf(C(6), C(7), wx), wy);
    val[ch] = lerpf(a, b, wz) * s;
    const float dx0 = lerpf(C(1) - C(0), C(3) - C(2), wy), dx1 = lerpf(C(5) - C(4), C(7) - C(6), wy);
    gx[ch] = lerpf(dx0, dx1, wz) * s * (float)N;
    const float dy0 = lerpf(C(2), C(3), wx) - lerpf(C(0), C(1), wx);
    const float dy1 = lerpf(C(6), C(7), wx) - lerpf(C(4), C(5), wx);
    gy[ch] = lerpf(dy0, dy1, wz) * s * (float)N;
    gz[ch] = (b - a) * s * (float)N;
  }
  return {chain3(val[0], gx[0], gy[0], gz[0], u, v, w), chain3(val[1], gx[1], gy[1], gz[1], u, v, w),
          chain3(val[2], gx[2], gy[2], gz[2], u, v, w), chain3(val[3], gx[3], gy[3], gz[3], u, v, w)};
}

// curl_sample (128^2 RG8, repeat, bilinear) with its gradient
__device__ __forceinline__ void curl_d(const uint8_t* curl, const DV& u, const DV& v, DV& r, DV& g) {
  const float x = u.v * 128.0f - 0.5f, y = v.v * 128.0f - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const uint32_t x0 = (uint32_t)ix & 127u, x1 = (uint32_t)(ix + 1) & 127u;
  const uint32_t y0 = (uint32_t)iy & 127u, y1 = (uint32_t)(iy + 1) & 127u;
  const uint16_t* c = reinterpret_cast<const uint16_t*>(curl);
  const uint32_t t00 = __ldg(c + y0 * 128 + x0), t10 = __ldg(c + y0 * 128 + x1);
  const uint32_t t01 = __ldg(c + y1 * 128 + x0), t11 = __ldg(c + y1 * 128 + x1);
  DV out[2];
#pragma unroll
  for (int ch = 0; ch < 2; ++ch) {
    const uint32_t sel = ch ? 0x7541u : 0x7540u;
    const float a00 = byte_to_float(t00, sel), a10 = byte_to_float(t10, sel);
    const float a01 = byte_to_float(t01, sel), a11 = byte_to_float(t11, sel);
    const float val = lerpf(lerpf(a00, a10, wx), lerpf(a01, a11, wx), wy) * (1.0f / 255.0f);
    const float gxv = lerpf(a10 - a00, a11 - a01, wy) * (128.0f / 255.0f);
    const float gyv = (lerpf(a01, a11, wx) - lerpf(a00, a10, wx)) * (128.0f / 255.0f);
    out[ch] = chain3(val, gxv, gyv, 0.0f, u, v, u);
  }
  r = out[0];
  g = out[1];
}

// weather_sample (R channel, W x H floats, repeat, bilinear) with its gradient
__device__ __forceinline__ DV weather_d(const float* wm, uint32_t W, uint32_t H, const DV& u, const DV& v) {
  const float x = u.v * (float)W - 0.5f, y = v.v * (float)H - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const int x0 = wrap_mod(ix, (int)W), x1 = wrap_mod(ix + 1, (int)W);
  const int y0 = wrap_mod(iy, (int)H), y1 = wrap_mod(iy + 1, (int)H);
  const float a00 = __ldg(wm + y0 * W + x0), a10 = __ldg(wm + y0 * W + x1);
  const float a01 = __ldg(wm + y1 * W + x0), a11 = __ldg(wm + y1 * W + x1);
  const float val = lerpf(lerpf(a00, a10, wx), lerpf(a01, a11, wx), wy);
  const float gxv = lerpf(a10 - a00, a11 - a01, wy) * (float)W;
  const float gyv = (lerpf(a01, a11, wx) - lerpf(a00, a10, wx)) * (float)H;
  return chain3(val, gxv, gyv, 0.0f, u, v, u);
}

// lut2d (RGBA, clamp-to-edge, bilinear) of the RGB channels with gradients
__device__ __forceinline__ DV3 lut2d_d(const float4* lut, int W, int H, const DV& u, const DV& v) {
  const float x = u.v * (float)W - 0.5f, y = v.v * (float)H - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const int x0 = clamp_idx(ix, W), x1 = clamp_idx(ix + 1, W);
  const int y0 = clamp_idx(iy, H), y1 = clamp_idx(iy + 1, H);
  const float4 t00 = __ldg(lut + y0 * W + x0), t10 = __ldg(lut + y0 * W + x1);
  const float4 t01 = __ldg(lut + y1 * W + x0), t11 = __ldg(lut + y1 * W + x1);
  const float c00[3] = {t00.x, t00.y, t00.z}, c10[3] = {t10.x, t10.y, t10.z};
  const float c01[3] = {t01.x, t01.y, t01.z}, c11[3] = {t11.x, t11.y, t11.z};
  DV out[3];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float a = lerpf(c00[ch], c10[ch], wx), b = lerpf(c01[ch], c11[ch], wx);
    const float gxv = lerpf(c10[ch] - c00[ch], c11[ch] - c01[ch], wy) * (float)W;
    out[ch] = chain3(lerpf(a, b, wy), gxv, (b - a) * (float)H, 0.0f, u, v, u);
  }
  return {out[0], out[1], out[2]};
}

// Aerial-perspective LUT (lut_ap) and its derivative along the distance
// coordinate w (trilinear: d/dw = 64 (upper - lower z plane)).
__device__ __forceinline__ void lut_ap_dw(const float4* lut, float u, float v, float w, float4& val, float4& dw) {
  const float x = u * 32.0f - 0.5f, y = v * 32.0f - 0.5f, z = w * 64.0f - 0.5f;
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  const float wx = x - fx, wy = y - fy, wz = z - fz;
  const int x0 = clamp_idx(ix, 32), x1 = clamp_idx(ix + 1, 32);
  const int y0 = clamp_idx(iy, 32), y1 = clamp_idx(iy + 1, 32);
  const int z0 = clamp_idx(iz, 64), z1 = clamp_idx(iz + 1, 64);
  auto at = [&](int xx, int yy, int zz) { return __ldg(lut + (zz * 32 + yy) * 32 + xx); };
  const float4 a = lerp4(lerp4(at(x0, y0, z0), at(x1, y0, z0), wx), lerp4(at(x0, y1, z0), at(x1, y1, z0), wx), wy);
  const float4 b = lerp4(lerp4(at(x0, y0, z1), at(x1, y0, z1), wx), lerp4(at(x0, y1, z1), at(x1, y1, z1), wx), wy);
  val = lerp4(a, b, wz);
  dw = make_float4((b.x - a.x) * 64.0f, (b.y - a.y) * 64.0f, (b.z - a.z) * 64.0f, (b.w - a.w) * 64.0f);
}

// ------------------------------------------------ march pieces, carried
// ndf (cloud_density_common.wgsl:49-91) of a carried height
__device__ __forceinline__ DV ndf_d(const DV& h, uint32_t t, float anvil_bias) {
  switch (t) {
    case 0: return dsmooth(0.0f, 0.07f, h) * dsmooth(1.0f, 0.2f, h);
    case 1: return dsmooth(0.0f, 0.10f, h) * (1.0f - dsmooth(0.6f, 1.0f, h));
    case 2: return dsmooth(0.0f, 0.15f, h) * dsmooth(1.0f, 0.4f, h);
    case 3: return dsmooth(0.0f, 0.20f, h) * dsmooth(1.0f, 0.3f, h);
    case 4: return dsmooth(0.0f, 0.30f, h) * (1.0f - dsmooth(0.7f, 1.0f, h));
    case 5: return dsmooth(0.0f, 0.40f, h) * (1.0f - dsmooth(0.6f, 1.0f, h));
    case 6: return dsmooth(0.0f, 0.50f, h) * (1.0f - dsmooth(0.8f, 1.0f, h));
    case 7: {
      const DV base = dsmooth(0.0f, 0.05f, h);
      const DV mid = dsmooth(0.95f, 0.5f, h);
      const DV anvil = dsmooth(0.7f, 0.9f, h) * (1.5f * clampf(anvil_bias, 0.0f, 2.0f));
      const DV mt = dsmooth(0.65f, 0.8f, h);
      return base * dmix(mid, anvil, mt);
    }
    default: return dc(0.0f);
  }
}

// altitude_from_entry (march_plain.cuh) of a carried point and distance
__device__ __forceinline__ DV altitude_d(const MarchUniforms& u, const DV3& p, const DV& r0, const DV& cv,
                                         const DV& h0, const DV& t) {
  const DV yy = p.y + u.planet_r;
  const DV len = dsqrt((p.x * p.x + yy * yy) + p.z * p.z);
  const DV num = 2.0f * t * r0 * cv + t * t;
  return h0 + num / (dmax(r0, 1.0f) + len);
}

// The carried layer's own record: its parameters with their slots, and the
// wind-cache quantities that move with its base and top.
struct LayerD {
  DV base, top, coverage, density_scale, lf_bias, layer_detail;
  DV wind_x, wind_z, skew_x, skew_z, skew_thickness;
};

// density_at with every input carried (the carried layer) or not
template <int ST, bool LIGHT>
__device__ DV density_d(const MarchUniforms& u, const LayerConst& L, const LayerD* cd, const DV3& p, const DV& alt,
                        const DV& wr, uint32_t type) {
  if (!cd)
    return dc(density_at<ST, PSC_FILTER_EXACT, LIGHT>(u, L, p.x.v, p.y.v, p.z.v, alt.v, wr.v, type, nullptr));
  const LayerD& D = *cd;
  const DV h = (alt - D.base) / dmax(D.top - D.base, 1.0f);
  if (h.v < 0.0f || h.v > 1.0f) return dc(0.0f);
  const DV eff = dclamp01(wr * D.coverage);
  if (eff.v < 0.01f) return dc(0.0f);
  const DV sk = h * D.skew_thickness;
  const DV ax = (p.x - D.wind_x) - D.skew_x * sk;
  const DV ay = p.y;
  const DV az = (p.z - D.wind_z) - D.skew_z * sk;
  const DV4 b = trilinear_d<ST, 128>(u.noise_base, ax / u.base_scale, ay / u.base_scale, az / u.base_scale,
                                     u.noise_scale);
  const DV lf = dclamp01(((b.y * 0.625f + b.z * 0.25f) + b.w * 0.125f) + D.lf_bias);
  const DV base_cloud = dremap01(b.x, -(1.0f - lf));
  DV cloud = base_cloud * ndf_d(h, type, L.anvil_bias);
  cloud = dremap01(cloud, 1.0f - eff) * eff;
  if (!LIGHT && cloud.v > 0.0f) {
    DV c2x, c2y;
    curl_d(u.curl, ax / u.detail_scale, az / u.detail_scale, c2x, c2y);
    const DV cx = c2x * 2.0f - 1.0f, cz = c2y * 2.0f - 1.0f;
    const DV dx = ax + (cx * u.curl_strength) * u.detail_scale;
    const DV dy = ay + (0.0f * u.curl_strength) * u.detail_scale;
    const DV dz = az + (cz * u.curl_strength) * u.detail_scale;
    const DV4 det = trilinear_d<ST, 32>(u.noise_detail, dx / u.detail_scale, dy / u.detail_scale,
                                        dz / u.detail_scale, u.noise_scale);
    const DV hf = (det.x * 0.625f + det.y * 0.25f) + det.z * 0.125f;
    const DV dmod = dmix(hf, 1.0f - hf, dclamp01(h * 10.0f));
    cloud = dremap01(cloud, dmod * D.layer_detail);
  }
  return dclamp01(cloud) * D.density_scale;
}

// march_to_light (march_plain.cuh) with everything carried
template <int ST>
__device__ DV light_od_d(const MarchUniforms& u, const LayerConst& L, const LayerD* cd, const DV3& p, const DV& alt,
                         const DV& wr, uint32_t type) {
  const float sx = u.sun[0], sy = u.sun[1], sz = u.sun[2];
  const DV r0 = alt + u.planet_r;
  const DV inv = dc(1.0f) / dmax(r0, 1.0f);
  const DV cv = ((p.x * inv) * sx + ((p.y + u.planet_r) * inv) * sy) + (p.z * inv) * sz;
  const float cos_sun = fmaxf(sy, 0.05f);
  const DV top = cd ? cd->top : dc(L.top_m);
  const DV dist = dmax((top - alt) / cos_sun, 1.0f);
  DV od = dc(0.0f);
  if (u.cone) {  // cloud_march.wgsl:599-666
    const float K[6][3] = {{0.38051305f, 0.92453449f, -0.02111345f},
                           {-0.50625799f, -0.03590792f, -0.86163418f},
                           {-0.32509218f, -0.94557439f, 0.01428793f},
                           {0.09026238f, -0.27376545f, 0.95755165f},
                           {0.28128598f, 0.42443639f, -0.86065785f},
                           {-0.16852403f, 0.14748697f, 0.97460106f}};
    const DV step = dist / 5.0f;
    for (int i = 0; i < 5; ++i) {
      const DV t = ((float)i + 0.5f) * step;
      const DV sc = step * ((float)i + 1.0f) / 5.0f;
      const DV3 q = {(t * sx + p.x) + K[i][0] * sc, (t * sy + p.y) + K[i][1] * sc, (t * sz + p.z) + K[i][2] * sc};
      const DV a = altitude_d(u, q, r0, cv, alt, t);
      od = od + density_d<ST, true>(u, L, cd, q, a, wr, type) * step;
    }
    const DV tf = dist * 3.0f;
    const DV3 q = {(tf * sx + p.x) + K[5][0] * (step * 3.0f), (tf * sy + p.y) + K[5][1] * (step * 3.0f),
                   (tf * sz + p.z) + K[5][2] * (step * 3.0f)};
    const DV a = altitude_d(u, q, r0, cv, alt, tf);
    return od + density_d<ST, true>(u, L, cd, q, a, wr, type) * step * 3.0f;
  }
  const DV step = dist / (float)u.light_steps;
  for (uint32_t i = 0; i < u.light_steps; ++i) {
    const DV t = ((float)i + 0.5f) * step;
    const DV3 q = {t * sx + p.x, t * sy + p.y, t * sz + p.z};
    const DV a = altitude_d(u, q, r0, cv, alt, t);
    od = od + density_d<ST, true>(u, L, cd, q, a, wr, type) * step;
  }
  return od;
}

// sun_transmittance_at (march_plain.cuh) of a carried point
__device__ DV3 sun_transmittance_d(const MarchUniforms& u, const DV3& p) {
  const float R = u.planet_r;
  const DV ay = p.y + R;
  const DV len = dsqrt((p.x * p.x + ay * ay) + p.z * p.z);
  const DV r = dmax(len, R + 1.0f);
  const DV mu = dclamp(((p.x / r) * u.sun[0] + (ay / r) * u.sun[1]) + (p.z / r) * u.sun[2], -1.0f, 1.0f);
  const DV ratio = dc(R) / r;
  const DV sin_h = -dsqrt(dmax(1.0f - ratio * ratio, 0.0f));
  if (mu.v <= sin_h.v) return {dc(0.0f), dc(0.0f), dc(0.0f)};
  const float ht = u.atmo_top;
  const float bh = sqrtf(fmaxf(ht * ht - R * R, 0.0f));
  const DV rho = dsqrt(dmax(r * r - R * R, 0.0f));
  const DV disc = r * r * (mu * mu - 1.0f) + ht * ht;
  const DV d = dmax(-r * mu + dsqrt(dmax(disc, 0.0f)), 0.0f);
  const DV d_min = ht - r, d_max = rho + bh;
  const DV xm = dclamp01((d - d_min) / dmax(d_max - d_min, 1.0f));
  const DV xr = rho / fmaxf(bh, 1.0f);
  return lut2d_d(u.lut_trans, 256, 64, xm, xr);
}

// sky_ambient (march_plain.cuh) of a carried point
__device__ DV3 sky_ambient_d(const MarchUniforms& u, const DV3& p, float sun_az) {
  const DV ay = p.y + u.planet_r;
  const DV cam_r = dsqrt((p.x * p.x + ay * ay) + p.z * p.z);
  const DV ux = p.x / cam_r, uy = ay / cam_r, uz = p.z / cam_r;
  const DV vza = datan2(dsqrt(ux * ux + uz * uz), uy);
  const DV sin_h = dclamp01(dc(u.planet_r) / cam_r);
  const DV zha = kPi - dasin(sin_h);
  DV vv;
  if (vza.v < zha.v) {
    vv = dsqrt(dclamp01(vza / dmax(zha, 1e-6f))) * 0.5f;
  } else {
    const DV br = dmax(kPi - zha, 1e-6f);
    vv = 0.5f + dsqrt(dclamp01((vza - zha) / br)) * 0.5f;
  }
  const DV vaz = datan2(ux, uz);
  DV du = (vaz - sun_az) / (2.0f * kPi);
  du = du - floorf(du.v);
  const DV3 s = lut2d_d(u.lut_sky, 192, 108, du, vv);
  return {s.x * u.sun_illum[0], s.y * u.sun_illum[1], s.z * u.sun_illum[2]};
}

// The distance t of a shell crossing with its derivatives with respect to the
// carried layer's base and top: a t on the sphere at planet radius + base
// (or + top) moves by dt/dr = r / (t + b), b = o.d; t = 0 (inside the layer)
// or a depth clip does not move.
__device__ DV shell_distance_d(const MarchUniforms& u, const LayerConst& L, const double oc[3], const double d[3],
                               float t) {
  DV r = dc(t);
  if (!(t > 0.0f)) return r;
  const double td = (double)t;
  const double px = oc[0] + d[0] * td, py = oc[1] + d[1] * td, pz = oc[2] + d[2] * td;
  const double rr = sqrt(px * px + py * py + pz * pz);
  const double b = oc[0] * d[0] + oc[1] * d[1] + oc[2] * d[2];
  const double eb = fabs(rr - L.r_bottom), et = fabs(rr - L.r_top);
  const double tol = 0.1 + 1e-6 * td;  // float rounding of t
  if (fmin(eb, et) > tol || fabs(td + b) < 1e-9) return r;
  const double k = (eb <= et ? L.r_bottom : L.r_top) / (td + b);
  r.d[eb <= et ? kBase : kTop] = (float)k;
  return r;
}

// One ray of the PLAIN march (k_march_plain) with its tangents; adds this
// pixel's loss and d loss / d parameter (before the 1 / N) to `acc`.
template <int ST>
__device__ void param_grad_pixel(const MarchUniforms& u, const ViewDev& v, const ParamGradDev& g, uint32_t px,
                                 uint32_t py, float acc[kP + 1]) {
  RaySetup rs;
  setup_ray(u, v, px, py, rs);
  const float dx = rs.dir[0], dy = rs.dir[1], dz = rs.dir[2];
  const float cx = u.cam[0], cy = u.cam[1], cz = u.cam[2];
  const float cos_theta = (dx * u.sun[0] + dy * u.sun[1]) + dz * u.sun[2];
  const float fwd = smoothstepf(0.0f, 1.0f, fmaxf(cos_theta, 0.0f));
  const float sun_az = atan2f(u.sun[0], u.sun[2]);
  uint32_t sx = (px + v.x_off) & 63u, sy = (py + v.y_off) & 63u;
  if (u.temporal_jitter) {
    const uint32_t ph = u.frame_index & 15u;
    sx = (sx ^ ((ph * 11u + 7u) & 63u)) & 63u;
    sy = (sy ^ ((ph * 23u + 13u) & 63u)) & 63u;
  }
  const float jitter = __ldg(u.blue + sy * 64u + sx);
  const double oc[3] = {(double)u.cam[0], (double)u.cam[1] + u.planet_r_d, (double)u.cam[2]};

  // the carried layer's parameters and wind quantities with their slots
  LayerD cdl;
  {
    const LayerConst& L = u.layers[g.layer];
    auto with = [](float v0, int slot, float k) {
      DV r = dc(v0);
      r.d[slot] = k;
      return r;
    };
    auto bt = [](float v0, float kb, float kt) {
      DV r = dc(v0);
      r.d[kBase] = kb;
      r.d[kTop] = kt;
      return r;
    };
    cdl.base = with(L.base_m, kBase, 1.0f);
    cdl.top = with(L.top_m, kTop, 1.0f);
    cdl.coverage = with(L.coverage, 0, 1.0f);
    cdl.lf_bias = with(L.lf_bias, 1, g.dlf_dshape);
    cdl.layer_detail = with(L.layer_detail, 2, g.dld_ddetail);
    cdl.density_scale = with(L.density_scale, 3, 1.0f);
    cdl.wind_x = bt(L.wind_off_x, g.dwind[0][0], g.dwind[0][1]);
    cdl.wind_z = bt(L.wind_off_z, g.dwind[1][0], g.dwind[1][1]);
    cdl.skew_x = bt(L.skew_x, g.dskew[0][0], g.dskew[0][1]);
    cdl.skew_z = bt(L.skew_z, g.dskew[1][0], g.dskew[1][1]);
    cdl.skew_thickness = bt(L.skew_thickness, g.dskew[2][0], g.dskew[2][1]);
  }

  DV Lc[3] = {dc(0.0f), dc(0.0f), dc(0.0f)}, T[3] = {dc(1.0f), dc(1.0f), dc(1.0f)};
  DV tw = dc(0.0f), twn = dc(0.0f);
  const float lum[3] = {0.2126f, 0.7152f, 0.0722f};
  const DV r0c = dc(rs.r0), cvc = dc(rs.cos_view), h0c = dc(rs.h0);
  for (uint32_t k = 0; k < u.layer_count; ++k) {
    if (fmaxf(T[0].v, fmaxf(T[1].v, T[2].v)) < 0.01f) break;
    const uint32_t li = (rs.order >> (4u * k)) & 15u;
    if (!((rs.hit_mask >> li) & 1u) || li >= 8u) continue;
    float t0f = 0.0f, t1f = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if ((uint32_t)j == li) {
        t0f = rs.t0[j];
        t1f = rs.t1[j];
      }
    const LayerConst& L = u.layers[li];
    const LayerD* cd = li == g.layer ? &cdl : nullptr;
    if (t1f - t0f <= 0.0f) continue;
    const DV t0 = cd ? shell_distance_d(u, L, oc, rs.dird, t0f) : dc(t0f);
    const DV t1 = cd ? shell_distance_d(u, L, oc, rs.dird, t1f) : dc(t1f);
    const DV step = (t1 - t0) / (float)u.cloud_steps;
    const float st[3] = {L.sigma_t[0], L.sigma_t[1], L.sigma_t[2]};
    for (uint32_t s = 0; s < u.cloud_steps; ++s) {
      const DV t = t0 + step * ((float)s + jitter);
      const DV3 p = {t * dx + cx, t * dy + cy, t * dz + cz};
      const DV alt = altitude_d(u, p, r0c, cvc, h0c, t);
      const DV wind_x = cd ? cd->wind_x : dc(L.wind_off_x), wind_z = cd ? cd->wind_z : dc(L.wind_off_z);
      const DV wsx = p.x - wind_x, wsz = p.z - wind_z;
      const DV wr = weather_d(u.weather, u.weather_w, u.weather_h, wsx / u.weather_scale + 0.5f,
                              wsz / u.weather_scale + 0.5f);
      const uint32_t type = effective_type(u, wsx.v, wsz.v, L.cloud_type);
      const DV density = density_d<ST, false>(u, L, cd, p, alt, wr, type);
      if (density.v > 1e-3f) {
        const DV od = light_od_d<ST>(u, L, cd, p, alt, wr, type);
        const DV base = cd ? cd->base : dc(L.base_m), top = cd ? cd->top : dc(L.top_m);
        const DV hn = dclamp01((alt - base) / dmax(top - base, 1.0f));
        PhaseConst pc;
        if (L.cloud_type == 7u) {  // the carried layer is not Cumulonimbus under approx-Mie
          const float mt = smoothstepf(0.60f, 0.85f, hn.v);
          pc = phase_consts_from_d(mixf(L.droplet_um, 50.0f, mt), u.droplet_bias);
        } else {
          pc = PhaseConst{L.g_hg, L.g_d, L.alpha, L.w_d, L.ice};
        }
        const DV3 stv = sun_transmittance_d(u, p);
        const DV3 sky = sky_ambient_d(u, p, sun_az);
        const DV ag = dmix(0.3f, 1.0f, hn) * u.ambient;
        DV lw = dc(0.0f);
        if (u.lightning_radius > 0.0f) {
          const DV ddx = p.x - u.lightning_origin_x, ddz = p.z - u.lightning_origin_z;
          const DV fo = dclamp01(1.0f - dsqrt(ddx * ddx + ddz * ddz) / u.lightning_radius);
          lw = fo * fo * (3.0f - 2.0f * fo);
        }
        const DV tsun[3] = {stv.x, stv.y, stv.z}, skyc[3] = {sky.x, sky.y, sky.z};
        const float f = u.forward_bias > 0.0f ? 1.0f + u.forward_bias * fwd : 1.0f;
        DV sl[3], sm[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const DV bb = dexp(od * -st[c]);
          const DV pw = 1.0f - dexp(od * (-2.0f * st[c]));
          const DV e = dmix(bb, bb * pw * 2.0f, u.powder);
          DV S = dc(0.0f);
          float a = 1.0f, b = 1.0f, cc = 1.0f;
          for (uint32_t o = 0; o < u.octaves; ++o) {
            const float ph = phase_with(u, cos_theta, cc, pc);
            S = S + dexp((od * -st[c]) * b) * tsun[c] * ((a * u.sun_illum[c]) * ph);
            a *= u.ms_a;
            b *= u.ms_b;
            cc *= u.ms_c;
          }
          if (u.forward_bias > 0.0f) S = S * f;
          const DV is = (density * u.sigma_s[c]) * ((S * e + skyc[c] * ag) + lw * u.lightning_rgb[c]);
          const DV ls = dmax(density * st[c], 1e-6f);
          sm[c] = dexp(ls * step * -1.0f);
          sl[c] = T[c] * ((is - is * sm[c]) / ls);
        }
        const DV sw = (sl[0] * lum[0] + sl[1] * lum[1]) + sl[2] * lum[2];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          Lc[c] = Lc[c] + sl[c];
          T[c] = T[c] * sm[c];
        }
        tw = tw + sw * t;
        twn = twn + sw;
      }
      if (fmaxf(T[0].v, fmaxf(T[1].v, T[2].v)) < 0.01f) break;
    }
  }

  // aerial perspective (cloud_march.wgsl:1016-1048)
  const DV t_lum = (T[0] * lum[0] + T[1] * lum[1]) + T[2] * lum[2];
  const DV opacity = 1.0f - t_lum;
  DV O[3] = {Lc[0], Lc[1], Lc[2]};
  if (opacity.v > 1e-4f) {
    const DV t_cloud = tw / dmax(twn, 1e-6f);
    const DV ds = dmax(t_cloud, 50.0f);
    const DV azd = dclamp01(dlog(ds * (1.0f / 50.0f)) * (1.0f / logf(100000.0f / 50.0f)));
    float4 ap, dap;
    lut_ap_dw(u.lut_ap, ((float)(px + v.x_off) + 0.5f) / u.vp_w, ((float)(py + v.y_off) + 0.5f) / u.vp_h, azd.v,
              ap, dap);
    const DV apw = along(ap.w, dap.w, azd);
    const DV apc[3] = {along(ap.x, dap.x, azd), along(ap.y, dap.y, azd), along(ap.z, dap.z, azd)};
#pragma unroll
    for (int c = 0; c < 3; ++c) O[c] = Lc[c] * apw + apc[c] * opacity;
  }
  const size_t idx = (size_t)py * v.width + px;
  const float4 bgp = __ldg(g.bg + idx), tg = __ldg(g.target + idx);
  const float bgc[3] = {bgp.x, bgp.y, bgp.z}, tgc[3] = {tg.x, tg.y, tg.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const DV I = O[c] + T[c] * bgc[c];
    const float r = I.v - tgc[c];
    acc[0] = fmaf(r, r, acc[0]);
#pragma unroll
    for (int i = 0; i < kP; ++i) acc[1 + i] = fmaf(2.0f * r, I.d[i], acc[1 + i]);
  }
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// out[0..5] += d loss / d (coverage, shape_bias, detail_bias, density_scale,
// base_m, top_m); loss (nullable) += the loss.
template <int ST>
__global__ void __launch_bounds__(kThreads) k_march_param_grad(const __grid_constant__ MarchUniforms u,
                                                               const __grid_constant__ ViewDev v,
                                                               const __grid_constant__ ParamGradDev g, double* out,
                                                               double* loss) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * kTileW + (warp & 1u) * 8u + (lane & 7u);
  const uint32_t py = blockIdx.y * kTileH + (warp >> 1) * 4u + (lane >> 3);
  float acc[kP + 1];
#pragma unroll
  for (int i = 0; i < kP + 1; ++i) acc[i] = 0.0f;
  if (px < v.width && py < v.height) param_grad_pixel<ST>(u, v, g, px, py, acc);
  __shared__ double s_red[kP + 1][kThreads / 32];
#pragma unroll
  for (int i = 0; i < kP + 1; ++i) {
    const double w = warp_sum((double)acc[i] * (double)g.inv_n);
    if (lane == 0) s_red[i][warp] = w;
  }
  __syncthreads();
  if (threadIdx.x < kP + 1) {
    double a = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) a += s_red[threadIdx.x][w];
    if (threadIdx.x == 0) {
      if (loss) atomicAdd(loss, a);
    } else {
      atomicAdd(out + threadIdx.x - 1, a);
    }
  }
}

template <int ST>
cudaError_t launch_st(const MarchUniforms& u, const ViewDev& v, const ParamGradDev& g, double* out, double* loss,
                      cudaStream_t s) {
  const dim3 grid((v.width + kTileW - 1) / kTileW, (v.height + kTileH - 1) / kTileH);
  k_march_param_grad<ST><<<grid, kThreads, 0, s>>>(u, v, g, out, loss);
  return cudaGetLastError();
}

}  // namespace

int launch_march_param_grad(const MarchUniforms& u, const ViewDev& v, const ParamGradDev& g, uint32_t storage,
                            double* out, double* loss, cudaStream_t s) {
  if (g.layer >= u.layer_count || g.layer >= 8u) return PSC_ERR_INVALID_ARGUMENT;
  cudaError_t e;
  switch (storage) {
    case PSC_STORAGE_U8: e = launch_st<PSC_STORAGE_U8>(u, v, g, out, loss, s); break;
    case PSC_STORAGE_F32: e = launch_st<PSC_STORAGE_F32>(u, v, g, out, loss, s); break;
    case PSC_STORAGE_F16: e = launch_st<PSC_STORAGE_F16>(u, v, g, out, loss, s); break;
    case PSC_STORAGE_BF16: e = launch_st<PSC_STORAGE_BF16>(u, v, g, out, loss, s); break;
    case PSC_STORAGE_FP8: e = launch_st<PSC_STORAGE_FP8>(u, v, g, out, loss, s); break;
    default: return PSC_ERR_INVALID_ARGUMENT;
  }
  return e == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

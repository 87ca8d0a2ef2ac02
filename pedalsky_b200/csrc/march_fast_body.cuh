// FAST schedule of the cloud march: the per-ray body shared by the
// single-view kernel (march_fast.cu) and the persistent batched kernel
// (march_batch.cu).  Same mathematics as the plain
// restatement (cloud_march.wgsl:731-1054), rearranged for the SM:
//   * per ray and layer: the phase lobes of every octave are evaluated once
//     (they depend only on cos(view, sun) and the layer's droplet size, except
//     for Cumulonimbus, whose diameter varies with height);
//   * per dense sample: the octave exponentials exp(-sigma*od*b^n) for
//     b = 1/2 come from one exponential and repeated squaring, which also
//     yields Beer (n = 0) and the powder term exp(-2*sigma*od);
//   * the transmittance-LUT and sky-view lookups share one altitude geometry
//     in well-conditioned forms (r = R + alt, rho = sqrt(alt*(2R + alt)),
//     zenith angles via atan2) with a polynomial arctangent;
//   * texel floors and indices come from one round-down add (floor_bits);
//   * weather/type fetches are skipped where the height gate already
//     returns zero density;
//   * texel coordinates are formed with one FMA per axis.
//   * smoothsteps multiply by precomputed reciprocals, and this translation
//     unit is built with approximate division and square root (a few ulp);
//   * F16 storage reads the channel-folded volumes (noise_bake.cu:k_fold_*):
//     the base volume as (R, 0.625G + 0.25B + 0.125A) and the detail volume
//     as 0.625R + 0.25G + 0.125B, the only combinations the density uses, so
//     an exact trilinear tap is two 16-byte (base) or 8-byte (detail) quad
//     loads and a texture tap filters two channels (or one) instead of four;
//   * the texture-unit light march reduces the tap geometry to per-sample
//     constants (altitude from a quadratic in t, texture coordinates affine
//     in t and h) and computes every tap position of a batch of up to four
//     taps and issues their fetches before it combines any of them, so the
//     fetches overlap instead of each waiting for the previous one;
//   * in the primary step the weather, type and base-shape fetches are
//     independent of each other and are issued together, with the curl
//     fetch of the detail erosion (a 2x2 quad, one 16-byte load); a uniform
//     weather map (the reference's synthesis writes R = 1) is not sampled;
//   * in the filtered forms (HYBRID, TEXTURE) the transmittance and sky-view
//     LUTs go through the texture unit, as the reference's linear sampler
//     does; EXACT keeps FP32 weights for them.
// Octave counts up to 4 are handled here; the host falls back to the plain
// kernel beyond that.  FULL = false (the lean form) compiles out the paths a
// common scene does not use: Cumulonimbus (the height-dependent phase of the
// octaves, the anvil profile of the light march), the cloud-type grid, Kahan
// sums, cone light sampling and lightning.  The host picks the lean form
// when none of them is in use (needs_full_paths): the hot loop is shorter and
// spills less.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "march_common.cuh"
#include "march_ray.cuh"
#include "psc_internal.h"

namespace psc {
namespace {

constexpr int kMaxOct = 4;

// atan(a), a in [0, 1]: a * P(a^2), P fitted by iteratively reweighted least
// squares on Chebyshev nodes (max abs error 3.3e-7 rad in FP32).
__device__ __forceinline__ float atan01(float a) {
  const float s = a * a;
  float p = 6.811792605e-03f;
  p = fmaf(p, s, -3.360421914e-02f);
  p = fmaf(p, s, 7.962367187e-02f);
  p = fmaf(p, s, -1.323334217e-01f);
  p = fmaf(p, s, 1.980781563e-01f);
  p = fmaf(p, s, -3.331736807e-01f);
  p = fmaf(p, s, 9.999961116e-01f);
  return p * a;
}
// atan2(y, x) with the same quadrant conventions as the C library.
__device__ __forceinline__ float fast_atan2(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  const float a = mx > 0.0f ? __fdividef(mn, mx) : 0.0f;
  float r = atan01(a);
  if (ay > ax) r = 1.57079632679f - r;
  if (x < 0.0f) r = 3.14159265359f - r;
  return copysignf(r, y);
}

// Texel coordinates already in texel units (x = p * N/scale - 0.5).
template <int ST, int N>
__device__ __forceinline__ float4 trilinear_texel(const void* vol, float x, float y, float z,
                                                  float volume_scale) {
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  const float wx = x - fx, wy = y - fy, wz = z - fz;
  const uint32_t x0 = (uint32_t)ix & (N - 1), x1 = (uint32_t)(ix + 1) & (N - 1);
  const uint32_t y0 = (uint32_t)iy & (N - 1), y1 = (uint32_t)(iy + 1) & (N - 1);
  const uint32_t z0 = (uint32_t)iz & (N - 1), z1 = (uint32_t)(iz + 1) & (N - 1);
  const uint32_t r00 = (z0 * N + y0) * N, r10 = (z0 * N + y1) * N;
  const uint32_t r01 = (z1 * N + y0) * N, r11 = (z1 * N + y1) * N;
  const float4 c000 = load_texel<ST>(vol, r00 + x0), c100 = load_texel<ST>(vol, r00 + x1);
  const float4 c010 = load_texel<ST>(vol, r10 + x0), c110 = load_texel<ST>(vol, r10 + x1);
  const float4 c001 = load_texel<ST>(vol, r01 + x0), c101 = load_texel<ST>(vol, r01 + x1);
  const float4 c011 = load_texel<ST>(vol, r11 + x0), c111 = load_texel<ST>(vol, r11 + x1);
  const float4 a = lerp4p(lerp4p(c000, c100, wx), lerp4p(c010, c110, wx), wy);
  const float4 b = lerp4p(lerp4p(c001, c101, wx), lerp4p(c011, c111, wx), wy);
  float4 r = lerp4p(a, b, wz);
  const float s = storage_scale<ST>(volume_scale);
  r.x *= s;
  r.y *= s;
  r.z *= s;
  r.w *= s;
  return r;
}

// floor(x) and its integer bits for |x| < 2^22: one round-down add puts
// 1.5 * 2^23 + floor(x) in a float whose low mantissa bits are floor(x)
// (two's complement, so masks wrap negative indices), and subtracting the
// constant back is exact.  Larger |x| (millions of texels, far beyond any
// ray here) still yields masked, in-bounds indices.
struct FloorBits {
  float f;
  uint32_t i;
};
__device__ __forceinline__ FloorBits floor_bits(float x) {
  const float s = __fadd_rd(x, 12582912.0f);
  return {s - 12582912.0f, __float_as_uint(s)};
}

__device__ __forceinline__ float2 h2f(uint32_t w) {
  return __half22float2(*reinterpret_cast<const __half2*>(&w));
}

// Exact trilinear tap of the folded base volume (128^3 quads, repeat),
// coordinates in texel units: one 16-byte quad load per slab, FP32 weights.
// Returns the stored scale (255 R, 2040 (0.625G + 0.25B + 0.125A)); the
// shape function folds the 1/255 and 1/2040 into its FMAs.
__device__ __forceinline__ float2 base_quad_tap(const uint4* q, float x, float y, float z) {
  const FloorBits bx = floor_bits(x), by = floor_bits(y), bz = floor_bits(z);
  const float wx = x - bx.f, wy = y - by.f, wz = z - bz.f;
  const uint32_t r = (by.i & 127u) * 128u + (bx.i & 127u);
  const uint32_t z0 = bz.i & 127u, z1 = (bz.i + 1u) & 127u;
  const uint4 a = __ldg(q + z0 * 16384u + r);
  const uint4 b = __ldg(q + z1 * 16384u + r);
  const float2 tx = make_float2(wx, wx), ty = make_float2(wy, wy);
  const float2 sa = lerp2(lerp2(h2f(a.x), h2f(a.y), tx), lerp2(h2f(a.z), h2f(a.w), tx), ty);
  const float2 sb = lerp2(lerp2(h2f(b.x), h2f(b.y), tx), lerp2(h2f(b.z), h2f(b.w), tx), ty);
  return lerp2(sa, sb, make_float2(wz, wz));
}

// Exact trilinear tap of the folded detail volume (32^3 quads, repeat):
// one 8-byte quad load per slab; the two slabs ride the two FP32x2 lanes.
// Returns 0.625R + 0.25G + 0.125B in [0, 1].
__device__ __forceinline__ float detail_quad_tap(const uint2* q, float x, float y, float z) {
  const FloorBits bx = floor_bits(x), by = floor_bits(y), bz = floor_bits(z);
  const float wx = x - bx.f, wy = y - by.f, wz = z - bz.f;
  const uint32_t r = (by.i & 31u) * 32u + (bx.i & 31u);
  const uint32_t z0 = bz.i & 31u, z1 = (bz.i + 1u) & 31u;
  const uint2 a = __ldg(q + z0 * 1024u + r);
  const uint2 b = __ldg(q + z1 * 1024u + r);
  const float2 a0 = h2f(a.x), a1 = h2f(a.y), b0 = h2f(b.x), b1 = h2f(b.y);
  const float2 tx = make_float2(wx, wx), ty = make_float2(wy, wy);
  const float2 s = lerp2(lerp2(make_float2(a0.x, b0.x), make_float2(a0.y, b0.y), tx),
                         lerp2(make_float2(a1.x, b1.x), make_float2(a1.y, b1.y), tx), ty);
  return lerpf(s.x, s.y, wz) * (1.0f / 2040.0f);
}

// Read-only 16-byte load that stays where it is written: the compiler may not
// sink it into the branch that consumes it, so it is in flight while the
// code before that branch runs.
__device__ __forceinline__ uint4 ldg_v4_early(const uint4* p) {
  uint4 r;
  asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}

// Bilinear curl tap (128^2, repeat) from the quad form, in two halves: the
// fetch (issued with the base-shape fetch, before it is known whether the
// detail erosion needs it) and the FP32-weight blend; (R, G) in [0, 1].
struct CurlFetch {
  uint4 q;
  float wx, wy;
};
__device__ __forceinline__ CurlFetch curl_fetch(const uint4* q, float x, float y) {
  const FloorBits bx = floor_bits(x), by = floor_bits(y);
  CurlFetch c;
  c.q = ldg_v4_early(q + (by.i & 127u) * 128u + (bx.i & 127u));
  c.wx = x - bx.f;
  c.wy = y - by.f;
  return c;
}
__device__ __forceinline__ float2 curl_blend(const CurlFetch& c) {
  const float2 tx = make_float2(c.wx, c.wx);
  const float2 v = lerp2(lerp2(h2f(c.q.x), h2f(c.q.y), tx), lerp2(h2f(c.q.z), h2f(c.q.w), tx),
                         make_float2(c.wy, c.wy));
  return make_float2(v.x * (1.0f / 255.0f), v.y * (1.0f / 255.0f));
}

// Scale of a base tap's two values: F16 taps return the stored integers
// (255 R, 2040 fbm), the other forms the values themselves.
template <int ST>
struct BaseScale {
  static constexpr float x = ST == PSC_STORAGE_F16 ? 1.0f / 255.0f : 1.0f;
  static constexpr float y = ST == PSC_STORAGE_F16 ? 1.0f / 2040.0f : 1.0f;
};

// Base-noise tap: (R, 0.625G + 0.25B + 0.125A) times BaseScale's inverse.
// LIGHT taps use the texture unit in the HYBRID form.
template <int ST, int FILT, bool LIGHT>
__device__ __forceinline__ float2 base_tap(const MarchUniforms& u, float ax, float ay, float az) {
  constexpr bool kTex = FILT == PSC_FILTER_TEXTURE || (FILT == PSC_FILTER_HYBRID && LIGHT);
  if constexpr (ST == PSC_STORAGE_F16) {
    if constexpr (kTex) {
      return tex3D<float2>(u.tex_base, ax * u.inv_base_scale, ay * u.inv_base_scale,
                           az * u.inv_base_scale);
    } else {
      const float k = u.base_texel_scale;
      return base_quad_tap(u.base_quad, fmaf(ax, k, -0.5f), fmaf(ay, k, -0.5f), fmaf(az, k, -0.5f));
    }
  } else {
    float4 b;
    if constexpr (kTex) {
      b = tex3D<float4>(u.tex_base, ax * u.inv_base_scale, ay * u.inv_base_scale,
                        az * u.inv_base_scale);
    } else {
      const float k = u.base_texel_scale;
      b = trilinear_texel<ST, 128>(u.noise_base, fmaf(ax, k, -0.5f), fmaf(ay, k, -0.5f),
                                   fmaf(az, k, -0.5f), u.noise_scale);
    }
    return make_float2(b.x, fmaf(b.w, 0.125f, fmaf(b.z, 0.25f, b.y * 0.625f)));
  }
}

// Detail-noise tap: 0.625R + 0.25G + 0.125B (cloud_march.wgsl:512-515).
template <int ST, int FILT>
__device__ __forceinline__ float detail_tap(const MarchUniforms& u, float dx, float dy, float dz) {
  if constexpr (ST == PSC_STORAGE_F16) {
    if constexpr (FILT == PSC_FILTER_TEXTURE) {
      return tex3D<float>(u.tex_detail, dx * u.inv_detail_scale, dy * u.inv_detail_scale,
                          dz * u.inv_detail_scale) * (1.0f / 2040.0f);
    } else {
      const float k = u.detail_texel_scale;
      return detail_quad_tap(u.detail_quad, fmaf(dx, k, -0.5f), fmaf(dy, k, -0.5f), fmaf(dz, k, -0.5f));
    }
  } else {
    float4 d;
    if constexpr (FILT == PSC_FILTER_TEXTURE) {
      d = tex3D<float4>(u.tex_detail, dx * u.inv_detail_scale, dy * u.inv_detail_scale,
                        dz * u.inv_detail_scale);
    } else {
      const float k = u.detail_texel_scale;
      d = trilinear_texel<ST, 32>(u.noise_detail, fmaf(dx, k, -0.5f), fmaf(dy, k, -0.5f),
                                  fmaf(dz, k, -0.5f), u.noise_scale);
    }
    return fmaf(d.z, 0.125f, fmaf(d.y, 0.25f, d.x * 0.625f));
  }
}

// smoothstep with the reciprocal of (e1 - e0) precomputed (a multiply, not
// a division); e0 > e1 gives the reversed ramps of cloud_density_common.wgsl.
// t = clamp01(x * inv_w + b) with b = -e0 * inv_w is one saturating FMA.
__device__ __forceinline__ float ssr_b(float inv_w, float b, float x) {
  const float t = __saturatef(fmaf(x, inv_w, b));
  return t * t * fmaf(-2.0f, t, 3.0f);
}
__device__ __forceinline__ float ssr(float e0, float inv_w, float x) { return ssr_b(inv_w, -e0 * inv_w, x); }
// ndf (cloud_density_common.wgsl:49-91) with reciprocal smoothsteps.
__device__ __forceinline__ float ndf_fast(float h, uint32_t t, float anvil_bias) {
  switch (t) {
    case 0: return ssr(0.0f, 1.0f / 0.07f, h) * ssr(1.0f, 1.0f / -0.8f, h);
    case 1: return ssr(0.0f, 1.0f / 0.10f, h) * (1.0f - ssr(0.6f, 1.0f / 0.4f, h));
    case 2: return ssr(0.0f, 1.0f / 0.15f, h) * ssr(1.0f, 1.0f / -0.6f, h);
    case 3: return ssr(0.0f, 1.0f / 0.20f, h) * ssr(1.0f, 1.0f / -0.7f, h);
    case 4: return ssr(0.0f, 1.0f / 0.30f, h) * (1.0f - ssr(0.7f, 1.0f / 0.3f, h));
    case 5: return ssr(0.0f, 1.0f / 0.40f, h) * (1.0f - ssr(0.6f, 1.0f / 0.4f, h));
    case 6: return ssr(0.0f, 1.0f / 0.50f, h) * (1.0f - ssr(0.8f, 1.0f / 0.2f, h));
    case 7: {
      const float base = ssr(0.0f, 1.0f / 0.05f, h);
      const float mid = ssr(0.95f, 1.0f / -0.45f, h);
      const float anvil = ssr(0.7f, 1.0f / 0.2f, h) * 1.5f * clampf(anvil_bias, 0.0f, 2.0f);
      const float mt = ssr(0.65f, 1.0f / 0.15f, h);
      return base * mixf(mid, anvil, mt);
    }
    default: return 0.0f;
  }
}

// Base-shape part shared by the primary and light densities
// (cloud_march.wgsl:463-494) from a base tap `b` = (R, low-frequency fbm)
// scaled by 1/(sx, sy) and the profile value `nd` = ndf(h, type).  With
// c = 1 - lf = clamp01(lf_c - fbm), lf_c = 1 - lf_bias, the remapped base is
// (R + c) / (1 + c).  The coverage remap remap(cloud, 1 - eff, 1, 0, 1) * eff
// equals cloud - (1 - eff) wherever the density is not gated off
// (eff >= 0.01), and 1 + c >= 1, so neither needs its guard.
template <int ST>
__device__ __forceinline__ float shape_from(float2 b, float lf_c, float nd, float one_minus_eff) {
  const float c = __saturatef(fmaf(b.y, -BaseScale<ST>::y, lf_c));
  const float base_cloud = __fdividef(fmaf(b.x, BaseScale<ST>::x, c), c + 1.0f);
  return fmaf(base_cloud, nd, -one_minus_eff);
}

// ndf_fast for types 0..6 as two reciprocal smoothsteps with per-type
// constants: ssr(0, inv_a, h) * g, g = ssr(e1, inv_w1, h) or 1 - that.
// Chosen once per dense sample, so the light taps carry no switch.
// b1 = -e1 * inv_w1 (the saturating-FMA form of ssr); the falling form
// 1 - S(t) is S(1 - t), the ramp with slope -inv_w1 and offset 1 - b1.  For
// these types the profile is exactly 0 outside h in [0, 1] (the rising ramp
// starts at 0 and the second factor reaches 0 at h = 1).
struct NdfCoef {
  float inv_a, b1, inv_w1;
};
__device__ __forceinline__ NdfCoef ndf_row(float a, float e1, float w1, bool flip) {
  const float inv_w1 = 1.0f / w1;
  const float b1 = -e1 * inv_w1;
  return flip ? NdfCoef{1.0f / a, 1.0f - b1, -inv_w1} : NdfCoef{1.0f / a, b1, inv_w1};
}
__device__ __forceinline__ NdfCoef ndf_coef(uint32_t t) {
  switch (t) {
    case 0: return ndf_row(0.07f, 1.0f, -0.8f, false);
    case 1: return ndf_row(0.10f, 0.6f, 0.4f, true);
    case 2: return ndf_row(0.15f, 1.0f, -0.6f, false);
    case 3: return ndf_row(0.20f, 1.0f, -0.7f, false);
    case 4: return ndf_row(0.30f, 0.7f, 0.3f, true);
    case 5: return ndf_row(0.40f, 0.6f, 0.4f, true);
    case 6: return ndf_row(0.50f, 0.8f, 0.2f, true);
    default: return {0.0f, 0.0f, 0.0f};  // unknown types: ndf = 0
  }
}
__device__ __forceinline__ float ndf_eval(const NdfCoef& k, float h) {
  return ssr_b(k.inv_a, 0.0f, h) * ssr_b(k.inv_w1, k.b1, h);
}

template <int ST, int FILT>
__device__ __forceinline__ float density_light(const MarchUniforms& u, const LayerConst& L, float qx,
                                               float qy, float qz, float alt, float eff,
                                               uint32_t type) {
  const float h = (alt - L.base_m) * L.inv_thickness;
  if (h < 0.0f || h > 1.0f) return 0.0f;
  const float ax = fmaf(-L.skew_kx, h, qx - L.wind_off_x);
  const float az = fmaf(-L.skew_kz, h, qz - L.wind_off_z);
  const float2 b = base_tap<ST, FILT, true>(u, ax, qy, az);
  return clamp01(shape_from<ST>(b, L.lf_c, ndf_fast(h, type, L.anvil_bias), 1.0f - eff)) *
         L.density_scale;
}

__device__ __forceinline__ float alt_from(const MarchUniforms& u, float qx, float qy, float qz,
                                          float r0, float cv, float h0, float t) {
  const float yy = qy + u.planet_r;
  const float len = sqrtf(fmaf(qx, qx, fmaf(yy, yy, qz * qz)));
  const float num = fmaf(2.0f * t * r0, cv, t * t);
  return h0 + __fdividef(num, r0 + len);
}

template <int ST, int FILT>
__device__ __noinline__ float light_cone(const MarchUniforms& u, const LayerConst& L, float px,
                                         float py, float pz, float alt, float eff, uint32_t type,
                                         float r0, float cv, float dist) {
  const float K[6][3] = {{0.38051305f, 0.92453449f, -0.02111345f},
                         {-0.50625799f, -0.03590792f, -0.86163418f},
                         {-0.32509218f, -0.94557439f, 0.01428793f},
                         {0.09026238f, -0.27376545f, 0.95755165f},
                         {0.28128598f, 0.42443639f, -0.86065785f},
                         {-0.16852403f, 0.14748697f, 0.97460106f}};
  const float sx = u.sun[0], sy = u.sun[1], sz = u.sun[2];
  const float step = dist * 0.2f;
  float od = 0.0f;
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const float t = ((float)i + 0.5f) * step;
    const float sc = step * ((float)i + 1.0f) * 0.2f;
    const float qx = fmaf(sx, t, px) + K[i][0] * sc;
    const float qy = fmaf(sy, t, py) + K[i][1] * sc;
    const float qz = fmaf(sz, t, pz) + K[i][2] * sc;
    od += density_light<ST, FILT>(u, L, qx, qy, qz, alt_from(u, qx, qy, qz, r0, cv, alt, t), eff,
                                  type) * step;
  }
  const float tf = dist * 3.0f;
  const float qx = fmaf(sx, tf, px) + K[5][0] * (step * 3.0f);
  const float qy = fmaf(sy, tf, py) + K[5][1] * (step * 3.0f);
  const float qz = fmaf(sz, tf, pz) + K[5][2] * (step * 3.0f);
  od += density_light<ST, FILT>(u, L, qx, qy, qz, alt_from(u, qx, qy, qz, r0, cv, alt, tf), eff,
                                type) * step * 3.0f;
  return od;
}

// Light march through the texture unit.  Per dense sample the tap geometry
// is reduced to constants: the distance from the planet centre along the
// sun ray is r(t)^2 = A + t (B + t) with A = r0^2, B = 2 r0 cos(up, sun),
// so alt(t) = h0 + t (B + t) / (r0 + r(t)) (the stable form alt_from
// uses), and the texture coordinates of a tap are affine in t and h.  For
// light paths up to 20 km (POLY) the normalised height comes instead from
// the Taylor series of r(t) - r0 in s = t / r0,
//   t cv + t^2 (1 - cv^2) / (2 r0) - t^3 cv (1 - cv^2) / (2 r0^2) + O(t^4 / (8 r0^3)),
// cv = cos(up, sun), as a cubic in t: the truncation error is below 1e-4 m at
// 20 km, smaller than the FP32 rounding of the altitude, and the square root
// and division per tap are gone.  Longer paths (low sun, thick layers) keep
// the exact form.  Six taps (the reference default) run as one batch, other
// counts in batches of 4, then 2, then 1 (no padded slots): every position and
// fetch of a batch first, then the densities and the optical-depth sum in
// tap order, plain or compensated as in the one-tap-at-a-time loop.  A tap
// outside the layer's height range is fetched but adds zero, as
// density_light returns for it.
struct LightRay {
  float A, B, r0, h0;  // geometry above
  float ih, hb;        // h = alt * ih - hb
  float px, py, pz;    // texture coordinates of the sample, wind removed
  float sx, sy, sz;    // sun direction in texture units per metre
  float kx, kz;        // skew shift in texture units per unit of h
  float step, one_minus_eff;
  float c0, c1, c2, c3;  // h(t) = c0 + t (c1 + t (c2 + t c3))
};

// ndf of a non-Cumulonimbus type from its coefficients, and of Cumulonimbus.
struct NdfGeneral {
  NdfCoef k;
  __device__ __forceinline__ float operator()(float h) const { return ndf_eval(k, h); }
};
// ndf of a non-Cumulonimbus type on taps that are all past the bottom ramp
// (h * inv_a >= 1, so its smoothstep is exactly 1): the top factor alone.
struct NdfTop {
  NdfCoef k;
  __device__ __forceinline__ float operator()(float h) const { return ssr_b(k.inv_w1, k.b1, h); }
};
struct NdfCb {
  float anvil_bias;
  __device__ __forceinline__ float operator()(float h) const { return ndf_fast(h, 7u, anvil_bias); }
};

// Base-noise tap of the light march at normalised texture coordinates
// (scaled as base_tap's).
template <int ST>
__device__ __forceinline__ float2 light_tex_tap(const MarchUniforms& u, float x, float y, float z) {
  if constexpr (ST == PSC_STORAGE_F16) {
    return tex3D<float2>(u.tex_base, x, y, z);
  } else {
    const float4 b = tex3D<float4>(u.tex_base, x, y, z);
    return make_float2(b.x, fmaf(b.w, 0.125f, fmaf(b.z, 0.25f, b.y * 0.625f)));
  }
}

// Normalised height of the light-march tap at distance t (as light_taps
// computes it): the cubic for POLY, the exact geometry otherwise.
template <bool POLY>
__device__ __forceinline__ float light_tap_h(const LightRay& lr, float t) {
  if constexpr (POLY) {
    return fmaf(t, fmaf(t, fmaf(t, lr.c3, lr.c2), lr.c1), lr.c0);
  } else {
    const float bt_t = lr.B + t;
    const float r = sqrtf(fmaf(t, bt_t, lr.A));
    const float alt = lr.h0 + __fdividef(t * bt_t, lr.r0 + r);
    return fmaf(alt, lr.ih, -lr.hb);
  }
}

// HCHECK: zero taps outside the layer's height range (Cumulonimbus; the
// other profiles are exactly 0 there already).
template <int ST, class Prof, bool HCHECK, uint32_t NB, bool POLY, bool FULL>
__device__ __forceinline__ void light_taps(const MarchUniforms& u, const LayerConst& L,
                                           const LightRay& lr, const Prof& prof, uint32_t i0,
                                           float& od, float& comp) {
  float2 bt[NB];
  float hh[NB];
  const float tb = ((float)i0 + 0.5f) * lr.step;
#pragma unroll
  for (uint32_t j = 0; j < NB; ++j) {
    const float t = fmaf((float)j, lr.step, tb);
    const float h = light_tap_h<POLY>(lr, t);
    hh[j] = h;
    bt[j] = light_tex_tap<ST>(u, fmaf(-lr.kx, h, fmaf(lr.sx, t, lr.px)), fmaf(lr.sy, t, lr.py),
                              fmaf(-lr.kz, h, fmaf(lr.sz, t, lr.pz)));
  }
  const float ds_step = L.density_scale * lr.step;
#pragma unroll
  for (uint32_t j = 0; j < NB; ++j) {
    const float h = hh[j];
    float d = __saturatef(shape_from<ST>(bt[j], L.lf_c, prof(h), lr.one_minus_eff));
    if (HCHECK && !(h >= 0.0f && h <= 1.0f)) d = 0.0f;
    if (FULL && u.kahan) {
      const float y = d * ds_step - comp;
      const float tt = od + y;
      comp = (tt - od) - y;
      od = tt;
    } else {
      od = fmaf(d, ds_step, od);
    }
  }
}

// LB: taps per fetch batch (PscMarchOptions.light_batch).  0: six taps (the
// reference default) in one batch, other counts in batches of 4, 2, 1; 3 or
// 2: batches of that many, then 2, 1.  The taps are summed in the same order
// whatever the batching.
//
// `rising` (lean form, six taps): the tap heights rise along the path, so
// once a tap is above L.light_h_dead every later tap adds exactly 0; when
// that holds from tap 2 (or 4) on for every lane of the warp, only the
// first 2 (or 4) taps are fetched and summed, which gives the same sum.
// `taps`, when given, receives the number of taps fetched in that case.
template <int ST, class Prof, bool HCHECK, bool POLY, bool FULL, int LB = 0>
__device__ __forceinline__ float light_march_tex(const MarchUniforms& u, const LayerConst& L,
                                                 const LightRay& lr, const Prof& prof,
                                                 bool rising = false, uint32_t* taps = nullptr) {
  const uint32_t n = u.light_steps;
  float od = 0.0f, comp = 0.0f;
  uint32_t i = 0;
  if constexpr (LB == 0) {
    if (n == 6u) {  // the reference default: all six fetches in one batch
      if constexpr (!FULL && POLY) {
        const unsigned act = __activemask();
        const float tb = 0.5f * lr.step;
        const bool dead2 = rising && light_tap_h<POLY>(lr, fmaf(2.0f, lr.step, tb)) > L.light_h_dead;
        const bool dead4 = rising && light_tap_h<POLY>(lr, fmaf(4.0f, lr.step, tb)) > L.light_h_dead;
        if (__all_sync(act, dead2)) {
          light_taps<ST, Prof, HCHECK, 2, POLY, FULL>(u, L, lr, prof, 0u, od, comp);
          if (taps) *taps = 2u;
          return od;
        }
        if (__all_sync(act, dead4)) {
          light_taps<ST, Prof, HCHECK, 4, POLY, FULL>(u, L, lr, prof, 0u, od, comp);
          if (taps) *taps = 4u;
          return od;
        }
      }
      light_taps<ST, Prof, HCHECK, 6, POLY, FULL>(u, L, lr, prof, 0u, od, comp);
      return od;
    }
    for (; i + 4u <= n; i += 4u) light_taps<ST, Prof, HCHECK, 4, POLY, FULL>(u, L, lr, prof, i, od, comp);
  } else {
    for (; i + (uint32_t)LB <= n; i += (uint32_t)LB)
      light_taps<ST, Prof, HCHECK, (uint32_t)LB, POLY, FULL>(u, L, lr, prof, i, od, comp);
  }
  if (i + 2u <= n) {
    light_taps<ST, Prof, HCHECK, 2, POLY, FULL>(u, L, lr, prof, i, od, comp);
    i += 2u;
  }
  if (i < n) light_taps<ST, Prof, HCHECK, 1, POLY, FULL>(u, L, lr, prof, i, od, comp);
  return od;
}

// Optical depth toward the sun (cloud_march.wgsl:543-578).  `taps`, when
// given, is lowered to the number of taps fetched where the lean form's
// light march stops early.
template <int ST, int FILT, bool FULL = true, int LB = 0>
__device__ __forceinline__ float light_od(const MarchUniforms& u, const LayerConst& L, float px,
                                          float py, float pz, float alt, float eff, uint32_t type,
                                          float ux, float uy, float uz, uint32_t* taps = nullptr) {
  const float r0 = u.planet_r + alt;
  const float cv = fmaf(ux, u.sun[0], fmaf(uy, u.sun[1], uz * u.sun[2]));
  const float dist = fmaxf((L.top_m - alt) * u.inv_cos_sun, 1.0f);
  if (FULL && u.cone) return light_cone<ST, FILT>(u, L, px, py, pz, alt, eff, type, r0, cv, dist);
  const float step = __fdividef(dist, (float)u.light_steps);
  if constexpr (FILT != PSC_FILTER_EXACT) {
    const float k = u.inv_base_scale;
    LightRay lr;
    lr.A = r0 * r0;
    lr.B = 2.0f * r0 * cv;
    lr.r0 = r0;
    lr.h0 = alt;
    lr.ih = L.inv_thickness;
    lr.hb = L.base_m * L.inv_thickness;
    lr.px = (px - L.wind_off_x) * k;
    lr.py = py * k;
    lr.pz = (pz - L.wind_off_z) * k;
    lr.sx = u.sun[0] * k;
    lr.sy = u.sun[1] * k;
    lr.sz = u.sun[2] * k;
    lr.kx = L.skew_kx * k;
    lr.kz = L.skew_kz * k;
    lr.step = step;
    lr.one_minus_eff = 1.0f - eff;
    const NdfGeneral gen{(FULL && u.type_grid) ? ndf_coef(type) : NdfCoef{L.ndf_inv_a, L.ndf_b1, L.ndf_inv_w1}};
    if (dist <= 20000.0f) {
      const float s2 = fmaf(-cv, cv, 1.0f) * __fdividef(0.5f, r0);
      lr.c0 = fmaf(alt, lr.ih, -lr.hb);
      lr.c1 = cv * lr.ih;
      lr.c2 = s2 * lr.ih;
      lr.c3 = -cv * __fdividef(s2, r0) * lr.ih;
      if (FULL && type == 7u) return light_march_tex<ST, NdfCb, true, true, FULL, LB>(u, L, lr, NdfCb{L.anvil_bias});
      // heights rise along the light path when cos(up, sun) >= 0 (the cubic's
      // slope stays positive over 20 km), so the first tap bounds them all
      const float t_first = 0.5f * step;
      const float h_first = fmaf(t_first, fmaf(t_first, fmaf(t_first, lr.c3, lr.c2), lr.c1), lr.c0);
      const bool rising = !FULL && cv >= 0.0f;
      if (rising && h_first * gen.k.inv_a >= 1.0001f)  // lean form only
        return light_march_tex<ST, NdfTop, false, true, FULL, LB>(u, L, lr, NdfTop{gen.k}, true, taps);
      return light_march_tex<ST, NdfGeneral, false, true, FULL, LB>(u, L, lr, gen, rising, taps);
    }
    if (FULL && type == 7u) return light_march_tex<ST, NdfCb, true, false, FULL, LB>(u, L, lr, NdfCb{L.anvil_bias});
    return light_march_tex<ST, NdfGeneral, false, false, FULL, LB>(u, L, lr, gen);
  }
  float od = 0.0f, comp = 0.0f;
  for (uint32_t i = 0; i < u.light_steps; ++i) {
    const float t = ((float)i + 0.5f) * step;
    const float qx = fmaf(u.sun[0], t, px), qy = fmaf(u.sun[1], t, py), qz = fmaf(u.sun[2], t, pz);
    const float term =
        density_light<ST, FILT>(u, L, qx, qy, qz, alt_from(u, qx, qy, qz, r0, cv, alt, t), eff, type) *
        step;
    if (FULL && u.kahan) {
      const float y = term - comp;
      const float tt = od + y;
      comp = (tt - od) - y;
      od = tt;
    } else {
      od += term;
    }
  }
  return od;
}

// atan2(y, x) for y >= 0 (the zenith angle of a direction), as fast_atan2.
__device__ __forceinline__ float atan2_upper(float y, float x) {
  const float ax = fabsf(x);
  const float a = __fdividef(fminf(ax, y), fmaxf(fmaxf(ax, y), 1e-30f));
  float r = atan01(a);
  if (y > ax) r = 1.57079632679f - r;
  return x < 0.0f ? 3.14159265359f - r : r;
}

// The two LUT lookups of a dense sample, sharing the altitude geometry
// (r = R + alt and rho = sqrt(alt (2R + alt)) instead of differences of
// squares at 6e6 m):
//  * transmittance toward the sun (cloud_march.wgsl:328-354): earth shadow,
//    then the Bruneton uv with a = max(alt, 1);
//  * sky-view ambient at the local up (cloud_march.wgsl:672-700): zenith
//    angle, horizon angle pi/2 + atan2(rho, R) (rho < R below 2600 km) and
//    azimuth; scaled by the sun illuminance.
// Returns whether the transmittance LUT was fetched (not in the earth's
// shadow), which only the fetch tally reads.
__device__ __forceinline__ bool lut_lookups(const MarchUniforms& u, float alt, float ux, float uy,
                                            float uz, float3& trans, float3& sky) {
  const float R = u.planet_r;
  const float a0 = fmaxf(alt, 0.0f);
  const float rho0 = sqrtf(a0 * (2.0f * R + a0));
  // transmittance
  const float a = fmaxf(alt, 1.0f);
  const float r = R + a;
  const float rho = alt >= 1.0f ? rho0 : u.rho_1m;
  const float mu = clampf(fmaf(ux, u.sun[0], fmaf(uy, u.sun[1], uz * u.sun[2])), -1.0f, 1.0f);
  const bool lit = !(mu <= -__fdividef(rho, r));
  if (!lit) {
    trans = make_float3(0.0f, 0.0f, 0.0f);
  } else {
    const float top = u.atmo_top;
    const float rm = r * mu;
    const float disc = fmaf(rm, rm, (top - r) * (top + r));
    const float d = fmaxf(sqrtf(fmaxf(disc, 0.0f)) - rm, 0.0f);
    const float d_min = top - r, d_max = rho + u.big_h;
    const float xm = __saturatef(__fdividef(d - d_min, fmaxf(d_max - d_min, 1.0f)));
    const float xr = rho * u.inv_big_h;
    const float4 t = u.tex_trans ? tex2D<float4>(u.tex_trans, xm, xr) : lut2d(u.lut_trans, 256, 64, xm, xr);
    trans = make_float3(t.x, t.y, t.z);
  }
  // sky view
  const float vza = atan2_upper(sqrtf(fmaf(ux, ux, uz * uz)), uy);
  const float zha = 1.57079632679f + atan01(fminf(rho0 * u.inv_planet_r, 1.0f));
  const bool below = vza < zha;
  const float num = below ? vza : vza - zha;
  const float den = below ? zha : kPi - zha;
  const float vv = fmaf(0.5f, sqrtf(__saturatef(__fdividef(num, fmaxf(den, 1e-6f)))), below ? 0.0f : 0.5f);
  float du = (fast_atan2(ux, uz) - u.sun_az) * (1.0f / (2.0f * kPi));
  du = du - floorf(du);
  const float4 sk = u.tex_sky ? tex2D<float4>(u.tex_sky, du, vv) : lut2d(u.lut_sky, 192, 108, du, vv);
  sky = make_float3(sk.x * u.sun_illum[0], sk.y * u.sun_illum[1], sk.z * u.sun_illum[2]);
  return lit;
}

// Weather R channel, repeat + bilinear; a uniform map is its value, power-of-
// two sizes wrap with a mask, and up to 1024^2 read one 16-byte 2x2
// footprint per tap.
__device__ __forceinline__ float weather_fast(const MarchUniforms& u, float uu, float vv) {
  const uint32_t W = u.weather_w, H = u.weather_h;
  if (u.weather_uniform) return u.weather_value;  // bilinear of a constant is the constant
  if (u.weather_quad) {
    const float x = fmaf(uu, (float)W, -0.5f), y = fmaf(vv, (float)H, -0.5f);
    const FloorBits bx = floor_bits(x), by = floor_bits(y);
    const float4 q = __ldg(u.weather_quad + (by.i & (H - 1)) * W + (bx.i & (W - 1)));
    return lerpf(lerpf(q.x, q.y, x - bx.f), lerpf(q.z, q.w, x - bx.f), y - by.f);
  }
  if (((W & (W - 1)) | (H & (H - 1))) != 0) return weather_sample(u.weather, W, H, uu, vv);
  const float x = fmaf(uu, (float)W, -0.5f), y = fmaf(vv, (float)H, -0.5f);
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const uint32_t x0 = (uint32_t)ix & (W - 1), x1 = (uint32_t)(ix + 1) & (W - 1);
  const uint32_t y0 = (uint32_t)iy & (H - 1), y1 = (uint32_t)(iy + 1) & (H - 1);
  const float a = lerpf(__ldg(u.weather + y0 * W + x0), __ldg(u.weather + y0 * W + x1), wx);
  const float b = lerpf(__ldg(u.weather + y1 * W + x0), __ldg(u.weather + y1 * W + x1), wx);
  return lerpf(a, b, wy);
}

// The primary steps of a ray's layer segment that can pass the profile test
// (no type grid): those whose altitude lies in the layer's band
// [live_lo, live_hi] (LayerConst), found from the ray's geometry instead of
// stepping through the rest.  Along the ray, |o + t d| = R + a at
// t = tv -/+ sqrt((R + a)^2 - rp^2) with tv = -r0 cos(up, d) and rp the
// line's closest distance to the planet centre, so the altitude stays at or
// below a_hi on [tv - sqrt(q_hi), tv + sqrt(q_hi)] and falls below a_lo only
// inside (tv - sqrt(q_lo), tv + sqrt(q_lo)); the hull of what remains in
// [t0, t1] becomes step indices.  In FP64 from the FP32 r0 and cos(up, d)
// the ray carries (their rounding moves t by about 1 m at most), with the
// band widened by 3 m more and the index range by 2-3 steps: every step that
// could pass the test is inside [s_begin, s_end), and the steps outside add
// nothing and leave the transmittance as it is, so skipping them is exact.
// Returns false when no step of the segment can pass.
__device__ __forceinline__ bool live_step_range(float r0f, float ray_B, const LayerConst& L, float R,
                                                float t0, float t1, float step, float jitter,
                                                uint32_t n, uint32_t& s_begin, uint32_t& s_end) {
  const double r0 = r0f, cv = (double)ray_B / (2.0 * fmax(r0, 1.0));
  const double tv = -r0 * cv;
  const double rp2 = r0 * r0 * fmax(1.0 - cv * cv, 0.0);
  const double rh = (double)R + ((double)L.live_hi + 3.0), rl = (double)R + ((double)L.live_lo - 3.0);
  const double qh = rh * rh - rp2;
  if (qh < 0.0) return false;  // the line stays above the band
  const double sh = sqrt(qh);
  double lo = fmax((double)t0, tv - sh), hi = fmin((double)t1, tv + sh);
  if (lo > hi) return false;
  const double ql = rl * rl - rp2;
  if (ql > 0.0) {  // the open interval where the altitude is below the band
    const double sl = sqrt(ql), c = tv - sl, d = tv + sl;
    const bool p1 = lo <= fmin(hi, c), p2 = fmax(lo, d) <= hi;
    if (!p1 && !p2) return false;
    const double nlo = p1 ? lo : fmax(lo, d), nhi = p2 ? hi : fmin(hi, c);
    lo = nlo;
    hi = nhi;
  }
  const double is = 1.0 / (double)step;
  const double fb = floor((lo - (double)t0) * is - (double)jitter) - 2.0;
  const double fe = ceil((hi - (double)t0) * is - (double)jitter) + 3.0;
  s_begin = fb <= 0.0 ? 0u : (fb >= (double)n ? n : (uint32_t)fb);
  s_end = fe <= 0.0 ? 0u : (fe >= (double)n ? n : (uint32_t)fe);
  return s_begin < s_end;
}

// 1 - exp(-y) without cancellation for small y.
__device__ __forceinline__ float one_minus_exp_neg(float y, float e) {
  return y < 0.03f ? y * fmaf(y, fmaf(y, fmaf(y, -1.0f / 24.0f, 1.0f / 6.0f), -0.5f), 1.0f)
                   : 1.0f - e;
}

// Per-thread shared-memory words of march_pixel_fast beyond the layer
// intervals, all touched at most once per dense sample and so kept out of
// the registers the step loop needs: the per-layer octave coefficients (two
// sets for a Cumulonimbus layer: its own droplet size and 50 um), the
// compensated optical depths of the Kahan form, the radiance, the
// aerial-perspective distance weights and (lean form) the ray's layer order
// and hit mask.
constexpr uint32_t kAuxWords = 2 * kMaxOct + 6 + 5 + 2;

// Fetch tally of the instrumented build (TALLY = true): per ray, the
// fetches march_pixel_fast issues, by kind, in the order of PscFetchCounts.
// The last two count, for the dense-sample body (LUT lookups, light march,
// octaves, radiance), the warp passes through it and the lanes active in
// them: their ratio over 32 is the body's SIMT efficiency.
enum TallyKind : uint32_t {
  kTallyRays, kTallySteps, kTallyLive, kTallyWeather, kTallyType, kTallyDetail, kTallyDense,
  kTallyLight, kTallyTrans, kTallySky, kTallyAp, kTallyDepth, kTallyDensePasses, kTallyDenseLanes,
  kTallyKinds
};
static_assert(kTallyKinds == kFetchTallyKinds, "one tally counter per PscFetchCounts field");

// One primary ray of the FAST schedule.  `s_t0/s_t1` are this CTA's shared
// arrays of per-layer entry/exit distances, laid out [layer][slot] with
// `stride` slots; `slot` is this thread's column.  `s_aux` holds kAuxWords
// words per thread, laid out the same way.
// TALLY = true is the instrumented build behind psc_count_fetches: the same
// arithmetic, and `tc` (kTallyKinds counters of this thread) counts every
// fetch issued; the timed kernels are built with TALLY = false, where `tc`
// is unused and the counting compiles away.  LB is the light-march fetch
// batch (light_march_tex).
template <int ST, int FILT, bool FULL = true, bool TALLY = false, int LB = 0>
__device__ __forceinline__ void march_pixel_fast(const MarchUniforms& u, const ViewDev& v, uint32_t px,
                                                 uint32_t py, float* s_t0, float* s_t1, float* s_aux,
                                                 uint32_t stride, uint32_t slot, uint32_t* tc = nullptr) {
  if constexpr (TALLY) {
    ++tc[kTallyRays];
    if (v.depth) ++tc[kTallyDepth];
  }

  // Per-lane layer intervals live in shared memory for the march, so the 16
  // entry/exit distances do not occupy registers across the loop.
  RaySetup rs;
  setup_ray(u, v, px, py, rs);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    if ((uint32_t)j < u.layer_count) {  // the arrays hold layer_count rows
      s_t0[j * stride + slot] = rs.t0[j];
      s_t1[j * stride + slot] = rs.t1[j];
    }
  }
  // the lean form keeps the layer order and hit mask in shared memory too,
  // and recomputes cos(view, sun) and the forward gain per layer: values
  // that the step loop does not read stay out of its registers (1080p
  // frame 3.949 -> 3.898 ms, the same image; the full form is left as it
  // was, where the change measured 0.8 % slower on the 4K frames)
  uint32_t* const s_ord = reinterpret_cast<uint32_t*>(s_aux + (kAuxWords - 2) * stride);
  const uint32_t order = FULL ? rs.order : 0u, hit_mask = FULL ? rs.hit_mask : 0u;
  if constexpr (!FULL) {
    s_ord[slot] = rs.order;
    s_ord[stride + slot] = rs.hit_mask;
  }
  const float ray_r0 = rs.r0, ray_h0 = rs.h0;
  // distance from the planet centre along the ray: r(t)^2 = A + t (B + t)
  const float ray_A = ray_r0 * ray_r0, ray_B = 2.0f * ray_r0 * rs.cos_view;
  const float dx = rs.dir[0], dy = rs.dir[1], dz = rs.dir[2];
  const float cx = u.cam[0], cy = u.cam[1], cz = u.cam[2];
  const float cos_theta_r = fmaf(dx, u.sun[0], fmaf(dy, u.sun[1], dz * u.sun[2]));
  const float fwd_gain_r =
      u.forward_bias > 0.0f ? 1.0f + u.forward_bias * smoothstepf(0.0f, 1.0f, fmaxf(cos_theta_r, 0.0f))
                            : 1.0f;
  uint32_t sx = (px + v.x_off) & 63u, sy = (py + v.y_off) & 63u;
  if (u.temporal_jitter) {
    const uint32_t ph = u.frame_index & 15u;
    sx = (sx ^ ((ph * 11u + 7u) & 63u)) & 63u;
    sy = (sy ^ ((ph * 23u + 13u) & 63u)) & 63u;
  }
  const float jitter = __ldg(u.blue + sy * 64u + sx);
  const uint32_t noct = u.octaves;

  float* const s_coef = s_aux;                         // [kMaxOct][stride]
  float* const s_coef_hi = s_aux + kMaxOct * stride;   // Cumulonimbus at 50 um, [kMaxOct][stride]
  float* const s_kahan = s_coef_hi + kMaxOct * stride; // od r,g,b then comp r,g,b
  float* const s_acc = s_kahan + 6 * stride;        // L r,g,b, sum(w t), sum(w)
  if (FULL && u.kahan) {
#pragma unroll
    for (int c = 0; c < 6; ++c) s_kahan[c * stride + slot] = 0.0f;
  }
#pragma unroll
  for (int c = 0; c < 5; ++c) s_acc[c * stride + slot] = 0.0f;

  float Tr = 1.0f, Tg = 1.0f, Tb = 1.0f;
  const uint32_t nl = u.layer_count;

  for (uint32_t k = 0; k < nl; ++k) {
    if (fmaxf(Tr, fmaxf(Tg, Tb)) < 0.01f) break;
    const uint32_t li = ((FULL ? order : s_ord[slot]) >> (4u * k)) & 15u;
    if (!(((FULL ? hit_mask : s_ord[stride + slot]) >> li) & 1u)) continue;
    const float t0 = s_t0[li * stride + slot], t1 = s_t1[li * stride + slot];
    const LayerConst& L = u.layers[li];
    const float segment = t1 - t0;
    if (segment <= 0.0f) continue;
    const float step = __fdividef(segment, (float)u.cloud_steps);
    uint32_t s_begin = 0u, s_end = u.cloud_steps;
    // lean form: the profile test depends on the altitude alone (no type
    // grid).  The full form keeps every step (the range costs it more than it
    // saves on the 4K stress frames: 91.6 ms against 88.1 ms).
    if constexpr (!FULL) {
      if (!(L.live_lo <= L.live_hi)) continue;  // no step of this layer can pass it
      if (!live_step_range(ray_r0, ray_B, L, u.planet_r, t0, t1, step, jitter, u.cloud_steps, s_begin,
                           s_end))
        continue;
    }
    const bool cb = FULL && L.cloud_type == 7u && u.phase_mode == PSC_PHASE_APPROX_MIE;
    const float cos_theta = FULL ? cos_theta_r : fmaf(dx, u.sun[0], fmaf(dy, u.sun[1], dz * u.sun[2]));
    const float fwd_gain =
        FULL ? fwd_gain_r
             : (u.forward_bias > 0.0f ? 1.0f + u.forward_bias * smoothstepf(0.0f, 1.0f, fmaxf(cos_theta, 0.0f))
                                      : 1.0f);

    // per ray and layer: a^n * phase_n * forward gain (shared memory)
    if (u.phase_mode == PSC_PHASE_DUAL_LOBE_HG) {
#pragma unroll
      for (int n = 0; n < kMaxOct; ++n) {
        const float c = u.cpow[n];
        s_coef[n * stride + slot] =
            (n < (int)noct) ? u.apow[n] * fwd_gain *
                                  mixf(hg_phase(cos_theta, u.hg_f * c), hg_phase(cos_theta, u.hg_b * c), u.hg_w)
                            : 0.0f;
      }
    } else if (!cb) {
      const PhaseConst pc{L.g_hg, L.g_d, L.alpha, L.w_d, L.ice};
#pragma unroll
      for (int n = 0; n < kMaxOct; ++n)
        s_coef[n * stride + slot] =
            (n < (int)noct) ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], pc) : 0.0f;
    } else {
      // Cumulonimbus: the droplet diameter blends from the layer's to 50 um
      // with mt = smoothstep(0.60, 0.85, h); mt is exactly 0 below the band
      // and exactly 1 once its clamp saturates, where mix(d, 50, mt) is
      // exactly d or exactly 50, so those two coefficient sets are
      // evaluated once here with the same expressions as the per-sample form
      const PhaseConst lo = phase_consts_from_d(mixf(L.droplet_um, 50.0f, 0.0f), u.droplet_bias);
      const PhaseConst hi = phase_consts_from_d(mixf(L.droplet_um, 50.0f, 1.0f), u.droplet_bias);
#pragma unroll
      for (int n = 0; n < kMaxOct; ++n) {
        const bool on = n < (int)noct;
        s_coef[n * stride + slot] = on ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], lo) : 0.0f;
        s_coef_hi[n * stride + slot] = on ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], hi) : 0.0f;
      }
    }

    for (uint32_t s = s_begin; s < s_end; ++s) {
      if constexpr (TALLY) ++tc[kTallySteps];
      const float t = fmaf((float)s + jitter, step, t0);
      const float px3 = fmaf(dx, t, cx), py3 = fmaf(dy, t, cy), pz3 = fmaf(dz, t, cz);
      const float bt = ray_B + t;
      const float alt = ray_h0 + __fdividef(t * bt, ray_r0 + sqrtf(fmaf(t, bt, ray_A)));
      const float h = (alt - L.base_m) * L.inv_thickness;
      // Profile test before any fetch (no type grid: the profile depends on h
      // alone).  The base shape is at most 1 and the detail erosion only
      // lowers it, so the density is at most (nd - (1 - eff)) * density_scale
      // (up to rounding, which skip_k and the 1.000001 absorb); at or below
      // the 1e-3 threshold the step adds nothing and its fetches are skipped.
      bool live = h >= 0.0f && h <= 1.0f;
      float nd = 0.0f;
      if (live && !(FULL && u.type_grid)) {
        // the lean form has no Cumulonimbus layer, so ndf_mode 0 there means
        // an unknown type, whose profile is 0
        nd = L.ndf_mode ? ndf_eval(NdfCoef{L.ndf_inv_a, L.ndf_b1, L.ndf_inv_w1}, h)
                        : (FULL ? ndf_fast(h, L.cloud_type, L.anvil_bias) : 0.0f);
        live = fmaf(nd, 1.000001f, -L.skip_k) * L.density_scale > 1e-3f;
      }
      if (live) {
        if constexpr (TALLY) {
          ++tc[kTallyLive];  // base-shape and curl fetches
          if (!u.weather_uniform) ++tc[kTallyWeather];
          if (FULL && u.type_grid) ++tc[kTallyType];
        }
        const float wsx = px3 - L.wind_off_x, wsz = pz3 - L.wind_off_z;
        const float ax = fmaf(-L.skew_kx, h, wsx);
        const float az = fmaf(-L.skew_kz, h, wsz);
        // weather, type and base fetches do not depend on each other
        const float wr = weather_fast(u, fmaf(wsx, u.inv_weather_scale, 0.5f),
                                      fmaf(wsz, u.inv_weather_scale, 0.5f));
        const uint32_t type = FULL ? effective_type(u, wsx, wsz, L.cloud_type) : L.cloud_type;
        const float2 bs = base_tap<ST, FILT, false>(u, ax, py3, az);
        const CurlFetch cf = curl_fetch(u.curl_quad, fmaf(ax, u.curl_texel_scale, -0.5f),
                                        fmaf(az, u.curl_texel_scale, -0.5f));
        const float eff = clamp01(wr * L.coverage);
        if (FULL && u.type_grid) nd = ndf_fast(h, type, L.anvil_bias);
        float cloud = shape_from<ST>(bs, L.lf_c, nd, 1.0f - eff);
        if (eff >= 0.01f) {  // coverage gate (cloud_march.wgsl:450-451)
          if (cloud > 0.0f) {  // curl-perturbed detail erosion (:502-527)
            if constexpr (TALLY) ++tc[kTallyDetail];
            const float2 c2 = curl_blend(cf);
            const float ddx = fmaf(fmaf(c2.x, 2.0f, -1.0f), u.curl_offset_scale, ax);
            const float ddz = fmaf(fmaf(c2.y, 2.0f, -1.0f), u.curl_offset_scale, az);
            const float hf = detail_tap<ST, FILT>(u, ddx, py3, ddz);
            const float dmod = mixf(hf, 1.0f - hf, clamp01(h * 10.0f));
            const float lo = dmod * L.layer_detail;
            cloud = __fdividef(cloud - lo, fmaxf(1.0f - lo, 1e-5f));
          }
          const float density = clamp01(cloud) * L.density_scale;

          if (density > 1e-3f) {
            const float yy = py3 + u.planet_r;
            const float inv_r = __fdividef(1.0f, u.planet_r + alt);
            const float ux = px3 * inv_r, uy = yy * inv_r, uz = pz3 * inv_r;
            // the two LUT fetches go out before the light march's, so all of
            // a dense sample's texture fetches are in flight together
            float3 ts, sky;
            [[maybe_unused]] const bool trans_fetched = lut_lookups(u, alt, ux, uy, uz, ts, sky);
            if constexpr (TALLY) {
              const uint32_t act = __activemask();
              if ((threadIdx.x & 31u) == (uint32_t)__ffs(act) - 1u) {
                ++tc[kTallyDensePasses];
                tc[kTallyDenseLanes] += (uint32_t)__popc(act);
              }
              ++tc[kTallyDense];
              ++tc[kTallySky];
              tc[kTallyTrans] += trans_fetched ? 1u : 0u;
            }
            uint32_t light_taps_done = (FULL && u.cone) ? 6u : u.light_steps;
            const float od = light_od<ST, FILT, FULL, LB>(u, L, px3, py3, pz3, alt, eff, type, ux, uy, uz,
                                                          TALLY ? &light_taps_done : nullptr);
            if constexpr (TALLY) tc[kTallyLight] += light_taps_done;
            const float st_r = L.sigma_t[0], st_g = L.sigma_t[1], st_b = L.sigma_t[2];
            const float xr = st_r * od, xg = st_g * od, xb = st_b * od;
            // e[n] = exp(-x * b^n); with b = 1/2 one exponential at n = 3 and
            // repeated squaring give every lower octave (octaves past the
            // count carry zero coefficients).
            float er[kMaxOct], eg[kMaxOct], eb[kMaxOct];
            const int m = (int)noct - 1;
            if (u.b_half) {
              float vr = __expf(xr * -0.125f), vg = __expf(xg * -0.125f), vb = __expf(xb * -0.125f);
#pragma unroll
              for (int n = kMaxOct - 1; n >= 0; --n) {
                er[n] = vr;
                eg[n] = vg;
                eb[n] = vb;
                vr *= vr;
                vg *= vg;
                vb *= vb;
              }
            } else {
#pragma unroll
              for (int n = 0; n < kMaxOct; ++n) {
                const bool live = n <= m;
                er[n] = live ? __expf(-xr * u.bpow[n]) : 0.0f;
                eg[n] = live ? __expf(-xg * u.bpow[n]) : 0.0f;
                eb[n] = live ? __expf(-xb * u.bpow[n]) : 0.0f;
              }
            }
            // Beer-powder mix(b, 2 b (1 - b^2), w) = b (1 + w (1 - 2 b^2)), b = e[0]
            const float br = er[0], bg = eg[0], bb = eb[0];
            const float enr = br * fmaf(u.powder, fmaf(-2.0f * br, br, 1.0f), 1.0f);
            const float eng = bg * fmaf(u.powder, fmaf(-2.0f * bg, bg, 1.0f), 1.0f);
            const float enb = bb * fmaf(u.powder, fmaf(-2.0f * bb, bb, 1.0f), 1.0f);
            float cf[kMaxOct];
            const float mt = cb ? smoothstepf(0.60f, 0.85f, h) : 0.0f;
            if (cb && mt > 0.0f && mt < 1.0f) {  // inside the blend band
              const PhaseConst pc = phase_consts_from_d(mixf(L.droplet_um, 50.0f, mt), u.droplet_bias);
#pragma unroll
              for (int n = 0; n < kMaxOct; ++n)
                cf[n] = (n < (int)noct) ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], pc) : 0.0f;
            } else if (cb && mt >= 1.0f) {
#pragma unroll
              for (int n = 0; n < kMaxOct; ++n) cf[n] = s_coef_hi[n * stride + slot];
            } else {
#pragma unroll
              for (int n = 0; n < kMaxOct; ++n) cf[n] = s_coef[n * stride + slot];
            }
            float sr = 0.0f, sg = 0.0f, sb = 0.0f;
#pragma unroll
            for (int n = 0; n < kMaxOct; ++n) {
              sr = fmaf(cf[n], er[n], sr);
              sg = fmaf(cf[n], eg[n], sg);
              sb = fmaf(cf[n], eb[n], sb);
            }
            sr *= u.sun_illum[0] * ts.x;
            sg *= u.sun_illum[1] * ts.y;
            sb *= u.sun_illum[2] * ts.z;
            const float ag = mixf(0.3f, 1.0f, clamp01(h)) * u.ambient;
            float lr = 0.0f, lg = 0.0f, lb = 0.0f;
            if (FULL && u.lightning_radius > 0.0f) {
              const float ddx = px3 - u.lightning_origin_x, ddz = pz3 - u.lightning_origin_z;
              const float fo = clamp01(1.0f - sqrtf(ddx * ddx + ddz * ddz) / u.lightning_radius);
              const float wgt = fo * fo * (3.0f - 2.0f * fo);
              lr = u.lightning_rgb[0] * wgt;
              lg = u.lightning_rgb[1] * wgt;
              lb = u.lightning_rgb[2] * wgt;
            }
            const float isr = density * u.sigma_s[0] * fmaf(sr, enr, fmaf(sky.x, ag, lr));
            const float isg = density * u.sigma_s[1] * fmaf(sg, eng, fmaf(sky.y, ag, lg));
            const float isb = density * u.sigma_s[2] * fmaf(sb, enb, fmaf(sky.z, ag, lb));
            const float lsr = fmaxf(density * st_r, 1e-6f), lsg = fmaxf(density * st_g, 1e-6f),
                        lsb = fmaxf(density * st_b, 1e-6f);
            const float yr = lsr * step, yg = lsg * step, yb = lsb * step;
            const float smr = __expf(-yr), smg = __expf(-yg), smb = __expf(-yb);
            const float slr = Tr * isr * __fdividef(one_minus_exp_neg(yr, smr), lsr);
            const float slg = Tg * isg * __fdividef(one_minus_exp_neg(yg, smg), lsg);
            const float slb = Tb * isb * __fdividef(one_minus_exp_neg(yb, smb), lsb);
            const float sw = fmaf(slb, 0.0722f, fmaf(slg, 0.7152f, slr * 0.2126f));
            s_acc[0 * stride + slot] += slr;
            s_acc[1 * stride + slot] += slg;
            s_acc[2 * stride + slot] += slb;
            s_acc[3 * stride + slot] = fmaf(sw, t, s_acc[3 * stride + slot]);
            s_acc[4 * stride + slot] += sw;
            if (FULL && u.kahan) {  // T = exp(-sum), the sum compensated (shared memory)
              const float y3[3] = {yr, yg, yb};
              float T3[3];
#pragma unroll
              for (int c = 0; c < 3; ++c) {
                const float od = s_kahan[c * stride + slot], kc = s_kahan[(3 + c) * stride + slot];
                const float a = y3[c] - kc;
                const float nsum = od + a;
                s_kahan[(3 + c) * stride + slot] = (nsum - od) - a;
                s_kahan[c * stride + slot] = nsum;
                T3[c] = __expf(-nsum);
              }
              Tr = T3[0];
              Tg = T3[1];
              Tb = T3[2];
            } else {
              Tr *= smr;
              Tg *= smg;
              Tb *= smb;
            }
          }
        }
      }
      if (fmaxf(Tr, fmaxf(Tg, Tb)) < 0.01f) break;
    }
  }

  const float t_lum = fmaf(Tb, 0.0722f, fmaf(Tg, 0.7152f, Tr * 0.2126f));
  const float opacity = 1.0f - t_lum;
  const float Lr = s_acc[0 * stride + slot], Lg = s_acc[1 * stride + slot], Lb = s_acc[2 * stride + slot];
  const float tw = s_acc[3 * stride + slot], twn = s_acc[4 * stride + slot];
  float Or = Lr, Og = Lg, Ob = Lb;
  if (opacity > 1e-4f) {
    if constexpr (TALLY) ++tc[kTallyAp];
    const float t_cloud = __fdividef(tw, fmaxf(twn, 1e-6f));
    const float ds = fmaxf(t_cloud, 50.0f);
    const float az = clamp01(__logf(ds * (1.0f / 50.0f)) * (1.0f / 7.6009024595f));  // ln 2000
    const float4 ap = lut_ap(u.lut_ap, ((float)(px + v.x_off) + 0.5f) / u.vp_w,
                             ((float)(py + v.y_off) + 0.5f) / u.vp_h, az);
    Or = fmaf(Lr, ap.w, ap.x * opacity);
    Og = fmaf(Lg, ap.w, ap.y * opacity);
    Ob = fmaf(Lb, ap.w, ap.z * opacity);
  }
  const size_t idx = (size_t)py * v.width + px;
  const float4 lo = make_float4(Or, Og, Ob, 1.0f);
  const float4 to = make_float4(Tr, Tg, Tb, 1.0f);
  if (v.out_l) v.out_l[idx] = lo;
  if (v.out_t) v.out_t[idx] = to;
  if (u.composite && v.hdr) {
    const float4 d = v.hdr[idx];
    v.hdr[idx] = make_float4(fmaf(d.x, to.x, lo.x), fmaf(d.y, to.y, lo.y), fmaf(d.z, to.z, lo.z),
                             fmaf(d.w, to.w, lo.w));
  }
}

}  // namespace
}  // namespace psc

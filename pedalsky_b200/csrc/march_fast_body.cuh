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
//   * the transmittance-LUT and sky-view lookups use well-conditioned forms
//     (r = R + alt, rho = sqrt(alt*(2R + alt)), zenith angles via atan2) with
//     a polynomial arctangent;
//   * weather/type fetches are skipped where the height gate already
//     returns zero density;
//   * texel coordinates are formed with one FMA per axis.
//   * smoothsteps multiply by precomputed reciprocals, and this translation
//     unit is built with approximate division and square root (a few ulp).
// Octave counts up to 4 are handled here; the host falls back to the plain
// kernel beyond that.
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

template <int ST, int FILT, bool LIGHT>
__device__ __forceinline__ float4 base_tap(const MarchUniforms& u, float ax, float ay, float az) {
  if constexpr (FILT == PSC_FILTER_TEXTURE || (FILT == PSC_FILTER_HYBRID && LIGHT)) {
    float4 r = tex3D<float4>(u.tex_base, ax * u.inv_base_scale, ay * u.inv_base_scale,
                             az * u.inv_base_scale);
    if constexpr (ST == PSC_STORAGE_F16) {
      r.x *= (1.0f / 255.0f);
      r.y *= (1.0f / 255.0f);
      r.z *= (1.0f / 255.0f);
      r.w *= (1.0f / 255.0f);
    }
    return r;
  } else {
    const float k = u.base_texel_scale;
    return trilinear_texel<ST, 128>(u.noise_base, fmaf(ax, k, -0.5f), fmaf(ay, k, -0.5f),
                                    fmaf(az, k, -0.5f), u.noise_scale);
  }
}

template <int ST, int FILT>
__device__ __forceinline__ float4 detail_tap(const MarchUniforms& u, float dx, float dy, float dz) {
  if constexpr (FILT == PSC_FILTER_TEXTURE) {
    float4 r = tex3D<float4>(u.tex_detail, dx * u.inv_detail_scale, dy * u.inv_detail_scale,
                             dz * u.inv_detail_scale);
    if constexpr (ST == PSC_STORAGE_F16) {
      r.x *= (1.0f / 255.0f);
      r.y *= (1.0f / 255.0f);
      r.z *= (1.0f / 255.0f);
      r.w *= (1.0f / 255.0f);
    }
    return r;
  } else {
    const float k = u.detail_texel_scale;
    return trilinear_texel<ST, 32>(u.noise_detail, fmaf(dx, k, -0.5f), fmaf(dy, k, -0.5f),
                                   fmaf(dz, k, -0.5f), u.noise_scale);
  }
}

// smoothstep with the reciprocal of (e1 - e0) precomputed (a multiply, not
// a division); e0 > e1 gives the reversed ramps of cloud_density_common.wgsl.
__device__ __forceinline__ float ssr(float e0, float inv_w, float x) {
  const float t = clamp01((x - e0) * inv_w);
  return t * t * fmaf(-2.0f, t, 3.0f);
}
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
// (cloud_march.wgsl:463-494).  `h` in [0,1], `eff` >= 0.01 already checked.
template <int ST, int FILT, bool LIGHT>
__device__ __forceinline__ float base_shape(const MarchUniforms& u, const LayerConst& L, float ax,
                                            float ay, float az, float h, float eff, uint32_t type) {
  const float4 b = base_tap<ST, FILT, LIGHT>(u, ax, ay, az);
  const float lf = clamp01(fmaf(b.w, 0.125f, fmaf(b.z, 0.25f, b.y * 0.625f)) + L.lf_bias);
  const float base_cloud = __fdividef(b.x + (1.0f - lf), fmaxf(2.0f - lf, 1e-5f));
  const float cloud = base_cloud * ndf_fast(h, type, L.anvil_bias);
  return __fdividef(cloud - (1.0f - eff), fmaxf(eff, 1e-5f)) * eff;
}

template <int ST, int FILT>
__device__ __forceinline__ float density_light(const MarchUniforms& u, const LayerConst& L, float qx,
                                               float qy, float qz, float alt, float eff,
                                               uint32_t type) {
  const float h = (alt - L.base_m) * L.inv_thickness;
  if (h < 0.0f || h > 1.0f) return 0.0f;
  const float sk = h * L.skew_thickness;
  const float ax = fmaf(-L.skew_x, sk, qx - L.wind_off_x);
  const float az = fmaf(-L.skew_z, sk, qz - L.wind_off_z);
  return clamp01(base_shape<ST, FILT, true>(u, L, ax, qy, az, h, eff, type)) * L.density_scale;
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

// Optical depth toward the sun (cloud_march.wgsl:543-578).
template <int ST, int FILT>
__device__ __forceinline__ float light_od(const MarchUniforms& u, const LayerConst& L, float px,
                                          float py, float pz, float alt, float eff, uint32_t type,
                                          float ux, float uy, float uz) {
  const float r0 = u.planet_r + alt;
  const float cv = fmaf(ux, u.sun[0], fmaf(uy, u.sun[1], uz * u.sun[2]));
  const float dist = fmaxf((L.top_m - alt) * u.inv_cos_sun, 1.0f);
  if (u.cone) return light_cone<ST, FILT>(u, L, px, py, pz, alt, eff, type, r0, cv, dist);
  const float step = __fdividef(dist, (float)u.light_steps);
  float od = 0.0f, comp = 0.0f;
  for (uint32_t i = 0; i < u.light_steps; ++i) {
    const float t = ((float)i + 0.5f) * step;
    const float qx = fmaf(u.sun[0], t, px), qy = fmaf(u.sun[1], t, py), qz = fmaf(u.sun[2], t, pz);
    const float term =
        density_light<ST, FILT>(u, L, qx, qy, qz, alt_from(u, qx, qy, qz, r0, cv, alt, t), eff, type) *
        step;
    if (u.kahan) {
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

// Transmittance-LUT lookup (cloud_march.wgsl:328-354) with r = R + alt and
// rho = sqrt(alt*(2R + alt)) instead of differences of squares at 6e6 m.
__device__ __forceinline__ float3 sun_trans_fast(const MarchUniforms& u, float alt, float ux,
                                                 float uy, float uz) {
  const float R = u.planet_r;
  const float a = fmaxf(alt, 1.0f);
  const float r = R + a;
  const float rho = sqrtf(a * (2.0f * R + a));
  const float mu = clampf(fmaf(ux, u.sun[0], fmaf(uy, u.sun[1], uz * u.sun[2])), -1.0f, 1.0f);
  if (mu <= -__fdividef(rho, r)) return make_float3(0.0f, 0.0f, 0.0f);
  const float top = u.atmo_top;
  const float rm = r * mu;
  const float disc = fmaf(rm, rm, (top - r) * (top + r));
  const float d = fmaxf(sqrtf(fmaxf(disc, 0.0f)) - rm, 0.0f);
  const float d_min = top - r, d_max = rho + u.big_h;
  const float xm = clamp01(__fdividef(d - d_min, fmaxf(d_max - d_min, 1.0f)));
  const float xr = __fdividef(rho, fmaxf(u.big_h, 1.0f));
  const float4 t = lut2d(u.lut_trans, 256, 64, xm, xr);
  return make_float3(t.x, t.y, t.z);
}

// Sky-view ambient (cloud_march.wgsl:672-700): local up, zenith angle and
// horizon angle through atan2 (pi - asin(R/r) = pi/2 + atan2(rho, R)).
__device__ __forceinline__ float3 sky_fast(const MarchUniforms& u, float alt, float ux, float uy,
                                           float uz) {
  const float R = u.planet_r;
  const float a = fmaxf(alt, 0.0f);
  const float rho = sqrtf(a * (2.0f * R + a));
  const float vza = fast_atan2(sqrtf(fmaf(ux, ux, uz * uz)), uy);
  const float zha = 1.57079632679f + fast_atan2(rho, R);
  float vv;
  if (vza < zha) {
    vv = sqrtf(clamp01(__fdividef(vza, fmaxf(zha, 1e-6f)))) * 0.5f;
  } else {
    vv = 0.5f + sqrtf(clamp01(__fdividef(vza - zha, fmaxf(kPi - zha, 1e-6f)))) * 0.5f;
  }
  float du = (fast_atan2(ux, uz) - u.sun_az) * (1.0f / (2.0f * kPi));
  du = du - floorf(du);
  const float4 s = lut2d(u.lut_sky, 192, 108, du, vv);
  return make_float3(s.x * u.sun_illum[0], s.y * u.sun_illum[1], s.z * u.sun_illum[2]);
}

// Weather R channel, repeat + bilinear; power-of-two sizes wrap with a mask.
__device__ __forceinline__ float weather_fast(const MarchUniforms& u, float uu, float vv) {
  const uint32_t W = u.weather_w, H = u.weather_h;
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

// 1 - exp(-y) without cancellation for small y.
__device__ __forceinline__ float one_minus_exp_neg(float y, float e) {
  return y < 0.03f ? y * fmaf(y, fmaf(y, fmaf(y, -1.0f / 24.0f, 1.0f / 6.0f), -0.5f), 1.0f)
                   : 1.0f - e;
}

// One primary ray of the FAST schedule.  `s_t0/s_t1` are this CTA's shared
// arrays of per-layer entry/exit distances, laid out [layer][slot] with
// `stride` slots; `slot` is this thread's column.
template <int ST, int FILT>
__device__ __forceinline__ void march_pixel_fast(const MarchUniforms& u, const ViewDev& v, uint32_t px,
                                                 uint32_t py, float* s_t0, float* s_t1,
                                                 uint32_t stride, uint32_t slot) {

  // Per-lane layer intervals live in shared memory for the march, so the 16
  // entry/exit distances do not occupy registers across the loop.
  RaySetup rs;
  setup_ray(u, v, px, py, rs);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    s_t0[j * stride + slot] = rs.t0[j];
    s_t1[j * stride + slot] = rs.t1[j];
  }
  const uint32_t order = rs.order, hit_mask = rs.hit_mask;
  const float ray_r0 = rs.r0, ray_cv = rs.cos_view, ray_h0 = rs.h0;
  const float dx = rs.dir[0], dy = rs.dir[1], dz = rs.dir[2];
  const float cx = u.cam[0], cy = u.cam[1], cz = u.cam[2];
  const float cos_theta = fmaf(dx, u.sun[0], fmaf(dy, u.sun[1], dz * u.sun[2]));
  const float fwd_gain =
      u.forward_bias > 0.0f ? 1.0f + u.forward_bias * smoothstepf(0.0f, 1.0f, fmaxf(cos_theta, 0.0f))
                            : 1.0f;
  uint32_t sx = (px + v.x_off) & 63u, sy = (py + v.y_off) & 63u;
  if (u.temporal_jitter) {
    const uint32_t ph = u.frame_index & 15u;
    sx = (sx ^ ((ph * 11u + 7u) & 63u)) & 63u;
    sy = (sy ^ ((ph * 23u + 13u) & 63u)) & 63u;
  }
  const float jitter = __ldg(u.blue + sy * 64u + sx);
  const uint32_t noct = u.octaves;

  // Dual-lobe HG lobes do not depend on the layer: evaluate once per ray.
  float hg_coef[kMaxOct];
  if (u.phase_mode == PSC_PHASE_DUAL_LOBE_HG) {
#pragma unroll
    for (int n = 0; n < kMaxOct; ++n) {
      const float c = u.cpow[n];
      hg_coef[n] = (n < (int)noct) ? u.apow[n] * fwd_gain *
                                         mixf(hg_phase(cos_theta, u.hg_f * c),
                                              hg_phase(cos_theta, u.hg_b * c), u.hg_w)
                                   : 0.0f;
    }
  }

  float Lr = 0.0f, Lg = 0.0f, Lb = 0.0f, Tr = 1.0f, Tg = 1.0f, Tb = 1.0f;
  float odr = 0.0f, odg = 0.0f, odb = 0.0f, kr = 0.0f, kg = 0.0f, kb = 0.0f;
  float tw = 0.0f, twn = 0.0f;
  const uint32_t nl = u.layer_count;

  for (uint32_t k = 0; k < nl; ++k) {
    if (fmaxf(Tr, fmaxf(Tg, Tb)) < 0.01f) break;
    const uint32_t li = (order >> (4u * k)) & 15u;
    if (!((hit_mask >> li) & 1u)) continue;
    const float t0 = s_t0[li * stride + slot], t1 = s_t1[li * stride + slot];
    const LayerConst& L = u.layers[li];
    const float segment = t1 - t0;
    if (segment <= 0.0f) continue;
    const float step = __fdividef(segment, (float)u.cloud_steps);
    const bool cb = L.cloud_type == 7u && u.phase_mode == PSC_PHASE_APPROX_MIE;

    // per ray and layer: a^n * phase_n * forward gain
    float coef[kMaxOct];
    if (u.phase_mode == PSC_PHASE_DUAL_LOBE_HG) {
#pragma unroll
      for (int n = 0; n < kMaxOct; ++n) coef[n] = hg_coef[n];
    } else if (!cb) {
      const PhaseConst pc{L.g_hg, L.g_d, L.alpha, L.w_d, L.ice};
#pragma unroll
      for (int n = 0; n < kMaxOct; ++n)
        coef[n] = (n < (int)noct) ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], pc) : 0.0f;
    }

    for (uint32_t s = 0; s < u.cloud_steps; ++s) {
      const float t = fmaf((float)s + jitter, step, t0);
      const float px3 = fmaf(dx, t, cx), py3 = fmaf(dy, t, cy), pz3 = fmaf(dz, t, cz);
      const float alt = alt_from(u, px3, py3, pz3, ray_r0, ray_cv, ray_h0, t);
      const float h = (alt - L.base_m) * L.inv_thickness;
      if (h >= 0.0f && h <= 1.0f) {
        const float wsx = px3 - L.wind_off_x, wsz = pz3 - L.wind_off_z;
        const float wr = weather_fast(u, fmaf(wsx, u.inv_weather_scale, 0.5f),
                                      fmaf(wsz, u.inv_weather_scale, 0.5f));
        const float eff = clamp01(wr * L.coverage);
        if (eff >= 0.01f) {
          const uint32_t type = effective_type(u, wsx, wsz, L.cloud_type);
          const float sk = h * L.skew_thickness;
          const float ax = fmaf(-L.skew_x, sk, wsx);
          const float az = fmaf(-L.skew_z, sk, wsz);
          float cloud = base_shape<ST, FILT, false>(u, L, ax, py3, az, h, eff, type);
          if (cloud > 0.0f) {  // curl-perturbed detail erosion (:502-527)
            const float2 c2 = curl_sample(u.curl, ax * u.inv_detail_scale, az * u.inv_detail_scale);
            const float ddx = fmaf(fmaf(c2.x, 2.0f, -1.0f), u.curl_offset_scale, ax);
            const float ddz = fmaf(fmaf(c2.y, 2.0f, -1.0f), u.curl_offset_scale, az);
            const float4 det = detail_tap<ST, FILT>(u, ddx, py3, ddz);
            const float hf = fmaf(det.z, 0.125f, fmaf(det.y, 0.25f, det.x * 0.625f));
            const float dmod = mixf(hf, 1.0f - hf, clamp01(h * 10.0f));
            const float lo = dmod * L.layer_detail;
            cloud = __fdividef(cloud - lo, fmaxf(1.0f - lo, 1e-5f));
          }
          const float density = clamp01(cloud) * L.density_scale;

          if (density > 1e-3f) {
            const float yy = py3 + u.planet_r;
            const float inv_r = __frcp_rn(u.planet_r + alt);
            const float ux = px3 * inv_r, uy = yy * inv_r, uz = pz3 * inv_r;
            const float od = light_od<ST, FILT>(u, L, px3, py3, pz3, alt, eff, type, ux, uy, uz);
            const float st_r = L.sigma_t[0], st_g = L.sigma_t[1], st_b = L.sigma_t[2];
            const float xr = st_r * od, xg = st_g * od, xb = st_b * od;
            // e[n] = exp(-x * b^n); with b = 1/2 one exponential at the last live
            // octave m and repeated squaring give every lower octave.
            float er[kMaxOct], eg[kMaxOct], eb[kMaxOct];
            const int m = (int)noct - 1;
            if (u.b_half) {
              const float bl = u.bpow[m];
              float vr = __expf(-xr * bl), vg = __expf(-xg * bl), vb = __expf(-xb * bl);
#pragma unroll
              for (int n = kMaxOct - 1; n >= 0; --n) {
                const bool live = n <= m;
                er[n] = live ? vr : 0.0f;
                eg[n] = live ? vg : 0.0f;
                eb[n] = live ? vb : 0.0f;
                if (live) {
                  vr *= vr;
                  vg *= vg;
                  vb *= vb;
                }
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
            const float br = er[0], bg = eg[0], bb = eb[0];  // Beer, n = 0
            const float pr = 1.0f - br * br, pg = 1.0f - bg * bg, pb = 1.0f - bb * bb;
            const float enr = mixf(br, br * pr * 2.0f, u.powder);
            const float eng = mixf(bg, bg * pg * 2.0f, u.powder);
            const float enb = mixf(bb, bb * pb * 2.0f, u.powder);
            float cf[kMaxOct];
            if (cb) {
              const float mt = smoothstepf(0.60f, 0.85f, h);
              const PhaseConst pc = phase_consts_from_d(mixf(L.droplet_um, 50.0f, mt), u.droplet_bias);
#pragma unroll
              for (int n = 0; n < kMaxOct; ++n)
                cf[n] = (n < (int)noct) ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], pc) : 0.0f;
            } else {
#pragma unroll
              for (int n = 0; n < kMaxOct; ++n) cf[n] = coef[n];
            }
            float sr = 0.0f, sg = 0.0f, sb = 0.0f;
#pragma unroll
            for (int n = 0; n < kMaxOct; ++n) {
              sr = fmaf(cf[n], er[n], sr);
              sg = fmaf(cf[n], eg[n], sg);
              sb = fmaf(cf[n], eb[n], sb);
            }
            const float3 ts = sun_trans_fast(u, alt, ux, uy, uz);
            sr *= u.sun_illum[0] * ts.x;
            sg *= u.sun_illum[1] * ts.y;
            sb *= u.sun_illum[2] * ts.z;
            const float3 sky = sky_fast(u, alt, ux, uy, uz);
            const float ag = mixf(0.3f, 1.0f, clamp01(h)) * u.ambient;
            float lr = 0.0f, lg = 0.0f, lb = 0.0f;
            if (u.lightning_radius > 0.0f) {
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
            Lr += slr;
            Lg += slg;
            Lb += slb;
            tw = fmaf(sw, t, tw);
            twn += sw;
            if (u.kahan) {
              const float ar = yr - kr, ag2 = yg - kg, ab = yb - kb;
              const float nr = odr + ar, ng = odg + ag2, nb = odb + ab;
              kr = (nr - odr) - ar;
              kg = (ng - odg) - ag2;
              kb = (nb - odb) - ab;
              odr = nr;
              odg = ng;
              odb = nb;
              Tr = __expf(-odr);
              Tg = __expf(-odg);
              Tb = __expf(-odb);
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
  float Or = Lr, Og = Lg, Ob = Lb;
  if (opacity > 1e-4f) {
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

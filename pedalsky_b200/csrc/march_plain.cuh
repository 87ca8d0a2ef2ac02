// Device functions of the PLAIN march (march.cu) shared with its tangent
// form (march_param_grad.cu): the density kernel, the altitude along a ray,
// the light march, and the sun transmittance / sky-view ambient lookups.
// FP32 as the reference (cloud_march.wgsl, cloud_density_common.wgsl).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "march_common.cuh"
#include "psc_internal.h"

namespace psc {
namespace {

// Density (cloud_march.wgsl:432-530; light variant cloud_density_common.wgsl:266-305).
template <int ST, int FILT, bool LIGHT>
__device__ __forceinline__ float density_at(const MarchUniforms& u, const LayerConst& L, float px,
                                            float py, float pz, float alt, float wr,
                                            uint32_t type, int* chk) {
  const float h = (alt - L.base_m) / fmaxf(L.top_m - L.base_m, 1.0f);
  if (h < 0.0f || h > 1.0f) return 0.0f;
  const float eff = clamp01(wr * L.coverage);
  if (eff < 0.01f) return 0.0f;
  const float sk = h * L.skew_thickness;
  const float ax = (px - L.wind_off_x) - L.skew_x * sk;
  const float ay = py;
  const float az = (pz - L.wind_off_z) - L.skew_z * sk;
  const float4 b = Noise<ST, FILT>::base(u, ax / u.base_scale, ay / u.base_scale, az / u.base_scale, chk);
  const float lf = clamp01(((b.y * 0.625f + b.z * 0.25f) + b.w * 0.125f) + L.lf_bias);
  const float base_cloud = remapf(b.x, -(1.0f - lf), 1.0f, 0.0f, 1.0f);
  float cloud = base_cloud * ndf(h, type, L.anvil_bias);
  cloud = remapf(cloud, 1.0f - eff, 1.0f, 0.0f, 1.0f) * eff;
  if (!LIGHT && cloud > 0.0f) {
    const float2 c2 = Noise<ST, FILT>::curl(u, ax / u.detail_scale, az / u.detail_scale, chk);
    const float cx = c2.x * 2.0f - 1.0f, cz = c2.y * 2.0f - 1.0f;
    const float dx = ax + (cx * u.curl_strength) * u.detail_scale;
    const float dy = ay + (0.0f * u.curl_strength) * u.detail_scale;
    const float dz = az + (cz * u.curl_strength) * u.detail_scale;
    const float4 det = Noise<ST, FILT>::detail(u, dx / u.detail_scale, dy / u.detail_scale,
                                               dz / u.detail_scale, chk);
    const float hf = (det.x * 0.625f + det.y * 0.25f) + det.z * 0.125f;
    const float dmod = mixf(hf, 1.0f - hf, clamp01(h * 10.0f));
    cloud = remapf(cloud, dmod * L.layer_detail, 1.0f, 0.0f, 1.0f);
  }
  return clamp01(cloud) * L.density_scale;
}

__device__ __forceinline__ float altitude_from_entry(const MarchUniforms& u, float px, float py,
                                                     float pz, float r0, float cos_view, float h0,
                                                     float t) {
  const float yy = py + u.planet_r;
  const float len = sqrtf((px * px + yy * yy) + pz * pz);
  const float num = 2.0f * t * r0 * cos_view + t * t;
  return h0 + num / (fmaxf(r0, 1.0f) + len);
}

template <int ST, int FILT>
__device__ float march_to_light(const MarchUniforms& u, const LayerConst& L, float px, float py,
                                float pz, float alt, float wr, uint32_t type, int* chk) {
  const float sx = u.sun[0], sy = u.sun[1], sz = u.sun[2];
  const float r0 = u.planet_r + alt;
  const float inv = 1.0f / fmaxf(r0, 1.0f);
  const float cv = ((px * inv) * sx + ((py + u.planet_r) * inv) * sy) + (pz * inv) * sz;
  const float cos_sun = fmaxf(sy, 0.05f);
  const float dist = fmaxf((L.top_m - alt) / cos_sun, 1.0f);
  float od = 0.0f, comp = 0.0f;
  if (u.cone) {  // cloud_march.wgsl:599-666
    const float K[6][3] = {{0.38051305f, 0.92453449f, -0.02111345f},
                           {-0.50625799f, -0.03590792f, -0.86163418f},
                           {-0.32509218f, -0.94557439f, 0.01428793f},
                           {0.09026238f, -0.27376545f, 0.95755165f},
                           {0.28128598f, 0.42443639f, -0.86065785f},
                           {-0.16852403f, 0.14748697f, 0.97460106f}};
    const float step = dist / 5.0f;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const float t = ((float)i + 0.5f) * step;
      const float sc = step * ((float)i + 1.0f) / 5.0f;
      const float qx = fmaf(sx, t, px) + K[i][0] * sc;
      const float qy = fmaf(sy, t, py) + K[i][1] * sc;
      const float qz = fmaf(sz, t, pz) + K[i][2] * sc;
      const float a = altitude_from_entry(u, qx, qy, qz, r0, cv, alt, t);
      od += density_at<ST, FILT, true>(u, L, qx, qy, qz, a, wr, type, chk) * step;
    }
    const float tf = dist * 3.0f;
    const float qx = fmaf(sx, tf, px) + K[5][0] * (step * 3.0f);
    const float qy = fmaf(sy, tf, py) + K[5][1] * (step * 3.0f);
    const float qz = fmaf(sz, tf, pz) + K[5][2] * (step * 3.0f);
    const float a = altitude_from_entry(u, qx, qy, qz, r0, cv, alt, tf);
    od += density_at<ST, FILT, true>(u, L, qx, qy, qz, a, wr, type, chk) * step * 3.0f;
    return od;
  }
  const float step = dist / (float)u.light_steps;
  for (uint32_t i = 0; i < u.light_steps; ++i) {
    const float t = ((float)i + 0.5f) * step;
    const float qx = fmaf(sx, t, px), qy = fmaf(sy, t, py), qz = fmaf(sz, t, pz);
    const float a = altitude_from_entry(u, qx, qy, qz, r0, cv, alt, t);
    const float term = density_at<ST, FILT, true>(u, L, qx, qy, qz, a, wr, type, chk) * step;
    if (u.kahan) {  // compensated sum
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

// cloud_march.wgsl:328-354
__device__ float3 sun_transmittance_at(const MarchUniforms& u, float px, float py, float pz, int* chk) {
  const float R = u.planet_r;
  const float ay = py + R;
  const float len = sqrtf((px * px + ay * ay) + pz * pz);
  const float r = fmaxf(len, R + 1.0f);
  const float mu = clampf(((px / r) * u.sun[0] + (ay / r) * u.sun[1]) + (pz / r) * u.sun[2], -1.0f, 1.0f);
  const float ratio = R / r;
  const float sin_h = -sqrtf(fmaxf(1.0f - ratio * ratio, 0.0f));
  if (mu <= sin_h) return make_float3(0.0f, 0.0f, 0.0f);
  const float ht = u.atmo_top;
  const float bh = sqrtf(fmaxf(ht * ht - R * R, 0.0f));
  const float rho = sqrtf(fmaxf(r * r - R * R, 0.0f));
  const float disc = r * r * (mu * mu - 1.0f) + ht * ht;
  const float d = fmaxf(-r * mu + sqrtf(fmaxf(disc, 0.0f)), 0.0f);
  const float d_min = ht - r, d_max = rho + bh;
  const float xm = clamp01((d - d_min) / fmaxf(d_max - d_min, 1.0f));
  const float xr = rho / fmaxf(bh, 1.0f);
  const float4 t = lut2d(u.lut_trans, 256, 64, xm, xr, chk, kChkTrans);
  return make_float3(t.x, t.y, t.z);
}

// cloud_march.wgsl:672-700.  The zenith angle uses atan2(|xz|, y), the
// well-conditioned form of acos(y) for directions near local up.
__device__ float3 sky_ambient(const MarchUniforms& u, float px, float py, float pz, float sun_az,
                              int* chk) {
  const float ay = py + u.planet_r;
  const float cam_r = sqrtf((px * px + ay * ay) + pz * pz);
  const float ux = px / cam_r, uy = ay / cam_r, uz = pz / cam_r;
  const float vza = atan2f(sqrtf(ux * ux + uz * uz), uy);
  const float sin_h = clamp01(u.planet_r / cam_r);
  const float zha = kPi - asinf(sin_h);
  float vv;
  if (vza < zha) {
    vv = sqrtf(clamp01(vza / fmaxf(zha, 1e-6f))) * 0.5f;
  } else {
    const float br = fmaxf(kPi - zha, 1e-6f);
    vv = 0.5f + sqrtf(clamp01((vza - zha) / br)) * 0.5f;
  }
  const float vaz = atan2f(ux, uz);
  float du = (vaz - sun_az) / (2.0f * kPi);
  du = du - floorf(du);
  const float4 s = lut2d(u.lut_sky, 192, 108, du, vv, chk, kChkSky);
  return make_float3(s.x * u.sun_illum[0], s.y * u.sun_illum[1], s.z * u.sun_illum[2]);
}

}  // namespace
}  // namespace psc

// Gradient of the procedural march's image loss with respect to one cloud
// layer's density parameters: coverage, shape_bias, detail_bias and
// density_scale.
//
// The four parameters enter the march only through sample_density
// (cloud_march.wgsl:432-530; march_plain.cuh:density_at): the coverage gate
// and remap (eff = clamp(weather.r * coverage, 0, 1)), the low-frequency
// erosion (lf = clamp(fbm + shape_bias * diurnal / 2, 0, 1)), the detail
// erosion (clamp(detail_strength + detail_bias * diurnal, 0, 1)) and the
// final scale.  Every quantity downstream of a density — the light march's
// optical depth, Beer-powder and the multi-scatter octaves, the in-scattered
// step integral, the transmittance, the luminance-weighted cloud distance and
// the aerial-perspective blend it selects — is carried here as a value with
// its four derivatives (forward mode), one thread per ray, in the PLAIN
// march's FP32 arithmetic and order with exact (FP32-weight) filtering of
// the context's noise storage.  The branch decisions (the 1e-3 density
// threshold, the 0.01 coverage gate, the early exit) are taken on the values
// and are constant under the derivative, as in the reference's own
// differentiable limit.  With the Kahan option the values are summed plainly
// (the derivative of a compensated sum is the plain sum of derivatives).
//
// The loss is the adjoint's: sum((I - target)^2) / (3 * viewport pixels),
// I = L + background * T per pixel and channel, over the view's rectangle;
// each ray adds its 2 (I - target) / N . dI to the four results.
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
constexpr int kP = 4;  // coverage, shape_bias, detail_bias, density_scale

struct D4 {
  float v;
  float d[kP];
};
__device__ __forceinline__ D4 dc(float v) { return {v, {0.0f, 0.0f, 0.0f, 0.0f}}; }
__device__ __forceinline__ D4 operator+(const D4& x, const D4& y) {
  D4 r{x.v + y.v};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] + y.d[i];
  return r;
}
__device__ __forceinline__ D4 operator-(const D4& x, const D4& y) {
  D4 r{x.v - y.v};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] - y.d[i];
  return r;
}
__device__ __forceinline__ D4 operator-(float s, const D4& x) {
  D4 r{s - x.v};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = -x.d[i];
  return r;
}
__device__ __forceinline__ D4 operator-(const D4& x) {
  D4 r{-x.v};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = -x.d[i];
  return r;
}
__device__ __forceinline__ D4 operator*(const D4& x, float s) {
  D4 r{x.v * s};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] * s;
  return r;
}
__device__ __forceinline__ D4 operator*(float s, const D4& x) {
  D4 r{s * x.v};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = x.d[i] * s;
  return r;
}
__device__ __forceinline__ D4 operator*(const D4& x, const D4& y) {
  D4 r{x.v * y.v};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = fmaf(x.d[i], y.v, x.v * y.d[i]);
  return r;
}
__device__ __forceinline__ D4 operator/(const D4& x, const D4& y) {
  const float q = x.v / y.v, iy = 1.0f / y.v;
  D4 r{q};
#pragma unroll
  for (int i = 0; i < kP; ++i) r.d[i] = (x.d[i] - q * y.d[i]) * iy;
  return r;
}
__device__ __forceinline__ D4 dexp(const D4& x) {
  const float e = expf(x.v);
  return {e, {x.d[0] * e, x.d[1] * e, x.d[2] * e, x.d[3] * e}};
}
__device__ __forceinline__ D4 dlog(const D4& x) {
  const float k = 1.0f / x.v;
  return {logf(x.v), {x.d[0] * k, x.d[1] * k, x.d[2] * k, x.d[3] * k}};
}
__device__ __forceinline__ D4 dmax(const D4& x, float m) { return x.v > m ? x : dc(fmaxf(x.v, m)); }
__device__ __forceinline__ D4 dclamp01(const D4& x) { return (x.v > 0.0f && x.v < 1.0f) ? x : dc(clamp01(x.v)); }
// mixf(a, b, t) = a (1 - t) + b t for a constant t
__device__ __forceinline__ D4 dmix(const D4& a, const D4& b, float t) { return a * (1.0f - t) + b * t; }
// remapf(v, a, 1, 0, 1) = 0 + ((v - a) * 1) / max(1 - a, 1e-5)
__device__ __forceinline__ D4 dremap01(const D4& v, const D4& a) {
  return (v - a) * 1.0f / dmax(1.0f - a, 1e-5f);
}

// Density of a sample (density_at) with its derivatives with respect to the
// differentiated layer's four parameters; `carried` is false for the other
// layers, whose densities are constants.
template <int ST, bool LIGHT>
__device__ __forceinline__ D4 density_d(const MarchUniforms& u, const LayerConst& L, const ParamGradDev& g,
                                        bool carried, float px, float py, float pz, float alt, float wr,
                                        uint32_t type) {
  if (!carried) return dc(density_at<ST, PSC_FILTER_EXACT, LIGHT>(u, L, px, py, pz, alt, wr, type, nullptr));
  const float h = (alt - L.base_m) / fmaxf(L.top_m - L.base_m, 1.0f);
  if (h < 0.0f || h > 1.0f) return dc(0.0f);
  const float eff_raw = wr * L.coverage;
  D4 eff = dc(clamp01(eff_raw));
  if (eff_raw > 0.0f && eff_raw < 1.0f) eff.d[0] = wr;
  if (eff.v < 0.01f) return dc(0.0f);
  const float sk = h * L.skew_thickness;
  const float ax = (px - L.wind_off_x) - L.skew_x * sk;
  const float ay = py;
  const float az = (pz - L.wind_off_z) - L.skew_z * sk;
  const float4 b = Noise<ST, PSC_FILTER_EXACT>::base(u, ax / u.base_scale, ay / u.base_scale, az / u.base_scale);
  const float lf_raw = ((b.y * 0.625f + b.z * 0.25f) + b.w * 0.125f) + L.lf_bias;
  D4 lf = dc(clamp01(lf_raw));
  if (lf_raw > 0.0f && lf_raw < 1.0f) lf.d[1] = g.dlf_dshape;
  const D4 base_cloud = dremap01(dc(b.x), -(1.0f - lf));
  D4 cloud = base_cloud * ndf(h, type, L.anvil_bias);
  cloud = dremap01(cloud, 1.0f - eff) * eff;
  if (!LIGHT && cloud.v > 0.0f) {
    const float2 c2 = Noise<ST, PSC_FILTER_EXACT>::curl(u, ax / u.detail_scale, az / u.detail_scale);
    const float cx = c2.x * 2.0f - 1.0f, cz = c2.y * 2.0f - 1.0f;
    const float dx = ax + (cx * u.curl_strength) * u.detail_scale;
    const float dy = ay + (0.0f * u.curl_strength) * u.detail_scale;
    const float dz = az + (cz * u.curl_strength) * u.detail_scale;
    const float4 det = Noise<ST, PSC_FILTER_EXACT>::detail(u, dx / u.detail_scale, dy / u.detail_scale,
                                                           dz / u.detail_scale);
    const float hf = (det.x * 0.625f + det.y * 0.25f) + det.z * 0.125f;
    const float dmod = mixf(hf, 1.0f - hf, clamp01(h * 10.0f));
    D4 ld = dc(L.layer_detail);
    ld.d[2] = g.dld_ddetail;
    cloud = dremap01(cloud, dmod * ld);
  }
  const D4 c = dclamp01(cloud);
  D4 r = c * L.density_scale;
  r.d[3] += c.v;
  return r;
}

// march_to_light (march_plain.cuh) with the densities carried.
template <int ST>
__device__ D4 light_od_d(const MarchUniforms& u, const LayerConst& L, const ParamGradDev& g, bool carried,
                         float px, float py, float pz, float alt, float wr, uint32_t type) {
  const float sx = u.sun[0], sy = u.sun[1], sz = u.sun[2];
  const float r0 = u.planet_r + alt;
  const float inv = 1.0f / fmaxf(r0, 1.0f);
  const float cv = ((px * inv) * sx + ((py + u.planet_r) * inv) * sy) + (pz * inv) * sz;
  const float cos_sun = fmaxf(sy, 0.05f);
  const float dist = fmaxf((L.top_m - alt) / cos_sun, 1.0f);
  D4 od = dc(0.0f);
  if (u.cone) {  // cloud_march.wgsl:599-666
    const float K[6][3] = {{0.38051305f, 0.92453449f, -0.02111345f},
                           {-0.50625799f, -0.03590792f, -0.86163418f},
                           {-0.32509218f, -0.94557439f, 0.01428793f},
                           {0.09026238f, -0.27376545f, 0.95755165f},
                           {0.28128598f, 0.42443639f, -0.86065785f},
                           {-0.16852403f, 0.14748697f, 0.97460106f}};
    const float step = dist / 5.0f;
    for (int i = 0; i < 5; ++i) {
      const float t = ((float)i + 0.5f) * step;
      const float sc = step * ((float)i + 1.0f) / 5.0f;
      const float qx = fmaf(sx, t, px) + K[i][0] * sc;
      const float qy = fmaf(sy, t, py) + K[i][1] * sc;
      const float qz = fmaf(sz, t, pz) + K[i][2] * sc;
      const float a = altitude_from_entry(u, qx, qy, qz, r0, cv, alt, t);
      od = od + density_d<ST, true>(u, L, g, carried, qx, qy, qz, a, wr, type) * step;
    }
    const float tf = dist * 3.0f;
    const float qx = fmaf(sx, tf, px) + K[5][0] * (step * 3.0f);
    const float qy = fmaf(sy, tf, py) + K[5][1] * (step * 3.0f);
    const float qz = fmaf(sz, tf, pz) + K[5][2] * (step * 3.0f);
    const float a = altitude_from_entry(u, qx, qy, qz, r0, cv, alt, tf);
    return od + density_d<ST, true>(u, L, g, carried, qx, qy, qz, a, wr, type) * step * 3.0f;
  }
  const float step = dist / (float)u.light_steps;
  for (uint32_t i = 0; i < u.light_steps; ++i) {
    const float t = ((float)i + 0.5f) * step;
    const float qx = fmaf(sx, t, px), qy = fmaf(sy, t, py), qz = fmaf(sz, t, pz);
    const float a = altitude_from_entry(u, qx, qy, qz, r0, cv, alt, t);
    od = od + density_d<ST, true>(u, L, g, carried, qx, qy, qz, a, wr, type) * step;
  }
  return od;
}

// Aerial-perspective LUT (lut_ap) and its derivative along the distance
// coordinate w (trilinear: d/dw = 64 (upper - lower z plane)).
__device__ __forceinline__ void lut_ap_dw(const float4* lut, float u, float v, float w, float4& val,
                                          float4& dw) {
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

__device__ __forceinline__ D4 along(float value, float slope, const D4& w) {
  return {value, {slope * w.d[0], slope * w.d[1], slope * w.d[2], slope * w.d[3]}};
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

  D4 Lc[3] = {dc(0.0f), dc(0.0f), dc(0.0f)}, T[3] = {dc(1.0f), dc(1.0f), dc(1.0f)};
  D4 tw = dc(0.0f), twn = dc(0.0f);
  const float lum[3] = {0.2126f, 0.7152f, 0.0722f};
  for (uint32_t k = 0; k < u.layer_count; ++k) {
    if (fmaxf(T[0].v, fmaxf(T[1].v, T[2].v)) < 0.01f) break;
    const uint32_t li = (rs.order >> (4u * k)) & 15u;
    if (!((rs.hit_mask >> li) & 1u) || li >= 8u) continue;
    float t0 = 0.0f, t1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if ((uint32_t)j == li) {
        t0 = rs.t0[j];
        t1 = rs.t1[j];
      }
    const LayerConst& L = u.layers[li];
    const bool carried = li == g.layer;
    const float segment = t1 - t0;
    if (segment <= 0.0f) continue;
    const float step = segment / (float)u.cloud_steps;
    const float st[3] = {L.sigma_t[0], L.sigma_t[1], L.sigma_t[2]};
    for (uint32_t s = 0; s < u.cloud_steps; ++s) {
      const float t = fmaf((float)s + jitter, step, t0);
      const float px3 = fmaf(dx, t, cx), py3 = fmaf(dy, t, cy), pz3 = fmaf(dz, t, cz);
      const float alt = altitude_from_entry(u, px3, py3, pz3, rs.r0, rs.cos_view, rs.h0, t);
      const float wsx = px3 - L.wind_off_x, wsz = pz3 - L.wind_off_z;
      const float wr =
          Noise<ST, PSC_FILTER_EXACT>::weather(u, wsx / u.weather_scale + 0.5f, wsz / u.weather_scale + 0.5f);
      const uint32_t type = effective_type(u, wsx, wsz, L.cloud_type);
      const D4 density = density_d<ST, false>(u, L, g, carried, px3, py3, pz3, alt, wr, type);
      if (density.v > 1e-3f) {
        const D4 od = light_od_d<ST>(u, L, g, carried, px3, py3, pz3, alt, wr, type);
        const float hn = clamp01((alt - L.base_m) / fmaxf(L.top_m - L.base_m, 1.0f));
        PhaseConst pc;
        if (L.cloud_type == 7u) {
          const float mt = smoothstepf(0.60f, 0.85f, hn);
          pc = phase_consts_from_d(mixf(L.droplet_um, 50.0f, mt), u.droplet_bias);
        } else {
          pc = PhaseConst{L.g_hg, L.g_d, L.alpha, L.w_d, L.ice};
        }
        const float3 stv = sun_transmittance_at(u, px3, py3, pz3, nullptr);
        const float3 sky = sky_ambient(u, px3, py3, pz3, sun_az, nullptr);
        const float ag = mixf(0.3f, 1.0f, hn) * u.ambient;
        float lgt[3] = {0.0f, 0.0f, 0.0f};
        if (u.lightning_radius > 0.0f) {
          const float ddx = px3 - u.lightning_origin_x, ddz = pz3 - u.lightning_origin_z;
          const float fo = clamp01(1.0f - sqrtf(ddx * ddx + ddz * ddz) / u.lightning_radius);
          const float wgt = fo * fo * (3.0f - 2.0f * fo);
          lgt[0] = u.lightning_rgb[0] * wgt;
          lgt[1] = u.lightning_rgb[1] * wgt;
          lgt[2] = u.lightning_rgb[2] * wgt;
        }
        const float tsun[3] = {stv.x, stv.y, stv.z}, skyc[3] = {sky.x, sky.y, sky.z};
        const float f = u.forward_bias > 0.0f ? 1.0f + u.forward_bias * fwd : 1.0f;
        D4 sl[3], sm[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const D4 bb = dexp(od * -st[c]);
          const D4 pw = 1.0f - dexp(od * (-2.0f * st[c]));
          const D4 e = dmix(bb, bb * pw * 2.0f, u.powder);
          D4 S = dc(0.0f);
          float a = 1.0f, b = 1.0f, cc = 1.0f;
          for (uint32_t o = 0; o < u.octaves; ++o) {
            const float ph = phase_with(u, cos_theta, cc, pc);
            S = S + dexp((od * -st[c]) * b) * (((a * u.sun_illum[c]) * tsun[c]) * ph);
            a *= u.ms_a;
            b *= u.ms_b;
            cc *= u.ms_c;
          }
          if (u.forward_bias > 0.0f) S = S * f;
          const D4 is = (density * u.sigma_s[c]) * ((S * e + dc(skyc[c] * ag)) + dc(lgt[c]));
          const D4 ls = dmax(density * st[c], 1e-6f);
          sm[c] = dexp(ls * -step);
          sl[c] = T[c] * ((is - is * sm[c]) / ls);
        }
        const D4 sw = (sl[0] * lum[0] + sl[1] * lum[1]) + sl[2] * lum[2];
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
  const D4 t_lum = (T[0] * lum[0] + T[1] * lum[1]) + T[2] * lum[2];
  const D4 opacity = 1.0f - t_lum;
  D4 O[3] = {Lc[0], Lc[1], Lc[2]};
  if (opacity.v > 1e-4f) {
    const D4 t_cloud = tw / dmax(twn, 1e-6f);
    const D4 ds = dmax(t_cloud, 50.0f);
    const D4 azd = dclamp01(dlog(ds * (1.0f / 50.0f)) * (1.0f / logf(100000.0f / 50.0f)));
    float4 ap, dap;
    lut_ap_dw(u.lut_ap, ((float)(px + v.x_off) + 0.5f) / u.vp_w, ((float)(py + v.y_off) + 0.5f) / u.vp_h, azd.v,
              ap, dap);
    const D4 apw = along(ap.w, dap.w, azd);
    const D4 apc[3] = {along(ap.x, dap.x, azd), along(ap.y, dap.y, azd), along(ap.z, dap.z, azd)};
#pragma unroll
    for (int c = 0; c < 3; ++c) O[c] = Lc[c] * apw + apc[c] * opacity;
  }
  const size_t idx = (size_t)py * v.width + px;
  const float4 bgp = __ldg(g.bg + idx), tg = __ldg(g.target + idx);
  const float bgc[3] = {bgp.x, bgp.y, bgp.z}, tgc[3] = {tg.x, tg.y, tg.z};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const D4 I = O[c] + T[c] * bgc[c];
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

// out[0..3] += d loss / d (coverage, shape_bias, detail_bias, density_scale);
// loss (nullable) += the loss.
template <int ST>
__global__ void __launch_bounds__(kThreads) k_march_param_grad(const __grid_constant__ MarchUniforms u,
                                                               const __grid_constant__ ViewDev v,
                                                               const __grid_constant__ ParamGradDev g, double* out,
                                                               double* loss) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * kTileW + (warp & 1u) * 8u + (lane & 7u);
  const uint32_t py = blockIdx.y * kTileH + (warp >> 1) * 4u + (lane >> 3);
  float acc[kP + 1] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
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

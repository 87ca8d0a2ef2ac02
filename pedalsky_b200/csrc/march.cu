// The cloud march kernels: one thread per primary ray (pixel), warps mapped
// to 8x4 pixel tiles so neighbouring rays share texel cache lines.
//
// Restates `fs_main` (shaders/clouds/cloud_march.wgsl:731-1054) with the
// density kernel of shaders/clouds/cloud_density_common.wgsl.  Arithmetic is
// FP32 as in the reference except for the per-ray set-up (view ray, planet-
// radius shell intersection, entry radius), which runs in FP64 because
// |oc|^2 - r^2 at r ~ 6.36e6 m cancels catastrophically in FP32, and the
// march position t = t0 + (s + jitter) * step, which is formed directly
// instead of by repeated addition.
//
// Schedules:
//   PSC_SCHED_PLAIN — the restatement, per dense sample, as the reference
//                     orders it;
//   PSC_SCHED_FAST  — same mathematics with per-ray/per-layer invariants
//                     hoisted (phase lobes per octave, exp merging for
//                     b = 0.5), fast SFU transcendentals and the dense
//                     shading reconverged across lanes.
#include <cuda_runtime.h>
#include <stdint.h>

#include "march_common.cuh"
#include "march_ray.cuh"
#include "psc_internal.h"

namespace psc {

namespace {

constexpr int kTileW = 16;  // pixels per CTA tile (x)
constexpr int kTileH = 8;   // pixels per CTA tile (y)
constexpr int kThreads = 128;

__device__ __forceinline__ void pixel_of(uint32_t& px, uint32_t& py) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  px = blockIdx.x * kTileW + (warp & 1u) * 8u + (lane & 7u);
  py = blockIdx.y * kTileH + (warp >> 1) * 4u + (lane >> 3);
}

__device__ __forceinline__ float max3f(float a, float b, float c) { return fmaxf(a, fmaxf(b, c)); }

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

// CK: options.debug_checks — every index is compared with its buffer's
// extent (march_common.cuh:idx_ok); without it the checks compile away.
template <int ST, int FILT, bool CK>
__global__ void __launch_bounds__(kThreads) k_march_plain(const __grid_constant__ MarchUniforms u,
                                                          const __grid_constant__ ViewDev v) {
  uint32_t px, py;
  pixel_of(px, py);
  if (px >= v.width || py >= v.height) return;
  int* const chk = CK ? u.error_word : nullptr;

  RaySetup rs;
  setup_ray(u, v, px, py, rs);
  const float dx = rs.dir[0], dy = rs.dir[1], dz = rs.dir[2];
  const float cx = u.cam[0], cy = u.cam[1], cz = u.cam[2];
  const float cos_theta = (dx * u.sun[0] + dy * u.sun[1]) + dz * u.sun[2];
  const float fwd = smoothstepf(0.0f, 1.0f, fmaxf(cos_theta, 0.0f));
  const float sun_az = atan2f(u.sun[0], u.sun[2]);

  // blue-noise jitter (cloud_march.wgsl:745-756)
  uint32_t sx = (px + v.x_off) & 63u, sy = (py + v.y_off) & 63u;
  if (u.temporal_jitter) {
    const uint32_t ph = u.frame_index & 15u;
    sx = (sx ^ ((ph * 11u + 7u) & 63u)) & 63u;
    sy = (sy ^ ((ph * 23u + 13u) & 63u)) & 63u;
  }
  const float jitter = idx_ok(chk, sy < 64u && sx < 64u, kChkBlue) ? __ldg(u.blue + sy * 64u + sx) : 0.0f;

  float Lr = 0.0f, Lg = 0.0f, Lb = 0.0f;
  float Tr = 1.0f, Tg = 1.0f, Tb = 1.0f;
  float odr = 0.0f, odg = 0.0f, odb = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;  // Kahan form
  float tw = 0.0f, twn = 0.0f;
  const uint32_t n = u.layer_count;

  for (uint32_t k = 0; k < n; ++k) {
    if (max3f(Tr, Tg, Tb) < 0.01f) break;
    const uint32_t li = (rs.order >> (4u * k)) & 15u;
    if (!((rs.hit_mask >> li) & 1u)) continue;
    if (!idx_ok(chk, li < 8u && li < u.layer_count, kChkLayer)) continue;
    float t0 = 0.0f, t1 = 0.0f;
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if ((uint32_t)j == li) {
        t0 = rs.t0[j];
        t1 = rs.t1[j];
      }
    const LayerConst& L = u.layers[li];
    const float segment = t1 - t0;
    if (segment <= 0.0f) continue;
    const float step = segment / (float)u.cloud_steps;
    const float st_r = L.sigma_t[0], st_g = L.sigma_t[1], st_b = L.sigma_t[2];

    for (uint32_t s = 0; s < u.cloud_steps; ++s) {
      const float t = fmaf((float)s + jitter, step, t0);
      const float px3 = fmaf(dx, t, cx), py3 = fmaf(dy, t, cy), pz3 = fmaf(dz, t, cz);
      const float alt = altitude_from_entry(u, px3, py3, pz3, rs.r0, rs.cos_view, rs.h0, t);
      const float wsx = px3 - L.wind_off_x, wsz = pz3 - L.wind_off_z;
      const float wr = Noise<ST, FILT>::weather(u, wsx / u.weather_scale + 0.5f,
                                                wsz / u.weather_scale + 0.5f, chk);
      const uint32_t type = effective_type(u, wsx, wsz, L.cloud_type, chk);
      const float density = density_at<ST, FILT, false>(u, L, px3, py3, pz3, alt, wr, type, chk);

      if (density > 1e-3f) {
        const float od = march_to_light<ST, FILT>(u, L, px3, py3, pz3, alt, wr, type, chk);
        const float br = expf(-st_r * od), bg = expf(-st_g * od), bb = expf(-st_b * od);
        const float pr = 1.0f - expf(-2.0f * st_r * od), pg = 1.0f - expf(-2.0f * st_g * od),
                    pb = 1.0f - expf(-2.0f * st_b * od);
        const float er = mixf(br, br * pr * 2.0f, u.powder);
        const float eg = mixf(bg, bg * pg * 2.0f, u.powder);
        const float eb = mixf(bb, bb * pb * 2.0f, u.powder);
        const float hn = clamp01((alt - L.base_m) / fmaxf(L.top_m - L.base_m, 1.0f));
        PhaseConst pc;
        if (L.cloud_type == 7u) {
          const float mt = smoothstepf(0.60f, 0.85f, hn);
          pc = phase_consts_from_d(mixf(L.droplet_um, 50.0f, mt), u.droplet_bias);
        } else {
          pc = PhaseConst{L.g_hg, L.g_d, L.alpha, L.w_d, L.ice};
        }
        const float3 st = sun_transmittance_at(u, px3, py3, pz3, chk);
        float sr = 0.0f, sg = 0.0f, sb = 0.0f;
        float a = 1.0f, b = 1.0f, c = 1.0f;
        for (uint32_t o = 0; o < u.octaves; ++o) {
          const float ph = phase_with(u, cos_theta, c, pc);
          sr += (((a * u.sun_illum[0]) * st.x) * ph) * expf((-st_r * od) * b);
          sg += (((a * u.sun_illum[1]) * st.y) * ph) * expf((-st_g * od) * b);
          sb += (((a * u.sun_illum[2]) * st.z) * ph) * expf((-st_b * od) * b);
          a *= u.ms_a;
          b *= u.ms_b;
          c *= u.ms_c;
        }
        if (u.forward_bias > 0.0f) {
          const float f = 1.0f + u.forward_bias * fwd;
          sr *= f;
          sg *= f;
          sb *= f;
        }
        const float3 sky = sky_ambient(u, px3, py3, pz3, sun_az, chk);
        const float ag = mixf(0.3f, 1.0f, hn) * u.ambient;
        float lr = 0.0f, lg = 0.0f, lb = 0.0f;
        if (u.lightning_radius > 0.0f) {
          const float ddx = px3 - u.lightning_origin_x, ddz = pz3 - u.lightning_origin_z;
          const float fo = clamp01(1.0f - sqrtf(ddx * ddx + ddz * ddz) / u.lightning_radius);
          const float wgt = fo * fo * (3.0f - 2.0f * fo);
          lr = u.lightning_rgb[0] * wgt;
          lg = u.lightning_rgb[1] * wgt;
          lb = u.lightning_rgb[2] * wgt;
        }
        const float isr = (density * u.sigma_s[0]) * ((sr * er + sky.x * ag) + lr);
        const float isg = (density * u.sigma_s[1]) * ((sg * eg + sky.y * ag) + lg);
        const float isb = (density * u.sigma_s[2]) * ((sb * eb + sky.z * ag) + lb);
        const float lsr = fmaxf(density * st_r, 1e-6f), lsg = fmaxf(density * st_g, 1e-6f),
                    lsb = fmaxf(density * st_b, 1e-6f);
        const float smr = expf(-lsr * step), smg = expf(-lsg * step), smb = expf(-lsb * step);
        const float slr = Tr * ((isr - isr * smr) / lsr);
        const float slg = Tg * ((isg - isg * smg) / lsg);
        const float slb = Tb * ((isb - isb * smb) / lsb);
        const float sw = (slr * 0.2126f + slg * 0.7152f) + slb * 0.0722f;
        Lr += slr;
        Lg += slg;
        Lb += slb;
        tw += sw * t;
        twn += sw;
        if (u.kahan) {  // T = exp(-sum(sigma*dt)), compensated sum
          const float xr = lsr * step - cr, xg = lsg * step - cg, xb = lsb * step - cb;
          const float nr = odr + xr, ng = odg + xg, nb = odb + xb;
          cr = (nr - odr) - xr;
          cg = (ng - odg) - xg;
          cb = (nb - odb) - xb;
          odr = nr;
          odg = ng;
          odb = nb;
          Tr = expf(-odr);
          Tg = expf(-odg);
          Tb = expf(-odb);
        } else {
          Tr *= smr;
          Tg *= smg;
          Tb *= smb;
        }
      }
      if (max3f(Tr, Tg, Tb) < 0.01f) break;
    }
  }

  // aerial perspective (cloud_march.wgsl:1016-1048)
  const float t_lum = (Tr * 0.2126f + Tg * 0.7152f) + Tb * 0.0722f;
  const float opacity = 1.0f - t_lum;
  const float t_cloud = tw / fmaxf(twn, 1e-6f);
  float Or = Lr, Og = Lg, Ob = Lb;
  if (opacity > 1e-4f) {
    const float ds = fmaxf(t_cloud, 50.0f);
    const float az = clamp01(logf(ds / 50.0f) / logf(100000.0f / 50.0f));
    const float4 ap = lut_ap(u.lut_ap, ((float)(px + v.x_off) + 0.5f) / u.vp_w,
                             ((float)(py + v.y_off) + 0.5f) / u.vp_h, az, chk);
    Or = Lr * ap.w + ap.x * opacity;
    Og = Lg * ap.w + ap.y * opacity;
    Ob = Lb * ap.w + ap.z * opacity;
  }
  const size_t idx = (size_t)py * v.width + px;
  if (!idx_ok(chk, px < v.width && py < v.height, kChkPixel)) return;
  const float4 lo = make_float4(Or, Og, Ob, 1.0f);
  const float4 to = make_float4(Tr, Tg, Tb, 1.0f);
  if (v.out_l) v.out_l[idx] = lo;
  if (v.out_t) v.out_t[idx] = to;
  if (u.composite && v.hdr) {  // cloud_composite.wgsl + blend One/Src1
    const float4 d = v.hdr[idx];
    v.hdr[idx] = make_float4(lo.x + d.x * to.x, lo.y + d.y * to.y, lo.z + d.z * to.z,
                             lo.w + d.w * to.w);
  }
}

__global__ void k_composite(const float4* __restrict__ l, const float4* __restrict__ t,
                            float4* __restrict__ hdr, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 a = __ldg(l + i), b = __ldg(t + i), d = hdr[i];
  hdr[i] = make_float4(a.x + d.x * b.x, a.y + d.y * b.y, a.z + d.z * b.z, a.w + d.w * b.w);
}

template <int ST, int FILT>
cudaError_t launch_plain(const MarchUniforms& u, const ViewDev& v, cudaStream_t s) {
  const dim3 grid((v.width + kTileW - 1) / kTileW, (v.height + kTileH - 1) / kTileH);
  if (u.debug_checks && u.error_word)
    k_march_plain<ST, FILT, true><<<grid, kThreads, 0, s>>>(u, v);
  else
    k_march_plain<ST, FILT, false><<<grid, kThreads, 0, s>>>(u, v);
  return cudaGetLastError();
}

}  // namespace

int launch_march(const MarchUniforms& u, const ViewDev& v, const PscMarchOptions& o,
                 cudaStream_t s) {
  cudaError_t e = cudaErrorInvalidValue;
  // the hybrid filter belongs to the FAST schedule; the checked debug form
  // runs it with exact filtering
  if (o.filter == PSC_FILTER_HYBRID && !(o.debug_checks && u.error_word)) return PSC_ERR_UNSUPPORTED;
  if (o.filter == PSC_FILTER_TEXTURE) {
    if (o.storage != PSC_STORAGE_U8) return PSC_ERR_UNSUPPORTED;
    e = launch_plain<PSC_STORAGE_U8, PSC_FILTER_TEXTURE>(u, v, s);
  } else {
    switch (o.storage) {
      case PSC_STORAGE_U8: e = launch_plain<PSC_STORAGE_U8, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_F32: e = launch_plain<PSC_STORAGE_F32, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_F16: e = launch_plain<PSC_STORAGE_F16, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_BF16: e = launch_plain<PSC_STORAGE_BF16, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_FP8: e = launch_plain<PSC_STORAGE_FP8, PSC_FILTER_EXACT>(u, v, s); break;
      default: return PSC_ERR_INVALID_ARGUMENT;
    }
  }
  return e == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_composite(const float4* l, const float4* t, float4* hdr, uint32_t n, cudaStream_t s) {
  if (n == 0) return PSC_OK;
  k_composite<<<(n + 255) / 256, 256, 0, s>>>(l, t, hdr, n);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

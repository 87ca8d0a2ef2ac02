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
#include "march_plain.cuh"
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

/*
 * ORACLE — test infrastructure, not product code.
 *
 * The templated march state shared by the procedural restatement
 * (oracle_march.cpp) and the voxel-grid form with its adjoint
 * (oracle_grid.cpp): samplers, layer records and the `March<R>` helpers
 * that restate shaders/clouds/cloud_march.wgsl and
 * shaders/clouds/cloud_density_common.wgsl.
 */
#ifndef PSC_ORACLE_MARCH_CORE_H
#define PSC_ORACLE_MARCH_CORE_H

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "oracle.h"
#include "oracle_common.h"

namespace oracle_core {

using namespace oracle;

template <class R>
struct V3 {
  R x, y, z;
};
template <class R>
inline V3<R> mk(R x, R y, R z) {
  return V3<R>{x, y, z};
}
template <class R>
inline V3<R> operator+(V3<R> a, V3<R> b) {
  return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class R>
inline V3<R> operator-(V3<R> a, V3<R> b) {
  return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class R>
inline V3<R> operator*(V3<R> a, V3<R> b) {
  return {a.x * b.x, a.y * b.y, a.z * b.z};
}
template <class R>
inline V3<R> operator*(V3<R> a, R s) {
  return {a.x * s, a.y * s, a.z * s};
}
template <class R>
inline V3<R> operator*(R s, V3<R> a) {
  return {s * a.x, s * a.y, s * a.z};
}
template <class R>
inline V3<R> operator/(V3<R> a, V3<R> b) {
  return {a.x / b.x, a.y / b.y, a.z / b.z};
}
template <class R>
inline V3<R> operator/(V3<R> a, R s) {
  return {a.x / s, a.y / s, a.z / s};
}
template <class R>
inline R dot(V3<R> a, V3<R> b) {
  return (a.x * b.x + a.y * b.y) + a.z * b.z;
}
template <class R>
inline R length(V3<R> a) {
  return std::sqrt(dot(a, a));
}
template <class R>
inline V3<R> normalize(V3<R> a) {
  return a / length(a);
}
template <class R>
inline V3<R> vexp(V3<R> a) {
  return {std::exp(a.x), std::exp(a.y), std::exp(a.z)};
}
template <class R>
inline V3<R> vmax(V3<R> a, R m) {
  return {std::fmax(a.x, m), std::fmax(a.y, m), std::fmax(a.z, m)};
}
template <class R>
inline R max3(V3<R> v) {  // math.wgsl:11
  return std::fmax(v.x, std::fmax(v.y, v.z));
}
template <class R>
inline R smoothstep(R e0, R e1, R x) {  // WGSL built-in; e0 > e1 gives a reversed ramp
  const R t = clampv<R>((x - e0) / (e1 - e0), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
template <class R>
inline R mix(R a, R b, R t) {  // WGSL built-in
  return a * (R(1) - t) + b * t;
}
template <class R>
inline R remap(R v, R a, R b, R c, R d) {  // math.wgsl:7-9
  return c + ((v - a) * (d - c)) / std::fmax(b - a, R(1e-5));
}

template <class R>
inline V3<R> load3(const float* p) {
  return {R(p[0]), R(p[1]), R(p[2])};
}

/* ----------------------------------------------------------- samplers */
template <class R>
struct Samplers {
  const OracleScene* s;
  int q8;

  // 3D RGBA8, repeat, trilinear (noise_sampler).
  void rgba8_3d(const uint8_t* d, int n, V3<R> uvw, R out[4]) const {
    const Axis<R> ax = axis_repeat<R>(uvw.x, n, q8);
    const Axis<R> ay = axis_repeat<R>(uvw.y, n, q8);
    const Axis<R> az = axis_repeat<R>(uvw.z, n, q8);
    auto t = [&](int x, int y, int z, int c) {
      return R(d[(((size_t)z * n + y) * n + x) * 4 + c]) / R(255);
    };
    for (int c = 0; c < 4; ++c) {
      const R x00 = lerp(t(ax.i0, ay.i0, az.i0, c), t(ax.i1, ay.i0, az.i0, c), ax.w);
      const R x10 = lerp(t(ax.i0, ay.i1, az.i0, c), t(ax.i1, ay.i1, az.i0, c), ax.w);
      const R x01 = lerp(t(ax.i0, ay.i0, az.i1, c), t(ax.i1, ay.i0, az.i1, c), ax.w);
      const R x11 = lerp(t(ax.i0, ay.i1, az.i1, c), t(ax.i1, ay.i1, az.i1, c), ax.w);
      out[c] = lerp(lerp(x00, x10, ay.w), lerp(x01, x11, ay.w), az.w);
    }
  }
  void curl(R u, R v, R out[2]) const {  // 128^2 RG8, repeat
    const Axis<R> ax = axis_repeat<R>(u, 128, q8);
    const Axis<R> ay = axis_repeat<R>(v, 128, q8);
    auto t = [&](int x, int y, int c) { return R(s->noise_curl[((size_t)y * 128 + x) * 2 + c]) / R(255); };
    for (int c = 0; c < 2; ++c)
      out[c] = lerp(lerp(t(ax.i0, ay.i0, c), t(ax.i1, ay.i0, c), ax.w),
                    lerp(t(ax.i0, ay.i1, c), t(ax.i1, ay.i1, c), ax.w), ay.w);
  }
  R weather_texel(int x, int y) const {
    const size_t i = (size_t)y * s->weather_w + x;
    switch (s->weather_format) {
      case PSC_WEATHER_RGBA16F:
        return R(f16_to_f32(((const uint16_t*)s->weather)[i * 4]));
      case PSC_WEATHER_RG8:
        return R(((const uint8_t*)s->weather)[i * 2]) / R(255);
      default:
        return R(((const float*)s->weather)[i]);
    }
  }
  R weather_r(R u, R v) const {  // repeat bilinear, R channel
    const Axis<R> ax = axis_repeat<R>(u, (int)s->weather_w, q8);
    const Axis<R> ay = axis_repeat<R>(v, (int)s->weather_h, q8);
    return lerp(lerp(weather_texel(ax.i0, ay.i0), weather_texel(ax.i1, ay.i0), ax.w),
                lerp(weather_texel(ax.i0, ay.i1), weather_texel(ax.i1, ay.i1), ax.w), ay.w);
  }
  // RGBA16F 2D, clamp, rgb (lut_sampler).
  V3<R> lut2d(const uint16_t* d, int w, int h, R u, R v) const {
    const Axis<R> ax = axis_clamp<R>(u, w, q8);
    const Axis<R> ay = axis_clamp<R>(v, h, q8);
    auto t = [&](int x, int y, int c) { return R(f16_to_f32(d[((size_t)y * w + x) * 4 + c])); };
    R o[3];
    for (int c = 0; c < 3; ++c)
      o[c] = lerp(lerp(t(ax.i0, ay.i0, c), t(ax.i1, ay.i0, c), ax.w),
                  lerp(t(ax.i0, ay.i1, c), t(ax.i1, ay.i1, c), ax.w), ay.w);
    return {o[0], o[1], o[2]};
  }
  void aerial(V3<R> uvw, R out[4]) const {  // 32x32x64 RGBA16F, clamp
    const uint16_t* d = s->lut_aerial;
    const Axis<R> ax = axis_clamp<R>(uvw.x, 32, q8);
    const Axis<R> ay = axis_clamp<R>(uvw.y, 32, q8);
    const Axis<R> az = axis_clamp<R>(uvw.z, 64, q8);
    auto t = [&](int x, int y, int z, int c) {
      return R(f16_to_f32(d[(((size_t)z * 32 + y) * 32 + x) * 4 + c]));
    };
    for (int c = 0; c < 4; ++c) {
      const R x00 = lerp(t(ax.i0, ay.i0, az.i0, c), t(ax.i1, ay.i0, az.i0, c), ax.w);
      const R x10 = lerp(t(ax.i0, ay.i1, az.i0, c), t(ax.i1, ay.i1, az.i0, c), ax.w);
      const R x01 = lerp(t(ax.i0, ay.i0, az.i1, c), t(ax.i1, ay.i0, az.i1, c), ax.w);
      const R x11 = lerp(t(ax.i0, ay.i1, az.i1, c), t(ax.i1, ay.i1, az.i1, c), ax.w);
      out[c] = lerp(lerp(x00, x10, ay.w), lerp(x01, x11, ay.w), az.w);
    }
  }
  // Wind field 32x16x32 RGBA16F, repeat (noise_sampler), xy channels.
  void wind(V3<R> uvw, R out[2]) const {
    const uint16_t* d = s->wind;
    const Axis<R> ax = axis_repeat<R>(uvw.x, 32, q8);
    const Axis<R> ay = axis_repeat<R>(uvw.y, 16, q8);
    const Axis<R> az = axis_repeat<R>(uvw.z, 32, q8);
    auto t = [&](int x, int y, int z, int c) {
      return R(f16_to_f32(d[(((size_t)z * 16 + y) * 32 + x) * 4 + c]));
    };
    for (int c = 0; c < 2; ++c) {
      const R x00 = lerp(t(ax.i0, ay.i0, az.i0, c), t(ax.i1, ay.i0, az.i0, c), ax.w);
      const R x10 = lerp(t(ax.i0, ay.i1, az.i0, c), t(ax.i1, ay.i1, az.i0, c), ax.w);
      const R x01 = lerp(t(ax.i0, ay.i0, az.i1, c), t(ax.i1, ay.i0, az.i1, c), ax.w);
      const R x11 = lerp(t(ax.i0, ay.i1, az.i1, c), t(ax.i1, ay.i1, az.i1, c), ax.w);
      out[c] = lerp(lerp(x00, x10, ay.w), lerp(x01, x11, ay.w), az.w);
    }
  }
};

/* --------------------------------------------------------- march state */
template <class R>
struct Layer {  // CloudLayerGpu in R
  R base, top, coverage, density_scale;
  uint32_t type;
  R shape_bias, detail_bias, anvil_bias, droplet;
};

template <class R>
struct WindCache {  // cloud_density_common.wgsl:137-149
  R off_x, off_z, skew_x, skew_z, skew_thickness;
};

enum { C_WEATHER = ORACLE_CNT_WEATHER };

template <class R>
struct March {
  const OracleScene* S;
  Samplers<R> tex;
  // uniforms in R
  R planet_r, atmo_top, sun_ang;
  V3<R> sun, cam, sun_illum, lightning_rgb, lightning_origin;
  R lightning_radius, sim_seconds;
  R vp_w, vp_h;
  R m_inv[4][4];
  V3<R> sigma_s, sigma_a;
  R droplet_bias, forward_bias, detail_strength, curl_strength, powder, ms_a, ms_b, ms_c,
      ambient, base_scale, detail_scale, weather_scale, drift, skew_strength, diurnal_strength;
  uint32_t light_steps, cloud_steps, octaves, layer_count, temporal_jitter, cone, frame_index;
  uint32_t phase_mode;
  R hg_f, hg_b, hg_w;
  Layer<R> layers[8];
  uint64_t* cnt;  // per-thread counters (may be null)

  void count(int k, uint64_t n = 1) const {
    if (cnt) cnt[k] += n;
  }

  void init(const OracleScene* s, int q8) {
    S = s;
    tex.s = s;
    tex.q8 = q8;
    const PscWorldUniformsGpu& w = s->world;
    const PscFrameUniformsGpu& f = s->frame;
    const PscCloudParamsGpu& p = s->params;
    planet_r = R(w.planet_radius_m);
    atmo_top = R(w.atmosphere_top_m);
    sun = load3<R>(f.sun_direction);
    sun_ang = R(f.sun_direction[3]);
    cam = load3<R>(f.camera_position_world);
    sun_illum = load3<R>(f.sun_illuminance);
    lightning_rgb = load3<R>(f.lightning_illuminance);
    lightning_radius = R(f.lightning_illuminance[3]);
    lightning_origin = load3<R>(f.lightning_origin_world);
    sim_seconds = R(f.simulated_seconds);
    frame_index = f.frame_index;
    vp_w = R(f.viewport_size[0]);
    vp_h = R(f.viewport_size[1]);
    for (int c = 0; c < 4; ++c)
      for (int r = 0; r < 4; ++r) m_inv[c][r] = R(f.inv_view_proj[c][r]);
    sigma_s = load3<R>(p.sigma_s);
    sigma_a = load3<R>(p.sigma_a);
    droplet_bias = R(p.droplet_diameter_bias);
    forward_bias = R(p.forward_bias);
    detail_strength = R(p.detail_strength);
    curl_strength = R(p.curl_strength);
    powder = R(p.powder_strength);
    ms_a = R(p.multi_scatter_a);
    ms_b = R(p.multi_scatter_b);
    ms_c = R(p.multi_scatter_c);
    ambient = R(p.ambient_strength);
    base_scale = R(p.base_scale_m);
    detail_scale = R(p.detail_scale_m);
    weather_scale = R(p.weather_scale_m);
    drift = R(p.wind_drift_strength);
    skew_strength = R(p.wind_skew_strength);
    diurnal_strength = R(p.diurnal_strength);
    light_steps = p.light_steps;
    cloud_steps = p.cloud_steps;
    octaves = p.multi_scatter_octaves;
    layer_count = std::min<uint32_t>(p.cloud_layer_count, 8u);
    temporal_jitter = p.temporal_jitter;
    cone = p.cone_light_sampling;
    phase_mode = s->options.phase_mode;
    hg_f = R(s->options.hg_g_forward);
    hg_b = R(s->options.hg_g_backward);
    hg_w = R(s->options.hg_blend);
    for (int i = 0; i < 8; ++i) {
      const PscCloudLayerGpu& l = s->layers[i];
      layers[i] = Layer<R>{R(l.base_m), R(l.top_m), R(l.coverage), R(l.density_scale),
                           l.cloud_type, R(l.shape_bias), R(l.detail_bias), R(l.anvil_bias),
                           R(l.droplet_diameter_um)};
    }
    cnt = nullptr;
  }

  V3<R> centre() const { return mk<R>(R(0), -planet_r, R(0)); }

  /* ---------------- cloud_density_common.wgsl ---------------- */
  R ndf(R h, uint32_t t, R anvil_bias) const {  // :49-91
    switch (t) {
      case 0: return smoothstep<R>(0, R(0.07), h) * smoothstep<R>(1, R(0.2), h);
      case 1: return smoothstep<R>(0, R(0.10), h) * (R(1) - smoothstep<R>(R(0.6), 1, h));
      case 2: return smoothstep<R>(0, R(0.15), h) * smoothstep<R>(1, R(0.4), h);
      case 3: return smoothstep<R>(0, R(0.20), h) * smoothstep<R>(1, R(0.3), h);
      case 4: return smoothstep<R>(0, R(0.30), h) * (R(1) - smoothstep<R>(R(0.7), 1, h));
      case 5: return smoothstep<R>(0, R(0.40), h) * (R(1) - smoothstep<R>(R(0.6), 1, h));
      case 6: return smoothstep<R>(0, R(0.50), h) * (R(1) - smoothstep<R>(R(0.8), 1, h));
      case 7: {
        const R base = smoothstep<R>(0, R(0.05), h);
        const R mid = smoothstep<R>(R(0.95), R(0.5), h);
        const R anvil = smoothstep<R>(R(0.7), R(0.9), h) * R(1.5) *
                        clampv<R>(anvil_bias, R(0), R(2));
        const R mix_t = smoothstep<R>(R(0.65), R(0.8), h);
        return base * mix<R>(mid, anvil, mix_t);
      }
      default: return R(0);
    }
  }

  WindCache<R> wind_cache(const Layer<R>& L) const {  // :154-183
    const R mid = (L.base + L.top) * R(0.5);
    const R u_y = clampv<R>(mid / R(12000), R(0), R(0.9999));
    R w[2];
    tex.wind(mk<R>(R(0.5), u_y, R(0.5)), w);
    count(ORACLE_CNT_WIND);
    WindCache<R> c;
    const R ds = drift * sim_seconds;
    c.off_x = w[0] * ds;
    c.off_z = w[1] * ds;
    c.skew_x = c.skew_z = c.skew_thickness = R(0);
    if (skew_strength != R(0)) {
      const R speed = std::sqrt(w[0] * w[0] + w[1] * w[1]);
      if (speed >= R(0.1)) {
        c.skew_x = w[0] / speed;
        c.skew_z = w[1] / speed;
        c.skew_thickness = std::fmax(L.top - L.base, R(1)) * skew_strength;
      }
    }
    return c;
  }

  R diurnal(uint32_t type) const {  // :204-219
    if (diurnal_strength == R(0)) return R(0);
    const bool conv = type == 0 || type == 2 || type == 3 || type == 7;
    if (!conv) return R(0);
    return smoothstep<R>(R(-0.1), R(0.4), sun.y) * diurnal_strength;
  }

  uint32_t effective_type(R px, R pz, const Layer<R>& L) const {  // :233-251
    count(ORACLE_CNT_TYPE);
    if (!S->type_grid) return L.type;
    const R half = R(32000) * R(0.5);
    const R u = (px + half) / R(32000);
    const R v = (pz + half) / R(32000);
    const int64_t tx_raw = (int64_t)std::floor(u * R(S->type_w));
    const int64_t ty_raw = (int64_t)std::floor(v * R(S->type_h));
    const int tx = wrap_index(tx_raw, (int)S->type_w);
    const int ty = wrap_index(ty_raw, (int)S->type_h);
    const uint32_t t = S->type_grid[(size_t)ty * S->type_w + tx];
    return t == 255u ? L.type : t;
  }

  R base_shape(V3<R> p_adv, R h, R eff_cov, const Layer<R>& L, uint32_t type, bool light) const {
    R base[4];
    tex.rgba8_3d(S->noise_base, 128, p_adv / std::fmax(base_scale, R(1)), base);
    count(light ? ORACLE_CNT_LIGHT : ORACLE_CNT_BASE);
    const R di = diurnal(L.type);
    const R esb = L.shape_bias * di;
    const R lf = clampv<R>(((base[1] * R(0.625) + base[2] * R(0.25)) + base[3] * R(0.125)) +
                               esb * R(0.5),
                           R(0), R(1));
    const R base_cloud = remap<R>(base[0], -(R(1) - lf), R(1), R(0), R(1));
    const R profile = ndf(h, type, L.anvil_bias);
    R cloud = base_cloud * profile;
    cloud = remap<R>(cloud, R(1) - eff_cov, R(1), R(0), R(1));
    return cloud * eff_cov;
  }

  R sample_density(V3<R> p, R alt, const Layer<R>& L, R weather_r, const WindCache<R>& w,
                   uint32_t type) const {  // cloud_march.wgsl:432-530
    const R h = (alt - L.base) / std::fmax(L.top - L.base, R(1));
    if (h < R(0) || h > R(1)) return R(0);
    const R eff = clampv<R>(weather_r * L.coverage, R(0), R(1));
    if (eff < R(0.01)) return R(0);
    const R sk = h * w.skew_thickness;
    const V3<R> p_adv = mk<R>((p.x - w.off_x) - w.skew_x * sk, (p.y - R(0)) - R(0),
                              (p.z - w.off_z) - w.skew_z * sk);
    R cloud = base_shape(p_adv, h, eff, L, type, false);
    if (cloud > R(0)) {
      const R ds1 = std::fmax(detail_scale, R(1));
      R c2[2];
      tex.curl(p_adv.x / ds1, p_adv.z / ds1, c2);
      count(ORACLE_CNT_CURL);
      const R cx = c2[0] * R(2) - R(1), cz = c2[1] * R(2) - R(1);
      const V3<R> dp = mk<R>(p_adv.x + (cx * curl_strength) * detail_scale,
                             p_adv.y + (R(0) * curl_strength) * detail_scale,
                             p_adv.z + (cz * curl_strength) * detail_scale);
      R det[4];
      tex.rgba8_3d(S->noise_detail, 32, dp / ds1, det);
      count(ORACLE_CNT_DETAIL);
      const R hf = (det[0] * R(0.625) + det[1] * R(0.25)) + det[2] * R(0.125);
      const R dmod = mix<R>(hf, R(1) - hf, clampv<R>(h * R(10), R(0), R(1)));
      const R edb = L.detail_bias * diurnal(L.type);
      const R ld = clampv<R>(detail_strength + edb, R(0), R(1));
      cloud = remap<R>(cloud, dmod * ld, R(1), R(0), R(1));
    }
    return clampv<R>(cloud, R(0), R(1)) * L.density_scale;
  }

  R sample_density_light(V3<R> p, R alt, const Layer<R>& L, R weather_r, const WindCache<R>& w,
                         uint32_t type) const {  // cloud_density_common.wgsl:266-305
    const R h = (alt - L.base) / std::fmax(L.top - L.base, R(1));
    if (h < R(0) || h > R(1)) return R(0);
    const R eff = clampv<R>(weather_r * L.coverage, R(0), R(1));
    if (eff < R(0.01)) return R(0);
    const R sk = h * w.skew_thickness;
    const V3<R> p_adv = mk<R>((p.x - w.off_x) - w.skew_x * sk, p.y,
                              (p.z - w.off_z) - w.skew_z * sk);
    const R cloud = base_shape(p_adv, h, eff, L, type, true);
    return clampv<R>(cloud, R(0), R(1)) * L.density_scale;
  }

  /* ---------------- cloud_march.wgsl ---------------- */
  R altitude_from_entry(V3<R> pw, R r0, R cos_view, R h0, R t) const {  // :360-365
    const V3<R> pi = pw - centre();
    const R num = R(2) * t * r0 * cos_view + t * t;
    return h0 + num / (std::fmax(r0, R(1)) + length(pi));
  }

  static bool ray_sphere(V3<R> ro, V3<R> rd, V3<R> c, R radius, R* t0, R* t1) {  // math:37-48
    const V3<R> oc = ro - c;
    const R b = dot(oc, rd);
    const R cc = dot(oc, oc) - radius * radius;
    const R disc = b * b - cc;
    if (disc < R(0)) return false;
    const R sq = std::sqrt(disc);
    *t0 = -b - sq;
    *t1 = -b + sq;
    return true;
  }

  bool layer_intersect(V3<R> ro, V3<R> rd, const Layer<R>& L, R* t0, R* t1) const {  // :370-416
    const V3<R> c = centre();
    const R rb = planet_r + L.base, rt = planet_r + L.top;
    R tt0 = 0, tt1 = 0, tb0 = 0, tb1 = 0;
    const bool hit_top = ray_sphere(ro, rd, c, rt, &tt0, &tt1);
    const bool hit_bot = ray_sphere(ro, rd, c, rb, &tb0, &tb1);
    if (!hit_top) return false;
    const R r_cam = length(ro - c);
    R ta, tb;
    if (r_cam < rb) {
      if (!hit_bot) return false;
      ta = std::fmax(tb1, R(0));
      tb = std::fmax(tt1, R(0));
    } else if (r_cam > rt) {
      ta = std::fmax(tt0, R(0));
      tb = (hit_bot && tb0 > R(0)) ? std::fmax(tb0, R(0)) : std::fmax(tt1, R(0));
    } else {
      ta = R(0);
      tb = (hit_bot && tb0 > R(0)) ? std::fmin(std::fmax(tt1, R(0)), tb0) : std::fmax(tt1, R(0));
    }
    *t0 = ta;
    *t1 = tb;
    return tb > ta;
  }

  V3<R> sun_transmittance_at(V3<R> p) const {  // :328-354
    const V3<R> pa = p - centre();
    const R r = std::fmax(length(pa), planet_r + R(1));
    const V3<R> up = pa / r;
    const R mu = clampv<R>(dot(up, sun), R(-1), R(1));
    const R ratio = planet_r / r;
    const R sin_h = -std::sqrt(std::fmax(R(1) - ratio * ratio, R(0)));
    if (mu <= sin_h) return mk<R>(0, 0, 0);
    const R ht = atmo_top;
    const R bh = std::sqrt(std::fmax(ht * ht - planet_r * planet_r, R(0)));
    const R rho = std::sqrt(std::fmax(r * r - planet_r * planet_r, R(0)));
    const R disc = r * r * (mu * mu - R(1)) + ht * ht;
    const R d = std::fmax(-r * mu + std::sqrt(std::fmax(disc, R(0))), R(0));
    const R d_min = ht - r, d_max = rho + bh;
    const R x_mu = clampv<R>((d - d_min) / std::fmax(d_max - d_min, R(1)), R(0), R(1));
    const R x_r = rho / std::fmax(bh, R(1));
    count(ORACLE_CNT_TRANS);
    return tex.lut2d(S->lut_transmittance, 256, 64, x_mu, x_r);
  }

  static R hg(R c, R g) {  // :151-155
    const R g2 = g * g;
    const R den = R(1) + g2 - R(2) * g * c;
    return (R(1) - g2) / (R(4) * R(3.14159265358979) * std::pow(std::fmax(den, R(1e-4)), R(1.5)));
  }
  static R draine(R c, R g, R alpha) {  // :161-168
    const R g2 = g * g;
    const R den = R(1) + g2 - R(2) * g * c;
    const R num = (R(1) - g2) * (R(1) + alpha * c * c);
    const R dd = R(4) * (R(1) + alpha * (R(1) + R(2) * g2) / R(3)) * R(3.14159265358979) *
                 std::pow(std::fmax(den, R(1e-4)), R(1.5));
    return num / std::fmax(dd, R(1e-6));
  }
  struct PhaseC {
    R g_hg, g_d, alpha, w_d, ice;
  };
  PhaseC phase_constants(const Layer<R>& L, R h) const {  // :256-272
    R d = L.droplet;
    if (L.type == 7u) {
      const R mt = smoothstep<R>(R(0.60), R(0.85), clampv<R>(h, R(0), R(1)));
      d = mix<R>(L.droplet, R(50), mt);
    }
    d = clampv<R>(d * droplet_bias, R(5), R(50));
    PhaseC c;
    c.g_hg = std::exp(R(-0.0990567) / (d - R(1.67154)));
    c.g_d = std::exp(R(-2.20679) / (d + R(3.91029))) - R(0.428934);
    c.alpha = std::exp(R(3.62489) - R(8.29288) / (d + R(5.52825)));
    c.w_d = std::exp(R(-0.599085) / (d - R(0.641583)) - R(0.665888));
    c.ice = smoothstep<R>(R(35), R(50), d);
    return c;
  }
  static R halo(R c, R peak, R width) {  // :229-236
    const R sc = width * std::sqrt(std::fmax(R(1) - peak * peak, R(1e-4)));
    const R dx = (c - peak) / std::fmax(sc, R(1e-4));
    return std::exp(R(-0.5) * dx * dx);
  }
  R phase_with(R cos_t, R g_scale, const PhaseC& c) const {  // :278-296
    if (phase_mode == PSC_PHASE_DUAL_LOBE_HG)
      return mix<R>(hg(cos_t, hg_f * g_scale), hg(cos_t, hg_b * g_scale), hg_w);
    const R p_hg = hg(cos_t, c.g_hg * g_scale);
    const R p_d = draine(cos_t, c.g_d * g_scale, c.alpha);
    R p = (R(1) - c.w_d) * p_hg + c.w_d * p_d;
    if (c.ice > R(0)) {
      const R width = (R(0.5) * (R(3.14159265358979) / R(180))) / std::fmax(g_scale, R(0.1));
      const R h22 = halo(cos_t, R(0.92718), width);
      const R h46 = halo(cos_t, R(0.69466), width);
      p = p + c.ice * (R(0.08) * h22 + R(0.03) * h46);
    }
    return p;
  }

  R march_to_light(V3<R> p, R alt, const Layer<R>& L, R wr, const WindCache<R>& w,
                   uint32_t type) const {  // :543-578
    if (cone) return march_to_light_cone(p, alt, L, wr, w, type);
    const R cos_sun = std::fmax(sun.y, R(0.05));
    const R dist = std::fmax((L.top - alt) / cos_sun, R(1));
    const R step = dist / R(light_steps);
    R od = 0;
    const R r0 = planet_r + alt;
    const R cos_view = dot((p - centre()) / std::fmax(r0, R(1)), sun);
    for (uint32_t i = 0; i < light_steps; ++i) {
      const R t = (R(i) + R(0.5)) * step;
      const V3<R> pi = p + sun * t;
      const R a = altitude_from_entry(pi, r0, cos_view, alt, t);
      od = od + sample_density_light(pi, a, L, wr, w, type) * step;
    }
    return od;
  }

  R march_to_light_cone(V3<R> p, R alt, const Layer<R>& L, R wr, const WindCache<R>& w,
                        uint32_t type) const {  // :599-666
    static const double K[6][3] = {{0.38051305, 0.92453449, -0.02111345},
                                   {-0.50625799, -0.03590792, -0.86163418},
                                   {-0.32509218, -0.94557439, 0.01428793},
                                   {0.09026238, -0.27376545, 0.95755165},
                                   {0.28128598, 0.42443639, -0.86065785},
                                   {-0.16852403, 0.14748697, 0.97460106}};
    auto kv = [&](int i) { return mk<R>(R((float)K[i][0]), R((float)K[i][1]), R((float)K[i][2])); };
    const R cos_sun = std::fmax(sun.y, R(0.05));
    const R dist = std::fmax((L.top - alt) / cos_sun, R(1));
    const R step = dist / R(5);
    const R r0 = planet_r + alt;
    const R cos_view = dot((p - centre()) / std::fmax(r0, R(1)), sun);
    R od = 0;
    for (uint32_t i = 0; i < 5; ++i) {
      const R t = (R(i) + R(0.5)) * step;
      const V3<R> off = ((kv((int)i) * step) * (R(i) + R(1))) / R(5);
      const V3<R> pi = (p + sun * t) + off;
      const R a = altitude_from_entry(pi, r0, cos_view, alt, t);
      od = od + sample_density_light(pi, a, L, wr, w, type) * step;
    }
    const R tf = dist * R(3);
    const V3<R> offf = kv(5) * (step * R(3));
    const V3<R> pf = (p + sun * tf) + offf;
    const R af = altitude_from_entry(pf, r0, cos_view, alt, tf);
    od = od + sample_density_light(pf, af, L, wr, w, type) * step * R(3);
    return od;
  }

  V3<R> sky_ambient(V3<R> p) const {  // :672-700
    const V3<R> rel = p - centre();
    const V3<R> up = normalize(rel);
    const R cam_r = length(rel);
    const R cos_v = clampv<R>(up.y, R(-1), R(1));
    const R vza = std::acos(cos_v);
    const R sin_h = clampv<R>(planet_r / cam_r, R(0), R(1));
    const R PI_ = R(3.14159265358979);
    const R zha = PI_ - std::asin(sin_h);
    R v;
    if (vza < zha) {
      v = std::sqrt(clampv<R>(vza / std::fmax(zha, R(1e-6)), R(0), R(1))) * R(0.5);
    } else {
      const R br = std::fmax(PI_ - zha, R(1e-6));
      v = R(0.5) + std::sqrt(clampv<R>((vza - zha) / br, R(0), R(1))) * R(0.5);
    }
    const R vaz = std::atan2(up.x, up.z);
    const R saz = std::atan2(sun.x, sun.z);
    R du = (vaz - saz) / (R(2) * PI_);
    du = du - std::floor(du);
    count(ORACLE_CNT_SKY);
    return tex.lut2d(S->lut_skyview, 192, 108, du, v) * sun_illum;
  }

  static V3<R> chromatic(R d) {  // :122-145
    const R t = clampv<R>(R(1) - d / R(20), R(0), R(1));
    if (t <= R(0)) return mk<R>(1, 1, 1);
    const R s = R(0.25) * t * t;
    return mk<R>(R(1) - R(0.5) * s, R(1), R(1) + s);
  }

  struct ViewRay {
    V3<R> org, dir;
    R cos_theta, fwd, jitter, depth_t_max;
  };

  // compute_view_ray (math.wgsl:23-33), the blue-noise jitter
  // (cloud_march.wgsl:745-756) and the depth clip (:764-775) of one pixel.
  ViewRay view_ray(uint32_t px, uint32_t py, const float* depth, uint32_t width) const {
    ViewRay r;
    const R fx = R(px) + R(0.5), fy = R(py) + R(0.5);
    const R nx = (fx / vp_w) * R(2) - R(1);
    const R ny = R(1) - (fy / vp_h) * R(2);
    R nh[4];
    for (int k = 0; k < 4; ++k)
      nh[k] = ((m_inv[0][k] * nx + m_inv[1][k] * ny) + m_inv[2][k] * R(1)) + m_inv[3][k] * R(1);
    const V3<R> near_p = mk<R>(nh[0] / nh[3], nh[1] / nh[3], nh[2] / nh[3]);
    r.dir = normalize(near_p - cam);
    r.org = cam;
    r.cos_theta = dot(r.dir, sun);
    r.fwd = smoothstep<R>(R(0), R(1), std::fmax(r.cos_theta, R(0)));

    int sx = (int)px & 63, sy = (int)py & 63;
    if (temporal_jitter) {
      const uint32_t ph = frame_index & 15u;
      const int ox = (int)((ph * 11u + 7u) & 63u), oy = (int)((ph * 23u + 13u) & 63u);
      sx = (sx ^ ox) & 63;
      sy = (sy ^ oy) & 63;
    }
    r.jitter = R(S->blue_noise[sy * 64 + sx]) / R(255);
    count(ORACLE_CNT_BLUE);

    r.depth_t_max = R(1e30);
    if (depth) {
      count(ORACLE_CNT_DEPTH);
      const R dn = R(depth[(size_t)py * width + px]);
      if (dn > R(0)) {
        R hh[4];
        for (int k = 0; k < 4; ++k)
          hh[k] = ((m_inv[0][k] * nx + m_inv[1][k] * ny) + m_inv[2][k] * dn) + m_inv[3][k];
        const V3<R> wp = mk<R>(hh[0] / hh[3], hh[1] / hh[3], hh[2] / hh[3]);
        r.depth_t_max = std::fmax(length(wp - r.org), R(0));
      }
    }
    return r;
  }

  // Branch-margin diagnostic (oracle_branch_margins): when not null, the
  // march lowers margin[0] to the smallest |max3(T) - 0.01| / 0.01 of its
  // early-exit tests and margin[1] to the smallest |density - 1e-3| / 1e-3
  // of its primary samples, the two tests whose outcome a last-bit change of
  // the operands can flip (cloud_march.wgsl:833,885,996).
  double* margin = nullptr;
  void note_exit(R tmax) const {
    if (margin) margin[0] = std::fmin(margin[0], std::fabs((double)tmax - 0.01) / 0.01);
  }
  void note_density(R d) const {
    if (margin) margin[1] = std::fmin(margin[1], std::fabs((double)d - 1e-3) / 1e-3);
  }

  // Branch tape (oracle_render_frozen): the outcomes of the march's tests
  // whose result jumps the image (the layer hits and their order, the early
  // exits, the 1e-3 density threshold, the aerial-perspective opacity test),
  // in the order they run.
  // tape_mode 1 appends each outcome to `tape`; 2 takes each outcome from
  // it instead of the comparison, so a march with other parameters follows
  // the recorded path (a replay that runs past the tape counts a miss and
  // uses the comparison).
  std::vector<uint8_t>* tape = nullptr;
  int tape_mode = 0;
  mutable size_t tape_pos = 0;
  mutable uint64_t tape_misses = 0;
  bool branch(bool outcome) const {
    if (tape_mode == 1) {
      tape->push_back(outcome ? 1 : 0);
    } else if (tape_mode == 2) {
      if (tape_pos < tape->size()) return (*tape)[tape_pos++] != 0;
      ++tape_misses;
    }
    return outcome;
  }

  void pixel(uint32_t px, uint32_t py, const float* depth, uint32_t width, R lum_out[4],
             R tr_out[4]) const {
    count(ORACLE_CNT_PIXELS);
    const R fx = R(px) + R(0.5), fy = R(py) + R(0.5);
    const ViewRay vr = view_ray(px, py, depth, width);
    const V3<R> dir = vr.dir, org = vr.org;
    const R cos_theta = vr.cos_theta, fwd = vr.fwd, jitter = vr.jitter,
            depth_t_max = vr.depth_t_max;

    struct Hit {
      uint32_t idx;
      R t0, t1;
      uint32_t hit;
    } hits[8];
    for (uint32_t l = 0; l < layer_count; ++l) {
      R t0 = 0, t1 = 0;
      const bool ok = branch(layer_intersect(org, dir, layers[l], &t0, &t1));
      uint32_t flag = 0;
      if (ok) {
        t1 = std::fmin(t1, depth_t_max);
        if (branch(t1 > t0)) flag = 1;
      }
      hits[l] = Hit{l, t0, t1, flag};
    }
    for (uint32_t i = 1; i < layer_count; ++i) {
      uint32_t j = i;
      while (j > 0 && branch(!(hits[j - 1].t0 <= hits[j].t0))) {
        std::swap(hits[j], hits[j - 1]);
        --j;
      }
    }

    V3<R> lum = mk<R>(0, 0, 0), trans = mk<R>(1, 1, 1);
    const V3<R> st_base = sigma_s + sigma_a;
    R tw = 0, twn = 0;
    const V3<R> lw = mk<R>(R(0.2126), R(0.7152), R(0.0722));

    for (uint32_t i = 0; i < layer_count; ++i) {
      note_exit(max3(trans));
      if (branch(max3(trans) < R(0.01))) break;
      const Hit lh = hits[i];
      if (!lh.hit) continue;
      const Layer<R>& L = layers[lh.idx];
      const V3<R> sigma_t = st_base * chromatic(L.droplet);
      const R segment = lh.t1 - lh.t0;
      if (segment <= R(0)) continue;
      const R step = segment / R(cloud_steps);
      R t = lh.t0 + jitter * step;
      const R r0 = length(org - centre());
      const R cos_view = dot((org - centre()) / std::fmax(r0, R(1)), dir);
      const R h0 = r0 - planet_r;
      const WindCache<R> w = wind_cache(L);
      for (uint32_t s = 0; s < cloud_steps; ++s) {
        count(ORACLE_CNT_STEPS);
        const V3<R> p = org + dir * t;
        const R alt = altitude_from_entry(p, r0, cos_view, h0, t);
        const R wsx = p.x - w.off_x, wsz = p.z - w.off_z;
        const R ws1 = std::fmax(weather_scale, R(1));
        const R wr = tex.weather_r(wsx / ws1 + R(0.5), wsz / ws1 + R(0.5));
        count(ORACLE_CNT_WEATHER);
        const uint32_t type = effective_type(wsx, wsz, L);
        const R density = sample_density(p, alt, L, wr, w, type);
        note_density(density);
        if (branch(density > R(1e-3))) {
          count(ORACLE_CNT_DENSE);
          const R od = march_to_light(p, alt, L, wr, w, type);
          const V3<R> beer = vexp(mk<R>(-sigma_t.x * od, -sigma_t.y * od, -sigma_t.z * od));
          const V3<R> pw = vexp(mk<R>(R(-2) * sigma_t.x * od, R(-2) * sigma_t.y * od,
                                      R(-2) * sigma_t.z * od));
          const V3<R> powder_v = mk<R>(R(1) - pw.x, R(1) - pw.y, R(1) - pw.z);
          const V3<R> bp = (beer * powder_v) * R(2);
          const V3<R> energy = mk<R>(mix<R>(beer.x, bp.x, powder), mix<R>(beer.y, bp.y, powder),
                                     mix<R>(beer.z, bp.z, powder));
          const R phase_h = clampv<R>((alt - L.base) / std::fmax(L.top - L.base, R(1)), R(0), R(1));
          const PhaseC pc = phase_constants(L, phase_h);
          const V3<R> st = sun_transmittance_at(p);
          V3<R> sun_in = mk<R>(0, 0, 0);
          R a = 1, b = 1, c = 1;
          for (uint32_t n = 0; n < octaves; ++n) {
            const R ph = phase_with(cos_theta, c, pc);
            const V3<R> e = vexp(mk<R>((-sigma_t.x * od) * b, (-sigma_t.y * od) * b,
                                       (-sigma_t.z * od) * b));
            sun_in = sun_in + (((a * sun_illum) * st) * ph) * e;
            a = a * ms_a;
            b = b * ms_b;
            c = c * ms_c;
          }
          if (forward_bias > R(0)) sun_in = sun_in * (R(1) + forward_bias * fwd);
          const R hn = clampv<R>((alt - L.base) / std::fmax(L.top - L.base, R(1)), R(0), R(1));
          const V3<R> amb = (sky_ambient(p) * ambient) * mix<R>(R(0.3), R(1), hn);
          V3<R> light = mk<R>(0, 0, 0);
          if (lightning_radius > R(0)) {
            const R dx = p.x - lightning_origin.x, dz = p.z - lightning_origin.z;
            const R d = std::sqrt(dx * dx + dz * dz);
            const R fo = clampv<R>(R(1) - d / lightning_radius, R(0), R(1));
            light = lightning_rgb * (fo * fo * (R(3) - R(2) * fo));
          }
          const V3<R> in_s = (density * sigma_s) * ((sun_in * energy + amb) + light);
          const V3<R> ls = vmax(density * sigma_t, R(1e-6));
          const V3<R> samp = vexp(mk<R>(-ls.x * step, -ls.y * step, -ls.z * step));
          const V3<R> s_int = (in_s - in_s * samp) / ls;
          const V3<R> step_lum = trans * s_int;
          const R sw = dot(step_lum, lw);
          lum = lum + step_lum;
          tw = tw + sw * t;
          twn = twn + sw;
          trans = trans * samp;
        }
        note_exit(max3(trans));
        if (branch(max3(trans) < R(0.01))) break;
        t = t + step;
      }
    }

    // AP (:1016-1048)
    const R t_lum = dot(trans, lw);
    const R opacity = R(1) - t_lum;
    const R t_cloud = tw / std::fmax(twn, R(1e-6));
    V3<R> lo = lum;
    if (branch(opacity > R(1e-4))) {
      const R ds = std::fmax(t_cloud, R(50));
      const R az = clampv<R>(std::log(ds / R(50)) / std::log(R(100000) / R(50)), R(0), R(1));
      R ap[4];
      tex.aerial(mk<R>(fx / vp_w, fy / vp_h, az), ap);
      count(ORACLE_CNT_AP);
      lo = lum * ap[3] + mk<R>(ap[0], ap[1], ap[2]) * opacity;
    }
    lum_out[0] = lo.x;
    lum_out[1] = lo.y;
    lum_out[2] = lo.z;
    lum_out[3] = R(1);
    tr_out[0] = trans.x;
    tr_out[1] = trans.y;
    tr_out[2] = trans.z;
    tr_out[3] = R(1);
  }
};


}  // namespace oracle_core

#endif

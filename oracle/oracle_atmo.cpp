/*
 * ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of the four atmosphere LUT bakes the cloud march samples
 * (transmittance, multi-scatter, sky-view, aerial perspective), in FP32 with
 * RGBA16F output like the reference's storage textures.
 *   shaders/common/atmosphere.wgsl:23-214
 *   shaders/common/atmosphere_lut_sampling.wgsl:5-38
 *   shaders/atmosphere/transmittance.comp.wgsl:18-31
 *   shaders/atmosphere/multiscatter.comp.wgsl:29-126
 *   shaders/atmosphere/skyview.comp.wgsl:47-174
 *   shaders/atmosphere/aerialperspective.comp.wgsl:42-127
 */
#include <cmath>
#include <cstdint>
#include <cstring>

#include "oracle.h"
#include "oracle_common.h"

using namespace oracle;

namespace {

const float PI_F = 3.14159265358979f;

struct V3 {
  float x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 mul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 mulv(V3 a, V3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline float length(V3 a) { return std::sqrt(dot(a, a)); }
inline V3 normalize(V3 a) {
  const float l = length(a);
  return {a.x / l, a.y / l, a.z / l};
}
inline V3 vexp(V3 a) { return {std::exp(a.x), std::exp(a.y), std::exp(a.z)}; }
inline V3 vmax(V3 a, float m) {
  return {std::fmax(a.x, m), std::fmax(a.y, m), std::fmax(a.z, m)};
}
inline V3 v4(const float* p) { return {p[0], p[1], p[2]}; }

struct Atmo {
  const PscWorldUniformsGpu* w;

  V3 density(float h) const {  // atmosphere.wgsl:23-31
    const float r = std::exp(-h / w->rayleigh_scale_height_m);
    const float m = std::exp(-h / w->mie_scale_height_m);
    const float half_t = w->ozone_thickness_m * 0.5f;
    const float dz = std::fabs(h - w->ozone_center_m);
    const float o = std::fmax(0.0f, 1.0f - dz / std::fmax(half_t, 1.0f));
    return {r, m, o};
  }
  V3 extinction(float h) const {  // :34-39
    const V3 d = density(h);
    return add(add(mul(v4(w->rayleigh_scattering), d.x),
                   mul(add(v4(w->mie_scattering), v4(w->mie_absorption)), d.y)),
               mul(v4(w->ozone_absorption), d.z));
  }
  V3 scattering(float h) const {  // :43-46
    const V3 d = density(h);
    return add(mul(v4(w->rayleigh_scattering), d.x), mul(v4(w->mie_scattering), d.y));
  }
  void scattering_pair(float h, V3* ray, V3* mie) const {  // :55-61
    const V3 d = density(h);
    *ray = mul(v4(w->rayleigh_scattering), d.x);
    *mie = mul(v4(w->mie_scattering), d.y);
  }
  static bool ray_sphere_origin(V3 ro, V3 rd, float r, float* t0, float* t1) {
    const float b = dot(ro, rd);
    const float c = dot(ro, ro) - r * r;
    const float disc = b * b - c;
    if (disc < 0.0f) return false;
    const float sq = std::sqrt(disc);
    *t0 = -b - sq;
    *t1 = -b + sq;
    return true;
  }
  float dist_to_top(V3 p, V3 dir) const {  // :112-116
    float t0, t1;
    if (!ray_sphere_origin(p, dir, w->atmosphere_top_m, &t0, &t1)) return 0.0f;
    return std::fmax(t1, 0.0f);
  }
  float dist_to_boundary(V3 p, V3 dir) const {  // :120-135
    float tt0, tt1, tp0, tp1;
    const bool hit_top = ray_sphere_origin(p, dir, w->atmosphere_top_m, &tt0, &tt1);
    const bool hit_planet = ray_sphere_origin(p, dir, w->planet_radius_m, &tp0, &tp1);
    if (!hit_top) return 0.0f;
    float t_max = tt1;
    if (hit_planet && tp0 > 0.0f) t_max = std::fmin(t_max, tp0);
    return std::fmax(t_max, 0.0f);
  }
  void trans_uv(V3 p, V3 dir, float* u, float* v) const {  // :149-163
    const float r = length(p);
    const float ht = w->atmosphere_top_m, hp = w->planet_radius_m;
    const float H = std::sqrt(std::fmax(ht * ht - hp * hp, 0.0f));
    const float rho = std::sqrt(std::fmax(r * r - hp * hp, 0.0f));
    const float d = std::fmax(dist_to_top(p, dir), 0.0f);
    const float d_min = ht - r;
    const float d_max = rho + H;
    *u = clampv((d - d_min) / std::fmax(d_max - d_min, 1.0f), 0.0f, 1.0f);
    *v = rho / std::fmax(H, 1.0f);
  }
  V3 integrate_od(V3 p, V3 dir, uint32_t n) const {  // :192-214
    const float t_max = dist_to_boundary(p, dir);
    if (t_max <= 0.0f) return {0, 0, 0};
    const float dt = t_max / (float)n;
    const float r0 = length(p);
    const float cos_view = dot(mul(p, 1.0f / std::fmax(r0, 1.0f)), dir);
    const float h0 = r0 - w->planet_radius_m;
    V3 od = {0, 0, 0};
    V3 prev = extinction(h0);
    for (uint32_t i = 1; i <= n; ++i) {
      const float t = (float)i * dt;
      const V3 pi = add(p, mul(dir, t));
      const float num = 2.0f * t * r0 * cos_view + t * t;
      const float rd = num / (std::fmax(r0, 1.0f) + length(pi));
      const V3 cur = extinction(h0 + rd);
      od = add(od, mul(mul(add(prev, cur), 0.5f), dt));
      prev = cur;
    }
    return od;
  }
};

/* `p / max(r, 1)` as written in WGSL is a vector divide; spelled as a
 * per-component divide to keep the rounding of the original. */
inline V3 div_s(V3 a, float s) { return {a.x / s, a.y / s, a.z / s}; }

struct Tex2D {  // RGBA16F, linear + clamp-to-edge (lut_sampler)
  const uint16_t* d;
  int w, h;
  V3 sample(float u, float v) const {
    const Axis<float> ax = axis_clamp<float>(u, w, 0);
    const Axis<float> ay = axis_clamp<float>(v, h, 0);
    auto t = [&](int x, int y, int c) { return f16_to_f32(d[((size_t)y * w + x) * 4 + c]); };
    V3 r;
    float* o = &r.x;
    for (int c = 0; c < 3; ++c) {
      const float a = lerp(t(ax.i0, ay.i0, c), t(ax.i1, ay.i0, c), ax.w);
      const float b = lerp(t(ax.i0, ay.i1, c), t(ax.i1, ay.i1, c), ax.w);
      o[c] = lerp(a, b, ay.w);
    }
    return r;
  }
};

V3 sample_trans_lut(const Atmo& A, const Tex2D& T, V3 p, V3 dir) {  // lut_sampling:5-22
  float t0, t1;
  if (Atmo::ray_sphere_origin(p, dir, A.w->planet_radius_m, &t0, &t1) && t0 > 0.0f)
    return {0, 0, 0};
  float u, v;
  A.trans_uv(p, dir, &u, &v);
  return T.sample(u, v);
}

inline float phase_rayleigh(float c) { return (3.0f / (16.0f * PI_F)) * (1.0f + c * c); }
inline float phase_mie(float c, float g) {
  const float g2 = g * g;
  const float den = 1.0f + g2 - 2.0f * g * c;
  return (1.0f - g2) / (4.0f * PI_F * std::pow(std::fmax(den, 1e-4f), 1.5f));
}

void store(uint16_t* o, V3 v, float a) {
  o[0] = f32_to_f16(v.x);
  o[1] = f32_to_f16(v.y);
  o[2] = f32_to_f16(v.z);
  o[3] = f32_to_f16(a);
}

inline V3 mat_mul_near(const float m[4][4], float x, float y, float* w_out) {
  // inv_view_proj * vec4(x, y, 1, 1), column-major.
  float r[4];
  for (int row = 0; row < 4; ++row)
    r[row] = ((m[0][row] * x + m[1][row] * y) + m[2][row] * 1.0f) + m[3][row] * 1.0f;
  *w_out = r[3];
  return {r[0], r[1], r[2]};
}

}  // namespace

extern "C" {

int oracle_bake_transmittance(const PscWorldUniformsGpu* world, uint16_t* out) {
  if (!world || !out) return -1;
  const Atmo A{world};
  const int W = 256, H = 64;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const float u = ((float)x + 0.5f) / (float)W, v = ((float)y + 0.5f) / (float)H;
      // transmittance_lut_uv_to_pos_dir, atmosphere.wgsl:166-184
      const float ht = world->atmosphere_top_m, hp = world->planet_radius_m;
      const float Hh = std::sqrt(std::fmax(ht * ht - hp * hp, 0.0f));
      const float rho = v * Hh;
      const float r = std::sqrt(rho * rho + hp * hp);
      const float d_min = ht - r, d_max = rho + Hh;
      const float d = d_min + u * (d_max - d_min);
      float mu = 1.0f;
      if (d != 0.0f)
        mu = clampv((Hh * Hh - rho * rho - d * d) / std::fmax(2.0f * r * d, 1e-6f), -1.0f, 1.0f);
      const V3 p = {0.0f, r, 0.0f};
      const float sin_t = std::sqrt(std::fmax(1.0f - mu * mu, 0.0f));
      const V3 dir = {sin_t, mu, 0.0f};
      const V3 od = A.integrate_od(p, dir, 40);
      store(out + ((size_t)y * W + x) * 4, vexp(mul(od, -1.0f)), 1.0f);
    }
  return 0;
}

int oracle_bake_multiscatter(const PscWorldUniformsGpu* world, const uint16_t* trans,
                             uint16_t* out) {
  if (!world || !trans || !out) return -1;
  const Atmo A{world};
  const Tex2D T{trans, 256, 64};
  const int W = 32, H = 32;
  const uint32_t N_DIRS = 64, N_STEPS = 20;
  for (int gy = 0; gy < H; ++gy)
    for (int gx = 0; gx < W; ++gx) {
      const float u = ((float)gx + 0.5f) / (float)W, v = ((float)gy + 0.5f) / (float)H;
      const float sun_cos = clampv(u * 2.0f - 1.0f, -1.0f, 1.0f);
      const float sun_sin = std::sqrt(std::fmax(1.0f - sun_cos * sun_cos, 0.0f));
      const float r = world->planet_radius_m +
                      v * (world->atmosphere_top_m - world->planet_radius_m);
      const V3 p0 = {0.0f, r, 0.0f};
      const V3 sun = {sun_sin, sun_cos, 0.0f};
      V3 l2 = {0, 0, 0}, fms = {0, 0, 0};
      const float h0 = r - world->planet_radius_m;
      for (uint32_t di = 0; di < N_DIRS; ++di) {
        // sphere_sample, multiscatter.comp.wgsl:29-35
        const float golden = 0.6180339887498949f;
        const float z = 1.0f - 2.0f * ((float)di + 0.5f) / (float)N_DIRS;
        const float rr = std::sqrt(std::fmax(1.0f - z * z, 0.0f));
        const float fr = (float)di * golden;
        const float phi = 2.0f * PI_F * (fr - std::floor(fr));
        const V3 vd = {rr * std::cos(phi), rr * std::sin(phi), z};
        const float t_max = A.dist_to_boundary(p0, vd);
        if (t_max <= 0.0f) continue;
        const float dt = t_max / (float)N_STEPS;
        const float cos_view = dot(div_s(p0, std::fmax(r, 1.0f)), vd);
        V3 tr = {1, 1, 1}, ld = {0, 0, 0}, fd = {0, 0, 0};
        for (uint32_t s = 0; s < N_STEPS; ++s) {
          const float t = ((float)s + 0.5f) * dt;
          const V3 p = add(p0, mul(vd, t));
          const float num = 2.0f * t * r * cos_view + t * t;
          const float rdl = num / (std::fmax(r, 1.0f) + length(p));
          const float h = h0 + rdl;
          const V3 st = A.extinction(h);
          const V3 ss = A.scattering(h);
          const V3 trs = vexp(mul(mul(st, -1.0f), dt));
          const float r_p = r + rdl;
          const float cos_sun = dot(p, sun) / std::fmax(r_p, 1.0f);
          V3 vis = {0, 0, 0};
          const float ratio = world->planet_radius_m / r_p;
          if (cos_sun > -std::sqrt(std::fmax(1.0f - ratio * ratio, 0.0f)))
            vis = sample_trans_lut(A, T, p, sun);
          const V3 in_s = mulv(ss, vis);
          const V3 safe = vmax(st, 1e-7f);
          const V3 s_int = {(in_s.x - in_s.x * trs.x) / safe.x, (in_s.y - in_s.y * trs.y) / safe.y,
                            (in_s.z - in_s.z * trs.z) / safe.z};
          ld = add(ld, mulv(tr, s_int));
          const V3 s_iso = {(ss.x - ss.x * trs.x) / safe.x, (ss.y - ss.y * trs.y) / safe.y,
                            (ss.z - ss.z * trs.z) / safe.z};
          fd = add(fd, mulv(tr, s_iso));
          tr = mulv(tr, trs);
        }
        l2 = add(l2, ld);
        fms = add(fms, fd);
      }
      const float norm = (4.0f * PI_F) / (float)N_DIRS;
      const float inv4pi = 1.0f / (4.0f * PI_F);
      const V3 L2 = mul(mul(l2, norm), inv4pi);
      const V3 F = mul(mul(fms, norm), inv4pi);
      const V3 fc = {clampv(F.x, 0.0f, 0.95f), clampv(F.y, 0.0f, 0.95f), clampv(F.z, 0.0f, 0.95f)};
      const V3 full = {L2.x / (1.0f - fc.x), L2.y / (1.0f - fc.y), L2.z / (1.0f - fc.z)};
      store(out + ((size_t)gy * W + gx) * 4, full, 1.0f);
    }
  return 0;
}

static V3 march_inscatter(const Atmo& A, const Tex2D& T, const Tex2D& MS, V3 p, float r,
                          V3 view_dir, V3 sun, float phase_r, float phase_m, float dt,
                          uint32_t n, bool stop_below_ground, const float* illum, V3* trans) {
  const PscWorldUniformsGpu* w = A.w;
  const float cos_view = dot(div_s(p, std::fmax(r, 1.0f)), view_dir);
  const float h0 = r - w->planet_radius_m;
  V3 lum = {0, 0, 0}, tr = {1, 1, 1};
  for (uint32_t s = 0; s < n; ++s) {
    const float t = ((float)s + 0.5f) * dt;
    const V3 pi = add(p, mul(view_dir, t));
    const float num = 2.0f * t * r * cos_view + t * t;
    const float rdl = num / (std::fmax(r, 1.0f) + length(pi));
    const float h = h0 + rdl;
    if (stop_below_ground && h < 0.0f) break;
    const V3 st = A.extinction(h);
    const V3 trs = vexp(mul(mul(st, -1.0f), dt));
    const V3 vis = sample_trans_lut(A, T, pi, sun);
    V3 sr, sm;
    A.scattering_pair(h, &sr, &sm);
    const V3 sun_in = mulv(add(mul(sr, phase_r), mul(sm, phase_m)), vis);
    const float r_p = r + rdl;
    const float h_norm =
        clampv(h / std::fmax(w->atmosphere_top_m - w->planet_radius_m, 1.0f), 0.0f, 1.0f);
    const float sun_cos = clampv(dot(div_s(pi, std::fmax(r_p, 1.0f)), sun), -1.0f, 1.0f);
    const V3 lms = MS.sample(sun_cos * 0.5f + 0.5f, h_norm);
    const V3 multi = mulv(add(sr, sm), lms);
    V3 in_s = add(sun_in, multi);
    if (illum) in_s = mulv(in_s, V3{illum[0], illum[1], illum[2]});
    const V3 safe = vmax(st, 1e-7f);
    const V3 s_int = {(in_s.x - in_s.x * trs.x) / safe.x, (in_s.y - in_s.y * trs.y) / safe.y,
                      (in_s.z - in_s.z * trs.z) / safe.z};
    lum = add(lum, mulv(tr, s_int));
    tr = mulv(tr, trs);
  }
  *trans = tr;
  return lum;
}

int oracle_bake_skyview(const PscFrameUniformsGpu* frame, const PscWorldUniformsGpu* world,
                        const uint16_t* trans, const uint16_t* ms, uint16_t* out) {
  if (!frame || !world || !trans || !ms || !out) return -1;
  const Atmo A{world};
  const Tex2D T{trans, 256, 64}, MS{ms, 32, 32};
  const int W = 192, H = 108;
  for (int gy = 0; gy < H; ++gy)
    for (int gx = 0; gx < W; ++gx) {
      const float u = ((float)gx + 0.5f) / (float)W, v = ((float)gy + 0.5f) / (float)H;
      const V3 pw = v4(frame->camera_position_world);
      V3 p = {pw.x, pw.y + world->planet_radius_m, pw.z};
      float r = length(p);
      if (r < world->planet_radius_m + 1.0f) {
        p = mul(normalize(p), world->planet_radius_m + 1.0f);
        r = world->planet_radius_m + 1.0f;
      }
      const float sin_h = clampv(world->planet_radius_m / r, 0.0f, 1.0f);
      const float zha = PI_F - std::asin(sin_h);
      float vza;
      if (v < 0.5f) {
        const float c = v * 2.0f;
        vza = c * c * zha;
      } else {
        const float c = (v - 0.5f) * 2.0f;
        vza = zha + c * c * (PI_F - zha);
      }
      const V3 sun = v4(frame->sun_direction);
      const float sun_az = std::atan2(sun.x, sun.z);
      const float az = sun_az + u * 2.0f * PI_F;
      const float cv = std::cos(vza), sv = std::sin(vza);
      const V3 vd = {sv * std::sin(az), cv, sv * std::cos(az)};
      const float ct = dot(vd, sun);
      const float pr = phase_rayleigh(ct), pm = phase_mie(ct, world->mie_g);
      const float t_max = A.dist_to_boundary(p, vd);
      uint16_t* o = out + ((size_t)gy * W + gx) * 4;
      if (t_max <= 0.0f) {
        store(o, V3{0, 0, 0}, 1.0f);
        continue;
      }
      const float dt = t_max / 32.0f;
      V3 tr;
      V3 lum = march_inscatter(A, T, MS, p, r, vd, sun, pr, pm, dt, 32, false, nullptr, &tr);
      float tp0, tp1;
      if (Atmo::ray_sphere_origin(p, vd, world->planet_radius_m, &tp0, &tp1) && tp0 > 0.0f) {
        const V3 pg = add(p, mul(vd, tp0));
        const V3 ng = normalize(pg);
        const V3 vis = sample_trans_lut(A, T, pg, sun);
        const float ndl = std::fmax(dot(ng, sun), 0.0f);
        const V3 bounce = mul(mul(mul(v4(world->ground_albedo), 1.0f / 3.14159265f), ndl), 1.0f);
        lum = add(lum, mulv(tr, mulv(bounce, vis)));
      }
      store(o, lum, 1.0f);
    }
  return 0;
}

int oracle_bake_aerial(const PscFrameUniformsGpu* frame, const PscWorldUniformsGpu* world,
                       const uint16_t* trans, const uint16_t* ms, uint16_t* out) {
  if (!frame || !world || !trans || !ms || !out) return -1;
  const Atmo A{world};
  const Tex2D T{trans, 256, 64}, MS{ms, 32, 32};
  const int W = 32, H = 32, D = 64;
  for (int gz = 0; gz < D; ++gz)
    for (int gy = 0; gy < H; ++gy)
      for (int gx = 0; gx < W; ++gx) {
        const float ux = ((float)gx + 0.5f) / (float)W, uy = ((float)gy + 0.5f) / (float)H;
        const float nx = ux * 2.0f - 1.0f, ny = uy * 2.0f - 1.0f;
        float hw;
        const V3 nh = mat_mul_near(frame->inv_view_proj, nx, -ny, &hw);
        const V3 np = div_s(nh, hw);
        const V3 vd = normalize(sub(np, v4(frame->camera_position_world)));
        const float zn = ((float)gz + 0.5f) / (float)D;
        const float t_target = 50.0f * std::pow(100000.0f / 50.0f, zn);
        const V3 pw = v4(frame->camera_position_world);
        const V3 p0 = {pw.x, pw.y + world->planet_radius_m, pw.z};
        const float r0 = length(p0);
        const V3 sun = v4(frame->sun_direction);
        const float ct = dot(vd, sun);
        const float pr = phase_rayleigh(ct), pm = phase_mie(ct, world->mie_g);
        const float dt = t_target / 16.0f;
        V3 tr;
        const V3 lum = march_inscatter(A, T, MS, p0, r0, vd, sun, pr, pm, dt, 16, true,
                                       frame->sun_illuminance, &tr);
        const float t_lum = (tr.x * 0.2126f + tr.y * 0.7152f) + tr.z * 0.0722f;
        store(out + (((size_t)gz * H + gy) * W + gx) * 4, lum, t_lum);
      }
  return 0;
}

}  // extern "C"

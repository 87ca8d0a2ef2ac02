// Voxel-grid form of the cloud march and its adjoint.
//
// Density comes from a trilinearly interpolated FP32 voxel grid (cell
// centres, zero outside) instead of the procedural Schneider density; the
// rest is the reference march loop (cloud_march.wgsl:808-1000): the 6-tap
// light march toward the sun (:543-578), Beer-powder and the Hillaire
// octaves (:888-927), the sun transmittance and sky-view ambient LUTs,
// approx-Mie or dual-lobe HG phase, lightning, and the energy-conserving
// step integral.  For differentiability every step contributes (no density
// gate) and the step integral is (1 - e^-x)/x without the 1e-6 floor; no
// aerial perspective is applied.
//
// Adjoint: one thread per ray runs the forward march keeping the
// transmittance at every k-th step, evaluates its pixel's loss term
// (I - target)^2 / N with I = L + background * T, then walks the checkpoint
// segments backwards: each segment is recomputed from its checkpoint,
// storing per step the primary and light-march grid sums and the prefix sum
// of the primary grid values within the segment, then traversed in reverse,
// carrying the adjoint of the transmittance.  The transmittance before a
// step is the checkpoint's times exp(-sigma_t * step * k * prefix).
// Checkpoints and segment buffers live
// in dynamic shared memory laid out [slot][thread], so every access is
// conflict-free and nothing is kept in local memory.  d loss / d density at the primary sample and d loss /
// d optical depth toward the sun are scattered into the gradient grid with
// atomic adds over the trilinear weights of the primary sample and of the
// six light taps.  Loss and d loss / d density_scale are reduced per CTA and
// added in double.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include "march_fast_body.cuh"

namespace psc {
namespace {

constexpr int kTileW = 16;
constexpr int kTileH = 8;
constexpr int kThreads = 128;
constexpr int kAdjointCtasDefault = 5;  // see adjoint_ctas_per_sm
constexpr int kMaxCp = 32;   // checkpoints per ray
constexpr int kMaxSeg = 32;  // steps per checkpoint segment

// Shared-memory words per thread of the adjoint: three transmittances per
// checkpoint, then a prefix sum, a primary grid value and a light sum per
// step of one segment.
__host__ __device__ constexpr uint32_t adjoint_words(uint32_t n_cp, uint32_t k_cp) {
  return 3u * n_cp + 3u * k_cp;
}

struct Tri {
  int x0, y0, z0;
  float wx, wy, wz;
};

__device__ __forceinline__ Tri grid_coords(const GridDev& g, float x, float alt, float z) {
  Tri t;
  const float fx = fmaf(x - g.min_x, g.inv_cell_x, -0.5f);
  const float fy = fmaf(alt - g.base, g.inv_cell_y, -0.5f);
  const float fz = fmaf(z - g.min_z, g.inv_cell_z, -0.5f);
  const float cx = floorf(fminf(fmaxf(fx, -2.0f), (float)g.nx + 1.0f));
  const float cy = floorf(fminf(fmaxf(fy, -2.0f), (float)g.ny + 1.0f));
  const float cz = floorf(fminf(fmaxf(fz, -2.0f), (float)g.nz + 1.0f));
  t.x0 = (int)cx;
  t.y0 = (int)cy;
  t.z0 = (int)cz;
  t.wx = fx - cx;
  t.wy = fy - cy;
  t.wz = fz - cz;
  return t;
}

// Trilinear fetch without per-corner branches: corner indices clamped into
// the grid (so every load is in bounds) and the weights of corners outside
// it zeroed, which gives the same sum as visiting the in-grid corners only;
// a sample with no corner inside the grid loads nothing.
// The four (x, z) corners of a y row come as one 16-byte quad
// (GridDev::quads, zero outside the grid), so x and z need neither clamping
// nor weight flags: x0 = -1 .. nx-1 and z0 = -1 .. nz-1 have a quad, any
// other no in-grid corner.  The sum equals the clamped per-corner form term
// for term (an outside corner adds weight x 0).
__device__ __forceinline__ float grid_fetch(const GridDev& g, const Tri& t) {
  const bool xin = (uint32_t)(t.x0 + 1) <= g.nx, zin = (uint32_t)(t.z0 + 1) <= g.nz;
  const bool y0 = (uint32_t)t.y0 < g.ny, y1 = (uint32_t)(t.y0 + 1) < g.ny;
  if (!(xin && zin && (y0 || y1))) return 0.0f;
  const float wx0 = 1.0f - t.wx, wx1 = t.wx;
  const float wz0 = 1.0f - t.wz, wz1 = t.wz;
  const float wy[2] = {y0 ? 1.0f - t.wy : 0.0f, y1 ? t.wy : 0.0f};
  const uint32_t k = (uint32_t)(t.x0 + 1), zk = (uint32_t)(t.z0 + 1), stride = g.nx + 1u;
  const uint32_t cy[2] = {(uint32_t)min(max(t.y0, 0), (int)g.ny - 1), (uint32_t)min(max(t.y0 + 1, 0), (int)g.ny - 1)};
  float v = 0.0f;
#pragma unroll
  for (int dy = 0; dy < 2; ++dy) {
    const float4 q = __ldg(g.quads + (cy[dy] * (g.nz + 1u) + zk) * stride + k);
    v = fmaf(wy[dy] * wz0, fmaf(wx1, q.y, wx0 * q.x), v);
    v = fmaf(wy[dy] * wz1, fmaf(wx1, q.w, wx0 * q.z), v);
  }
  return v;
}

// Adds val x the trilinear weights into the gradient grid: the corners'
// in-grid flags, clamped indices and weights as in grid_fetch, one atomic add
// per in-grid corner of non-zero weight (a corner outside the grid has
// weight zero and is skipped).
// (into the pair layout GridDev::grad_pairs: one 8-byte vector atomic add
// per in-grid (y, z) corner pair of non-zero weight; the pair slots outside
// the grid collect weight that the fold ignores)
__device__ __forceinline__ void grid_scatter(const GridDev& g, const Tri& t, float val) {
  if (val == 0.0f) return;
  const bool xin = (uint32_t)(t.x0 + 1) <= g.nx;
  const bool y0 = (uint32_t)t.y0 < g.ny, y1 = (uint32_t)(t.y0 + 1) < g.ny;
  const bool z0 = (uint32_t)t.z0 < g.nz, z1 = (uint32_t)(t.z0 + 1) < g.nz;
  if (!(xin && (y0 || y1) && (z0 || z1))) return;
  const float wx0 = (1.0f - t.wx) * val, wx1 = t.wx * val;
  const float wy[2] = {y0 ? 1.0f - t.wy : 0.0f, y1 ? t.wy : 0.0f};
  const float wz[2] = {z0 ? 1.0f - t.wz : 0.0f, z1 ? t.wz : 0.0f};
  const uint32_t k = (uint32_t)(t.x0 + 1), stride = g.nx + 1u;
  const uint32_t cy[2] = {(uint32_t)min(max(t.y0, 0), (int)g.ny - 1), (uint32_t)min(max(t.y0 + 1, 0), (int)g.ny - 1)};
  const uint32_t cz[2] = {(uint32_t)min(max(t.z0, 0), (int)g.nz - 1), (uint32_t)min(max(t.z0 + 1, 0), (int)g.nz - 1)};
#pragma unroll
  for (int dy = 0; dy < 2; ++dy)
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
      const float wyz = wy[dy] * wz[dz];
      if (wyz != 0.0f)
        atomicAdd(g.grad_pairs + (cy[dy] * g.nz + cz[dz]) * stride + k, make_float2(wyz * wx0, wyz * wx1));
    }
}

// Light march geometry (cloud_march.wgsl:543-578).
struct LightGeo {
  float r0, cv, delta;
};

__device__ __forceinline__ LightGeo light_geo(const MarchUniforms& u, const LayerConst& L, float alt,
                                              float ux, float uy, float uz) {
  LightGeo lg;
  lg.r0 = u.planet_r + alt;
  lg.cv = fmaf(ux, u.sun[0], fmaf(uy, u.sun[1], uz * u.sun[2]));
  lg.delta = __fdividef(fmaxf((L.top_m - alt) * u.inv_cos_sun, 1.0f), (float)u.light_steps);
  return lg;
}

__device__ __forceinline__ Tri light_tap(const MarchUniforms& u, const GridDev& g, const LightGeo& lg,
                                         float px3, float py3, float pz3, float alt, uint32_t j) {
  const float t = ((float)j + 0.5f) * lg.delta;
  const float qx = fmaf(u.sun[0], t, px3), qy = fmaf(u.sun[1], t, py3), qz = fmaf(u.sun[2], t, pz3);
  return grid_coords(g, qx, alt_from(u, qx, qy, qz, lg.r0, lg.cv, alt, t), qz);
}

__device__ __forceinline__ float light_sum(const MarchUniforms& u, const GridDev& g, const LightGeo& lg,
                                           float px3, float py3, float pz3, float alt) {
  float s = 0.0f;
  for (uint32_t j = 0; j < u.light_steps; ++j) s += grid_fetch(g, light_tap(u, g, lg, px3, py3, pz3, alt, j));
  return s * lg.delta;
}

// (1 - e^-x) / x with e = e^-x.
__device__ __forceinline__ float phi_of(float x, float e) {
  return fabsf(x) < 0.03f ? fmaf(x, fmaf(x, fmaf(x, -1.0f / 24.0f, 1.0f / 6.0f), -0.5f), 1.0f)
                          : __fdividef(1.0f - e, x);
}

// Per-position lighting of one sample: sun factor per channel (illuminance x
// sun transmittance), octave coefficients (a^n x forward gain x phase_n) and
// the ambient + lightning term.
struct Light {
  float sun[3], amb[3], cf[kMaxOct];
};

__device__ __forceinline__ void lighting(const MarchUniforms& u, const LayerConst& L, const float* coef,
                                         bool cb, float cos_theta, float fwd_gain, float px3, float pz3,
                                         float alt, float ux, float uy, float uz, Light& l) {
  const float h = clamp01((alt - L.base_m) * L.inv_thickness);
  if (cb) {
    const float mt = smoothstepf(0.60f, 0.85f, h);
    const PhaseConst pc = phase_consts_from_d(mixf(L.droplet_um, 50.0f, mt), u.droplet_bias);
#pragma unroll
    for (int n = 0; n < kMaxOct; ++n)
      l.cf[n] = (n < (int)u.octaves) ? u.apow[n] * fwd_gain * phase_with(u, cos_theta, u.cpow[n], pc) : 0.0f;
  } else {
#pragma unroll
    for (int n = 0; n < kMaxOct; ++n) l.cf[n] = coef[n];
  }
  float3 ts, sky;
  lut_lookups(u, alt, ux, uy, uz, ts, sky);
  l.sun[0] = u.sun_illum[0] * ts.x;
  l.sun[1] = u.sun_illum[1] * ts.y;
  l.sun[2] = u.sun_illum[2] * ts.z;
  const float ag = mixf(0.3f, 1.0f, h) * u.ambient;
  float lr = 0.0f, lg = 0.0f, lb = 0.0f;
  if (u.lightning_radius > 0.0f) {
    const float ddx = px3 - u.lightning_origin_x, ddz = pz3 - u.lightning_origin_z;
    const float fo = clamp01(1.0f - sqrtf(ddx * ddx + ddz * ddz) / u.lightning_radius);
    const float wgt = fo * fo * (3.0f - 2.0f * fo);
    lr = u.lightning_rgb[0] * wgt;
    lg = u.lightning_rgb[1] * wgt;
    lb = u.lightning_rgb[2] * wgt;
  }
  l.amb[0] = fmaf(sky.x, ag, lr);
  l.amb[1] = fmaf(sky.y, ag, lg);
  l.amb[2] = fmaf(sky.z, ag, lb);
}

// In-scatter source X(od) = sun(od) * energy(od) + ambient for channel c,
// and (DERIV) its derivative in the light optical depth.
template <bool DERIV>
__device__ __forceinline__ float source(const MarchUniforms& u, const Light& l, float st, int c, float od,
                                        float* dX) {
  float S = 0.0f, dS = 0.0f, B = 1.0f;
#pragma unroll
  for (int n = 0; n < kMaxOct; ++n) {
    if (n < (int)u.octaves) {
      const float e = __expf(-st * od * u.bpow[n]);
      if (n == 0) B = e;
      S = fmaf(l.cf[n], e, S);
      if (DERIV) dS = fmaf(-l.cf[n] * st * u.bpow[n], e, dS);
    }
  }
  S *= l.sun[c];
  const float P = 1.0f - B * B;  // 1 - exp(-2 * sigma_t * od)
  const float ps = u.powder;
  const float E = fmaf(ps, 2.0f * B * P - B, B);
  if (DERIV) {
    dS *= l.sun[c];
    const float dB = -st * B, dP = 2.0f * st * B * B;
    const float dE = fmaf(ps, 2.0f * (dB * P + B * dP) - dB, dB);
    *dX = fmaf(dS, E, S * dE);
  }
  return fmaf(S, E, l.amb[c]);
}

// `sm` is this thread's column of the adjoint's shared memory (stride
// kThreads words); unused by the forward form.
template <bool ADJ>
__device__ __forceinline__ void grid_pixel(const MarchUniforms& u, const ViewDev& v, const GridDev& g,
                                           uint32_t px, uint32_t py, float* sm, float& loss_out,
                                           float& dk_out) {
  RaySetup rs;
  setup_ray(u, v, px, py, rs);
  const LayerConst& L = u.layers[0];
  const float dx = rs.dir[0], dy = rs.dir[1], dz = rs.dir[2];
  const float cx = u.cam[0], cy = u.cam[1], cz = u.cam[2];
  const float ray_r0 = rs.r0, ray_cv = rs.cos_view, ray_h0 = rs.h0;
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
  const bool cb = L.cloud_type == 7u && u.phase_mode == PSC_PHASE_APPROX_MIE;
  float coef[kMaxOct];
  {
    const PhaseConst pc{L.g_hg, L.g_d, L.alpha, L.w_d, L.ice};
#pragma unroll
    for (int n = 0; n < kMaxOct; ++n) {
      float ph = 0.0f;
      if (n < (int)u.octaves) {
        ph = u.phase_mode == PSC_PHASE_DUAL_LOBE_HG
                 ? mixf(hg_phase(cos_theta, u.hg_f * u.cpow[n]), hg_phase(cos_theta, u.hg_b * u.cpow[n]), u.hg_w)
                 : (cb ? 0.0f : phase_with(u, cos_theta, u.cpow[n], pc));
      }
      coef[n] = u.apow[n] * fwd_gain * ph;
    }
  }
  const float st[3] = {L.sigma_t[0], L.sigma_t[1], L.sigma_t[2]};
  const float ss[3] = {u.sigma_s[0], u.sigma_s[1], u.sigma_s[2]};

  float Lc[3] = {0.0f, 0.0f, 0.0f}, T[3] = {1.0f, 1.0f, 1.0f};
  const float t0 = rs.t0[0], t1 = rs.t1[0];
  const bool hit = (rs.hit_mask & 1u) && t1 > t0;
  const float step = hit ? __fdividef(t1 - t0, (float)u.cloud_steps) : 0.0f;
  const uint32_t kcp = g.k_cp;
  uint32_t n_exec = 0;
  // shared-memory slots: checkpoint transmittances, then the segment's
  // prefix sums, primary grid values and light sums
  float* const s_cp = sm;
  float* const s_pre = sm + 3u * ((u.cloud_steps + kcp - 1u) / kcp) * kThreads;
  float* const s_gv = s_pre + kcp * kThreads;
  float* const s_gl = s_gv + kcp * kThreads;

  auto position = [&](uint32_t s, float& px3, float& py3, float& pz3, float& alt, float& ux, float& uy,
                      float& uz) {
    const float t = fmaf((float)s + jitter, step, t0);
    px3 = fmaf(dx, t, cx);
    py3 = fmaf(dy, t, cy);
    pz3 = fmaf(dz, t, cz);
    alt = alt_from(u, px3, py3, pz3, ray_r0, ray_cv, ray_h0, t);
    const float inv_r = __frcp_rn(u.planet_r + alt);
    ux = px3 * inv_r;
    uy = (py3 + u.planet_r) * inv_r;
    uz = pz3 * inv_r;
  };

  if (hit) {
    for (uint32_t s = 0; s < u.cloud_steps; ++s) {
      if constexpr (ADJ) {
        if (s % kcp == 0) {
          const uint32_t c0 = 3u * (s / kcp) * kThreads;
          s_cp[c0] = T[0];
          s_cp[c0 + kThreads] = T[1];
          s_cp[c0 + 2u * kThreads] = T[2];
        }
      }
      float px3, py3, pz3, alt, ux, uy, uz;
      position(s, px3, py3, pz3, alt, ux, uy, uz);
      const float gv = grid_fetch(g, grid_coords(g, px3, alt, pz3));
      const LightGeo lg = light_geo(u, L, alt, ux, uy, uz);
      const float gl = light_sum(u, g, lg, px3, py3, pz3, alt);
      const float rho = g.k * gv, od = g.k * gl;
      Light l;
      lighting(u, L, coef, cb, cos_theta, fwd_gain, px3, pz3, alt, ux, uy, uz, l);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float X = source<false>(u, l, st[c], c, od, nullptr);
        const float x = rho * st[c] * step;
        const float e = __expf(-x);
        Lc[c] = fmaf(T[c], rho * ss[c] * X * step * phi_of(x, e), Lc[c]);
        T[c] *= e;
      }
      n_exec = s + 1;
      if (fmaxf(T[0], fmaxf(T[1], T[2])) < g.exit_t) break;
    }
  }

  const size_t idx = (size_t)py * v.width + px;
  const float4 lo = make_float4(Lc[0], Lc[1], Lc[2], 1.0f);
  const float4 to = make_float4(T[0], T[1], T[2], 1.0f);
  if (v.out_l) v.out_l[idx] = lo;
  if (v.out_t) v.out_t[idx] = to;
  if constexpr (!ADJ) {
    if (u.composite && v.hdr) {
      const float4 d = v.hdr[idx];
      v.hdr[idx] = make_float4(fmaf(d.x, to.x, lo.x), fmaf(d.y, to.y, lo.y), fmaf(d.z, to.z, lo.z),
                               fmaf(d.w, to.w, lo.w));
    }
  } else {

  // ---- loss term and reverse sweep ----
  const float4 bgp = __ldg(g.bg + idx), tg = __ldg(g.target + idx);
  const float bgc[3] = {bgp.x, bgp.y, bgp.z}, tgc[3] = {tg.x, tg.y, tg.z};
  float gI[3], lam[3], loss = 0.0f;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float d = fmaf(bgc[c], T[c], Lc[c]) - tgc[c];
    loss = fmaf(d * d, g.inv_n, loss);
    gI[c] = 2.0f * d * g.inv_n;
    lam[c] = gI[c] * bgc[c];
  }
  loss_out = loss;
  float dk = 0.0f;
  if (n_exec > 0) {
    const float kstep = g.k * step;
    for (int seg = (int)((n_exec - 1) / kcp); seg >= 0; --seg) {
      const uint32_t s0 = (uint32_t)seg * kcp;
      const uint32_t s1 = min(s0 + kcp, n_exec);
      float pre = 0.0f;
      for (uint32_t s = s0; s < s1; ++s) {  // recompute the segment
        float px3, py3, pz3, alt, ux, uy, uz;
        position(s, px3, py3, pz3, alt, ux, uy, uz);
        const float gv = grid_fetch(g, grid_coords(g, px3, alt, pz3));
        const float gl = light_sum(u, g, light_geo(u, L, alt, ux, uy, uz), px3, py3, pz3, alt);
        const uint32_t b = (s - s0) * kThreads;
        s_pre[b] = pre;
        s_gv[b] = gv;
        s_gl[b] = gl;
        pre += gv;
      }
      const uint32_t c0 = 3u * (uint32_t)seg * kThreads;
      const float cp3[3] = {s_cp[c0], s_cp[c0 + kThreads], s_cp[c0 + 2u * kThreads]};
      for (uint32_t s = s1; s-- > s0;) {  // reverse
        const uint32_t b = (s - s0) * kThreads;
        float px3, py3, pz3, alt, ux, uy, uz;
        position(s, px3, py3, pz3, alt, ux, uy, uz);
        const float gv = s_gv[b], gl = s_gl[b];
        const float p_od = kstep * s_pre[b];  // optical depth per unit sigma_t since the checkpoint
        const float bT[3] = {cp3[0] * __expf(-st[0] * p_od), cp3[1] * __expf(-st[1] * p_od),
                             cp3[2] * __expf(-st[2] * p_od)};
        const float rho = g.k * gv, od = g.k * gl;
        Light l;
        lighting(u, L, coef, cb, cos_theta, fwd_gain, px3, pz3, alt, ux, uy, uz, l);
        float drho = 0.0f, dod = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          float dX;
          const float X = source<true>(u, l, st[c], c, od, &dX);
          const float x = rho * st[c] * step;
          const float e = __expf(-x), ph = phi_of(x, e);
          const float s_int = rho * ss[c] * X * step * ph;
          const float gT = gI[c] * bT[c];
          drho = fmaf(gT, ss[c] * X * step * e, drho);
          drho = fmaf(lam[c] * bT[c], -st[c] * step * e, drho);
          dod = fmaf(gT * rho * ss[c] * step * ph, dX, dod);
          lam[c] = fmaf(lam[c], e, gI[c] * s_int);
        }
        grid_scatter(g, grid_coords(g, px3, alt, pz3), g.k * drho);
        const LightGeo lg = light_geo(u, L, alt, ux, uy, uz);
        const float vl = g.k * lg.delta * dod;
        if (vl != 0.0f)
          for (uint32_t j = 0; j < u.light_steps; ++j)
            grid_scatter(g, light_tap(u, g, lg, px3, py3, pz3, alt, j), vl);
        dk = fmaf(gv, drho, fmaf(gl, dod, dk));
      }
    }
  }
  dk_out = dk;
  }
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// MINB: CTAs per SM the register allocation is bounded for (0: unbounded,
// 96 registers, 5 CTAs per SM).
template <bool ADJ, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) k_grid_march(const __grid_constant__ MarchUniforms u,
                                                               const __grid_constant__ ViewDev v,
                                                               const __grid_constant__ GridDev g) {
  extern __shared__ float s_adj[];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * kTileW + (warp & 1u) * 8u + (lane & 7u);
  const uint32_t py = blockIdx.y * kTileH + (warp >> 1) * 4u + (lane >> 3);
  float loss = 0.0f, dk = 0.0f;
  if (px < v.width && py < v.height) grid_pixel<ADJ>(u, v, g, px, py, s_adj + threadIdx.x, loss, dk);
  if (!ADJ) return;
  __shared__ double s_red[2][kThreads / 32];
  const double ls = warp_sum((double)loss), ks = warp_sum((double)dk);
  if (lane == 0) {
    s_red[0][warp] = ls;
    s_red[1][warp] = ks;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      a += s_red[0][w];
      b += s_red[1][w];
    }
    atomicAdd(g.loss, a);
    atomicAdd(g.grad_scale, b * (double)g.inv_sigma_bar);
  }
}

// The adjoint's CTAs per SM: PSC_ADJOINT_CTAS_PER_SM (5, 6 or 8) overrides
// the measured default, read once per process.
int adjoint_ctas_per_sm() {
  static const int n = [] {
    const char* e = getenv("PSC_ADJOINT_CTAS_PER_SM");
    const int v = e ? atoi(e) : 0;
    return (v == 5 || v == 6 || v == 8) ? v : kAdjointCtasDefault;
  }();
  return n;
}

template <int MINB>
cudaError_t launch_adjoint(const MarchUniforms& u, const ViewDev& v, const GridDev& g, dim3 grid,
                           size_t smem, cudaStream_t s) {
  if (smem > 48u * 1024u) {
    const cudaError_t e = cudaFuncSetAttribute(k_grid_march<true, MINB>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  k_grid_march<true, MINB><<<grid, kThreads, smem, s>>>(u, v, g);
  return cudaGetLastError();
}

__global__ void k_grid_quads(const float* __restrict__ v, float4* __restrict__ q, uint32_t nx, uint32_t ny,
                             uint32_t nz) {
  const uint32_t sx = nx + 1u, sz = nz + 1u;
  const uint64_t n = (uint64_t)ny * sz * sx;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t xk = (uint32_t)(i % sx), zk = (uint32_t)((i / sx) % sz), y = (uint32_t)(i / ((uint64_t)sx * sz));
    auto at = [&](uint32_t z, uint32_t x) {  // z, x shifted by one: 0 is outside
      return (z >= 1u && z <= nz && x >= 1u && x <= nx) ? __ldg(v + ((size_t)y * nz + (z - 1u)) * nx + (x - 1u)) : 0.0f;
    };
    q[i] = make_float4(at(zk, xk), at(zk, xk + 1u), at(zk + 1u, xk), at(zk + 1u, xk + 1u));
  }
}

__global__ void k_grid_fold(const float2* __restrict__ gp, float* __restrict__ grad, uint32_t nx, uint32_t rows) {
  const uint64_t n = (uint64_t)rows * nx;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(i / nx), x = (uint32_t)(i % nx);
    const float2* row = gp + (size_t)r * (nx + 1u);
    grad[i] += __ldg(row + x + 1u).x + __ldg(row + x).y;
  }
}

}  // namespace

int launch_grid_quads(const float* values, float4* quads, uint32_t nx, uint32_t ny, uint32_t nz, cudaStream_t s) {
  k_grid_quads<<<148u * 8u, 256, 0, s>>>(values, quads, nx, ny, nz);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_grid_fold(const float2* grad_pairs, float* grad, uint32_t nx, uint32_t rows, cudaStream_t s) {
  k_grid_fold<<<148u * 8u, 256, 0, s>>>(grad_pairs, grad, nx, rows);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_grid_march(const MarchUniforms& u, const ViewDev& v, const GridDev& g, bool adjoint,
                      cudaStream_t s) {
  if (!g.quads || (adjoint && !g.grad_pairs)) return PSC_ERR_INVALID_ARGUMENT;
  if (u.octaves == 0 || u.octaves > (uint32_t)kMaxOct) return PSC_ERR_UNSUPPORTED;
  if (adjoint && (g.k_cp == 0 || g.k_cp > (uint32_t)kMaxSeg ||
                  (u.cloud_steps + g.k_cp - 1) / g.k_cp > (uint32_t)kMaxCp))
    return PSC_ERR_INVALID_ARGUMENT;
  const dim3 grid((v.width + kTileW - 1) / kTileW, (v.height + kTileH - 1) / kTileH);
  if (adjoint) {
    // at most 3 x 32 + 3 x 32 words per thread (96 KiB per CTA)
    const uint32_t n_cp = (u.cloud_steps + g.k_cp - 1) / g.k_cp;
    const size_t smem = (size_t)adjoint_words(n_cp, g.k_cp) * kThreads * sizeof(float);
    const int ctas = adjoint_ctas_per_sm();
    const cudaError_t e = ctas == 8   ? launch_adjoint<8>(u, v, g, grid, smem, s)
                          : ctas == 6 ? launch_adjoint<6>(u, v, g, grid, smem, s)
                                      : launch_adjoint<0>(u, v, g, grid, smem, s);
    return e == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
  }
  k_grid_march<false, 0><<<grid, kThreads, 0, s>>>(u, v, g);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

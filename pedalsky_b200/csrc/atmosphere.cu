// Atmosphere LUT bakes the cloud march samples, on the device:
//   transmittance 256x64   (shaders/atmosphere/transmittance.comp.wgsl:18-31)
//   multi-scatter 32x32    (shaders/atmosphere/multiscatter.comp.wgsl:36-126)
//   sky-view     192x108   (shaders/atmosphere/skyview.comp.wgsl:47-174)
//   aerial persp. 32x32x64 (shaders/atmosphere/aerialperspective.comp.wgsl:42-127)
// with the shared helpers of shaders/common/atmosphere.wgsl:23-214 and
// atmosphere_lut_sampling.wgsl:5-22.  Output is RGBA16F like the reference's
// storage textures, with the float4 copy the march samples written beside it
// (the same RGBA16F-rounded values).  The sky-view and aerial LUTs depend on
// the camera and sun, so they are re-baked per frame; transmittance and
// multi-scatter depend on the world only.
//
// Work split: the sky-view and aerial march of one texel runs on a group of
// lanes, one step per lane (32 and 16), with the transmittance in front of
// each step the group's exclusive prefix product and the luminance the
// group's sum; the multi-scatter texel runs on a 64-thread block, one
// direction per thread, summed over the block.  The sums and products are
// associated differently from the reference's sequential loops (a few FP32
// ulps), far inside the RGBA16F rounding of the output.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "psc_internal.h"

namespace psc {
namespace {

struct Atmo {
  float R, top, hr, hm;
  float3 ray_s, mie_s, mie_a, ozone;
  float oz_c, oz_t, mie_g;
  float3 albedo;
};

__device__ __forceinline__ float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot3(float3 a, float3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
__device__ __forceinline__ float len3(float3 a) { return sqrtf(dot3(a, a)); }
__device__ __forceinline__ float3 exp3(float3 a) { return f3(expf(a.x), expf(a.y), expf(a.z)); }
__device__ __forceinline__ float3 max3s(float3 a, float m) { return f3(fmaxf(a.x, m), fmaxf(a.y, m), fmaxf(a.z, m)); }
__device__ __forceinline__ float clampf(float x, float a, float b) { return fminf(fmaxf(x, a), b); }

__device__ __forceinline__ float3 density(const Atmo& A, float h) {  // atmosphere.wgsl:23-31
  const float r = expf(-h / A.hr);
  const float m = expf(-h / A.hm);
  const float dz = fabsf(h - A.oz_c);
  const float o = fmaxf(0.0f, 1.0f - dz / fmaxf(A.oz_t * 0.5f, 1.0f));
  return f3(r, m, o);
}
__device__ __forceinline__ float3 extinction(const Atmo& A, float h) {
  const float3 d = density(A, h);
  return (A.ray_s * d.x + (A.mie_s + A.mie_a) * d.y) + A.ozone * d.z;
}
__device__ __forceinline__ void scat_pair(const Atmo& A, float h, float3& r, float3& m) {
  const float3 d = density(A, h);
  r = A.ray_s * d.x;
  m = A.mie_s * d.y;
}
__device__ __forceinline__ bool sphere0(float3 ro, float3 rd, float r, float& t0, float& t1) {
  const float b = dot3(ro, rd);
  const float c = dot3(ro, ro) - r * r;
  const float disc = b * b - c;
  if (disc < 0.0f) return false;
  const float sq = sqrtf(disc);
  t0 = -b - sq;
  t1 = -b + sq;
  return true;
}
__device__ __forceinline__ float dist_boundary(const Atmo& A, float3 p, float3 d) {  // :120-135
  float tt0, tt1, tp0, tp1;
  if (!sphere0(p, d, A.top, tt0, tt1)) return 0.0f;
  float tm = tt1;
  if (sphere0(p, d, A.R, tp0, tp1) && tp0 > 0.0f) tm = fminf(tm, tp0);
  return fmaxf(tm, 0.0f);
}

__device__ __forceinline__ float3 texel_rgb(uint2 w) {
  const __half2 lo = *reinterpret_cast<const __half2*>(&w.x), hi = *reinterpret_cast<const __half2*>(&w.y);
  return f3(__low2float(lo), __high2float(lo), __low2float(hi));
}

__device__ float3 sample_rgba16f(const uint16_t* lut, int W, int H, float u, float v) {
  const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const float wx = x - fx, wy = y - fy;
  const int x0 = min(max((int)fx, 0), W - 1), x1 = min(max((int)fx + 1, 0), W - 1);
  const int y0 = min(max((int)fy, 0), H - 1), y1 = min(max((int)fy + 1, 0), H - 1);
  // one 8-byte load per texel (RGBA16F), RGB used
  const uint2* q = reinterpret_cast<const uint2*>(lut);
  const float3 a = texel_rgb(q[y0 * W + x0]), b = texel_rgb(q[y0 * W + x1]);
  const float3 cc = texel_rgb(q[y1 * W + x0]), d = texel_rgb(q[y1 * W + x1]);
  const float ta[3] = {a.x, a.y, a.z}, tb[3] = {b.x, b.y, b.z}, tc[3] = {cc.x, cc.y, cc.z},
              td[3] = {d.x, d.y, d.z};
  float o[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float top = fmaf(wx, tb[c] - ta[c], ta[c]), bot = fmaf(wx, td[c] - tc[c], tc[c]);
    o[c] = fmaf(wy, bot - top, top);
  }
  return f3(o[0], o[1], o[2]);
}

__device__ float3 trans_lut(const Atmo& A, const uint16_t* T, float3 p, float3 dir) {  // lut_sampling:5-22
  float t0, t1;
  if (sphere0(p, dir, A.R, t0, t1) && t0 > 0.0f) return f3(0.0f, 0.0f, 0.0f);
  const float r = len3(p);
  const float H = sqrtf(fmaxf(A.top * A.top - A.R * A.R, 0.0f));
  const float rho = sqrtf(fmaxf(r * r - A.R * A.R, 0.0f));
  float tt0, tt1;
  float d = 0.0f;
  if (sphere0(p, dir, A.top, tt0, tt1)) d = fmaxf(tt1, 0.0f);
  const float d_min = A.top - r, d_max = rho + H;
  const float u = clampf((d - d_min) / fmaxf(d_max - d_min, 1.0f), 0.0f, 1.0f);
  const float v = rho / fmaxf(H, 1.0f);
  return sample_rgba16f(T, 256, 64, u, v);
}

// Texel i of a LUT: RGBA16F into `oh`, the same rounded values as float4
// into `of`.
__device__ __forceinline__ void store_lut(uint16_t* oh, float4* of, int i, float3 v, float a) {
  __half2 lo = __floats2half2_rn(v.x, v.y), hi = __floats2half2_rn(v.z, a);
  uint2 w;
  w.x = *reinterpret_cast<uint32_t*>(&lo);
  w.y = *reinterpret_cast<uint32_t*>(&hi);
  *reinterpret_cast<uint2*>(oh + (size_t)i * 4) = w;
  of[i] = make_float4(__low2float(lo), __high2float(lo), __low2float(hi), __high2float(hi));
}

// Sums, prefix products and broadcasts over a group of G consecutive lanes
// (G = 16 or 32, aligned to G lanes of the warp; every lane of the warp
// takes part).
template <int G>
__device__ __forceinline__ float3 shfl_up3(float3 v, int d) {
  return f3(__shfl_up_sync(0xffffffffu, v.x, d, G), __shfl_up_sync(0xffffffffu, v.y, d, G),
            __shfl_up_sync(0xffffffffu, v.z, d, G));
}
template <int G>
__device__ __forceinline__ float3 sum_group3(float3 v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o, G);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o, G);
    v.z += __shfl_xor_sync(0xffffffffu, v.z, o, G);
  }
  return v;
}
template <int G>
__device__ __forceinline__ float3 lane3(float3 v, int src) {
  return f3(__shfl_sync(0xffffffffu, v.x, src, G), __shfl_sync(0xffffffffu, v.y, src, G),
            __shfl_sync(0xffffffffu, v.z, src, G));
}

__global__ void k_transmittance(const Atmo A, uint16_t* out, float4* out_f) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= 256 || y >= 64) return;
  const float u = ((float)x + 0.5f) / 256.0f, v = ((float)y + 0.5f) / 64.0f;
  const float H = sqrtf(fmaxf(A.top * A.top - A.R * A.R, 0.0f));
  const float rho = v * H;
  const float r = sqrtf(rho * rho + A.R * A.R);
  const float d_min = A.top - r, d_max = rho + H;
  const float d = d_min + u * (d_max - d_min);
  float mu = 1.0f;
  if (d != 0.0f) mu = clampf((H * H - rho * rho - d * d) / fmaxf(2.0f * r * d, 1e-6f), -1.0f, 1.0f);
  const float3 p = f3(0.0f, r, 0.0f);
  const float3 dir = f3(sqrtf(fmaxf(1.0f - mu * mu, 0.0f)), mu, 0.0f);
  // integrate_optical_depth, atmosphere.wgsl:192-214 (40 trapezoid steps)
  float3 od = f3(0.0f, 0.0f, 0.0f);
  const float tmax = dist_boundary(A, p, dir);
  if (tmax > 0.0f) {
    const float dt = tmax / 40.0f;
    const float r0 = len3(p);
    const float cv = dot3(p * (1.0f / fmaxf(r0, 1.0f)), dir);
    const float h0 = r0 - A.R;
    float3 prev = extinction(A, h0);
    for (int i = 1; i <= 40; ++i) {
      const float t = (float)i * dt;
      const float3 pi = p + dir * t;
      const float rd = (2.0f * t * r0 * cv + t * t) / (fmaxf(r0, 1.0f) + len3(pi));
      const float3 cur = extinction(A, h0 + rd);
      od = od + (prev + cur) * 0.5f * dt;
      prev = cur;
    }
  }
  store_lut(out, out_f, y * 256 + x, exp3(od * -1.0f), 1.0f);
}

// One texel per 64-thread block (grid 32 x 32), one of the 64 directions
// per thread, the directions' sums reduced over the block.
__global__ void __launch_bounds__(64) k_multiscatter(const Atmo A, const uint16_t* T, uint16_t* out,
                                                     float4* out_f) {
  const int gx = blockIdx.x, gy = blockIdx.y, di = (int)threadIdx.x;
  const float u = ((float)gx + 0.5f) / 32.0f, v = ((float)gy + 0.5f) / 32.0f;
  const float sc = clampf(u * 2.0f - 1.0f, -1.0f, 1.0f);
  const float ss = sqrtf(fmaxf(1.0f - sc * sc, 0.0f));
  const float r = A.R + v * (A.top - A.R);
  const float3 p0 = f3(0.0f, r, 0.0f), sun = f3(ss, sc, 0.0f);
  const float h0 = r - A.R;
  float3 ld = f3(0, 0, 0), fd = f3(0, 0, 0);
  const float z = 1.0f - 2.0f * ((float)di + 0.5f) / 64.0f;
  const float rr = sqrtf(fmaxf(1.0f - z * z, 0.0f));
  const float fr = (float)di * 0.6180339887498949f;
  const float phi = 2.0f * kPi * (fr - floorf(fr));
  const float3 vd = f3(rr * cosf(phi), rr * sinf(phi), z);
  const float tmax = dist_boundary(A, p0, vd);
  if (tmax > 0.0f) {
    const float dt = tmax / 20.0f;
    const float cv = dot3(p0 * (1.0f / fmaxf(r, 1.0f)), vd);
    float3 tr = f3(1, 1, 1);
    for (int s = 0; s < 20; ++s) {
      const float t = ((float)s + 0.5f) * dt;
      const float3 p = p0 + vd * t;
      const float rdl = (2.0f * t * r * cv + t * t) / (fmaxf(r, 1.0f) + len3(p));
      const float h = h0 + rdl;
      const float3 st = extinction(A, h);
      float3 sr, sm;
      scat_pair(A, h, sr, sm);
      const float3 ssum = sr + sm;
      const float3 trs = exp3(st * -dt);
      const float r_p = r + rdl;
      const float ratio = A.R / r_p;
      float3 vis = f3(0, 0, 0);
      if (dot3(p, sun) / fmaxf(r_p, 1.0f) > -sqrtf(fmaxf(1.0f - ratio * ratio, 0.0f)))
        vis = trans_lut(A, T, p, sun);
      const float3 in_s = ssum * vis;
      const float3 safe = max3s(st, 1e-7f);
      ld = ld + tr * f3((in_s.x - in_s.x * trs.x) / safe.x, (in_s.y - in_s.y * trs.y) / safe.y,
                        (in_s.z - in_s.z * trs.z) / safe.z);
      fd = fd + tr * f3((ssum.x - ssum.x * trs.x) / safe.x, (ssum.y - ssum.y * trs.y) / safe.y,
                        (ssum.z - ssum.z * trs.z) / safe.z);
      tr = tr * trs;
    }
  }
  ld = sum_group3<32>(ld);
  fd = sum_group3<32>(fd);
  __shared__ float3 part[2][2];
  if ((di & 31) == 0) {
    part[di >> 5][0] = ld;
    part[di >> 5][1] = fd;
  }
  __syncthreads();
  if (di != 0) return;
  const float3 l2 = part[0][0] + part[1][0], fms = part[0][1] + part[1][1];
  const float norm = (4.0f * kPi) / 64.0f, inv4pi = 1.0f / (4.0f * kPi);
  const float3 L2 = l2 * norm * inv4pi, F = fms * norm * inv4pi;
  const float3 full = f3(L2.x / (1.0f - clampf(F.x, 0.0f, 0.95f)), L2.y / (1.0f - clampf(F.y, 0.0f, 0.95f)),
                         L2.z / (1.0f - clampf(F.z, 0.0f, 0.95f)));
  store_lut(out, out_f, gy * 32 + gx, full, 1.0f);
}

__device__ __forceinline__ float phase_r(float c) { return (3.0f / (16.0f * kPi)) * (1.0f + c * c); }
__device__ __forceinline__ float phase_m(float c, float g) {
  const float g2 = g * g, den = fmaxf(1.0f + g2 - 2.0f * g * c, 1e-4f);
  return (1.0f - g2) / (4.0f * kPi * (den * sqrtf(den)));
}

// Shared single+multi-scatter march of the sky-view and AP bakes over a
// group of G lanes (G = the step count): lane s of the group takes step s.
// The transmittance in front of a step is the exclusive prefix product of
// the steps' transmittances over the group, the luminance the group's sum of
// each step's term weighted by it; with `stop`, the steps from the first one
// below the ground on add nothing and pass light unchanged (the sequential
// march's break).  Every lane returns the group's luminance and `tr`.
template <int G>
__device__ float3 inscatter_group(const Atmo& A, const uint16_t* T, const uint16_t* MS, float3 p, float r,
                                  float3 vd, float3 sun, float pr, float pm, float dt, bool stop,
                                  float3 illum, float3& tr) {
  const int s = (int)(threadIdx.x & (unsigned)(G - 1));
  const float cv = dot3(p * (1.0f / fmaxf(r, 1.0f)), vd);
  const float h0 = r - A.R;
  const float t = ((float)s + 0.5f) * dt;
  const float3 pi = p + vd * t;
  const float rdl = (2.0f * t * r * cv + t * t) / (fmaxf(r, 1.0f) + len3(pi));
  const float h = h0 + rdl;
  const unsigned below = __ballot_sync(0xffffffffu, stop && h < 0.0f);
  unsigned mine;
  if constexpr (G == 32) {
    mine = below;
  } else {
    mine = (below >> ((threadIdx.x & 31u) & ~(unsigned)(G - 1))) & ((1u << G) - 1u);
  }
  const int first = mine ? __ffs((int)mine) - 1 : G;
  float3 trs = f3(1, 1, 1), term = f3(0, 0, 0);
  if (s < first) {
    const float3 st = extinction(A, h);
    trs = exp3(st * -dt);
    const float3 vis = trans_lut(A, T, pi, sun);
    float3 sr, sm;
    scat_pair(A, h, sr, sm);
    const float3 sun_in = (sr * pr + sm * pm) * vis;
    const float r_p = r + rdl;
    const float hn = clampf(h / fmaxf(A.top - A.R, 1.0f), 0.0f, 1.0f);
    const float scos = clampf(dot3(pi * (1.0f / fmaxf(r_p, 1.0f)), sun), -1.0f, 1.0f);
    const float3 lms = sample_rgba16f(MS, 32, 32, scos * 0.5f + 0.5f, hn);
    const float3 in_s = (sun_in + (sr + sm) * lms) * illum;
    const float3 safe = max3s(st, 1e-7f);
    term = f3((in_s.x - in_s.x * trs.x) / safe.x, (in_s.y - in_s.y * trs.y) / safe.y,
              (in_s.z - in_s.z * trs.z) / safe.z);
  }
  float3 inc = trs;  // inclusive prefix product over the group
#pragma unroll
  for (int off = 1; off < G; off <<= 1) {
    const float3 o = shfl_up3<G>(inc, off);
    if (s >= off) inc = o * inc;
  }
  float3 ex = shfl_up3<G>(inc, 1);
  if (s == 0) ex = f3(1, 1, 1);
  tr = lane3<G>(inc, G - 1);
  return sum_group3<G>(ex * term);
}

struct FrameLite {
  float inv_vp[4][4];
  float3 cam, sun, illum;
};

// Sky-view texel (gx, gy) of frame F, by one warp (32 steps, one per lane).
__device__ float3 skyview_texel(const Atmo& A, const FrameLite& F, const uint16_t* T, const uint16_t* MS,
                                int gx, int gy) {
  const float u = ((float)gx + 0.5f) / 192.0f, v = ((float)gy + 0.5f) / 108.0f;
  float3 p = f3(F.cam.x, F.cam.y + A.R, F.cam.z);
  float r = len3(p);
  if (r < A.R + 1.0f) {
    p = p * ((A.R + 1.0f) / r);
    r = A.R + 1.0f;
  }
  const float zha = kPi - asinf(clampf(A.R / r, 0.0f, 1.0f));
  float vza;
  if (v < 0.5f) {
    const float c = v * 2.0f;
    vza = c * c * zha;
  } else {
    const float c = (v - 0.5f) * 2.0f;
    vza = zha + c * c * (kPi - zha);
  }
  const float az = atan2f(F.sun.x, F.sun.z) + u * 2.0f * kPi;
  const float3 vd = f3(sinf(vza) * sinf(az), cosf(vza), sinf(vza) * cosf(az));
  const float ct = dot3(vd, F.sun);
  const float tmax = dist_boundary(A, p, vd);
  if (tmax <= 0.0f) return f3(0, 0, 0);  // the same for the whole warp
  float3 tr;
  float3 lum = inscatter_group<32>(A, T, MS, p, r, vd, F.sun, phase_r(ct), phase_m(ct, A.mie_g),
                                   tmax / 32.0f, false, f3(1, 1, 1), tr);
  float tp0, tp1;
  if (sphere0(p, vd, A.R, tp0, tp1) && tp0 > 0.0f) {
    const float3 pg = p + vd * tp0;
    const float3 ng = pg * (1.0f / len3(pg));
    const float3 vis = trans_lut(A, T, pg, F.sun);
    const float ndl = fmaxf(dot3(ng, F.sun), 0.0f);
    lum = lum + tr * (A.albedo * (1.0f / 3.14159265f) * ndl * vis);
  }
  return lum;
}

// Aerial-perspective texel `texel` ((gz * 32 + gy) * 32 + gx) of frame F, by
// a group of 16 lanes (16 steps, one per lane); RGB luminance, A the
// luminance-weighted transmittance.
__device__ float4 aerial_texel(const Atmo& A, const FrameLite& F, const uint16_t* T, const uint16_t* MS,
                               int texel) {
  const int gx = texel & 31, gy = (texel >> 5) & 31, gz = texel >> 10;
  const float nx = (((float)gx + 0.5f) / 32.0f) * 2.0f - 1.0f;
  const float ny = -((((float)gy + 0.5f) / 32.0f) * 2.0f - 1.0f);
  float h[4];
#pragma unroll
  for (int rr = 0; rr < 4; ++rr)
    h[rr] = ((F.inv_vp[0][rr] * nx + F.inv_vp[1][rr] * ny) + F.inv_vp[2][rr]) + F.inv_vp[3][rr];
  float3 vd = f3(h[0] / h[3] - F.cam.x, h[1] / h[3] - F.cam.y, h[2] / h[3] - F.cam.z);
  vd = vd * (1.0f / len3(vd));
  const float zn = ((float)gz + 0.5f) / 64.0f;
  const float t_target = 50.0f * powf(100000.0f / 50.0f, zn);
  const float3 p0 = f3(F.cam.x, F.cam.y + A.R, F.cam.z);
  const float r0 = len3(p0);
  const float ct = dot3(vd, F.sun);
  float3 tr;
  const float3 lum = inscatter_group<16>(A, T, MS, p0, r0, vd, F.sun, phase_r(ct), phase_m(ct, A.mie_g),
                                         t_target / 16.0f, true, F.illum, tr);
  const float tl = (tr.x * 0.2126f + tr.y * 0.7152f) + tr.z * 0.0722f;
  return make_float4(lum.x, lum.y, lum.z, tl);
}

constexpr int kSkyTexels = 192 * 108;      // 2592 blocks of 8 warps
constexpr int kApTexels = 32 * 32 * 64;    // 4096 blocks of 16 lane groups

__global__ void __launch_bounds__(256) k_skyview(const Atmo A, const FrameLite F, const uint16_t* T,
                                                 const uint16_t* MS, uint16_t* out, float4* out_f) {
  const int texel = (int)blockIdx.x * 8 + (int)(threadIdx.x >> 5);
  if (texel >= kSkyTexels) return;  // whole warps
  const float3 lum = skyview_texel(A, F, T, MS, texel % 192, texel / 192);
  if ((threadIdx.x & 31u) == 0) store_lut(out, out_f, texel, lum, 1.0f);
}

__global__ void __launch_bounds__(256) k_aerial(const Atmo A, const FrameLite F, const uint16_t* T,
                                                const uint16_t* MS, uint16_t* out, float4* out_f) {
  const int texel = (int)blockIdx.x * 16 + (int)(threadIdx.x >> 4);
  if (texel >= kApTexels) return;  // whole warps
  const float4 v = aerial_texel(A, F, T, MS, texel);
  if ((threadIdx.x & 15u) == 0) store_lut(out, out_f, texel, f3(v.x, v.y, v.z), v.w);
}

__device__ __forceinline__ float4 f16_rounded(float3 v, float a) {
  return make_float4(__half2float(__float2half_rn(v.x)), __half2float(__float2half_rn(v.y)),
                     __half2float(__float2half_rn(v.z)), __half2float(__float2half_rn(a)));
}

// Per-view sky-view LUTs for a batch (blockIdx.y = view).  Output float4
// holding the RGBA16F-rounded values the single-view path reads.
__global__ void __launch_bounds__(256) k_skyview_batch(const Atmo A, const FrameLite* __restrict__ frames,
                                                       const uint16_t* T, const uint16_t* MS, float4* out) {
  const int texel = (int)blockIdx.x * 8 + (int)(threadIdx.x >> 5);
  if (texel >= kSkyTexels) return;
  const float3 lum = skyview_texel(A, frames[blockIdx.y], T, MS, texel % 192, texel / 192);
  if ((threadIdx.x & 31u) == 0) out[(size_t)blockIdx.y * kSkyTexels + texel] = f16_rounded(lum, 1.0f);
}

// Per-view aerial-perspective LUTs (blockIdx.y = view).
__global__ void __launch_bounds__(256) k_aerial_batch(const Atmo A, const FrameLite* __restrict__ frames,
                                                      const uint16_t* T, const uint16_t* MS, float4* out) {
  const int texel = (int)blockIdx.x * 16 + (int)(threadIdx.x >> 4);
  if (texel >= kApTexels) return;
  const float4 v = aerial_texel(A, frames[blockIdx.y], T, MS, texel);
  if ((threadIdx.x & 15u) == 0)
    out[(size_t)blockIdx.y * kApTexels + texel] = f16_rounded(f3(v.x, v.y, v.z), v.w);
}

Atmo atmo_from(const PscWorldUniformsGpu& w) {
  Atmo A;
  A.R = w.planet_radius_m;
  A.top = w.atmosphere_top_m;
  A.hr = w.rayleigh_scale_height_m;
  A.hm = w.mie_scale_height_m;
  A.ray_s = make_float3(w.rayleigh_scattering[0], w.rayleigh_scattering[1], w.rayleigh_scattering[2]);
  A.mie_s = make_float3(w.mie_scattering[0], w.mie_scattering[1], w.mie_scattering[2]);
  A.mie_a = make_float3(w.mie_absorption[0], w.mie_absorption[1], w.mie_absorption[2]);
  A.ozone = make_float3(w.ozone_absorption[0], w.ozone_absorption[1], w.ozone_absorption[2]);
  A.oz_c = w.ozone_center_m;
  A.oz_t = w.ozone_thickness_m;
  A.mie_g = w.mie_g;
  A.albedo = make_float3(w.ground_albedo[0], w.ground_albedo[1], w.ground_albedo[2]);
  return A;
}

}  // namespace

void frame_lite_from(const PscFrameUniformsGpu& f, void* out) {
  FrameLite F;
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) F.inv_vp[c][r] = f.inv_view_proj[c][r];
  F.cam = make_float3(f.camera_position_world[0], f.camera_position_world[1], f.camera_position_world[2]);
  F.sun = make_float3(f.sun_direction[0], f.sun_direction[1], f.sun_direction[2]);
  F.illum = make_float3(f.sun_illuminance[0], f.sun_illuminance[1], f.sun_illuminance[2]);
  *static_cast<FrameLite*>(out) = F;
}
size_t frame_lite_size() { return sizeof(FrameLite); }

int launch_view_lut_bakes(const PscWorldUniformsGpu& w, const void* d_frames, uint32_t n,
                          const uint16_t* trans, const uint16_t* ms, float4* sky, float4* ap,
                          cudaStream_t s) {
  if (n == 0) return PSC_OK;
  if (n > 65535u) return PSC_ERR_INVALID_ARGUMENT;
  const Atmo A = atmo_from(w);
  const FrameLite* F = static_cast<const FrameLite*>(d_frames);
  k_skyview_batch<<<dim3(kSkyTexels / 8, n), 256, 0, s>>>(A, F, trans, ms, sky);
  k_aerial_batch<<<dim3(kApTexels / 16, n), 256, 0, s>>>(A, F, trans, ms, ap);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_lut_bakes(const PscWorldUniformsGpu& w, const PscFrameUniformsGpu& f, bool statics,
                     uint16_t* const lut_f16[4], float4* const lut_f32[4], cudaStream_t s) {
  const Atmo A = atmo_from(w);
  FrameLite F;
  frame_lite_from(f, &F);
  if (statics) {
    k_transmittance<<<dim3(32, 8), dim3(8, 8), 0, s>>>(A, lut_f16[0], lut_f32[0]);
    k_multiscatter<<<dim3(32, 32), 64, 0, s>>>(A, lut_f16[0], lut_f16[1], lut_f32[1]);
  }
  k_skyview<<<kSkyTexels / 8, 256, 0, s>>>(A, F, lut_f16[0], lut_f16[1], lut_f16[2], lut_f32[2]);
  k_aerial<<<kApTexels / 16, 256, 0, s>>>(A, F, lut_f16[0], lut_f16[1], lut_f16[3], lut_f32[3]);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

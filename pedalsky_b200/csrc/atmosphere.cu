// Atmosphere LUT bakes the cloud march samples, on the device:
//   transmittance 256x64   (shaders/atmosphere/transmittance.comp.wgsl:18-31)
//   multi-scatter 32x32    (shaders/atmosphere/multiscatter.comp.wgsl:36-126)
//   sky-view     192x108   (shaders/atmosphere/skyview.comp.wgsl:47-174)
//   aerial persp. 32x32x64 (shaders/atmosphere/aerialperspective.comp.wgsl:42-127)
// with the shared helpers of shaders/common/atmosphere.wgsl:23-214 and
// atmosphere_lut_sampling.wgsl:5-22.  Output is RGBA16F like the reference's
// storage textures.  The sky-view and aerial LUTs depend on the camera and
// sun, so they are re-baked per frame.
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

__device__ float3 sample_rgba16f(const uint16_t* lut, int W, int H, float u, float v) {
  const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const float wx = x - fx, wy = y - fy;
  const int x0 = min(max((int)fx, 0), W - 1), x1 = min(max((int)fx + 1, 0), W - 1);
  const int y0 = min(max((int)fy, 0), H - 1), y1 = min(max((int)fy + 1, 0), H - 1);
  const __half* h = reinterpret_cast<const __half*>(lut);
  float o[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float a = __half2float(h[(y0 * W + x0) * 4 + c]), b = __half2float(h[(y0 * W + x1) * 4 + c]);
    const float cc = __half2float(h[(y1 * W + x0) * 4 + c]), d = __half2float(h[(y1 * W + x1) * 4 + c]);
    const float top = fmaf(wx, b - a, a), bot = fmaf(wx, d - cc, cc);
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

__device__ __forceinline__ void store_h4(uint16_t* o, float3 v, float a) {
  __half2 lo = __floats2half2_rn(v.x, v.y), hi = __floats2half2_rn(v.z, a);
  uint2 w;
  w.x = *reinterpret_cast<uint32_t*>(&lo);
  w.y = *reinterpret_cast<uint32_t*>(&hi);
  *reinterpret_cast<uint2*>(o) = w;
}

__global__ void k_transmittance(const Atmo A, uint16_t* out) {
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
  store_h4(out + (y * 256 + x) * 4, exp3(od * -1.0f), 1.0f);
}

__global__ void k_multiscatter(const Atmo A, const uint16_t* T, uint16_t* out) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= 32 || gy >= 32) return;
  const float u = ((float)gx + 0.5f) / 32.0f, v = ((float)gy + 0.5f) / 32.0f;
  const float sc = clampf(u * 2.0f - 1.0f, -1.0f, 1.0f);
  const float ss = sqrtf(fmaxf(1.0f - sc * sc, 0.0f));
  const float r = A.R + v * (A.top - A.R);
  const float3 p0 = f3(0.0f, r, 0.0f), sun = f3(ss, sc, 0.0f);
  const float h0 = r - A.R;
  float3 l2 = f3(0, 0, 0), fms = f3(0, 0, 0);
  for (int di = 0; di < 64; ++di) {
    const float z = 1.0f - 2.0f * ((float)di + 0.5f) / 64.0f;
    const float rr = sqrtf(fmaxf(1.0f - z * z, 0.0f));
    const float fr = (float)di * 0.6180339887498949f;
    const float phi = 2.0f * kPi * (fr - floorf(fr));
    const float3 vd = f3(rr * cosf(phi), rr * sinf(phi), z);
    const float tmax = dist_boundary(A, p0, vd);
    if (tmax <= 0.0f) continue;
    const float dt = tmax / 20.0f;
    const float cv = dot3(p0 * (1.0f / fmaxf(r, 1.0f)), vd);
    float3 tr = f3(1, 1, 1), ld = f3(0, 0, 0), fd = f3(0, 0, 0);
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
      const float3 one_m = f3(1.0f - trs.x, 1.0f - trs.y, 1.0f - trs.z);
      ld = ld + tr * f3((in_s.x - in_s.x * trs.x) / safe.x, (in_s.y - in_s.y * trs.y) / safe.y,
                        (in_s.z - in_s.z * trs.z) / safe.z);
      fd = fd + tr * f3((ssum.x - ssum.x * trs.x) / safe.x, (ssum.y - ssum.y * trs.y) / safe.y,
                        (ssum.z - ssum.z * trs.z) / safe.z);
      (void)one_m;
      tr = tr * trs;
    }
    l2 = l2 + ld;
    fms = fms + fd;
  }
  const float norm = (4.0f * kPi) / 64.0f, inv4pi = 1.0f / (4.0f * kPi);
  const float3 L2 = l2 * norm * inv4pi, F = fms * norm * inv4pi;
  const float3 full = f3(L2.x / (1.0f - clampf(F.x, 0.0f, 0.95f)), L2.y / (1.0f - clampf(F.y, 0.0f, 0.95f)),
                         L2.z / (1.0f - clampf(F.z, 0.0f, 0.95f)));
  store_h4(out + (gy * 32 + gx) * 4, full, 1.0f);
}

__device__ __forceinline__ float phase_r(float c) { return (3.0f / (16.0f * kPi)) * (1.0f + c * c); }
__device__ __forceinline__ float phase_m(float c, float g) {
  const float g2 = g * g, den = fmaxf(1.0f + g2 - 2.0f * g * c, 1e-4f);
  return (1.0f - g2) / (4.0f * kPi * (den * sqrtf(den)));
}

// Shared single+multi-scatter march of the sky-view and AP bakes.
__device__ float3 inscatter(const Atmo& A, const uint16_t* T, const uint16_t* MS, float3 p, float r,
                            float3 vd, float3 sun, float pr, float pm, float dt, int n, bool stop,
                            float3 illum, float3& tr) {
  const float cv = dot3(p * (1.0f / fmaxf(r, 1.0f)), vd);
  const float h0 = r - A.R;
  float3 lum = f3(0, 0, 0);
  tr = f3(1, 1, 1);
  for (int s = 0; s < n; ++s) {
    const float t = ((float)s + 0.5f) * dt;
    const float3 pi = p + vd * t;
    const float rdl = (2.0f * t * r * cv + t * t) / (fmaxf(r, 1.0f) + len3(pi));
    const float h = h0 + rdl;
    if (stop && h < 0.0f) break;
    const float3 st = extinction(A, h);
    const float3 trs = exp3(st * -dt);
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
    lum = lum + tr * f3((in_s.x - in_s.x * trs.x) / safe.x, (in_s.y - in_s.y * trs.y) / safe.y,
                        (in_s.z - in_s.z * trs.z) / safe.z);
    tr = tr * trs;
  }
  return lum;
}

struct FrameLite {
  float inv_vp[4][4];
  float3 cam, sun, illum;
};

__global__ void k_skyview(const Atmo A, const FrameLite F, const uint16_t* T, const uint16_t* MS,
                          uint16_t* out) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= 192 || gy >= 108) return;
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
  uint16_t* o = out + (gy * 192 + gx) * 4;
  if (tmax <= 0.0f) {
    store_h4(o, f3(0, 0, 0), 1.0f);
    return;
  }
  float3 tr;
  float3 lum = inscatter(A, T, MS, p, r, vd, F.sun, phase_r(ct), phase_m(ct, A.mie_g), tmax / 32.0f,
                         32, false, f3(1, 1, 1), tr);
  float tp0, tp1;
  if (sphere0(p, vd, A.R, tp0, tp1) && tp0 > 0.0f) {
    const float3 pg = p + vd * tp0;
    const float3 ng = pg * (1.0f / len3(pg));
    const float3 vis = trans_lut(A, T, pg, F.sun);
    const float ndl = fmaxf(dot3(ng, F.sun), 0.0f);
    lum = lum + tr * (A.albedo * (1.0f / 3.14159265f) * ndl * vis);
  }
  store_h4(o, lum, 1.0f);
}

__global__ void k_aerial(const Atmo A, const FrameLite F, const uint16_t* T, const uint16_t* MS,
                         uint16_t* out) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  const int gz = blockIdx.z * blockDim.z + threadIdx.z;
  if (gx >= 32 || gy >= 32 || gz >= 64) return;
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
  const float3 lum = inscatter(A, T, MS, p0, r0, vd, F.sun, phase_r(ct), phase_m(ct, A.mie_g),
                               t_target / 16.0f, 16, true, F.illum, tr);
  const float tl = (tr.x * 0.2126f + tr.y * 0.7152f) + tr.z * 0.0722f;
  store_h4(out + ((gz * 32 + gy) * 32 + gx) * 4, lum, tl);
}

__device__ __forceinline__ float4 f16_rounded(float3 v, float a) {
  return make_float4(__half2float(__float2half_rn(v.x)), __half2float(__float2half_rn(v.y)),
                     __half2float(__float2half_rn(v.z)), __half2float(__float2half_rn(a)));
}

// Per-view sky-view LUTs for a batch (blockIdx.z = view).  Output float4
// holding the RGBA16F-rounded values the single-view path reads.
__global__ void k_skyview_batch(const Atmo A, const FrameLite* __restrict__ frames,
                                const uint16_t* T, const uint16_t* MS, float4* out) {
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  if (gx >= 192 || gy >= 108) return;
  const FrameLite& F = frames[blockIdx.z];
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
  float4* o = out + (size_t)blockIdx.z * (192 * 108) + gy * 192 + gx;
  if (tmax <= 0.0f) {
    *o = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    return;
  }
  float3 tr;
  float3 lum = inscatter(A, T, MS, p, r, vd, F.sun, phase_r(ct), phase_m(ct, A.mie_g), tmax / 32.0f,
                         32, false, f3(1, 1, 1), tr);
  float tp0, tp1;
  if (sphere0(p, vd, A.R, tp0, tp1) && tp0 > 0.0f) {
    const float3 pg = p + vd * tp0;
    const float3 ng = pg * (1.0f / len3(pg));
    const float3 vis = trans_lut(A, T, pg, F.sun);
    const float ndl = fmaxf(dot3(ng, F.sun), 0.0f);
    lum = lum + tr * (A.albedo * (1.0f / 3.14159265f) * ndl * vis);
  }
  *o = f16_rounded(lum, 1.0f);
}

// Per-view aerial-perspective LUTs (blockIdx.z = view * 16 + z block).
__global__ void k_aerial_batch(const Atmo A, const FrameLite* __restrict__ frames, const uint16_t* T,
                               const uint16_t* MS, float4* out) {
  const int view = blockIdx.z / 16;
  const int gx = blockIdx.x * blockDim.x + threadIdx.x, gy = blockIdx.y * blockDim.y + threadIdx.y;
  const int gz = (blockIdx.z % 16) * blockDim.z + threadIdx.z;
  if (gx >= 32 || gy >= 32 || gz >= 64) return;
  const FrameLite& F = frames[view];
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
  const float3 lum = inscatter(A, T, MS, p0, r0, vd, F.sun, phase_r(ct), phase_m(ct, A.mie_g),
                               t_target / 16.0f, 16, true, F.illum, tr);
  const float tl = (tr.x * 0.2126f + tr.y * 0.7152f) + tr.z * 0.0722f;
  out[(size_t)view * (32 * 32 * 64) + (gz * 32 + gy) * 32 + gx] = f16_rounded(lum, tl);
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
  const Atmo A = atmo_from(w);
  const FrameLite* F = static_cast<const FrameLite*>(d_frames);
  k_skyview_batch<<<dim3(24, 14, n), dim3(8, 8), 0, s>>>(A, F, trans, ms, sky);
  k_aerial_batch<<<dim3(8, 8, 16 * n), dim3(4, 4, 4), 0, s>>>(A, F, trans, ms, ap);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_lut_bakes(const PscWorldUniformsGpu& w, const PscFrameUniformsGpu& f, uint16_t* trans,
                     uint16_t* ms, uint16_t* sky, uint16_t* ap, cudaStream_t s) {
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
  FrameLite F;
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) F.inv_vp[c][r] = f.inv_view_proj[c][r];
  F.cam = make_float3(f.camera_position_world[0], f.camera_position_world[1], f.camera_position_world[2]);
  F.sun = make_float3(f.sun_direction[0], f.sun_direction[1], f.sun_direction[2]);
  F.illum = make_float3(f.sun_illuminance[0], f.sun_illuminance[1], f.sun_illuminance[2]);
  k_transmittance<<<dim3(32, 8), dim3(8, 8), 0, s>>>(A, trans);
  k_multiscatter<<<dim3(4, 4), dim3(8, 8), 0, s>>>(A, trans, ms);
  k_skyview<<<dim3(24, 14), dim3(8, 8), 0, s>>>(A, F, trans, ms, sky);
  k_aerial<<<dim3(8, 8, 16), dim3(4, 4, 4), 0, s>>>(A, F, trans, ms, ap);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

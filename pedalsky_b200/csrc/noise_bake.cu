// Noise-volume bakes on the device: base shape 128^3 RGBA8, detail 32^3
// RGBA8, curl 128^2 RG8 (shaders/clouds/noise_base.comp.wgsl,
// noise_detail.comp.wgsl, noise_curl.comp.wgsl), and the conversion of the
// RGBA8 volumes into the march's storage forms.
//
// This file is compiled with -fmad=false: every FP32 operation rounds on its
// own, in the order written, so the output is byte-identical to a CPU bake
// that evaluates the same expressions in IEEE binary32 (division and sqrt are
// IEEE-rounded by default).  WGSL built-ins are spelled out the same way:
// length(v) = sqrt((x*x + y*y) + z*z), normalize(v) = v / length(v),
// mix(a, b, t) = a*(1-t) + b*t, dot = (a.x*b.x + a.y*b.y) + a.z*b.z.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "psc_internal.h"

namespace psc {
namespace {

__device__ __forceinline__ uint32_t hash3(uint32_t x, uint32_t y, uint32_t z) {
  uint32_t h = x * 0x27d4eb2du + y * 0x165667b1u + z * 0x9e3779b9u;
  h = (h ^ (h >> 15)) * 0x2c1b3c6du;
  h = (h ^ (h >> 12)) * 0x297a2d39u;
  return h ^ (h >> 15);
}
__device__ __forceinline__ float unit16(uint32_t h) { return (float)(h & 0xffffu) / 65535.0f; }
__device__ __forceinline__ uint32_t wrapc(int32_t c, int32_t f) {
  return (uint32_t)(((c % f) + f) % f);
}
__device__ __forceinline__ float len3(float x, float y, float z) {
  const float xx = x * x, yy = y * y, zz = z * z;
  return sqrtf((xx + yy) + zz);
}
__device__ __forceinline__ float mixw(float a, float b, float t) { return a * (1.0f - t) + b * t; }
__device__ __forceinline__ float fade(float t) {
  return ((t * t) * t) * (t * (t * 6.0f - 15.0f) + 10.0f);
}
__device__ __forceinline__ uint8_t to_unorm8(float v) {
  return (uint8_t)rintf(fminf(fmaxf(v, 0.0f), 1.0f) * 255.0f);
}

// Worley cell noise, 27 neighbours, tileable at `freq` (noise_base:45-70).
__device__ float worley(float px, float py, float pz, uint32_t freq, bool detail_offset) {
  const float fq = (float)freq;
  const float sx = px * fq, sy = py * fq, sz = pz * fq;
  const float flx = floorf(sx), fly = floorf(sy), flz = floorf(sz);
  const int32_t cx = (int32_t)flx, cy = (int32_t)fly, cz = (int32_t)flz;
  const float fx = sx - flx, fy = sy - fly, fz = sz - flz;
  const int32_t f = (int32_t)freq;
  float min_d = 1.0f;
  for (int32_t dz = -1; dz <= 1; ++dz)
    for (int32_t dy = -1; dy <= 1; ++dy)
      for (int32_t dx = -1; dx <= 1; ++dx) {
        uint32_t wx = wrapc(cx + dx, f), wy = wrapc(cy + dy, f), wz = wrapc(cz + dz, f);
        if (detail_offset) {  // noise_detail.comp.wgsl:49
          wx += 73u;
          wy += 19u;
          wz += 41u;
        }
        const float jx = unit16(hash3(wx, wy, wz));
        const float jy = unit16(hash3(wx + 1u, wy, wz));
        const float jz = unit16(hash3(wx, wy + 1u, wz));
        const float d = len3(((float)dx + jx) - fx, ((float)dy + jy) - fy, ((float)dz + jz) - fz);
        min_d = fminf(min_d, d);
      }
  return fminf(fmaxf(1.0f - min_d, 0.0f), 1.0f);
}

__device__ float worley_fbm(float x, float y, float z, uint32_t f, bool off) {
  const float a = worley(x, y, z, f, off);
  const float b = worley(x, y, z, f * 2u, off);
  const float c = worley(x, y, z, f * 4u, off);
  return (a * 0.625f + b * 0.25f) + c * 0.125f;
}

__device__ float perlin3(float px, float py, float pz, uint32_t freq) {  // noise_base:92-115
  const float fq = (float)freq;
  const float sx = px * fq, sy = py * fq, sz = pz * fq;
  const float flx = floorf(sx), fly = floorf(sy), flz = floorf(sz);
  const int32_t cx = (int32_t)flx, cy = (int32_t)fly, cz = (int32_t)flz;
  const float fx = sx - flx, fy = sy - fly, fz = sz - flz;
  const float ux = fade(fx), uy = fade(fy), uz = fade(fz);
  const int32_t f = (int32_t)freq;
  float dots[8];
#pragma unroll
  for (int iz = 0; iz < 2; ++iz)
#pragma unroll
    for (int iy = 0; iy < 2; ++iy)
#pragma unroll
      for (int ix = 0; ix < 2; ++ix) {
        const uint32_t wx = wrapc(cx + ix, f), wy = wrapc(cy + iy, f), wz = wrapc(cz + iz, f);
        const float vx = unit16(hash3(wx, wy, wz)) * 2.0f - 1.0f;
        const float vy = unit16(hash3(wx + 1u, wy, wz)) * 2.0f - 1.0f;
        const float vz = unit16(hash3(wx, wy + 1u, wz)) * 2.0f - 1.0f;
        const float l = len3(vx, vy, vz);
        const float gx = vx / l, gy = vy / l, gz = vz / l;
        const float ddx = fx - (float)ix, ddy = fy - (float)iy, ddz = fz - (float)iz;
        dots[ix + iy * 2 + iz * 4] = (gx * ddx + gy * ddy) + gz * ddz;
      }
  const float x00 = mixw(dots[0], dots[1], ux), x10 = mixw(dots[2], dots[3], ux);
  const float x01 = mixw(dots[4], dots[5], ux), x11 = mixw(dots[6], dots[7], ux);
  const float y0 = mixw(x00, x10, uy), y1 = mixw(x01, x11, uy);
  return mixw(y0, y1, uz) * 0.5f + 0.5f;
}

__global__ void k_bake_base(uint8_t* __restrict__ out) {  // noise_base.comp.wgsl:124-139
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= 128u || y >= 128u || z >= 128u) return;
  const float px = ((float)x + 0.5f) / 128.0f, py = ((float)y + 0.5f) / 128.0f,
              pz = ((float)z + 0.5f) / 128.0f;
  const float p1 = perlin3(px, py, pz, 4u), p2 = perlin3(px, py, pz, 8u),
              p3 = perlin3(px, py, pz, 16u);
  const float perlin = (p1 * 0.5f + p2 * 0.25f) + p3 * 0.125f;
  const float wl = worley_fbm(px, py, pz, 4u, false);
  const float a = wl - 1.0f;
  const float pw = fminf(fmaxf(0.0f + ((perlin - a) * (1.0f - 0.0f)) / fmaxf(1.0f - a, 1e-5f), 0.0f), 1.0f);
  uchar4 t;
  t.x = to_unorm8(pw);
  t.y = to_unorm8(worley_fbm(px, py, pz, 2u, false));
  t.z = to_unorm8(worley_fbm(px, py, pz, 8u, false));
  t.w = to_unorm8(worley_fbm(px, py, pz, 14u, false));
  reinterpret_cast<uchar4*>(out)[(z * 128u + y) * 128u + x] = t;
}

__global__ void k_bake_detail(uint8_t* __restrict__ out) {  // noise_detail.comp.wgsl:62-72
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= 32u || y >= 32u || z >= 32u) return;
  const float px = ((float)x + 0.5f) / 32.0f, py = ((float)y + 0.5f) / 32.0f,
              pz = ((float)z + 0.5f) / 32.0f;
  uchar4 t;
  t.x = to_unorm8(worley_fbm(px, py, pz, 2u, true));
  t.y = to_unorm8(worley_fbm(px, py, pz, 8u, true));
  t.z = to_unorm8(worley_fbm(px, py, pz, 16u, true));
  t.w = 0;
  reinterpret_cast<uchar4*>(out)[(z * 32u + y) * 32u + x] = t;
}

__device__ __forceinline__ uint32_t hash2(uint32_t x, uint32_t y) {
  uint32_t h = x * 0x27d4eb2du + y * 0x165667b1u;
  h = (h ^ (h >> 15)) * 0x2c1b3c6du;
  h = (h ^ (h >> 12)) * 0x297a2d39u;
  return h ^ (h >> 15);
}

__device__ float perlin2(float px, float py, uint32_t freq) {  // noise_curl.comp.wgsl:36-56
  const float fq = (float)freq;
  const float sx = px * fq, sy = py * fq;
  const float flx = floorf(sx), fly = floorf(sy);
  const int32_t cx = (int32_t)flx, cy = (int32_t)fly;
  const float fx = sx - flx, fy = sy - fly;
  const float ux = fade(fx), uy = fade(fy);
  const int32_t f = (int32_t)freq;
  float d[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int ox = k & 1, oy = k >> 1;
    const uint32_t wx = wrapc(cx + ox, f), wy = wrapc(cy + oy, f);
    const float rx = (float)(hash2(wx, wy) & 0xffffu) / 65535.0f * 2.0f - 1.0f;
    const float ry = (float)(hash2(wx + 1u, wy) & 0xffffu) / 65535.0f * 2.0f - 1.0f;
    const float l = sqrtf(rx * rx + ry * ry);
    d[k] = (rx / l) * (fx - (float)ox) + (ry / l) * (fy - (float)oy);
  }
  const float x0 = mixw(d[0], d[1], ux), x1 = mixw(d[2], d[3], ux);
  return mixw(x0, x1, uy);
}

__device__ __forceinline__ float potential(float x, float y) {
  return perlin2(x, y, 4u) + 0.5f * perlin2(x, y, 8u);
}

__global__ void k_bake_curl(uint8_t* __restrict__ out) {  // noise_curl.comp.wgsl:62-74
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= 128u || y >= 128u) return;
  const float px = ((float)x + 0.5f) / 128.0f, py = ((float)y + 0.5f) / 128.0f;
  const float eps = 1.0f / 128.0f;
  const float dpdx = (potential(px + eps, py + 0.0f) - potential(px - eps, py - 0.0f)) / (2.0f * eps);
  const float dpdy = (potential(px + 0.0f, py + eps) - potential(px - 0.0f, py - eps)) / (2.0f * eps);
  const float cx = dpdy, cy = -dpdx;
  out[(y * 128u + x) * 2u + 0u] = to_unorm8(fminf(fmaxf(cx * 0.5f + 0.5f, 0.0f), 1.0f));
  out[(y * 128u + x) * 2u + 1u] = to_unorm8(fminf(fmaxf(cy * 0.5f + 0.5f, 0.0f), 1.0f));
}

// RGBA8 texels -> storage form.  F16/BF16 hold the byte value itself
// (integers 0..255 are exact in both); FP8 e4m3 holds v/255 * fp8_scale.
__global__ void k_convert(const uint32_t* __restrict__ src, void* __restrict__ dst, uint32_t n,
                          int storage, float fp8_scale) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t w = src[i];
  const float c[4] = {(float)(w & 0xffu), (float)((w >> 8) & 0xffu), (float)((w >> 16) & 0xffu),
                      (float)(w >> 24)};
  if (storage == PSC_STORAGE_F32) {
    reinterpret_cast<float4*>(dst)[i] =
        make_float4(c[0] / 255.0f, c[1] / 255.0f, c[2] / 255.0f, c[3] / 255.0f);
  } else if (storage == PSC_STORAGE_F16) {
    __half2 a = __floats2half2_rn(c[0], c[1]), b = __floats2half2_rn(c[2], c[3]);
    uint2 o;
    o.x = *reinterpret_cast<uint32_t*>(&a);
    o.y = *reinterpret_cast<uint32_t*>(&b);
    reinterpret_cast<uint2*>(dst)[i] = o;
  } else if (storage == PSC_STORAGE_BF16) {
    __nv_bfloat162 a = __floats2bfloat162_rn(c[0], c[1]), b = __floats2bfloat162_rn(c[2], c[3]);
    uint2 o;
    o.x = *reinterpret_cast<uint32_t*>(&a);
    o.y = *reinterpret_cast<uint32_t*>(&b);
    reinterpret_cast<uint2*>(dst)[i] = o;
  } else if (storage == PSC_STORAGE_FP8) {
    uint32_t o = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const __nv_fp8_e4m3 q(c[k] / 255.0f * fp8_scale);
      o |= (uint32_t)(*reinterpret_cast<const uint8_t*>(&q)) << (8 * k);
    }
    reinterpret_cast<uint32_t*>(dst)[i] = o;
  } else {
    reinterpret_cast<uint32_t*>(dst)[i] = w;
  }
}

// Channel-folded FP16 forms of the noise volumes, read by the FAST schedule.
// The march uses the base volume only through R and the low-frequency fbm
// 0.625 G + 0.25 B + 0.125 A, and the detail volume only through
// 0.625 R + 0.25 G + 0.125 B (cloud_march.wgsl:463-470, 512-515).  Filtering
// is linear, so filtering the folded channel equals folding the filtered
// channels.  On bytes the folds are integers: base (R, 5G + 2B + A) and
// detail 5R + 2G + B, at most 2040, which FP16 holds exactly; the kernels
// rescale by 1/255 and 1/2040 after filtering.
//   fold: one texel per entry (source of the texture arrays);
//   quad: the 2x2 footprint (x, x+1) x (y, y+1) of slab z, repeat-wrapped,
//         per entry, so an exact trilinear tap is one load per slab.
__device__ __forceinline__ uint32_t fold_base_texel(uint32_t w) {
  const uint32_t r = w & 0xffu, g = (w >> 8) & 0xffu, b = (w >> 16) & 0xffu, a = w >> 24;
  const __half2 h = __floats2half2_rn((float)r, (float)(5u * g + 2u * b + a));
  return *reinterpret_cast<const uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t fold_detail_texel(uint32_t w) {
  const uint32_t r = w & 0xffu, g = (w >> 8) & 0xffu, b = (w >> 16) & 0xffu;
  return __half_as_ushort(__float2half_rn((float)(5u * r + 2u * g + b)));
}

template <uint32_t N>
__global__ void k_fold_base(const uint32_t* __restrict__ src, uint32_t* __restrict__ fold,
                            uint4* __restrict__ quad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * N * N) return;
  const uint32_t x = i % N, y = (i / N) % N, z = i / (N * N);
  const uint32_t x1 = (x + 1u) & (N - 1u), y1 = (y + 1u) & (N - 1u);
  const uint32_t row0 = (z * N + y) * N, row1 = (z * N + y1) * N;
  fold[i] = fold_base_texel(src[i]);
  quad[i] = make_uint4(fold_base_texel(src[row0 + x]), fold_base_texel(src[row0 + x1]),
                       fold_base_texel(src[row1 + x]), fold_base_texel(src[row1 + x1]));
}

template <uint32_t N>
__global__ void k_fold_detail(const uint32_t* __restrict__ src, uint16_t* __restrict__ fold,
                              uint2* __restrict__ quad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N * N * N) return;
  const uint32_t x = i % N, y = (i / N) % N, z = i / (N * N);
  const uint32_t x1 = (x + 1u) & (N - 1u), y1 = (y + 1u) & (N - 1u);
  const uint32_t row0 = (z * N + y) * N, row1 = (z * N + y1) * N;
  fold[i] = (uint16_t)fold_detail_texel(src[i]);
  quad[i] = make_uint2(fold_detail_texel(src[row0 + x]) | (fold_detail_texel(src[row0 + x1]) << 16),
                       fold_detail_texel(src[row1 + x]) | (fold_detail_texel(src[row1 + x1]) << 16));
}

// Curl tile (128^2 RG8) as 2x2 quads of (R, G) half pairs, repeat-wrapped:
// a bilinear curl tap is one 16-byte load.  Bytes are exact in FP16.
__global__ void k_curl_quads(const uint16_t* __restrict__ src, uint4* __restrict__ quad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 128u * 128u) return;
  const uint32_t x = i & 127u, y = i >> 7, x1 = (x + 1u) & 127u, y1 = (y + 1u) & 127u;
  auto pair = [&](uint32_t xx, uint32_t yy) {
    const uint32_t t = src[yy * 128u + xx];
    const __half2 h = __floats2half2_rn((float)(t & 0xffu), (float)(t >> 8));
    return *reinterpret_cast<const uint32_t*>(&h);
  };
  quad[i] = make_uint4(pair(x, y), pair(x1, y), pair(x, y1), pair(x1, y1));
}

}  // namespace

int launch_curl_quads(const uint8_t* curl, uint4* quad, cudaStream_t s) {
  k_curl_quads<<<128u * 128u / 256u, 256, 0, s>>>(reinterpret_cast<const uint16_t*>(curl), quad);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_fold_storage(const uint8_t* base_u8, const uint8_t* detail_u8, uint32_t* base_fold,
                        uint4* base_quad, uint16_t* detail_fold, uint2* detail_quad, cudaStream_t s) {
  k_fold_base<128><<<128u * 128u * 128u / 256u, 256, 0, s>>>(
      reinterpret_cast<const uint32_t*>(base_u8), base_fold, base_quad);
  k_fold_detail<32><<<32u * 32u * 32u / 256u, 256, 0, s>>>(
      reinterpret_cast<const uint32_t*>(detail_u8), detail_fold, detail_quad);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_noise_bakes(uint8_t* base, uint8_t* detail, uint8_t* curl, cudaStream_t s) {
  k_bake_base<<<dim3(32, 32, 32), dim3(4, 4, 4), 0, s>>>(base);
  k_bake_detail<<<dim3(8, 8, 8), dim3(4, 4, 4), 0, s>>>(detail);
  k_bake_curl<<<dim3(16, 16), dim3(8, 8), 0, s>>>(curl);
  if (cudaGetLastError() != cudaSuccess) return PSC_ERR_CUDA;
  return cudaStreamSynchronize(s) == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_convert_storage(const uint8_t* src, void* dst, uint32_t n_texels, int storage,
                           float fp8_scale, cudaStream_t s) {
  k_convert<<<(n_texels + 255) / 256, 256, 0, s>>>(reinterpret_cast<const uint32_t*>(src), dst,
                                                    n_texels, storage, fp8_scale);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

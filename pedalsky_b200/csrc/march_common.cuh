// Device helpers for the cloud march: texel decoding for every noise storage
// form, exact (FP32-weight) and texture-unit filtering, LUT sampling, and the
// density / phase functions of the reference
// (shaders/clouds/cloud_density_common.wgsl, shaders/clouds/cloud_march.wgsl).
//
// Index safety: every texel index is produced by a power-of-two mask, an
// explicit modulo or a clamp, so all loads stay inside their buffers for any
// coordinate value (NaN converts to 0, huge values saturate), which is why
// the kernels carry no per-load bounds checks.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "psc_internal.h"

namespace psc {

// ---------------------------------------------------------------- basics
__device__ __forceinline__ float clamp01(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
__device__ __forceinline__ float clampf(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}
// WGSL smoothstep; e0 > e1 is a reversed ramp (cloud_density_common.wgsl:58).
__device__ __forceinline__ float smoothstepf(float e0, float e1, float x) {
  const float t = clamp01((x - e0) / (e1 - e0));
  return t * t * (3.0f - 2.0f * t);
}
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.0f - t) + b * t; }
// math.wgsl:7-9
__device__ __forceinline__ float remapf(float v, float a, float b, float c, float d) {
  return c + ((v - a) * (d - c)) / fmaxf(b - a, 1e-5f);
}
__device__ __forceinline__ float lerpf(float a, float b, float t) { return fmaf(t, b - a, a); }
__device__ __forceinline__ float4 lerp4(float4 a, float4 b, float t) {
  return make_float4(lerpf(a.x, b.x, t), lerpf(a.y, b.y, t), lerpf(a.z, b.z, t),
                     lerpf(a.w, b.w, t));
}

// Packed FP32x2 arithmetic (sm_100 `fma.rn.f32x2` / `sub.rn.f32x2`): two
// IEEE-rounded lanes per instruction, bit-identical to the scalar forms.
__device__ __forceinline__ unsigned long long f2_bits(float2 v) {
  return *reinterpret_cast<unsigned long long*>(&v);
}
__device__ __forceinline__ float2 bits_f2(unsigned long long b) {
  return *reinterpret_cast<float2*>(&b);
}
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return bits_f2(d);
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)), "l"(f2_bits(c)));
  return bits_f2(d);
}
// fma(t, b - a, a) on two lanes
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 tt) {
  return fma2(tt, sub2(b, a), a);
}
__device__ __forceinline__ float4 lerp4p(float4 a, float4 b, float t) {
  const float2 tt = make_float2(t, t);
  const float2 lo = lerp2(make_float2(a.x, a.y), make_float2(b.x, b.y), tt);
  const float2 hi = lerp2(make_float2(a.z, a.w), make_float2(b.z, b.w), tt);
  return make_float4(lo.x, lo.y, hi.x, hi.y);
}

__device__ __forceinline__ int wrap_mod(int i, int n) {
  int m = i % n;
  return m < 0 ? m + n : m;
}
__device__ __forceinline__ int clamp_idx(int i, int n) { return min(max(i, 0), n - 1); }

// ---------------------------------------------------- debug index checks
// options.debug_checks: every index the PLAIN kernel forms is compared with
// its buffer's extent; a violation records its site code in the device
// word (first one wins) and the access is skipped.  With chk == nullptr
// (every other caller) the test folds away at compile time.
enum CheckSite : int {
  kChkBase = 1, kChkDetail = 2, kChkCurl = 3, kChkWeather = 4, kChkType = 5, kChkTrans = 6,
  kChkSky = 7, kChkAerial = 8, kChkBlue = 9, kChkPixel = 10, kChkLayer = 11
};
__device__ __forceinline__ bool idx_ok(int* chk, bool ok, int site) {
  if (chk != nullptr && !ok) {
    atomicCAS(chk, 0, site);
    return false;
  }
  return true;
}

// ---------------------------------------------------- texel decoding
// Exact unorm8 -> float: the byte placed in the mantissa of 2^23.
__device__ __forceinline__ float byte_to_float(uint32_t word, uint32_t sel) {
  return __int_as_float(__byte_perm(word, 0x4B000000u, sel)) - 8388608.0f;
}
__device__ __forceinline__ float4 unpack_u8x4(uint32_t w) {
  return make_float4(byte_to_float(w, 0x7540u), byte_to_float(w, 0x7541u),
                     byte_to_float(w, 0x7542u), byte_to_float(w, 0x7543u));
}
__device__ __forceinline__ float4 unpack_h4(uint2 w) {
  const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
  const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
  return make_float4(a.x, a.y, b.x, b.y);
}
__device__ __forceinline__ float4 unpack_bf4(uint2 w) {
  return make_float4(__uint_as_float(w.x << 16), __uint_as_float(w.x & 0xffff0000u),
                     __uint_as_float(w.y << 16), __uint_as_float(w.y & 0xffff0000u));
}
__device__ __forceinline__ float4 unpack_e4m3x4(uint32_t w) {
  __nv_fp8x2_e4m3 lo, hi;
  lo.__x = (__nv_fp8x2_storage_t)(w & 0xffffu);
  hi.__x = (__nv_fp8x2_storage_t)(w >> 16);
  const float2 a = static_cast<float2>(lo);
  const float2 b = static_cast<float2>(hi);
  return make_float4(a.x, a.y, b.x, b.y);
}

// Raw texel (before the per-volume scale) for storage form ST.
template <int ST>
__device__ __forceinline__ float4 load_texel(const void* base, uint32_t idx) {
  if constexpr (ST == PSC_STORAGE_U8) {
    return unpack_u8x4(__ldg(reinterpret_cast<const uint32_t*>(base) + idx));
  } else if constexpr (ST == PSC_STORAGE_F32) {
    return __ldg(reinterpret_cast<const float4*>(base) + idx);
  } else if constexpr (ST == PSC_STORAGE_F16) {
    return unpack_h4(__ldg(reinterpret_cast<const uint2*>(base) + idx));
  } else if constexpr (ST == PSC_STORAGE_BF16) {
    return unpack_bf4(__ldg(reinterpret_cast<const uint2*>(base) + idx));
  } else {
    return unpack_e4m3x4(__ldg(reinterpret_cast<const uint32_t*>(base) + idx));
  }
}

template <int ST>
__device__ __forceinline__ float storage_scale(float volume_scale) {
  if constexpr (ST == PSC_STORAGE_F32) return 1.0f;
  else if constexpr (ST == PSC_STORAGE_FP8) return volume_scale;
  else return 1.0f / 255.0f;
}

// Trilinear, repeat addressing, N a power of two; texel centre at u*N - 0.5.
template <int ST, int N>
__device__ __forceinline__ float4 trilinear_repeat(const void* vol, float u, float v, float w,
                                                   float volume_scale, int* chk = nullptr,
                                                   int site = 0) {
  const float x = u * (float)N - 0.5f, y = v * (float)N - 0.5f, z = w * (float)N - 0.5f;
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  const float wx = x - fx, wy = y - fy, wz = z - fz;
  const uint32_t x0 = (uint32_t)ix & (N - 1), x1 = (uint32_t)(ix + 1) & (N - 1);
  const uint32_t y0 = (uint32_t)iy & (N - 1), y1 = (uint32_t)(iy + 1) & (N - 1);
  const uint32_t z0 = (uint32_t)iz & (N - 1), z1 = (uint32_t)(iz + 1) & (N - 1);
  if (!idx_ok(chk, x0 < N && x1 < N && y0 < N && y1 < N && z0 < N && z1 < N, site))
    return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const uint32_t r00 = (z0 * N + y0) * N, r10 = (z0 * N + y1) * N;
  const uint32_t r01 = (z1 * N + y0) * N, r11 = (z1 * N + y1) * N;
  const float4 c000 = load_texel<ST>(vol, r00 + x0), c100 = load_texel<ST>(vol, r00 + x1);
  const float4 c010 = load_texel<ST>(vol, r10 + x0), c110 = load_texel<ST>(vol, r10 + x1);
  const float4 c001 = load_texel<ST>(vol, r01 + x0), c101 = load_texel<ST>(vol, r01 + x1);
  const float4 c011 = load_texel<ST>(vol, r11 + x0), c111 = load_texel<ST>(vol, r11 + x1);
  const float4 a = lerp4(lerp4(c000, c100, wx), lerp4(c010, c110, wx), wy);
  const float4 b = lerp4(lerp4(c001, c101, wx), lerp4(c011, c111, wx), wy);
  float4 r = lerp4(a, b, wz);
  const float s = storage_scale<ST>(volume_scale);
  r.x *= s;
  r.y *= s;
  r.z *= s;
  r.w *= s;
  return r;
}

// Curl: 128^2 RG8, repeat, bilinear.
__device__ __forceinline__ float2 curl_sample(const uint8_t* curl, float u, float v,
                                              int* chk = nullptr) {
  const float x = u * 128.0f - 0.5f, y = v * 128.0f - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const uint32_t x0 = (uint32_t)ix & 127u, x1 = (uint32_t)(ix + 1) & 127u;
  const uint32_t y0 = (uint32_t)iy & 127u, y1 = (uint32_t)(iy + 1) & 127u;
  if (!idx_ok(chk, x0 < 128u && x1 < 128u && y0 < 128u && y1 < 128u, kChkCurl))
    return make_float2(0.5f, 0.5f);
  const uint16_t* c = reinterpret_cast<const uint16_t*>(curl);
  const uint32_t t00 = __ldg(c + y0 * 128 + x0), t10 = __ldg(c + y0 * 128 + x1);
  const uint32_t t01 = __ldg(c + y1 * 128 + x0), t11 = __ldg(c + y1 * 128 + x1);
  const float r = lerpf(lerpf(byte_to_float(t00, 0x7540u), byte_to_float(t10, 0x7540u), wx),
                        lerpf(byte_to_float(t01, 0x7540u), byte_to_float(t11, 0x7540u), wx), wy);
  const float g = lerpf(lerpf(byte_to_float(t00, 0x7541u), byte_to_float(t10, 0x7541u), wx),
                        lerpf(byte_to_float(t01, 0x7541u), byte_to_float(t11, 0x7541u), wx), wy);
  return make_float2(r * (1.0f / 255.0f), g * (1.0f / 255.0f));
}

// Weather R channel: W x H floats, repeat, bilinear.
__device__ __forceinline__ float weather_sample(const float* wm, uint32_t W, uint32_t H, float u,
                                                float v, int* chk = nullptr) {
  const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const int x0 = wrap_mod(ix, (int)W), x1 = wrap_mod(ix + 1, (int)W);
  const int y0 = wrap_mod(iy, (int)H), y1 = wrap_mod(iy + 1, (int)H);
  if (!idx_ok(chk, x0 >= 0 && x1 >= 0 && y0 >= 0 && y1 >= 0 && (uint32_t)x0 < W && (uint32_t)x1 < W &&
                       (uint32_t)y0 < H && (uint32_t)y1 < H, kChkWeather))
    return 0.0f;
  const float a = lerpf(__ldg(wm + y0 * W + x0), __ldg(wm + y0 * W + x1), wx);
  const float b = lerpf(__ldg(wm + y1 * W + x0), __ldg(wm + y1 * W + x1), wx);
  return lerpf(a, b, wy);
}

// RGBA LUT (float4), clamp-to-edge, bilinear.
__device__ __forceinline__ float4 lut2d(const float4* lut, int W, int H, float u, float v,
                                        int* chk = nullptr, int site = 0) {
  const float x = u * (float)W - 0.5f, y = v * (float)H - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const int ix = (int)fx, iy = (int)fy;
  const float wx = x - fx, wy = y - fy;
  const int x0 = clamp_idx(ix, W), x1 = clamp_idx(ix + 1, W);
  const int y0 = clamp_idx(iy, H), y1 = clamp_idx(iy + 1, H);
  if (!idx_ok(chk, x0 >= 0 && x1 < W && y0 >= 0 && y1 < H, site)) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const float4 a = lerp4(__ldg(lut + y0 * W + x0), __ldg(lut + y0 * W + x1), wx);
  const float4 b = lerp4(__ldg(lut + y1 * W + x0), __ldg(lut + y1 * W + x1), wx);
  return lerp4(a, b, wy);
}

// Aerial perspective 32x32x64, clamp-to-edge, trilinear.
__device__ __forceinline__ float4 lut_ap(const float4* lut, float u, float v, float w,
                                         int* chk = nullptr) {
  const float x = u * 32.0f - 0.5f, y = v * 32.0f - 0.5f, z = w * 64.0f - 0.5f;
  const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  const float wx = x - fx, wy = y - fy, wz = z - fz;
  const int x0 = clamp_idx(ix, 32), x1 = clamp_idx(ix + 1, 32);
  const int y0 = clamp_idx(iy, 32), y1 = clamp_idx(iy + 1, 32);
  const int z0 = clamp_idx(iz, 64), z1 = clamp_idx(iz + 1, 64);
  if (!idx_ok(chk, x0 >= 0 && x1 < 32 && y0 >= 0 && y1 < 32 && z0 >= 0 && z1 < 64, kChkAerial))
    return make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  auto at = [&](int xx, int yy, int zz) { return __ldg(lut + (zz * 32 + yy) * 32 + xx); };
  const float4 a = lerp4(lerp4(at(x0, y0, z0), at(x1, y0, z0), wx),
                         lerp4(at(x0, y1, z0), at(x1, y1, z0), wx), wy);
  const float4 b = lerp4(lerp4(at(x0, y0, z1), at(x1, y0, z1), wx),
                         lerp4(at(x0, y1, z1), at(x1, y1, z1), wx), wy);
  return lerp4(a, b, wz);
}

// --------------------------------------------- density profile (NDF)
// cloud_density_common.wgsl:49-91
__device__ __forceinline__ float ndf(float h, uint32_t t, float anvil_bias) {
  switch (t) {
    case 0: return smoothstepf(0.0f, 0.07f, h) * smoothstepf(1.0f, 0.2f, h);
    case 1: return smoothstepf(0.0f, 0.10f, h) * (1.0f - smoothstepf(0.6f, 1.0f, h));
    case 2: return smoothstepf(0.0f, 0.15f, h) * smoothstepf(1.0f, 0.4f, h);
    case 3: return smoothstepf(0.0f, 0.20f, h) * smoothstepf(1.0f, 0.3f, h);
    case 4: return smoothstepf(0.0f, 0.30f, h) * (1.0f - smoothstepf(0.7f, 1.0f, h));
    case 5: return smoothstepf(0.0f, 0.40f, h) * (1.0f - smoothstepf(0.6f, 1.0f, h));
    case 6: return smoothstepf(0.0f, 0.50f, h) * (1.0f - smoothstepf(0.8f, 1.0f, h));
    case 7: {
      const float base = smoothstepf(0.0f, 0.05f, h);
      const float mid = smoothstepf(0.95f, 0.5f, h);
      const float anvil = smoothstepf(0.7f, 0.9f, h) * 1.5f * clampf(anvil_bias, 0.0f, 2.0f);
      const float mt = smoothstepf(0.65f, 0.8f, h);
      return base * mixf(mid, anvil, mt);
    }
    default: return 0.0f;
  }
}

// -------------------------------------------------------- phase
// cloud_march.wgsl:151-168, 229-296.  pow(x, 1.5) is written x*sqrt(x).
__device__ __forceinline__ float pow15(float x) { return x * sqrtf(x); }
__device__ __forceinline__ float hg_phase(float c, float g) {
  const float g2 = g * g;
  const float den = 1.0f + g2 - 2.0f * g * c;
  return (1.0f - g2) / (4.0f * kPi * pow15(fmaxf(den, 1e-4f)));
}
__device__ __forceinline__ float draine_phase(float c, float g, float alpha) {
  const float g2 = g * g;
  const float den = 1.0f + g2 - 2.0f * g * c;
  const float num = (1.0f - g2) * (1.0f + alpha * c * c);
  const float dd = 4.0f * (1.0f + alpha * (1.0f + 2.0f * g2) / 3.0f) * kPi * pow15(fmaxf(den, 1e-4f));
  return num / fmaxf(dd, 1e-6f);
}
struct PhaseConst {
  float g_hg, g_d, alpha, w_d, ice;
};
__device__ __forceinline__ PhaseConst phase_consts_from_d(float d_um, float bias) {
  const float d = clampf(d_um * bias, 5.0f, 50.0f);
  PhaseConst c;
  c.g_hg = expf(-0.0990567f / (d - 1.67154f));
  c.g_d = expf(-2.20679f / (d + 3.91029f)) - 0.428934f;
  c.alpha = expf(3.62489f - 8.29288f / (d + 5.52825f));
  c.w_d = expf(-0.599085f / (d - 0.641583f) - 0.665888f);
  c.ice = smoothstepf(35.0f, 50.0f, d);
  return c;
}
__device__ __forceinline__ float halo_lobe(float c, float peak, float width) {
  const float sc = width * sqrtf(fmaxf(1.0f - peak * peak, 1e-4f));
  const float dx = (c - peak) / fmaxf(sc, 1e-4f);
  return expf(-0.5f * dx * dx);
}
__device__ __forceinline__ float phase_with(const MarchUniforms& u, float cos_t, float g_scale,
                                            const PhaseConst& c) {
  if (u.phase_mode == PSC_PHASE_DUAL_LOBE_HG)
    return mixf(hg_phase(cos_t, u.hg_f * g_scale), hg_phase(cos_t, u.hg_b * g_scale), u.hg_w);
  const float p_hg = hg_phase(cos_t, c.g_hg * g_scale);
  const float p_d = draine_phase(cos_t, c.g_d * g_scale, c.alpha);
  float p = (1.0f - c.w_d) * p_hg + c.w_d * p_d;
  if (c.ice > 0.0f) {
    const float width = (0.5f * (kPi / 180.0f)) / fmaxf(g_scale, 0.1f);
    p = p + c.ice * (0.08f * halo_lobe(cos_t, 0.92718f, width) +
                     0.03f * halo_lobe(cos_t, 0.69466f, width));
  }
  return p;
}

// ---------------------------------------------------- noise access
template <int ST, int FILT>
struct Noise {
  __device__ __forceinline__ static float4 base(const MarchUniforms& u, float x, float y, float z,
                                                int* chk = nullptr) {
    if constexpr (FILT == PSC_FILTER_TEXTURE) {
      return tex3D<float4>(u.tex_base, x, y, z);
    } else {
      return trilinear_repeat<ST, 128>(u.noise_base, x, y, z, u.noise_scale, chk, kChkBase);
    }
  }
  __device__ __forceinline__ static float4 detail(const MarchUniforms& u, float x, float y, float z,
                                                  int* chk = nullptr) {
    if constexpr (FILT == PSC_FILTER_TEXTURE) {
      return tex3D<float4>(u.tex_detail, x, y, z);
    } else {
      return trilinear_repeat<ST, 32>(u.noise_detail, x, y, z, u.noise_scale, chk, kChkDetail);
    }
  }
  // The 2D curl tile and the weather map are small and read at most once per
  // step; they always use the exact FP32-weight path.
  __device__ __forceinline__ static float2 curl(const MarchUniforms& u, float x, float y,
                                                int* chk = nullptr) {
    return curl_sample(u.curl, x, y, chk);
  }
  __device__ __forceinline__ static float weather(const MarchUniforms& u, float x, float y,
                                                  int* chk = nullptr) {
    return weather_sample(u.weather, u.weather_w, u.weather_h, x, y, chk);
  }
};

// cloud_density_common.wgsl:233-251; the grid spans 32 km centred on the
// origin, any size, double-modulo wrap, 255 = layer type.
__device__ __forceinline__ uint32_t effective_type(const MarchUniforms& u, float px, float pz,
                                                   uint32_t layer_type, int* chk = nullptr) {
  if (!u.type_grid) return layer_type;
  const float uu = (px + 16000.0f) / 32000.0f;
  const float vv = (pz + 16000.0f) / 32000.0f;
  const int tx = wrap_mod((int)floorf(uu * (float)u.type_w), (int)u.type_w);
  const int ty = wrap_mod((int)floorf(vv * (float)u.type_h), (int)u.type_h);
  if (!idx_ok(chk, tx >= 0 && ty >= 0 && (uint32_t)tx < u.type_w && (uint32_t)ty < u.type_h, kChkType))
    return layer_type;
  const uint32_t t = __ldg(u.type_grid + (uint32_t)ty * u.type_w + (uint32_t)tx);
  return t == PSC_TYPE_SENTINEL ? layer_type : t;
}

}  // namespace psc

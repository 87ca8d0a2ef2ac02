/*
 * ORACLE — test infrastructure, not product code.  Shared helpers for the
 * CPU restatement: IEEE half conversion and wgpu sampler emulation
 * (linear filtering, texel-centre convention `u*N - 0.5`, repeat / clamp
 * addressing as configured in crates/ps-clouds/src/noise.rs:178-187 and
 * crates/ps-core/src/atmosphere_luts.rs:132-135).
 */
#ifndef PSC_ORACLE_COMMON_H
#define PSC_ORACLE_COMMON_H

#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle {

inline float f16_to_f32(uint16_t h) {
  const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
  uint32_t exp = (h >> 10) & 0x1fu;
  uint32_t mant = h & 0x3ffu;
  uint32_t bits;
  if (exp == 0) {
    if (mant == 0) {
      bits = sign;
    } else {  // subnormal: normalise
      int e = -1;
      do {
        ++e;
        mant <<= 1;
      } while ((mant & 0x400u) == 0);
      mant &= 0x3ffu;
      bits = sign | ((uint32_t)(127 - 15 - e) << 23) | (mant << 13);
    }
  } else if (exp == 31) {
    bits = sign | 0x7f800000u | (mant << 13);
  } else {
    bits = sign | ((exp + 127 - 15) << 23) | (mant << 13);
  }
  float f;
  std::memcpy(&f, &bits, 4);
  return f;
}

/* Round-to-nearest-even f32 -> f16, the conversion the `half` crate's
 * `f16::from_f32` performs. */
inline uint16_t f32_to_f16(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  const uint32_t sign = (x >> 16) & 0x8000u;
  const uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) {  // inf / nan
    return (uint16_t)(sign | 0x7c00u | (ax > 0x7f800000u ? 0x200u : 0u));
  }
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // overflow -> inf
  if (ax < 0x38800000u) {  // result is subnormal or zero
    if (ax < 0x33000000u) return (uint16_t)sign;  // < half of min subnormal
    const uint32_t e = ax >> 23;
    const uint32_t m = (ax & 0x7fffffu) | 0x800000u;
    const uint32_t shift = 126u - e;  // 14..24
    uint32_t r = m >> shift;
    const uint32_t rem = m & ((1u << shift) - 1u);
    const uint32_t half = 1u << (shift - 1u);
    if (rem > half || (rem == half && (r & 1u))) ++r;
    return (uint16_t)(sign | r);
  }
  uint32_t e = (ax >> 23) - 127u + 15u;
  uint32_t m = ax & 0x7fffffu;
  uint32_t r = (e << 10) | (m >> 13);
  const uint32_t rem = m & 0x1fffu;
  if (rem > 0x1000u || (rem == 0x1000u && (r & 1u))) ++r;
  return (uint16_t)(sign | r);
}

template <class R>
inline R clampv(R x, R lo, R hi) {
  return std::fmin(std::fmax(x, lo), hi);
}

/* Filter weight: exact, or quantised to 8 fractional bits the way GPU
 * texture units store the interpolation weight (ORACLE_FILTER_Q8). */
template <class R>
inline R filter_weight(R frac, int q8) {
  if (!q8) return frac;
  return std::nearbyint(frac * R(256)) / R(256);
}

inline int wrap_index(int64_t i, int n) {
  int64_t m = i % n;
  if (m < 0) m += n;
  return (int)m;
}
inline int clamp_index(int64_t i, int n) {
  return (int)(i < 0 ? 0 : (i >= n ? n - 1 : i));
}

/* Axis set-up: texel coordinate x = u*N - 0.5, i0 = floor(x), frac. */
template <class R>
struct Axis {
  int i0, i1;
  R w;  // weight of i1
};

template <class R>
inline Axis<R> axis_repeat(R u, int n, int q8) {
  const R x = u * R(n) - R(0.5);
  const R fl = std::floor(x);
  Axis<R> a;
  a.i0 = wrap_index((int64_t)fl, n);
  a.i1 = wrap_index((int64_t)fl + 1, n);
  a.w = filter_weight<R>(x - fl, q8);
  return a;
}

template <class R>
inline Axis<R> axis_clamp(R u, int n, int q8) {
  const R x = u * R(n) - R(0.5);
  const R fl = std::floor(x);
  Axis<R> a;
  a.i0 = clamp_index((int64_t)fl, n);
  a.i1 = clamp_index((int64_t)fl + 1, n);
  a.w = filter_weight<R>(x - fl, q8);
  return a;
}

template <class R>
inline R lerp(R a, R b, R t) {
  return a + (b - a) * t;
}

}  // namespace oracle

#endif

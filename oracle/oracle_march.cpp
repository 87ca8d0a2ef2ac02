/*
 * ORACLE — test infrastructure, not product code.
 *
 * CPU restatement of the cloud march `fs_main`
 * (shaders/clouds/cloud_march.wgsl:731-1054), its density kernel
 * (shaders/clouds/cloud_density_common.wgsl:49-305) and helpers
 * (shaders/common/math.wgsl:7-48), templated on the arithmetic type:
 *   ORACLE_FP64 — every operation in double (the correctness reference);
 *   ORACLE_FP32 — every operation in float, the "WGSL mirror" (also the
 *                 timed CPU baseline).
 * Texel data are the same inputs in both (RGBA8 noise, RGBA16F LUTs and
 * wind); only the arithmetic differs.  ORACLE_FILTER_Q8 quantises filter
 * weights to 8 fractional bits to model GPU texture units.
 */
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle.h"
#include "oracle_common.h"
#include "oracle_march_core.h"

using namespace oracle;

using namespace oracle_core;

namespace {

bool scene_ok(const OracleScene* s) {
  return s && s->noise_base && s->noise_detail && s->noise_curl && s->blue_noise && s->weather &&
         s->weather_w && s->weather_h && s->wind && s->lut_transmittance && s->lut_skyview &&
         s->lut_aerial && (!s->type_grid || (s->type_w && s->type_h));
}

template <class R>
int render_t(const OracleScene* s, uint32_t w, uint32_t h, int filter, int threads, uint32_t row0,
             uint32_t row1, float* lum, float* tr, uint64_t* counters) {
  March<R> base;
  base.init(s, filter == ORACLE_FILTER_Q8);
  if (row1 == 0 || row1 > h) row1 = h;
  std::vector<uint64_t> total(ORACLE_CNT__COUNT, 0);
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
  {
    March<R> m = base;
    std::vector<uint64_t> local(ORACLE_CNT__COUNT, 0);
    m.cnt = counters ? local.data() : nullptr;
#pragma omp for schedule(dynamic, 1)
    for (int y = (int)row0; y < (int)row1; ++y) {
      for (uint32_t x = 0; x < w; ++x) {
        R l4[4], t4[4];
        m.pixel(x, (uint32_t)y, s->depth, w, l4, t4);
        const size_t o = ((size_t)y * w + x) * 4;
        for (int c = 0; c < 4; ++c) {
          lum[o + c] = (float)l4[c];
          tr[o + c] = (float)t4[c];
        }
      }
    }
    if (counters) {
#pragma omp critical
      for (int k = 0; k < ORACLE_CNT__COUNT; ++k) total[k] += local[k];
    }
  }
  if (counters)
    for (int k = 0; k < ORACLE_CNT__COUNT; ++k) counters[k] = total[k];
  return 0;
}

}  // namespace

extern "C" {

int oracle_render(const OracleScene* s, uint32_t w, uint32_t h, int precision, int filter,
                  int threads, uint32_t row0, uint32_t row1, float* lum, float* tr,
                  uint64_t* counters) {
  if (!scene_ok(s) || !w || !h || !lum || !tr) return -1;
  if (precision == ORACLE_FP64) return render_t<double>(s, w, h, filter, threads, row0, row1, lum, tr, counters);
  if (precision == ORACLE_FP32) return render_t<float>(s, w, h, filter, threads, row0, row1, lum, tr, counters);
  return -1;
}

int oracle_render_pixel(const OracleScene* s, uint32_t w, uint32_t h, uint32_t x, uint32_t y,
                        int precision, int filter, double* lum4, double* tr4) {
  if (!scene_ok(s) || x >= w || y >= h || !lum4 || !tr4) return -1;
  if (precision == ORACLE_FP64) {
    March<double> m;
    m.init(s, filter == ORACLE_FILTER_Q8);
    m.pixel(x, y, s->depth, w, lum4, tr4);
  } else {
    March<float> m;
    m.init(s, filter == ORACLE_FILTER_Q8);
    float l[4], t[4];
    m.pixel(x, y, s->depth, w, l, t);
    for (int c = 0; c < 4; ++c) {
      lum4[c] = l[c];
      tr4[c] = t[c];
    }
  }
  return 0;
}

// Test support: the FP64 march of rows [row0, row1) (all rows when row1 is
// 0) recording, per pixel, how close it came to its two data-dependent
// branches (March::margin): out_t the smallest |max3(T) - 0.01| / 0.01 over
// its early-exit tests, out_d the smallest |density - 1e-3| / 1e-3 over its
// primary samples; 1e30 where a test never ran.  A pixel whose margin is
// within the rounding of the operands can take the other branch under a
// last-bit change of its inputs.
int oracle_branch_margins(const OracleScene* s, uint32_t w, uint32_t h, int threads, uint32_t row0,
                          uint32_t row1, double* out_t, double* out_d) {
  if (!scene_ok(s) || !w || !h || !out_t || !out_d) return -1;
  March<double> base;
  base.init(s, false);
  if (row1 == 0 || row1 > h) row1 = h;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
  {
    March<double> m = base;
#pragma omp for schedule(dynamic, 1)
    for (int y = (int)row0; y < (int)row1; ++y) {
      for (uint32_t x = 0; x < w; ++x) {
        double mg[2] = {1e30, 1e30};
        m.margin = mg;
        double l4[4], t4[4];
        m.pixel(x, (uint32_t)y, s->depth, w, l4, t4);
        const size_t o = (size_t)y * w + x;
        out_t[o] = mg[0];
        out_d[o] = mg[1];
      }
    }
  }
  return 0;
}

// Test support: the FP64 march of `s` with the discontinuous tests' outcomes
// (layer hits and order, early exits, the 1e-3 density threshold, the AP
// opacity test) taken from
// the FP64 march of `ref` at the same pixel (March::branch), so that the
// image is a smooth function of the parameters that differ between the two
// scenes: its central differences converge to the derivative with the
// branches held, which is what a tangent or adjoint of the march computes.
// The image stays in double (central differences of millimetre steps need
// more than FP32's 7 digits).  Returns the number of outcomes a replay
// needed beyond its record (0 when both scenes march the same path), or -1
// on bad arguments.
long long oracle_render_frozen(const OracleScene* ref, const OracleScene* s, uint32_t w, uint32_t h,
                               int threads, double* lum, double* tr) {
  if (!scene_ok(ref) || !scene_ok(s) || !w || !h || !lum || !tr) return -1;
  March<double> base_ref, base;
  base_ref.init(ref, false);
  base.init(s, false);
  uint64_t misses = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel
  {
    March<double> mr = base_ref, m = base;
    std::vector<uint8_t> tape;
    mr.tape = &tape;
    mr.tape_mode = 1;
    m.tape = &tape;
    m.tape_mode = 2;
#pragma omp for schedule(dynamic, 1)
    for (int y = 0; y < (int)h; ++y) {
      for (uint32_t x = 0; x < w; ++x) {
        double l4[4], t4[4];
        tape.clear();
        mr.pixel(x, (uint32_t)y, ref->depth, w, l4, t4);
        m.tape_pos = 0;
        m.pixel(x, (uint32_t)y, s->depth, w, l4, t4);
        const size_t o = ((size_t)y * w + x) * 4;
        for (int c = 0; c < 4; ++c) {
          lum[o + c] = l4[c];
          tr[o + c] = t4[c];
        }
      }
    }
#pragma omp critical
    misses += m.tape_misses;
  }
  return (long long)misses;
}

// Test support: one primary density sample (sample_density,
// cloud_march.wgsl:432-530) in FP64 at world point p3 and altitude `alt`, in
// layer `li`, with weather R channel `weather_r`; also the layer's profile
// ndf(h) (cloud_density_common.wgsl:49-91) there.  The tests use it to check
// density <= max(ndf(h) - (1 - eff), 0) * density_scale, the bound the GPU
// march relies on to skip the fetches of steps that cannot be dense.
int oracle_density_sample(const OracleScene* s, uint32_t li, const double* p3, double alt,
                          double weather_r, double* density, double* profile) {
  if (!scene_ok(s) || li >= 8 || !p3 || !density || !profile) return -1;
  March<double> m;
  m.init(s, 0);
  const Layer<double>& L = m.layers[li];
  const WindCache<double> w = m.wind_cache(L);
  const uint32_t type = m.effective_type(p3[0], p3[2], L);
  *density = m.sample_density(mk<double>(p3[0], p3[1], p3[2]), alt, L, weather_r, w, type);
  const double h = (alt - L.base) / std::fmax(L.top - L.base, 1.0);
  *profile = m.ndf(h, type, L.anvil_bias);
  return 0;
}

int oracle_composite(const float* lum, const float* tr, float* hdr, uint32_t n) {
  if (!lum || !tr || !hdr) return -1;
  for (size_t i = 0; i < (size_t)n * 4; ++i) hdr[i] = lum[i] + hdr[i] * tr[i];
  return 0;
}

}  // extern "C"

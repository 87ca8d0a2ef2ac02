// Host side of the C ABI declared in include/psclouds.h.
//
// Mirrors the reference's `CloudsSubsystem` (crates/ps-clouds/src/lib.rs):
// it owns the device copies of the noise volumes, weather inputs and LUTs,
// keeps CloudParams / the layer array / the frame and world uniforms, and
// turns them into one flattened `MarchUniforms` block per launch.  Every
// entry point validates its arguments and reports failures as an int status
// plus a thread-local message; nothing throws across the boundary.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/psclouds.h"
#include "psc_ctx.h"
#include "psc_internal.h"

namespace psc {
int launch_convert_storage(const uint8_t* src, void* dst, uint32_t n_texels, int storage,
                           float fp8_scale, cudaStream_t s);
int launch_curl_quads(const uint8_t* curl, uint4* quad, cudaStream_t s);
int launch_fold_storage(const uint8_t* base_u8, const uint8_t* detail_u8, uint32_t* base_fold,
                        uint4* base_quad, uint16_t* detail_fold, uint2* detail_quad, cudaStream_t s);
}

namespace {
thread_local std::string g_last_error;
}  // namespace

#define PSC_CUDA(call, what)                    \
  do {                                          \
    cudaError_t e_ = (call);                    \
    if (e_ != cudaSuccess) return cuda_fail(e_, what); \
  } while (0)

namespace psc {
namespace host {

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? PSC_ERR_OUT_OF_MEMORY : PSC_ERR_CUDA, "%s: %s", what,
              cudaGetErrorString(e));
}

int ensure_device(psc_ctx* c) {
  int n = 0;
  PSC_CUDA(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
  if (c->device >= n) return fail(PSC_ERR_INVALID_ARGUMENT, "device %d not in [0,%d)", c->device, n);
  PSC_CUDA(cudaSetDevice(c->device), "cudaSetDevice");
  return PSC_OK;
}

}  // namespace host
}  // namespace psc

using psc::host::cuda_fail;
using psc::host::ensure_device;
using psc::host::fail;

namespace {

bool all_finite(const float* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

float half_bits_to_float(uint16_t h) {
  __half_raw r;
  r.x = h;
  return __half2float(__half(r));
}
uint16_t float_to_half_bits(float f) {
  __half_raw r = __half_raw(__float2half_rn(f));
  return r.x;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree((void*)p);
  p = nullptr;
}

}  // namespace


namespace {

const uint32_t kLutW[4] = {256, 32, 192, 32};
const uint32_t kLutH[4] = {64, 32, 108, 32};
const uint32_t kLutD[4] = {1, 1, 1, 64};

size_t lut_texels(int k) { return (size_t)kLutW[k] * kLutH[k] * kLutD[k]; }

int validate_params(const PscCloudParamsGpu& p) {
  const float* f = reinterpret_cast<const float*>(&p);
  // every float field (the u32 fields are checked by value below)
  const size_t float_fields[] = {0, 1, 2, 4, 5, 6, 7, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 25, 26, 27};
  for (size_t i : float_fields)
    if (!std::isfinite(f[i])) return fail(PSC_ERR_NOT_FINITE, "CloudParams field %zu is not finite", i);
  if (p.cloud_steps == 0 || p.cloud_steps > 4096)
    return fail(PSC_ERR_INVALID_ARGUMENT, "cloud_steps %u out of range [1,4096]", p.cloud_steps);
  if (p.light_steps == 0 || p.light_steps > 256)
    return fail(PSC_ERR_INVALID_ARGUMENT, "light_steps %u out of range [1,256]", p.light_steps);
  if (p.multi_scatter_octaves > 64)
    return fail(PSC_ERR_INVALID_ARGUMENT, "multi_scatter_octaves %u > 64", p.multi_scatter_octaves);
  if (p.cloud_layer_count > PSC_MAX_CLOUD_LAYERS)
    return fail(PSC_ERR_LAYERS, "cloud_layer_count %u > 8", p.cloud_layer_count);
  return PSC_OK;
}

int validate_layers(const PscCloudLayerGpu* l, uint32_t n) {
  if (n > PSC_MAX_CLOUD_LAYERS) return fail(PSC_ERR_LAYERS, "%u layers exceeds the maximum of 8", n);
  for (uint32_t i = 0; i < n; ++i) {
    const float f[] = {l[i].base_m, l[i].top_m, l[i].coverage, l[i].density_scale, l[i].shape_bias,
                       l[i].detail_bias, l[i].anvil_bias, l[i].droplet_diameter_um};
    if (!all_finite(f, 8)) return fail(PSC_ERR_NOT_FINITE, "layer %u has a non-finite field", i);
    if (!(l[i].top_m > l[i].base_m))
      return fail(PSC_ERR_LAYERS, "layer %u: top_m %g <= base_m %g", i, l[i].top_m, l[i].base_m);
    if (l[i].cloud_type > 7u) return fail(PSC_ERR_LAYERS, "layer %u: cloud_type %u > 7", i, l[i].cloud_type);
  }
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = i + 1; j < n; ++j)  // check_non_overlap, cloud_layers.rs:136-150
      if (l[i].base_m < l[j].top_m && l[j].base_m < l[i].top_m)
        return fail(PSC_ERR_LAYERS, "cloud layers %u and %u overlap", i, j);
  return PSC_OK;
}

float smoothstep_h(float e0, float e1, float x) {
  float t = (x - e0) / (e1 - e0);
  t = std::fmin(std::fmax(t, 0.0f), 1.0f);
  return t * t * (3.0f - 2.0f * t);
}

// LayerWindCache (cloud_density_common.wgsl:154-183): one trilinear, repeat
// sample of the wind field at (0.5, mid_alt / 12 km, 0.5).
void wind_cache(const psc_ctx* c, const PscCloudParamsGpu& p, const PscFrameUniformsGpu& f,
                const PscCloudLayerGpu& L, psc::LayerConst& o) {
  float wx = 0.0f, wz = 0.0f;
  if (c->h_wind.size() == 32u * 16u * 32u * 4u) {
    const float mid = (L.base_m + L.top_m) * 0.5f;
    const float uy = std::fmin(std::fmax(mid / 12000.0f, 0.0f), 0.9999f);
    auto axis = [](float u, int n, int& i0, int& i1, float& w) {
      const float x = u * (float)n - 0.5f;
      const float fl = std::floor(x);
      const int i = (int)fl;
      i0 = ((i % n) + n) % n;
      i1 = (((i + 1) % n) + n) % n;
      w = x - fl;
    };
    int x0, x1, y0, y1, z0, z1;
    float ax, ay, az;
    axis(0.5f, 32, x0, x1, ax);
    axis(uy, 16, y0, y1, ay);
    axis(0.5f, 32, z0, z1, az);
    auto tx = [&](int x, int y, int z, int ch) {
      return half_bits_to_float(c->h_wind[(((size_t)z * 16 + y) * 32 + x) * 4 + ch]);
    };
    float r[2];
    for (int ch = 0; ch < 2; ++ch) {
      auto l = [](float a, float b, float t) { return a + (b - a) * t; };
      const float a0 = l(l(tx(x0, y0, z0, ch), tx(x1, y0, z0, ch), ax),
                         l(tx(x0, y1, z0, ch), tx(x1, y1, z0, ch), ax), ay);
      const float a1 = l(l(tx(x0, y0, z1, ch), tx(x1, y0, z1, ch), ax),
                         l(tx(x0, y1, z1, ch), tx(x1, y1, z1, ch), ax), ay);
      r[ch] = l(a0, a1, az);
    }
    wx = r[0];
    wz = r[1];
  }
  const float drift = p.wind_drift_strength * f.simulated_seconds;
  o.wind_off_x = wx * drift;
  o.wind_off_z = wz * drift;
  o.skew_x = o.skew_z = o.skew_thickness = 0.0f;
  if (p.wind_skew_strength != 0.0f) {
    const float sp = std::sqrt(wx * wx + wz * wz);
    if (sp >= 0.1f) {
      o.skew_x = wx / sp;
      o.skew_z = wz / sp;
      o.skew_thickness = std::fmax(L.top_m - L.base_m, 1.0f) * p.wind_skew_strength;
    }
  }
}

// The wind field at the centre column and altitude `mid` (as wind_cache
// samples it, in double): its x and z components.
void wind_at_mid(const psc_ctx* c, double mid, double& wx, double& wz) {
  wx = wz = 0.0;
  if (c->h_wind.size() != 32u * 16u * 32u * 4u) return;
  const double uy = std::fmin(std::fmax(mid / 12000.0, 0.0), 0.9999);
  auto axis = [](double u, int n, int& i0, int& i1, double& w) {
    const double x = u * (double)n - 0.5;
    const double fl = std::floor(x);
    const int i = (int)fl;
    i0 = ((i % n) + n) % n;
    i1 = (((i + 1) % n) + n) % n;
    w = x - fl;
  };
  int x0, x1, y0, y1, z0, z1;
  double ax, ay, az;
  axis(0.5, 32, x0, x1, ax);
  axis(uy, 16, y0, y1, ay);
  axis(0.5, 32, z0, z1, az);
  auto tx = [&](int x, int y, int z, int ch) {
    return (double)half_bits_to_float(c->h_wind[(((size_t)z * 16 + y) * 32 + x) * 4 + ch]);
  };
  auto l = [](double a, double b, double t) { return a + (b - a) * t; };
  double r[2];
  for (int ch = 0; ch < 2; ++ch) {
    const double a0 = l(l(tx(x0, y0, z0, ch), tx(x1, y0, z0, ch), ax), l(tx(x0, y1, z0, ch), tx(x1, y1, z0, ch), ax), ay);
    const double a1 = l(l(tx(x0, y0, z1, ch), tx(x1, y0, z1, ch), ax), l(tx(x0, y1, z1, ch), tx(x1, y1, z1, ch), ax), ay);
    r[ch] = l(a0, a1, az);
  }
  wx = r[0];
  wz = r[1];
}

// Flatten one view's scene (params, layers, frame) plus the context's world,
// options and inputs into the kernel's uniform block.
// The layer's profile (cloud_density_common.wgsl:49-91) in double, as the
// FAST march evaluates it: types 0..6 through the coefficients in `o`,
// Cumulonimbus by its own formula, any other type 0.
double profile_h(const PscCloudLayerGpu& L, const psc::LayerConst& o, double h) {
  auto S = [](double t) {
    t = std::fmin(std::fmax(t, 0.0), 1.0);
    return t * t * (3.0 - 2.0 * t);
  };
  if (o.ndf_mode) return S(h * o.ndf_inv_a) * S(h * o.ndf_inv_w1 + o.ndf_b1);
  if (L.cloud_type != 7u) return 0.0;
  const double base = S(h / 0.05), mid = S((h - 0.95) / -0.45);
  const double anvil = S((h - 0.7) / 0.2) * 1.5 * std::fmin(std::fmax((double)L.anvil_bias, 0.0), 2.0);
  const double mt = S((h - 0.65) / 0.15);
  return base * (mid * (1.0 - mt) + anvil * mt);
}

// LayerConst::live_lo / live_hi: the hull of the normalised heights whose
// profile can pass the FAST march's test (nd * 1.000001 - skip_k) *
// density_scale > 1e-3, found on a 1/20000 grid with the threshold lowered by
// 1e-4 and widened by 1e-3 of the height and then 1 m of altitude, so that
// the kernel's FP32 evaluation of any passing step lies inside it.
// LayerConst::light_h_dead: above the last height where the profile can
// exceed skip_k (threshold lowered by 1e-4, widened by 2 grid cells and
// 1e-3) every light-march tap adds exactly 0: the base shape is at most 1
// and 1 - eff is at least skip_k.
// The scan is a pure function of the profile's inputs; the last results are
// kept per thread, so a frame stream whose layers do not change pays for it
// once instead of on every call.
void live_band(const PscCloudLayerGpu& L, psc::LayerConst& o) {
  struct Key {
    uint32_t mode, type;
    float inv_a, b1, inv_w1, anvil, skip_k, density_scale, inv_thickness, base_m;
    bool operator==(const Key& k) const { return std::memcmp(this, &k, sizeof(Key)) == 0; }
  };
  struct Entry {
    Key key;
    float live_lo, live_hi, light_h_dead;
  };
  Key key;
  std::memset(&key, 0, sizeof(key));
  key = Key{o.ndf_mode, L.cloud_type, o.ndf_inv_a, o.ndf_b1, o.ndf_inv_w1, L.anvil_bias,
            o.skip_k, o.density_scale, o.inv_thickness, o.base_m};
  thread_local Entry cache[32];
  thread_local uint32_t cache_n = 0, cache_next = 0;
  for (uint32_t i = 0; i < cache_n; ++i)
    if (cache[i].key == key) {
      o.live_lo = cache[i].live_lo;
      o.live_hi = cache[i].live_hi;
      o.light_h_dead = cache[i].light_h_dead;
      return;
    }
  const int M = 20000;
  int first = -1, last = -1, last_light = -1;
  for (int i = 0; i <= M; ++i) {
    const double nd = profile_h(L, o, (double)i / M);
    if ((nd * 1.000001 - o.skip_k) * o.density_scale > 1e-3 * (1.0 - 1e-4)) {
      if (first < 0) first = i;
      last = i;
    }
    if (nd * 1.000001 > (double)o.skip_k - 1e-4) last_light = i;
  }
  if (first < 0) {
    o.live_lo = 1.0f;
    o.live_hi = 0.0f;
    o.light_h_dead = 2.0f;  // no primary step is dense, so no light march runs
  } else {
    const double thick = 1.0 / (double)o.inv_thickness;
    o.light_h_dead = last_light < 0 ? -1.0f : (float)((double)(last_light + 2) / M + 1e-3);
    const double h_lo = std::fmax((double)(first - 2) / M - 1e-3, 0.0);
    const double h_hi = std::fmin((double)(last + 2) / M + 1e-3, 1.0);
    o.live_lo = (float)((double)o.base_m + h_lo * thick - 1.0);
    o.live_hi = (float)((double)o.base_m + h_hi * thick + 1.0);
  }
  cache[cache_next] = Entry{key, o.live_lo, o.live_hi, o.light_h_dead};
  cache_next = (cache_next + 1) % 32u;
  cache_n = std::min(cache_n + 1, 32u);
}

void build_uniforms_for(const psc_ctx* c, const PscCloudParamsGpu& p, const PscCloudLayerGpu* layers,
                        const PscFrameUniformsGpu& f, uint32_t width, uint32_t height,
                        psc::MarchUniforms& u) {
  std::memset(&u, 0, sizeof(u));
  const PscWorldUniformsGpu& w = c->world;
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      u.inv_vp[col][row] = f.inv_view_proj[col][row];
      u.inv_vp_d[col][row] = (double)f.inv_view_proj[col][row];
    }
  for (int k = 0; k < 3; ++k) {
    u.cam[k] = f.camera_position_world[k];
    u.sun[k] = f.sun_direction[k];
    u.sun_illum[k] = f.sun_illuminance[k];
    u.lightning_rgb[k] = f.lightning_illuminance[k];
    u.sigma_s[k] = p.sigma_s[k];
  }
  u.lightning_radius = f.lightning_illuminance[3];
  u.lightning_origin_x = f.lightning_origin_world[0];
  u.lightning_origin_z = f.lightning_origin_world[2];
  u.vp_w = (float)width;
  u.vp_h = (float)height;
  u.temporal_jitter = p.temporal_jitter;
  u.frame_index = f.frame_index;
  u.planet_r = w.planet_radius_m;
  u.planet_r_d = (double)w.planet_radius_m;
  u.atmo_top = w.atmosphere_top_m;
  u.droplet_bias = p.droplet_diameter_bias;
  u.forward_bias = p.forward_bias;
  u.detail_strength = p.detail_strength;
  u.curl_strength = p.curl_strength;
  u.powder = p.powder_strength;
  u.ms_a = p.multi_scatter_a;
  u.ms_b = p.multi_scatter_b;
  u.ms_c = p.multi_scatter_c;
  u.ambient = p.ambient_strength;
  u.base_scale = std::fmax(p.base_scale_m, 1.0f);
  u.detail_scale = std::fmax(p.detail_scale_m, 1.0f);
  u.weather_scale = std::fmax(p.weather_scale_m, 1.0f);
  u.light_steps = p.light_steps;
  u.cloud_steps = p.cloud_steps;
  u.octaves = p.multi_scatter_octaves;
  u.layer_count = std::min<uint32_t>(p.cloud_layer_count, 8u);
  u.cone = p.cone_light_sampling;
  u.phase_mode = c->opts.phase_mode;
  u.hg_f = c->opts.hg_g_forward;
  u.hg_b = c->opts.hg_g_backward;
  u.hg_w = c->opts.hg_blend;
  u.kahan = c->opts.kahan;
  u.composite = c->opts.composite;
  u.debug_checks = c->opts.debug_checks;
  u.error_word = nullptr;  // set by launch_view_march in the debug form

  u.base_texel_scale = 128.0f / u.base_scale;
  u.detail_texel_scale = 32.0f / u.detail_scale;
  u.curl_texel_scale = 128.0f / u.detail_scale;
  u.inv_base_scale = 1.0f / u.base_scale;
  u.inv_detail_scale = 1.0f / u.detail_scale;
  u.inv_weather_scale = 1.0f / u.weather_scale;
  u.curl_offset_scale = p.curl_strength * u.detail_scale;
  u.sun_az = std::atan2(f.sun_direction[0], f.sun_direction[2]);
  {
    const double top = w.atmosphere_top_m, R = w.planet_radius_m;
    u.big_h = (float)std::sqrt(std::max(top * top - R * R, 0.0));
    u.inv_big_h = 1.0f / std::fmax(u.big_h, 1.0f);
    u.inv_planet_r = 1.0f / (float)R;
    const float Rf = (float)R;
    u.rho_1m = std::sqrt(1.0f * (2.0f * Rf + 1.0f));
  }
  u.inv_cos_sun = 1.0f / std::fmax(f.sun_direction[1], 0.05f);
  u.b_half = p.multi_scatter_b == 0.5f ? 1u : 0u;
  {
    float a = 1.0f, b = 1.0f, cc = 1.0f;
    for (int n = 0; n < 8; ++n) {
      u.apow[n] = a;
      u.bpow[n] = b;
      u.cpow[n] = cc;
      a *= p.multi_scatter_a;
      b *= p.multi_scatter_b;
      cc *= p.multi_scatter_c;
    }
  }
  // diurnal_modulation (cloud_density_common.wgsl:204-219), per layer type
  const float bell = smoothstep_h(-0.1f, 0.4f, f.sun_direction[1]);
  for (uint32_t i = 0; i < 8; ++i) {
    const PscCloudLayerGpu& L = layers[i];
    psc::LayerConst& o = u.layers[i];
    o.base_m = L.base_m;
    o.top_m = L.top_m;
    o.inv_thickness = 1.0f / std::fmax(L.top_m - L.base_m, 1.0f);
    o.coverage = L.coverage;
    o.density_scale = L.density_scale;
    o.cloud_type = L.cloud_type;
    const uint32_t t = L.cloud_type;
    const bool conv = t == 0 || t == 2 || t == 3 || t == 7;
    const float di = (p.diurnal_strength == 0.0f || !conv) ? 0.0f : bell * p.diurnal_strength;
    o.lf_bias = (L.shape_bias * di) * 0.5f;
    o.layer_detail = std::fmin(std::fmax(p.detail_strength + L.detail_bias * di, 0.0f), 1.0f);
    o.anvil_bias = L.anvil_bias;
    o.droplet_um = L.droplet_diameter_um;
    // chromatic_mie_modulation, cloud_march.wgsl:122-145
    float cm[3] = {1.0f, 1.0f, 1.0f};
    const float tt = std::fmin(std::fmax(1.0f - L.droplet_diameter_um / 20.0f, 0.0f), 1.0f);
    if (tt > 0.0f) {
      const float s = 0.25f * tt * tt;
      cm[0] = 1.0f - 0.5f * s;
      cm[2] = 1.0f + s;
    }
    for (int k = 0; k < 3; ++k) o.sigma_t[k] = (p.sigma_s[k] + p.sigma_a[k]) * cm[k];
    wind_cache(c, p, f, L, o);
    // cloud_phase_constants (cloud_march.wgsl:256-272) for non-Cb layers
    const float d = std::fmin(std::fmax(L.droplet_diameter_um * p.droplet_diameter_bias, 5.0f), 50.0f);
    o.g_hg = std::exp(-0.0990567f / (d - 1.67154f));
    o.g_d = std::exp(-2.20679f / (d + 3.91029f)) - 0.428934f;
    o.alpha = std::exp(3.62489f - 8.29288f / (d + 5.52825f));
    o.w_d = std::exp(-0.599085f / (d - 0.641583f) - 0.665888f);
    o.ice = smoothstep_h(35.0f, 50.0f, d);
    // the FAST schedule's ndf coefficients (march_fast_body.cuh:ndf_coef,
    // cloud_density_common.wgsl:49-91): smoothstep(0, a) times a rising or
    // falling second smoothstep, for every type but Cumulonimbus
    static const float kA[7] = {0.07f, 0.10f, 0.15f, 0.20f, 0.30f, 0.40f, 0.50f};
    static const float kE1[7] = {1.0f, 0.6f, 1.0f, 1.0f, 0.7f, 0.6f, 0.8f};
    static const float kW1[7] = {-0.8f, 0.4f, -0.6f, -0.7f, 0.3f, 0.4f, 0.2f};
    static const uint32_t kMode[7] = {1, 2, 1, 1, 2, 2, 2};
    if (L.cloud_type < 7) {
      o.ndf_inv_a = 1.0f / kA[L.cloud_type];
      o.ndf_inv_w1 = 1.0f / kW1[L.cloud_type];
      o.ndf_b1 = -kE1[L.cloud_type] * o.ndf_inv_w1;
      o.ndf_mode = kMode[L.cloud_type];
      if (o.ndf_mode == 2) {  // 1 - S(t) = S(1 - t)
        o.ndf_inv_w1 = -o.ndf_inv_w1;
        o.ndf_b1 = 1.0f - o.ndf_b1;
      }
    } else {
      o.ndf_inv_a = o.ndf_b1 = o.ndf_inv_w1 = 0.0f;
      o.ndf_mode = 0;
    }
    o.lf_c = 1.0f - o.lf_bias;
    {
      // the largest eff any weather sample can give: bilinear taps stay
      // within the map's extremes, and eff = clamp01(weather * coverage)
      const float wext = L.coverage >= 0.0f ? c->weather_max : c->weather_min;
      const float eff_max = std::fmin(std::fmax(wext * L.coverage, 0.0f), 1.0f);
      o.skip_k = eff_max < 0.01f ? 4.0f : (1.0f - eff_max) - 1e-6f;
    }
    o.skew_kx = o.skew_x * o.skew_thickness;
    o.skew_kz = o.skew_z * o.skew_thickness;
    live_band(L, o);
    o.r_bottom = (double)w.planet_radius_m + (double)L.base_m;
    o.r_top = (double)w.planet_radius_m + (double)L.top_m;
  }

  u.noise_base = c->d_base_store;
  u.noise_detail = c->d_detail_store;
  u.noise_scale = 1.0f / c->fp8_scale;
  u.curl = c->d_curl;
  u.blue = c->d_blue;
  u.weather = c->d_weather;
  u.weather_quad = c->d_weather_quad;
  u.weather_uniform = c->weather_uniform ? 1u : 0u;
  u.weather_value = c->weather_value;
  u.weather_w = c->weather_w;
  u.weather_h = c->weather_h;
  u.type_grid = c->d_type;
  u.type_w = c->type_w;
  u.type_h = c->type_h;
  u.lut_trans = c->d_lut[PSC_LUT_TRANSMITTANCE];
  u.lut_sky = c->d_lut[PSC_LUT_SKYVIEW];
  u.lut_ap = c->d_lut[PSC_LUT_AERIAL];
  u.tex_base = c->tex_base;
  u.tex_detail = c->tex_detail;
  u.curl_quad = c->d_curl_quad;
  u.base_quad = c->d_base_quad;
  u.detail_quad = c->d_detail_quad;
  // texture-unit sampling of the transmittance LUT belongs to the filtered
  // forms; EXACT keeps FP32 weights everywhere
  u.tex_trans = c->opts.filter != PSC_FILTER_EXACT ? c->tex_lut[PSC_LUT_TRANSMITTANCE] : 0;
  u.tex_sky = c->opts.filter != PSC_FILTER_EXACT ? c->tex_lut[PSC_LUT_SKYVIEW] : 0;
}

void build_uniforms(const psc_ctx* c, uint32_t width, uint32_t height, psc::MarchUniforms& u) {
  build_uniforms_for(c, c->params, c->layers, c->frame, width, height, u);
}

int build_storage(psc_ctx* c) {
  if (!c->have_base || !c->have_detail) return PSC_OK;
  const int st = (int)c->opts.storage;
  if (st == c->store_form && c->d_base_store) return PSC_OK;
  const size_t tex_bytes[] = {4, 16, 8, 8, 4};
  dfree(c->d_base_store);
  dfree(c->d_detail_store);
  PSC_CUDA(cudaMalloc(&c->d_base_store, 128u * 128u * 128u * tex_bytes[st]), "cudaMalloc base storage");
  PSC_CUDA(cudaMalloc(&c->d_detail_store, 32u * 32u * 32u * tex_bytes[st]), "cudaMalloc detail storage");
  if (psc::launch_convert_storage(c->d_base_u8, c->d_base_store, 128u * 128u * 128u, st, c->fp8_scale, 0) ||
      psc::launch_convert_storage(c->d_detail_u8, c->d_detail_store, 32u * 32u * 32u, st, c->fp8_scale, 0))
    return fail(PSC_ERR_CUDA, "storage conversion launch failed");
  if (c->have_curl) {  // the FAST schedule reads the curl tile as quads
    if (!c->d_curl_quad) PSC_CUDA(cudaMalloc(&c->d_curl_quad, 128u * 128u * 16u), "cudaMalloc curl quads");
    if (psc::launch_curl_quads(c->d_curl, c->d_curl_quad, 0)) return fail(PSC_ERR_CUDA, "curl quad launch failed");
  }
  if (st == PSC_STORAGE_F16) {  // the FAST schedule reads the channel-folded forms
    if (!c->d_base_fold) PSC_CUDA(cudaMalloc(&c->d_base_fold, 128u * 128u * 128u * 4u), "cudaMalloc base fold");
    if (!c->d_base_quad) PSC_CUDA(cudaMalloc(&c->d_base_quad, 128u * 128u * 128u * 16u), "cudaMalloc base quads");
    if (!c->d_detail_fold) PSC_CUDA(cudaMalloc(&c->d_detail_fold, 32u * 32u * 32u * 2u), "cudaMalloc detail fold");
    if (!c->d_detail_quad) PSC_CUDA(cudaMalloc(&c->d_detail_quad, 32u * 32u * 32u * 8u), "cudaMalloc detail quads");
    if (psc::launch_fold_storage(c->d_base_u8, c->d_detail_u8, c->d_base_fold, c->d_base_quad, c->d_detail_fold,
                                 c->d_detail_quad, 0))
      return fail(PSC_ERR_CUDA, "channel fold launch failed");
  }
  PSC_CUDA(cudaDeviceSynchronize(), "storage conversion");
  c->store_form = st;
  return PSC_OK;
}

void destroy_textures(psc_ctx* c) {
  if (c->tex_base) cudaDestroyTextureObject(c->tex_base);
  if (c->tex_detail) cudaDestroyTextureObject(c->tex_detail);
  if (c->arr_base) cudaFreeArray(c->arr_base);
  if (c->arr_detail) cudaFreeArray(c->arr_detail);
  c->tex_base = c->tex_detail = 0;
  c->arr_base = c->arr_detail = nullptr;
  c->tex_dirty = true;
}

// 3D texture over an RGBA8 volume (read as normalised float) or a
// channel-folded FP16 volume (half2 base / half detail, read as stored),
// linear filtering, repeat addressing, normalised coordinates: the noise
// sampler of crates/ps-clouds/src/noise.rs:178-187.
int make_volume_texture(const void* d_src, uint32_t n, int half_channels, cudaArray_t* arr,
                        cudaTextureObject_t* tex) {
  const cudaChannelFormatDesc fmt = half_channels == 2   ? cudaCreateChannelDescHalf2()
                                    : half_channels == 1 ? cudaCreateChannelDescHalf1()
                                                         : cudaCreateChannelDesc<uchar4>();
  const size_t texel = half_channels ? 2u * half_channels : 4u;
  const cudaExtent ext = make_cudaExtent(n, n, n);
  PSC_CUDA(cudaMalloc3DArray(arr, &fmt, ext), "cudaMalloc3DArray");
  cudaMemcpy3DParms cp{};
  cp.srcPtr = make_cudaPitchedPtr((void*)d_src, n * texel, n, n);
  cp.dstArray = *arr;
  cp.extent = ext;
  cp.kind = cudaMemcpyDeviceToDevice;
  PSC_CUDA(cudaMemcpy3D(&cp), "cudaMemcpy3D volume");
  cudaResourceDesc rd{};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = *arr;
  cudaTextureDesc td{};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeWrap;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = half_channels ? cudaReadModeElementType : cudaReadModeNormalizedFloat;
  td.normalizedCoords = 1;
  PSC_CUDA(cudaCreateTextureObject(tex, &rd, &td, nullptr), "cudaCreateTextureObject");
  return PSC_OK;
}

int build_textures(psc_ctx* c) {
  if (c->opts.filter == PSC_FILTER_EXACT || !c->tex_dirty) return PSC_OK;
  destroy_textures(c);
  const bool f16 = c->opts.storage == PSC_STORAGE_F16;
  if (f16 && (!c->d_base_fold || !c->d_detail_fold))
    return fail(PSC_ERR_MISSING_INPUT, "folded F16 volumes were not built");
  int rc = make_volume_texture(f16 ? (const void*)c->d_base_fold : c->d_base_u8, 128, f16 ? 2 : 0,
                               &c->arr_base, &c->tex_base);
  if (rc) return rc;
  rc = make_volume_texture(f16 ? (const void*)c->d_detail_fold : c->d_detail_u8, 32, f16 ? 1 : 0,
                           &c->arr_detail, &c->tex_detail);
  if (rc) return rc;
  c->tex_dirty = false;
  return PSC_OK;
}

void destroy_batch_sky_textures(psc_ctx* c) {
  for (cudaTextureObject_t t : c->batch_sky_tex)
    if (t) cudaDestroyTextureObject(t);
  c->batch_sky_tex.clear();
}

void release_batch(psc_ctx* c) {
  destroy_batch_sky_textures(c);
  if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
  c->batch_exec = nullptr;
  c->batch_key.clear();
  for (int j = 0; j < psc_ctx::kBranches; ++j) {
    if (c->batch_branch[j]) cudaStreamDestroy(c->batch_branch[j]);
    if (c->batch_join[j]) cudaEventDestroy(c->batch_join[j]);
    c->batch_branch[j] = nullptr;
    c->batch_join[j] = nullptr;
  }
  if (c->batch_fork) cudaEventDestroy(c->batch_fork);
  c->batch_fork = nullptr;
  if (c->batch_stream) cudaStreamDestroy(c->batch_stream);
  if (c->batch_staged) cudaEventDestroy(c->batch_staged);
  c->batch_stream = nullptr;
  c->batch_staged = nullptr;
  dfree(c->d_bu);
  dfree(c->d_bv);
  dfree(c->d_bframes);
  dfree(c->d_bsky);
  dfree(c->d_bap);
  dfree(c->d_btiles);
  dfree(c->d_bcounter);
  if (c->h_bu) cudaFreeHost(c->h_bu);
  if (c->h_bv) cudaFreeHost(c->h_bv);
  if (c->h_bframes) cudaFreeHost(c->h_bframes);
  if (c->h_btiles) cudaFreeHost(c->h_btiles);
  c->h_bu = nullptr;
  c->h_bv = nullptr;
  c->h_bframes = nullptr;
  c->h_btiles = nullptr;
  c->batch_cap_views = c->batch_cap_tiles = 0;
}

// Grow the batch buffers; a growth invalidates any captured graph.
int reserve_batch(psc_ctx* c, uint32_t views, uint32_t tiles) {
  if (!c->batch_stream) {
    PSC_CUDA(cudaStreamCreateWithFlags(&c->batch_stream, cudaStreamNonBlocking), "batch stream");
    PSC_CUDA(cudaEventCreateWithFlags(&c->batch_staged, cudaEventDisableTiming), "batch event");
    PSC_CUDA(cudaMalloc(&c->d_bcounter, sizeof(uint32_t)), "cudaMalloc batch counter");
  }
  const size_t fl = psc::frame_lite_size();
  if (views > c->batch_cap_views) {
    cudaEventSynchronize(c->batch_staged);
    if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
    c->batch_exec = nullptr;
    destroy_batch_sky_textures(c);
    dfree(c->d_bu);
    dfree(c->d_bv);
    dfree(c->d_bframes);
    dfree(c->d_bsky);
    dfree(c->d_bap);
    if (c->h_bu) cudaFreeHost(c->h_bu);
    if (c->h_bv) cudaFreeHost(c->h_bv);
    if (c->h_bframes) cudaFreeHost(c->h_bframes);
    c->h_bu = nullptr;
    c->h_bv = nullptr;
    c->h_bframes = nullptr;
    PSC_CUDA(cudaMalloc(&c->d_bu, views * sizeof(psc::MarchUniforms)), "cudaMalloc batch uniforms");
    PSC_CUDA(cudaMalloc(&c->d_bv, views * sizeof(psc::ViewDev)), "cudaMalloc batch views");
    PSC_CUDA(cudaMalloc(&c->d_bframes, views * fl), "cudaMalloc batch frames");
    PSC_CUDA(cudaMalloc(&c->d_bsky, (size_t)views * 192 * 108 * sizeof(float4)), "cudaMalloc batch sky LUTs");
    PSC_CUDA(cudaMalloc(&c->d_bap, (size_t)views * 32 * 32 * 64 * sizeof(float4)), "cudaMalloc batch AP LUTs");
    PSC_CUDA(cudaMallocHost(&c->h_bu, views * sizeof(psc::MarchUniforms)), "pinned batch uniforms");
    PSC_CUDA(cudaMallocHost(&c->h_bv, views * sizeof(psc::ViewDev)), "pinned batch views");
    PSC_CUDA(cudaMallocHost(&c->h_bframes, views * fl), "pinned batch frames");
    // each view's sky-view LUT also behind a texture object (bilinear,
    // clamp, normalised coordinates), as the context's own sky-view LUT is
    c->batch_sky_tex.assign(views, 0);
    for (uint32_t i = 0; i < views; ++i) {
      cudaResourceDesc rd{};
      rd.resType = cudaResourceTypePitch2D;
      rd.res.pitch2D.devPtr = c->d_bsky + (size_t)i * PSC_SKYVIEW_W * PSC_SKYVIEW_H;
      rd.res.pitch2D.desc = cudaCreateChannelDesc<float4>();
      rd.res.pitch2D.width = PSC_SKYVIEW_W;
      rd.res.pitch2D.height = PSC_SKYVIEW_H;
      rd.res.pitch2D.pitchInBytes = (size_t)PSC_SKYVIEW_W * sizeof(float4);
      cudaTextureDesc td{};
      td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
      td.filterMode = cudaFilterModeLinear;
      td.readMode = cudaReadModeElementType;
      td.normalizedCoords = 1;
      PSC_CUDA(cudaCreateTextureObject(&c->batch_sky_tex[i], &rd, &td, nullptr), "batch sky-view texture");
    }
    c->batch_cap_views = views;
  }
  if (tiles > c->batch_cap_tiles) {
    cudaEventSynchronize(c->batch_staged);
    if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
    c->batch_exec = nullptr;
    dfree(c->d_btiles);
    if (c->h_btiles) cudaFreeHost(c->h_btiles);
    c->h_btiles = nullptr;
    PSC_CUDA(cudaMalloc(&c->d_btiles, tiles * sizeof(uint32_t)), "cudaMalloc batch tiles");
    PSC_CUDA(cudaMallocHost(&c->h_btiles, tiles * sizeof(uint32_t)), "pinned batch tiles");
    c->batch_cap_tiles = tiles;
  }
  return PSC_OK;
}

int validate_tuning(const PscBatchTuning& t) {
  if (t.form != PSC_BATCH_PERSISTENT && t.form != PSC_BATCH_PER_VIEW)
    return fail(PSC_ERR_INVALID_ARGUMENT, "batch form must be PSC_BATCH_PERSISTENT or PSC_BATCH_PER_VIEW");
  if (t.threads != 64 && t.threads != 128 && t.threads != 256)
    return fail(PSC_ERR_INVALID_ARGUMENT, "batch threads must be 64, 128 or 256 (got %u)", t.threads);
  const uint32_t warps = t.threads / 32;
  if (t.tile_w < 8 || t.tile_w % 8 || warps % (t.tile_w / 8))
    return fail(PSC_ERR_INVALID_ARGUMENT, "tile_w %u must be 8*k with k dividing %u", t.tile_w, warps);
  return PSC_OK;
}

// Host staging of one batch: per-view uniform blocks, view records, frame
// records for the LUT bakes and the cost-sorted tile list.
// Uniform block of one batch view: its own scene, and its own sky-view and
// aerial-perspective LUTs (baked per view into `sky` / `ap`; the context's
// sky-view texture belongs to its own frame).  `sky_tex`, when not 0, is a
// texture object over `sky`, used by the filtered forms as the single-view
// march uses the context's; 0 reads `sky` with plain loads.
void build_batch_view_uniforms(const psc_ctx* c, const PscBatchView& bv, float4* sky, float4* ap,
                               psc::MarchUniforms& u, cudaTextureObject_t sky_tex = 0) {
  PscCloudParamsGpu p = bv.params;
  p.cloud_layer_count = bv.n_layers;
  PscCloudLayerGpu layers[8];
  std::memset(layers, 0, sizeof(layers));
  for (uint32_t l = 0; l < bv.n_layers; ++l) layers[l] = bv.layers[l];
  build_uniforms_for(c, p, layers, bv.frame, bv.width, bv.height, u);
  u.lut_sky = sky;
  u.tex_sky = c->opts.filter != PSC_FILTER_EXACT ? sky_tex : 0;
  u.lut_ap = ap;
}

int stage_batch(psc_ctx* c, const PscBatchView* views, uint32_t n, uint32_t* n_tiles_out) {
  const PscBatchTuning& tu = c->batch_tuning;
  const bool per_view = tu.form == PSC_BATCH_PER_VIEW;
  const uint32_t tile_w = tu.tile_w, tile_h = (tu.threads / 32 / (tu.tile_w / 8)) * 4;
  uint64_t total = 0;
  for (uint32_t i = 0; i < n && !per_view; ++i) {
    const uint64_t tx = (views[i].width + tile_w - 1) / tile_w, ty = (views[i].height + tile_h - 1) / tile_h;
    if (tx > 4096 || ty > 4096) return fail(PSC_ERR_INVALID_ARGUMENT, "view %u has too many tiles", i);
    total += tx * ty;
  }
  if (total > (1u << 26)) return fail(PSC_ERR_INVALID_ARGUMENT, "batch of %llu tiles is too large", (unsigned long long)total);
  int rc = reserve_batch(c, n, (uint32_t)total);
  if (rc) return rc;
  // the previous enqueue must have consumed the pinned staging
  PSC_CUDA(cudaEventSynchronize(c->batch_staged), "batch staging wait");
  const size_t fl = psc::frame_lite_size();
  for (uint32_t i = 0; i < n; ++i) {
    const PscBatchView& bv = views[i];
    build_batch_view_uniforms(c, bv, c->d_bsky + (size_t)i * PSC_SKYVIEW_W * PSC_SKYVIEW_H,
                              c->d_bap + (size_t)i * PSC_AP_W * PSC_AP_H * PSC_AP_D, c->h_bu[i],
                              c->batch_sky_tex[i]);
    c->h_bv[i] = psc::ViewDev{bv.width, bv.height, 0, 0, bv.depth, reinterpret_cast<float4*>(bv.out_luminance),
                              reinterpret_cast<float4*>(bv.out_transmittance), reinterpret_cast<float4*>(bv.hdr)};
    psc::frame_lite_from(bv.frame, static_cast<char*>(c->h_bframes) + i * fl);
  }
  // views in descending estimated cost (primary steps x layers, then pixels)
  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; ++i) order[i] = i;
  auto cost = [&](uint32_t i) {
    return (double)views[i].params.cloud_steps * (double)std::max<uint32_t>(views[i].n_layers, 1);
  };
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const double ca = cost(a), cb = cost(b);
    if (ca != cb) return ca > cb;
    return (uint64_t)views[a].width * views[a].height > (uint64_t)views[b].width * views[b].height;
  });
  c->batch_order = order;
  uint32_t k = 0;
  for (uint32_t i : order) {
    if (per_view) break;
    const uint32_t tx = (views[i].width + tile_w - 1) / tile_w, ty = (views[i].height + tile_h - 1) / tile_h;
    for (uint32_t y = 0; y < ty; ++y)
      for (uint32_t x = 0; x < tx; ++x) c->h_btiles[k++] = (i << 24) | (x << 12) | y;
  }
  *n_tiles_out = k;
  return PSC_OK;
}

// The per-view form on `s`: frame records H2D, then per view, in descending
// cost over the branch streams (forked from and joined back into `s`), its
// sky-view / aerial-perspective LUT bake and its FAST kernel (uniforms by
// value), so a view's bake overlaps the other branches' marches.
int enqueue_batch_per_view(psc_ctx* c, uint32_t n, cudaStream_t s, bool capturing) {
  if (!c->batch_fork) {
    PSC_CUDA(cudaEventCreateWithFlags(&c->batch_fork, cudaEventDisableTiming), "batch fork event");
    for (int j = 0; j < psc_ctx::kBranches; ++j) {
      PSC_CUDA(cudaStreamCreateWithFlags(&c->batch_branch[j], cudaStreamNonBlocking), "batch branch stream");
      PSC_CUDA(cudaEventCreateWithFlags(&c->batch_join[j], cudaEventDisableTiming), "batch join event");
    }
  }
  const size_t fl = psc::frame_lite_size();
  PSC_CUDA(cudaMemcpyAsync(c->d_bframes, c->h_bframes, n * fl, cudaMemcpyHostToDevice, s), "batch frames H2D");
  PSC_CUDA(cudaEventRecordWithFlags(c->batch_staged, s, capturing ? cudaEventRecordExternal : 0),
           "batch event");
  const uint32_t nb = std::min<uint32_t>(n, (uint32_t)psc_ctx::kBranches);
  PSC_CUDA(cudaEventRecord(c->batch_fork, s), "batch fork");
  for (uint32_t j = 0; j < nb; ++j)
    PSC_CUDA(cudaStreamWaitEvent(c->batch_branch[j], c->batch_fork, 0), "batch fork wait");
  for (uint32_t k = 0; k < n; ++k) {
    const uint32_t i = c->batch_order[k];
    cudaStream_t br = c->batch_branch[k % nb];
    if (c->batch_bake[i] &&
        psc::launch_view_lut_bakes(c->world, static_cast<const char*>(c->d_bframes) + i * fl, 1,
                                   c->d_lut_h[PSC_LUT_TRANSMITTANCE], c->d_lut_h[PSC_LUT_MULTISCATTER],
                                   c->d_bsky + (size_t)i * PSC_SKYVIEW_W * PSC_SKYVIEW_H,
                                   c->d_bap + (size_t)i * PSC_AP_W * PSC_AP_H * PSC_AP_D, br))
      return fail(PSC_ERR_CUDA, "per-view LUT bake launch failed");
    int rc = psc::launch_march_fast(c->h_bu[i], c->h_bv[i], c->opts, br);
    if (rc == PSC_ERR_UNSUPPORTED) rc = psc::launch_march(c->h_bu[i], c->h_bv[i], c->opts, br);
    if (rc) return fail(rc, "per-view march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  }
  for (uint32_t j = 0; j < nb; ++j) {
    PSC_CUDA(cudaEventRecord(c->batch_join[j], c->batch_branch[j]), "batch join");
    PSC_CUDA(cudaStreamWaitEvent(s, c->batch_join[j], 0), "batch join wait");
  }
  return PSC_OK;
}

uint64_t fnv1a(const void* p, size_t n, uint64_t h = 1469598103934665603ull) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

// Copies, per-view LUT bakes, counter reset and the persistent march on `s`.
int enqueue_batch(psc_ctx* c, uint32_t n, uint32_t n_tiles, cudaStream_t s, bool capturing) {
  const size_t fl = psc::frame_lite_size();
  PSC_CUDA(cudaMemcpyAsync(c->d_bu, c->h_bu, n * sizeof(psc::MarchUniforms), cudaMemcpyHostToDevice, s), "batch uniforms H2D");
  PSC_CUDA(cudaMemcpyAsync(c->d_bv, c->h_bv, n * sizeof(psc::ViewDev), cudaMemcpyHostToDevice, s), "batch views H2D");
  PSC_CUDA(cudaMemcpyAsync(c->d_bframes, c->h_bframes, n * fl, cudaMemcpyHostToDevice, s), "batch frames H2D");
  PSC_CUDA(cudaMemcpyAsync(c->d_btiles, c->h_btiles, n_tiles * sizeof(uint32_t), cudaMemcpyHostToDevice, s), "batch tiles H2D");
  // Under capture the record must become an external event node so that the
  // next call can wait on it after a graph launch.
  PSC_CUDA(cudaEventRecordWithFlags(c->batch_staged, s, capturing ? cudaEventRecordExternal : 0),
           "batch event");
  const bool any_bake = std::find(c->batch_bake.begin(), c->batch_bake.begin() + n, 1) != c->batch_bake.begin() + n;
  if (any_bake && psc::launch_view_lut_bakes(c->world, c->d_bframes, n, c->d_lut_h[PSC_LUT_TRANSMITTANCE],
                                             c->d_lut_h[PSC_LUT_MULTISCATTER], c->d_bsky, c->d_bap, s))
    return fail(PSC_ERR_CUDA, "per-view LUT bake launch failed");
  PSC_CUDA(cudaMemsetAsync(c->d_bcounter, 0, sizeof(uint32_t), s), "batch counter reset");
  const int rc = psc::launch_march_batch(c->opts, (int)c->batch_tuning.threads, c->batch_tuning.tile_w,
                                         c->d_bu, c->d_bv, c->d_btiles, n_tiles, c->d_bcounter, c->sms,
                                         psc::needs_full_paths(c->h_bu, n), s);
  if (rc == PSC_ERR_UNSUPPORTED)
    return fail(rc, "batched march supports F16/U8/F32 exact, F16/U8 hybrid and U8 texture storage");
  if (rc) return fail(rc, "batched march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  return PSC_OK;
}

// The float4 copy of LUT `kind` and, for the transmittance and sky-view
// LUTs, the texture objects over it; created once per context.
int ensure_lut_float4(psc_ctx* c, int kind) {
  const size_t n = lut_texels(kind);
  if (!c->d_lut[kind]) {
    PSC_CUDA(cudaMalloc(&c->d_lut[kind], n * sizeof(float4)), "cudaMalloc LUT");
    if (kind == PSC_LUT_TRANSMITTANCE) {
      // bilinear, clamp-to-edge, normalised coordinates: the LUT sampler of
      // the reference (crates/ps-clouds/src/lib.rs:256-265), bound to the
      // float4 copy so later uploads and bakes need no new object
      const uint32_t w = PSC_TRANSMITTANCE_W, h = PSC_TRANSMITTANCE_H;
      cudaResourceDesc rd{};
      rd.resType = cudaResourceTypePitch2D;
      rd.res.pitch2D.devPtr = c->d_lut[kind];
      rd.res.pitch2D.desc = cudaCreateChannelDesc<float4>();
      rd.res.pitch2D.width = w;
      rd.res.pitch2D.height = h;
      rd.res.pitch2D.pitchInBytes = (size_t)w * sizeof(float4);
      cudaTextureDesc td{};
      td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
      td.filterMode = cudaFilterModeLinear;
      td.readMode = cudaReadModeElementType;
      td.normalizedCoords = 1;
      PSC_CUDA(cudaCreateTextureObject(&c->tex_lut[kind], &rd, &td, nullptr), "LUT texture object");
    }
  }
  if (kind == PSC_LUT_SKYVIEW) {
    // the sky-view LUT also lives in a float4 array behind a texture object
    // (bilinear, clamp, normalised coordinates), refreshed on every upload
    // and bake
    if (!c->arr_sky) {
      const cudaChannelFormatDesc fmt = cudaCreateChannelDesc<float4>();
      PSC_CUDA(cudaMallocArray(&c->arr_sky, &fmt, PSC_SKYVIEW_W, PSC_SKYVIEW_H), "cudaMallocArray sky-view");
      cudaResourceDesc rd{};
      rd.resType = cudaResourceTypeArray;
      rd.res.array.array = c->arr_sky;
      cudaTextureDesc td{};
      td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
      td.filterMode = cudaFilterModeLinear;
      td.readMode = cudaReadModeElementType;
      td.normalizedCoords = 1;
      PSC_CUDA(cudaCreateTextureObject(&c->tex_lut[kind], &rd, &td, nullptr), "sky-view texture object");
    }
  }
  return PSC_OK;
}

int upload_lut_float4(psc_ctx* c, int kind, const uint16_t* h16) {
  const size_t n = lut_texels(kind);
  std::vector<float> f(n * 4);
  for (size_t i = 0; i < n * 4; ++i) f[i] = half_bits_to_float(h16[i]);
  int rc = ensure_lut_float4(c, kind);
  if (rc) return rc;
  PSC_CUDA(cudaMemcpy(c->d_lut[kind], f.data(), n * sizeof(float4), cudaMemcpyHostToDevice), "LUT upload");
  if (kind == PSC_LUT_SKYVIEW) {
    const size_t row = PSC_SKYVIEW_W * sizeof(float4);
    PSC_CUDA(cudaMemcpy2DToArray(c->arr_sky, 0, 0, c->d_lut[kind], row, row, PSC_SKYVIEW_H,
                                 cudaMemcpyDeviceToDevice), "sky-view array copy");
  }
  c->have_lut[kind] = true;
  return PSC_OK;
}

// Grow-only device scratch of `n` elements of T.
template <class T>
int grow(T** p, size_t* cap, size_t n, const char* what) {
  if (*cap >= n && *p) return PSC_OK;
  dfree(*p);
  *cap = 0;
  PSC_CUDA(cudaMalloc(p, n * sizeof(T)), what);
  *cap = n;
  return PSC_OK;
}

void half_res_dims(uint32_t w, uint32_t h, uint32_t* rw, uint32_t* rh) {
  *rw = std::max(1u, (uint32_t)((float)w * 0.5f));  // lib.rs:751-758
  *rh = std::max(1u, (uint32_t)((float)h * 0.5f));
}

void free_taa_view(psc_ctx::TaaView& tv) {
  for (int k = 0; k < 2; ++k) {
    dfree(tv.l[k]);
    dfree(tv.t[k]);
  }
  tv.w = tv.h = 0;
  tv.valid = false;
}

// One TAA frame of the active view (lib.rs:776-825 bookkeeping, then the
// resolve pass): on the first active frame (the view's previous march was
// not resolved), after a resize or an invalidation the history is not valid
// and the resolve is the current sample; otherwise the write slot flips and
// the current sample weighs 1/8.  *res_l / *res_t point at the resolved pair
// (the new history slot).
int taa_step(psc_ctx* c, const float4* cur_l, const float4* cur_t, uint32_t w, uint32_t h,
             cudaStream_t s, const float4** res_l, const float4** res_t) {
  psc_ctx::TaaView& tv = c->taa[c->active_view];
  const bool just_enabled = tv.marches == 0 || tv.resolved_at != tv.marches - 1;
  tv.resolved_at = tv.marches;
  if (tv.w != w || tv.h != h || !tv.l[0]) {
    free_taa_view(tv);
    for (int k = 0; k < 2; ++k) {
      PSC_CUDA(cudaMalloc(&tv.l[k], (size_t)w * h * sizeof(float4)), "cudaMalloc TAA history");
      PSC_CUDA(cudaMalloc(&tv.t[k], (size_t)w * h * sizeof(float4)), "cudaMalloc TAA history");
    }
    tv.w = w;
    tv.h = h;
    tv.valid = false;
  }
  if (just_enabled) tv.valid = false;
  tv.write_slot = tv.valid ? (tv.write_slot ^ 1u) : 0u;
  const uint32_t ws = tv.write_slot;
  psc::TaaParams p{};
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      p.inv_vp[col][row] = c->frame.inv_view_proj[col][row];
      p.prev_vp[col][row] = c->frame.prev_view_proj[col][row];
    }
  for (int k = 0; k < 3; ++k) p.cam[k] = c->frame.camera_position_world[k];
  p.blend_weight = tv.valid ? 1.0f / 8.0f : 1.0f;  // TAA_BLEND_WEIGHT, lib.rs:42
  p.history_valid = tv.valid ? 1.0f : 0.0f;
  p.w = w;
  p.h = h;
  p.cur_l = cur_l;
  p.cur_t = cur_t;
  p.hist_l = tv.l[ws ^ 1u];
  p.hist_t = tv.t[ws ^ 1u];
  p.out_l = tv.l[ws];
  p.out_t = tv.t[ws];
  if (psc::launch_taa_resolve(p, s)) return fail(PSC_ERR_CUDA, "TAA launch failed");
  ++c->launches;
  tv.valid = true;
  *res_l = tv.l[ws];
  *res_t = tv.t[ws];
  return PSC_OK;
}

const char* check_site_name(int site) {
  static const char* names[] = {"?",         "base noise", "detail noise",     "curl",
                                "weather",   "type grid",  "transmittance LUT", "sky-view LUT",
                                "aerial LUT", "blue noise", "pixel",            "layer"};
  return (site > 0 && site < (int)(sizeof(names) / sizeof(names[0]))) ? names[site] : names[0];
}

// One view's march.  options.debug_checks runs the PLAIN schedule's checked
// kernel (exact filtering unless U8 texture): every index is compared with
// its buffer, the first violation is recorded in a device word and the call
// waits for the kernel to report it.
int launch_view_march(psc_ctx* c, psc::MarchUniforms& u, const psc::ViewDev& vd, cudaStream_t s) {
  if (c->opts.debug_checks) {
    if (!c->d_check) PSC_CUDA(cudaMalloc(&c->d_check, sizeof(int)), "cudaMalloc check word");
    PSC_CUDA(cudaMemsetAsync(c->d_check, 0, sizeof(int), s), "check word reset");
    u.error_word = c->d_check;
    PscMarchOptions o = c->opts;
    o.schedule = PSC_SCHED_PLAIN;
    if (!(o.filter == PSC_FILTER_TEXTURE && o.storage == PSC_STORAGE_U8)) o.filter = PSC_FILTER_EXACT;
    const int rc = psc::launch_march(u, vd, o, s);
    if (rc) return fail(rc, "checked march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
    ++c->launches;
    int site = 0;
    PSC_CUDA(cudaMemcpyAsync(&site, c->d_check, sizeof(int), cudaMemcpyDeviceToHost, s), "check word read");
    PSC_CUDA(cudaStreamSynchronize(s), "checked march");
    if (site) return fail(PSC_ERR_DEVICE_CHECK, "debug check: out-of-range %s index (skipped)", check_site_name(site));
    return PSC_OK;
  }
  int rc = PSC_ERR_UNSUPPORTED;
  if (c->opts.schedule == PSC_SCHED_FAST) rc = psc::launch_march_fast(u, vd, c->opts, s);
  if (rc == PSC_ERR_UNSUPPORTED) rc = psc::launch_march(u, vd, c->opts, s);
  if (rc) return fail(rc, "march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  ++c->launches;
  return PSC_OK;
}

// The half-res / TAA form of psc_render for one whole-viewport view: march
// into the cloud RT, resolve, copy out, composite.
int render_rt_view(psc_ctx* c, const PscView& v, cudaStream_t s) {
  const uint32_t W = v.width, H = v.height;
  uint32_t rw = W, rh = H;
  if (c->opts.half_res) half_res_dims(W, H, &rw, &rh);
  const size_t n_rt = (size_t)rw * rh;
  if (c->rt_cap < n_rt || !c->d_rt_l || !c->d_rt_t) {  // L and T grow together
    dfree(c->d_rt_l);
    dfree(c->d_rt_t);
    c->rt_cap = 0;
    PSC_CUDA(cudaMalloc(&c->d_rt_l, n_rt * sizeof(float4)), "cudaMalloc cloud RT");
    PSC_CUDA(cudaMalloc(&c->d_rt_t, n_rt * sizeof(float4)), "cudaMalloc cloud RT");
    c->rt_cap = n_rt;
  }
  int rc = PSC_OK;
  const float* depth = v.depth;
  if (c->opts.half_res && v.depth) {
    rc = grow(&c->d_rt_depth, &c->rt_depth_cap, n_rt, "cudaMalloc cloud-RT depth");
    if (rc) return rc;
    if (psc::launch_depth_halfres(v.depth, W, H, c->d_rt_depth, rw, rh, s))
      return fail(PSC_ERR_CUDA, "half-res depth launch failed");
    ++c->launches;
    depth = c->d_rt_depth;
  }
  psc::MarchUniforms u;
  build_uniforms(c, rw, rh, u);
  u.composite = 0;
  psc::ViewDev vd{rw, rh, 0, 0, depth, c->d_rt_l, c->d_rt_t, nullptr};
  rc = launch_view_march(c, u, vd, s);
  if (rc) return rc;
  const float4 *src_l = c->d_rt_l, *src_t = c->d_rt_t;
  if (c->opts.taa) {
    rc = taa_step(c, c->d_rt_l, c->d_rt_t, rw, rh, s, &src_l, &src_t);
    if (rc) return rc;
  }
  if (v.out_luminance)
    PSC_CUDA(cudaMemcpyAsync(v.out_luminance, src_l, n_rt * sizeof(float4), cudaMemcpyDeviceToDevice, s),
             "cloud RT copy");
  if (v.out_transmittance)
    PSC_CUDA(cudaMemcpyAsync(v.out_transmittance, src_t, n_rt * sizeof(float4), cudaMemcpyDeviceToDevice, s),
             "cloud RT copy");
  if (c->opts.composite) {
    const int e = c->opts.half_res
                      ? psc::launch_composite_halfres(src_l, src_t, rw, rh, reinterpret_cast<float4*>(v.hdr), W, H, s)
                      : psc::launch_composite(src_l, src_t, reinterpret_cast<float4*>(v.hdr), W * H, s);
    if (e) return fail(PSC_ERR_CUDA, "composite launch failed");
    ++c->launches;
  }
  return PSC_OK;
}

}  // namespace

namespace psc {
namespace host {

int validate_batch(psc_ctx* c, const PscBatchView* views, uint32_t n) {
  if (!c->have_base || !c->have_detail || !c->have_curl || !c->have_blue)
    return fail(PSC_ERR_MISSING_INPUT, "noise volumes missing (psc_bake_noise or psc_upload_noise)");
  if (!c->d_weather) return fail(PSC_ERR_MISSING_INPUT, "weather map missing (psc_upload_weather)");
  if (!c->d_lut_h[PSC_LUT_TRANSMITTANCE] || !c->d_lut_h[PSC_LUT_MULTISCATTER] || !c->have_lut[PSC_LUT_TRANSMITTANCE])
    return fail(PSC_ERR_MISSING_INPUT, "transmittance/multi-scatter LUTs missing (psc_bake_luts or psc_upload_lut)");
  if (c->opts.schedule != PSC_SCHED_FAST)
    return fail(PSC_ERR_UNSUPPORTED, "the batched kernel implements the FAST schedule (options.schedule)");
  if (c->opts.half_res || c->opts.taa || c->opts.debug_checks)
    return fail(PSC_ERR_UNSUPPORTED,
                "the batched kernel renders full-resolution views without TAA or debug checks");
  for (uint32_t i = 0; i < n; ++i) {
    const PscBatchView& v = views[i];
    if (!v.width || !v.height || v.width > 32768 || v.height > 32768)
      return fail(PSC_ERR_INVALID_ARGUMENT, "batch view %u: size %ux%u out of range", i, v.width, v.height);
    if (!v.out_luminance && !v.out_transmittance && !(c->opts.composite && v.hdr))
      return fail(PSC_ERR_INVALID_ARGUMENT, "batch view %u has no output buffer", i);
    if (c->opts.composite && !v.hdr) return fail(PSC_ERR_INVALID_ARGUMENT, "batch view %u: composite needs hdr", i);
    int rc = validate_layers(v.layers, v.n_layers);
    if (rc) return fail(rc, "batch view %u: %s", i, g_last_error.c_str());
    PscCloudParamsGpu p = v.params;
    p.cloud_layer_count = v.n_layers;
    rc = validate_params(p);
    if (rc) return fail(rc, "batch view %u: %s", i, g_last_error.c_str());
    if (p.multi_scatter_octaves == 0 || p.multi_scatter_octaves > 4)
      return fail(PSC_ERR_UNSUPPORTED, "batch view %u: the batched kernel handles 1..4 octaves", i);
    const float* ff = reinterpret_cast<const float*>(&v.frame);
    for (size_t k = 0; k < sizeof(v.frame) / 4; ++k)
      if (k != 94 && !std::isfinite(ff[k])) return fail(PSC_ERR_NOT_FINITE, "batch view %u: frame word %zu", i, k);
  }
  return PSC_OK;
}

uint64_t count_batch_tiles(const PscBatchView* views, uint32_t n, const PscBatchTuning& tu) {
  const uint32_t tile_w = tu.tile_w, tile_h = (tu.threads / 32 / (tu.tile_w / 8)) * 4;
  uint64_t total = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const uint64_t tx = (views[i].width + tile_w - 1) / tile_w, ty = (views[i].height + tile_h - 1) / tile_h;
    if (tx > 4096 || ty > 4096) return UINT64_MAX;
    total += tx * ty;
  }
  return total;
}

// Same records and tile order as the allocating batch path, written into
// caller-provided host arrays with no heap use (n <= PSC_MAX_BATCH_VIEWS;
// the view order is a stable insertion sort).
int fill_batch(const psc_ctx* c, const PscBatchView* views, uint32_t n, const PscBatchTuning& tu,
               MarchUniforms* hu, ViewDev* hv, void* hframes, uint32_t* htiles, uint32_t max_tiles,
               float4* sky, float4* ap, uint32_t* n_tiles_out) {
  const uint32_t tile_w = tu.tile_w, tile_h = (tu.threads / 32 / (tu.tile_w / 8)) * 4;
  const size_t fl = psc::frame_lite_size();
  for (uint32_t i = 0; i < n; ++i) {
    const PscBatchView& bv = views[i];
    build_batch_view_uniforms(c, bv, sky + (size_t)i * PSC_SKYVIEW_W * PSC_SKYVIEW_H,
                              ap + (size_t)i * PSC_AP_W * PSC_AP_H * PSC_AP_D, hu[i]);
    hv[i] = psc::ViewDev{bv.width, bv.height, 0, 0, bv.depth, reinterpret_cast<float4*>(bv.out_luminance),
                         reinterpret_cast<float4*>(bv.out_transmittance), reinterpret_cast<float4*>(bv.hdr)};
    psc::frame_lite_from(bv.frame, static_cast<char*>(hframes) + i * fl);
  }
  auto cost = [&](uint32_t i) {
    return (double)views[i].params.cloud_steps * (double)std::max<uint32_t>(views[i].n_layers, 1);
  };
  auto before = [&](uint32_t a, uint32_t b) {
    const double ca = cost(a), cb = cost(b);
    if (ca != cb) return ca > cb;
    return (uint64_t)views[a].width * views[a].height > (uint64_t)views[b].width * views[b].height;
  };
  uint32_t order[PSC_MAX_BATCH_VIEWS];
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t j = i;
    for (; j > 0 && before(i, order[j - 1]); --j) order[j] = order[j - 1];
    order[j] = i;
  }
  uint32_t k = 0;
  for (uint32_t oi = 0; oi < n; ++oi) {
    const uint32_t i = order[oi];
    const uint32_t tx = (views[i].width + tile_w - 1) / tile_w, ty = (views[i].height + tile_h - 1) / tile_h;
    if ((uint64_t)k + (uint64_t)tx * ty > max_tiles)
      return fail(PSC_ERR_INVALID_ARGUMENT, "batch needs more than %u tiles", max_tiles);
    for (uint32_t y = 0; y < ty; ++y)
      for (uint32_t x = 0; x < tx; ++x) htiles[k++] = (i << 24) | (x << 12) | y;
  }
  *n_tiles_out = k;
  return PSC_OK;
}

bool storage_ready(const psc_ctx* c) {
  const bool store = c->d_base_store && c->d_detail_store && c->store_form == (int)c->opts.storage;
  const bool tex = c->opts.filter == PSC_FILTER_EXACT || (!c->tex_dirty && c->tex_base && c->tex_detail);
  return store && tex;
}

}  // namespace host
}  // namespace psc

extern "C" {

const char* psc_last_error(void) { return g_last_error.c_str(); }
uint32_t psc_abi_version(void) { return PSC_ABI_VERSION; }

#ifndef PSC_BUILD_ID
#define PSC_BUILD_ID "unknown"
#endif
const char* psc_build_id(void) { return PSC_BUILD_ID; }
size_t psc_sizeof_params(void) { return sizeof(PscCloudParamsGpu); }
size_t psc_sizeof_layer(void) { return sizeof(PscCloudLayerGpu); }
size_t psc_sizeof_frame(void) { return sizeof(PscFrameUniformsGpu); }
size_t psc_sizeof_world(void) { return sizeof(PscWorldUniformsGpu); }

int psc_params_default(PscCloudParamsGpu* o) {  // params.rs:142-212
  if (!o) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  std::memset(o, 0, sizeof(*o));
  o->sigma_s[0] = 0.030f;
  o->sigma_s[1] = 0.040f;
  o->sigma_s[2] = 0.060f;
  o->droplet_diameter_bias = 1.0f;
  o->detail_strength = 0.05f;
  o->curl_strength = 0.1f;
  o->powder_strength = 1.0f;
  o->multi_scatter_a = o->multi_scatter_b = o->multi_scatter_c = 0.5f;
  o->ambient_strength = 1.0f;
  o->base_scale_m = 4500.0f;
  o->detail_scale_m = 800.0f;
  o->weather_scale_m = 32000.0f;
  o->light_steps = 6;
  o->cloud_steps = 192;
  o->multi_scatter_octaves = 4;
  o->wind_drift_strength = 1.0f;
  o->wind_skew_strength = 0.5f;
  o->diurnal_strength = 1.0f;
  return PSC_OK;
}

int psc_world_default(PscWorldUniformsGpu* o) {  // weather.rs:60-84
  if (!o) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  std::memset(o, 0, sizeof(*o));
  o->planet_radius_m = 6360000.0f;
  o->atmosphere_top_m = 6460000.0f;
  o->rayleigh_scale_height_m = 8000.0f;
  o->mie_scale_height_m = 1200.0f;
  const float ray[3] = {5.802e-6f, 13.558e-6f, 33.100e-6f};
  const float oz[3] = {0.650e-6f, 1.881e-6f, 0.085e-6f};
  for (int k = 0; k < 3; ++k) {
    o->rayleigh_scattering[k] = ray[k];
    o->mie_scattering[k] = 3.996e-6f;
    o->mie_absorption[k] = 4.4e-6f;
    o->ozone_absorption[k] = oz[k];
    o->ground_albedo[k] = 0.18f;
  }
  o->mie_g = 0.8f;
  o->ozone_center_m = 25000.0f;
  o->ozone_thickness_m = 30000.0f;
  return PSC_OK;
}

int psc_options_default(PscMarchOptions* o) {
  if (!o) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  std::memset(o, 0, sizeof(*o));
  o->phase_mode = PSC_PHASE_APPROX_MIE;
  o->hg_g_forward = 0.8f;
  o->hg_g_backward = -0.2f;
  o->hg_blend = 0.5f;
  o->storage = PSC_STORAGE_U8;
  o->filter = PSC_FILTER_EXACT;
  o->schedule = PSC_SCHED_PLAIN;
  return PSC_OK;
}

// cloud_layers.rs:106-126
static float remap_coverage(float sc) {
  const float lo = 0.40f, hi = 0.60f, knee = 0.10f;
  const float t = std::fmin(std::fmax(sc, 0.0f), 1.0f);
  if (t <= 0.0f) return 0.0f;
  if (t < knee) {
    const float s = t / knee;
    return (s * s * (3.0f - 2.0f * s)) * lo;
  }
  const float bt = std::fmin(std::fmax((t - knee) / (1.0f - knee), 0.0f), 1.0f);
  return lo + bt * (hi - lo);
}

int psc_synthesise_layers(const PscCloudLayerDesc* in, uint32_t n, PscCloudLayerGpu* out) {
  if ((n && !in) || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null layer pointer");
  if (n > PSC_MAX_CLOUD_LAYERS) return fail(PSC_ERR_LAYERS, "%u layers exceeds the maximum of 8", n);
  static const float dens[8] = {1.0f, 1.0f, 1.0f, 0.85f, 0.7f, 0.55f, 0.4f, 1.4f};  // scene.rs:293-302
  static const float drop[8] = {20.0f, 16.0f, 16.0f, 14.0f, 30.0f, 50.0f, 50.0f, 20.0f};  // :334-352
  for (uint32_t i = 0; i < n; ++i) {
    const PscCloudLayerDesc& d = in[i];
    if (d.cloud_type > 7) return fail(PSC_ERR_LAYERS, "layer %u: cloud_type %u > 7", i, d.cloud_type);
    PscCloudLayerGpu g{};
    g.base_m = d.base_m;
    g.top_m = d.top_m;
    g.coverage = remap_coverage(d.coverage);
    g.density_scale = d.density_scale >= 0.0f ? d.density_scale : dens[d.cloud_type];
    g.cloud_type = d.cloud_type;
    g.shape_bias = d.shape_octave_bias;
    g.detail_bias = d.detail_octave_bias;
    g.anvil_bias = d.anvil_bias >= 0.0f ? d.anvil_bias : (d.cloud_type == 7 ? 1.0f : 0.0f);
    g.droplet_diameter_um = d.droplet_diameter_um >= 0.0f ? d.droplet_diameter_um : drop[d.cloud_type];
    out[i] = g;
  }
  return validate_layers(out, n);
}

int psc_frame_from_camera(const PscFlyCamera* cam, uint32_t width, uint32_t height, float sun_alt,
                          float sun_az, float sun_ang, float lux, PscFrameUniformsGpu* o) {
  if (!cam || !o) return fail(PSC_ERR_INVALID_ARGUMENT, "null camera or output");
  if (!width || !height) return fail(PSC_ERR_INVALID_ARGUMENT, "zero-size viewport");
  const float vals[] = {cam->position[0], cam->position[1], cam->position[2], cam->pitch_rad,
                        cam->yaw_rad, cam->roll_rad, cam->fov_y_rad, cam->near_m, sun_alt, sun_az,
                        sun_ang, lux};
  if (!all_finite(vals, 12)) return fail(PSC_ERR_NOT_FINITE, "non-finite camera or sun value");
  if (!(cam->fov_y_rad > 0.0f && cam->fov_y_rad < 3.14159f) || !(cam->near_m > 0.0f))
    return fail(PSC_ERR_INVALID_ARGUMENT, "fov_y must be in (0, pi) and near_m > 0");
  std::memset(o, 0, sizeof(*o));
  // FlyCamera::forward / look_to_rh / perspective_infinite_reverse_rh
  const double yaw = cam->yaw_rad, pitch = cam->pitch_rad;
  double fw[3] = {std::cos(pitch) * std::sin(yaw), std::sin(pitch), -std::cos(pitch) * std::cos(yaw)};
  double n = std::sqrt(fw[0] * fw[0] + fw[1] * fw[1] + fw[2] * fw[2]);
  for (double& v : fw) v /= n;
  double rt[3] = {-fw[2], 0.0, fw[0]};  // forward x (0,1,0)
  n = std::sqrt(rt[0] * rt[0] + rt[2] * rt[2]);
  for (double& v : rt) v /= n;
  const double up[3] = {rt[1] * fw[2] - rt[2] * fw[1], rt[2] * fw[0] - rt[0] * fw[2],
                        rt[0] * fw[1] - rt[1] * fw[0]};
  const double eye[3] = {cam->position[0], cam->position[1], cam->position[2]};
  double V[4][4] = {};  // [col][row]
  for (int k = 0; k < 3; ++k) {
    V[k][0] = rt[k];
    V[k][1] = up[k];
    V[k][2] = -fw[k];
  }
  V[3][0] = -(eye[0] * rt[0] + eye[1] * rt[1] + eye[2] * rt[2]);
  V[3][1] = -(eye[0] * up[0] + eye[1] * up[1] + eye[2] * up[2]);
  V[3][2] = eye[0] * fw[0] + eye[1] * fw[1] + eye[2] * fw[2];
  V[3][3] = 1.0;
  if (cam->roll_rad != 0.0f) {  // Mat4::from_rotation_z(roll) * view
    const double cr = std::cos((double)cam->roll_rad), sr = std::sin((double)cam->roll_rad);
    double Rm[4][4] = {{cr, sr, 0, 0}, {-sr, cr, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
    double T[4][4];
    for (int col = 0; col < 4; ++col)
      for (int row = 0; row < 4; ++row) {
        double s = 0;
        for (int k = 0; k < 4; ++k) s += Rm[k][row] * V[col][k];
        T[col][row] = s;
      }
    std::memcpy(V, T, sizeof(V));
  }
  const double f = 1.0 / std::tan(0.5 * (double)cam->fov_y_rad);
  double P[4][4] = {};
  P[0][0] = f / ((double)width / (double)height);
  P[1][1] = f;
  P[2][3] = -1.0;
  P[3][2] = cam->near_m;
  double VP[4][4];
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      double s = 0;
      for (int k = 0; k < 4; ++k) s += P[k][row] * V[col][k];
      VP[col][row] = s;
    }
  // inverse via the adjugate (cofactor expansion in 2x2 minors)
  const double* m = &VP[0][0];  // m[col*4+row]
  auto a = [&](int row, int col) { return m[col * 4 + row]; };
  double s0 = a(0, 0) * a(1, 1) - a(1, 0) * a(0, 1), s1 = a(0, 0) * a(1, 2) - a(1, 0) * a(0, 2);
  double s2 = a(0, 0) * a(1, 3) - a(1, 0) * a(0, 3), s3 = a(0, 1) * a(1, 2) - a(1, 1) * a(0, 2);
  double s4 = a(0, 1) * a(1, 3) - a(1, 1) * a(0, 3), s5 = a(0, 2) * a(1, 3) - a(1, 2) * a(0, 3);
  double c5 = a(2, 2) * a(3, 3) - a(3, 2) * a(2, 3), c4 = a(2, 1) * a(3, 3) - a(3, 1) * a(2, 3);
  double c3 = a(2, 1) * a(3, 2) - a(3, 1) * a(2, 2), c2 = a(2, 0) * a(3, 3) - a(3, 0) * a(2, 3);
  double c1 = a(2, 0) * a(3, 2) - a(3, 0) * a(2, 2), c0 = a(2, 0) * a(3, 1) - a(3, 0) * a(2, 1);
  const double det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
  if (det == 0.0 || !std::isfinite(det)) return fail(PSC_ERR_INVALID_ARGUMENT, "singular view-projection");
  const double id = 1.0 / det;
  double inv[4][4];  // inv[row][col]
  inv[0][0] = (a(1, 1) * c5 - a(1, 2) * c4 + a(1, 3) * c3) * id;
  inv[0][1] = (-a(0, 1) * c5 + a(0, 2) * c4 - a(0, 3) * c3) * id;
  inv[0][2] = (a(3, 1) * s5 - a(3, 2) * s4 + a(3, 3) * s3) * id;
  inv[0][3] = (-a(2, 1) * s5 + a(2, 2) * s4 - a(2, 3) * s3) * id;
  inv[1][0] = (-a(1, 0) * c5 + a(1, 2) * c2 - a(1, 3) * c1) * id;
  inv[1][1] = (a(0, 0) * c5 - a(0, 2) * c2 + a(0, 3) * c1) * id;
  inv[1][2] = (-a(3, 0) * s5 + a(3, 2) * s2 - a(3, 3) * s1) * id;
  inv[1][3] = (a(2, 0) * s5 - a(2, 2) * s2 + a(2, 3) * s1) * id;
  inv[2][0] = (a(1, 0) * c4 - a(1, 1) * c2 + a(1, 3) * c0) * id;
  inv[2][1] = (-a(0, 0) * c4 + a(0, 1) * c2 - a(0, 3) * c0) * id;
  inv[2][2] = (a(3, 0) * s4 - a(3, 1) * s2 + a(3, 3) * s0) * id;
  inv[2][3] = (-a(2, 0) * s4 + a(2, 1) * s2 - a(2, 3) * s0) * id;
  inv[3][0] = (-a(1, 0) * c3 + a(1, 1) * c1 - a(1, 2) * c0) * id;
  inv[3][1] = (a(0, 0) * c3 - a(0, 1) * c1 + a(0, 2) * c0) * id;
  inv[3][2] = (-a(3, 0) * s3 + a(3, 1) * s1 - a(3, 2) * s0) * id;
  inv[3][3] = (a(2, 0) * s3 - a(2, 1) * s1 + a(2, 2) * s0) * id;
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      o->view[col][row] = (float)V[col][row];
      o->proj[col][row] = (float)P[col][row];
      o->view_proj[col][row] = (float)VP[col][row];
      o->prev_view_proj[col][row] = (float)VP[col][row];
      o->inv_view_proj[col][row] = (float)inv[row][col];
    }
  o->camera_position_world[0] = cam->position[0];
  o->camera_position_world[1] = std::fmax(cam->position[1], 0.1f);  // test_harness.rs:356
  o->camera_position_world[2] = cam->position[2];
  o->viewport_size[0] = (float)width;
  o->viewport_size[1] = (float)height;
  o->viewport_size[2] = 1.0f / (float)width;
  o->viewport_size[3] = 1.0f / (float)height;
  // altaz_to_world, world.rs:110-114
  const double sa = std::sin((double)sun_alt), ca = std::cos((double)sun_alt);
  const double sz = std::sin((double)sun_az), cz = std::cos((double)sun_az);
  o->sun_direction[0] = (float)(ca * sz);
  o->sun_direction[1] = (float)sa;
  o->sun_direction[2] = (float)(-ca * cz);
  o->sun_direction[3] = sun_ang;
  for (int k = 0; k < 4; ++k) o->sun_illuminance[k] = lux;
  return PSC_OK;
}

// Void-and-cluster blue noise (crates/ps-clouds/src/noise.rs:646-704).
int psc_generate_blue_noise(uint8_t* out) {
  if (!out) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  const int S = 64, N = S * S, rad = 6;
  const float sigma = 1.9f;
  const float k = 1.0f / ((2.0f * sigma) * sigma);
  // splat kernel, row-major over (dy, dx) in [-6, 6]^2
  float kern[13 * 13];
  for (int dy = -rad; dy <= rad; ++dy)
    for (int dx = -rad; dx <= rad; ++dx)
      kern[(dy + rad) * 13 + (dx + rad)] = std::exp(-(float)(dx * dx + dy * dy) * k) * 1.0f;
  std::vector<float> energy(N, 0.0f);
  std::vector<uint32_t> rank(N, 0);
  std::vector<uint8_t> placed(N, 0);
  for (int step = 0; step < N; ++step) {
    int best = 0;
    float be = INFINITY;
    for (int i = 0; i < N; ++i)
      if (!placed[i] && energy[i] < be) {
        be = energy[i];
        best = i;
      }
    placed[best] = 1;
    rank[best] = (uint32_t)step;
    const int cx = best % S, cy = best / S;
    for (int dy = -rad; dy <= rad; ++dy) {
      const int yy = ((cy + dy) % S + S) % S;
      for (int dx = -rad; dx <= rad; ++dx) {
        const int xx = ((cx + dx) % S + S) % S;
        energy[yy * S + xx] += kern[(dy + rad) * 13 + (dx + rad)];
      }
    }
  }
  const float maxr = (float)(N - 1);
  for (int i = 0; i < N; ++i) {
    const float v = std::round(((float)rank[i] / maxr) * 255.0f);
    out[i] = (uint8_t)std::fmin(std::fmax(v, 0.0f), 255.0f);
  }
  return PSC_OK;
}

// weather_map.rs:160-183
static float wm_hash2(int32_t x, int32_t y) {
  uint32_t h = (uint32_t)x * 2654435761u;
  h ^= (uint32_t)y * 2246822519u;
  h ^= h >> 16;
  h *= 2654435761u;
  h ^= h >> 13;
  return std::fmin(std::fmax((float)h / 4294967296.0f, 0.0f), 1.0f);
}
static float wm_value_noise(float x, float y) {
  const float xi = std::floor(x), yi = std::floor(y);
  const float xf = x - xi, yf = y - yi;
  const int32_t ix = (int32_t)xi, iy = (int32_t)yi;
  const float h00 = wm_hash2(ix, iy), h10 = wm_hash2(ix + 1, iy);
  const float h01 = wm_hash2(ix, iy + 1), h11 = wm_hash2(ix + 1, iy + 1);
  const float sx = xf * xf * (3.0f - 2.0f * xf), sy = yf * yf * (3.0f - 2.0f * yf);
  const float b = h00 + (h10 - h00) * sx, t = h01 + (h11 - h01) * sx;
  return b + (t - b) * sy;
}

int psc_synthesise_weather_map(uint32_t n_layers, float precip, float wet, const float* grid,
                               uint32_t gw, uint32_t gh, float gext, uint16_t* out) {
  if (!out) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  if (grid && (gw < 1 || gh < 1 || !(gext > 0.0f)))
    return fail(PSC_ERR_INVALID_ARGUMENT, "coverage grid needs w,h >= 1 and extent > 0");
  const float gate = n_layers ? 1.0f : 0.0f;
  const float alpha = std::fmax(std::fmin(std::fmax(precip / 50.0f, 0.0f), 1.0f),
                                std::fmin(std::fmax(wet, 0.0f), 1.0f));
  for (uint32_t y = 0; y < 128; ++y)
    for (uint32_t x = 0; x < 128; ++x) {
      float cov = gate;
      if (grid) {  // coverage_grid.rs:34-60, sample_world
        const float gx = (((float)x + 0.5f) / 128.0f) * 32000.0f - 16000.0f;
        const float gy = (((float)y + 0.5f) / 128.0f) * 32000.0f - 16000.0f;
        const float half = gext * 0.5f;
        const float u = std::fmin(std::fmax((gx + half) / gext, 0.0f), 1.0f);
        const float v = std::fmin(std::fmax((gy + half) / gext, 0.0f), 1.0f);
        const float fx = u * ((float)gw - 1.0f), fy = v * ((float)gh - 1.0f);
        const uint32_t x0 = (uint32_t)std::floor(fx), y0 = (uint32_t)std::floor(fy);
        const uint32_t x1 = std::min(x0 + 1, gw - 1), y1 = std::min(y0 + 1, gh - 1);
        const float tx = fx - (float)x0, ty = fy - (float)y0;
        const float b = grid[y0 * gw + x0] + (grid[y0 * gw + x1] - grid[y0 * gw + x0]) * tx;
        const float t = grid[y1 * gw + x0] + (grid[y1 * gw + x1] - grid[y1 * gw + x0]) * tx;
        cov = std::fmin(std::fmax(b + (t - b) * ty, 0.0f), 1.0f);
      }
      const float bias = wm_value_noise((float)x * 0.05f, (float)y * 0.05f) * 2.0f - 1.0f;
      uint16_t* t = out + (y * 128 + x) * 4;
      t[0] = float_to_half_bits(cov);
      t[1] = float_to_half_bits(0.0f);
      t[2] = float_to_half_bits(bias);
      t[3] = float_to_half_bits(alpha);
    }
  return PSC_OK;
}

int psc_synthesise_wind_field(float speed, float dir_deg, uint16_t* out) {  // wind_field.rs:150-170
  if (!out) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  if (!std::isfinite(speed) || !std::isfinite(dir_deg)) return fail(PSC_ERR_NOT_FINITE, "non-finite wind");
  const float pi = 3.14159265358979323846f;
  const float to_rad = (dir_deg + 180.0f) * (pi / 180.0f);
  const float ekman = 30.0f * pi / 180.0f;
  for (uint32_t z = 0; z < 32; ++z)
    for (uint32_t y = 0; y < 16; ++y)
      for (uint32_t x = 0; x < 32; ++x) {
        const float alt = ((float)y + 0.5f) / 16.0f * 12000.0f;
        const float sp = speed * std::pow(std::fmax(alt, 10.0f) / 10.0f, 0.143f);
        const float veer = std::pow(std::fmin(std::fmax(alt / 12000.0f, 0.0f), 1.0f), 0.7f);
        const float ang = to_rad + veer * ekman;
        uint16_t* t = out + ((z * 16 + y) * 32 + x) * 4;
        t[0] = float_to_half_bits(sp * std::sin(ang));
        t[1] = float_to_half_bits(sp * -std::cos(ang));
        t[2] = 0;
        t[3] = 0;
      }
  return PSC_OK;
}

int psc_create(int device, psc_ctx** out) {
  if (!out) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  *out = nullptr;
  // The device is bound lazily: host-side state and validation work without
  // a GPU, and the first call that touches the device checks the ordinal.
  if (device < 0) return fail(PSC_ERR_INVALID_ARGUMENT, "device %d is negative", device);
  psc_ctx* c = new (std::nothrow) psc_ctx();
  if (!c) return fail(PSC_ERR_OUT_OF_MEMORY, "context allocation");
  c->device = device;
  psc_params_default(&c->params);
  c->params.cloud_layer_count = 0;
  psc_world_default(&c->world);
  psc_options_default(&c->opts);
  *out = c;
  return PSC_OK;
}

int psc_destroy(psc_ctx* c) {
  if (!c) return PSC_OK;
  const bool touched = c->d_base_u8 || c->d_detail_u8 || c->d_curl || c->d_blue || c->d_weather ||
                       c->d_type || c->d_lut[0] || c->d_lut_h[0] || c->d_lut[2] || c->d_lut_h[3] ||
                       c->d_bu || c->batch_stream;
  if (!touched) {
    delete c;
    return PSC_OK;
  }
  cudaSetDevice(c->device);
  destroy_textures(c);
  dfree(c->d_base_u8);
  dfree(c->d_detail_u8);
  dfree(c->d_base_store);
  dfree(c->d_detail_store);
  dfree(c->d_base_fold);
  dfree(c->d_base_quad);
  dfree(c->d_detail_fold);
  dfree(c->d_detail_quad);
  dfree(c->d_curl_quad);
  dfree(c->d_curl);
  dfree(c->d_rt_l);
  dfree(c->d_rt_t);
  dfree(c->d_rt_depth);
  dfree(c->d_check);
  dfree(c->d_grid_quads);
  dfree(c->d_grad_pairs);
  for (auto& tv : c->taa) free_taa_view(tv);
  dfree(c->d_blue);
  dfree(c->d_weather);
  dfree(c->d_weather_quad);
  dfree(c->d_type);
  for (int k = 0; k < 4; ++k) {
    if (c->tex_lut[k]) cudaDestroyTextureObject(c->tex_lut[k]);
    if (k == PSC_LUT_SKYVIEW && c->arr_sky) cudaFreeArray(c->arr_sky);
    dfree(c->d_lut[k]);
    dfree(c->d_lut_h[k]);
  }
  release_batch(c);
  delete c;
  return PSC_OK;
}

int psc_set_march_steps(psc_ctx* c, uint32_t cloud, uint32_t light) {  // lib.rs:709-712
  if (!c) return fail(PSC_ERR_INVALID_ARGUMENT, "null context");
  c->params.cloud_steps = std::min(std::max(cloud, 8u), 256u);
  c->params.light_steps = std::min(std::max(light, 1u), 16u);
  return PSC_OK;
}

int psc_set_params(psc_ctx* c, const PscCloudParamsGpu* p) {
  if (!c || !p) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  PscCloudParamsGpu q = *p;
  q.cloud_layer_count = c->n_layers;  // owned by psc_set_layers
  const int rc = validate_params(q);
  if (rc) return rc;
  c->params = q;
  return PSC_OK;
}

int psc_get_params(psc_ctx* c, PscCloudParamsGpu* out) {
  if (!c || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  *out = c->params;
  return PSC_OK;
}

int psc_set_layers(psc_ctx* c, const PscCloudLayerGpu* l, uint32_t n) {
  if (!c || (n && !l)) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  const int rc = validate_layers(l, n);
  if (rc) return rc;
  std::memset(c->layers, 0, sizeof(c->layers));
  for (uint32_t i = 0; i < n; ++i) c->layers[i] = l[i];
  c->n_layers = n;
  c->params.cloud_layer_count = n;
  return PSC_OK;
}

int psc_set_frame(psc_ctx* c, const PscFrameUniformsGpu* f, const PscWorldUniformsGpu* w) {
  if (!c || !f || !w) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  const float* ff = reinterpret_cast<const float*>(f);
  for (size_t i = 0; i < sizeof(*f) / 4; ++i)
    if (i != 94 && !std::isfinite(ff[i]))  // word 94 = frame_index (u32)
      return fail(PSC_ERR_NOT_FINITE, "FrameUniforms word %zu is not finite", i);
  if (!all_finite(reinterpret_cast<const float*>(w), sizeof(*w) / 4))
    return fail(PSC_ERR_NOT_FINITE, "WorldUniforms has a non-finite field");
  if (!(w->planet_radius_m > 0.0f) || !(w->atmosphere_top_m > w->planet_radius_m))
    return fail(PSC_ERR_INVALID_ARGUMENT, "need 0 < planet_radius_m < atmosphere_top_m");
  c->frame = *f;
  c->world = *w;
  c->have_frame = true;
  return PSC_OK;
}

int psc_set_options(psc_ctx* c, const PscMarchOptions* o) {
  if (!c || !o) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (o->phase_mode > PSC_PHASE_DUAL_LOBE_HG) return fail(PSC_ERR_INVALID_ARGUMENT, "bad phase_mode");
  if (o->storage > PSC_STORAGE_FP8) return fail(PSC_ERR_INVALID_ARGUMENT, "bad storage");
  if (o->filter > PSC_FILTER_HYBRID) return fail(PSC_ERR_INVALID_ARGUMENT, "bad filter");
  if (o->filter == PSC_FILTER_HYBRID && o->schedule != PSC_SCHED_FAST)
    return fail(PSC_ERR_UNSUPPORTED, "the hybrid filter is implemented by the FAST schedule only");
  if (o->filter == PSC_FILTER_HYBRID && o->storage != PSC_STORAGE_U8 && o->storage != PSC_STORAGE_F16)
    return fail(PSC_ERR_UNSUPPORTED, "the hybrid filter reads RGBA8 or RGBA16F volumes only");
  if (o->schedule > PSC_SCHED_FAST) return fail(PSC_ERR_INVALID_ARGUMENT, "bad schedule");
  if (o->filter == PSC_FILTER_TEXTURE && o->storage != PSC_STORAGE_U8 && o->storage != PSC_STORAGE_F16)
    return fail(PSC_ERR_UNSUPPORTED, "texture filtering reads RGBA8 or RGBA16F volumes only");
  if (o->filter == PSC_FILTER_TEXTURE && o->storage == PSC_STORAGE_F16 && o->schedule != PSC_SCHED_FAST)
    return fail(PSC_ERR_UNSUPPORTED, "F16 texture volumes are read by the FAST schedule only");
  if (o->half_res > 1 || o->taa > 1) return fail(PSC_ERR_INVALID_ARGUMENT, "half_res and taa are 0 or 1");
  if (o->light_batch != 0 && o->light_batch != 2 && o->light_batch != 3)
    return fail(PSC_ERR_INVALID_ARGUMENT, "light_batch is 0, 2 or 3 (got %u)", o->light_batch);
  const float hv[] = {o->hg_g_forward, o->hg_g_backward, o->hg_blend};
  if (!all_finite(hv, 3)) return fail(PSC_ERR_NOT_FINITE, "non-finite HG lobe");
  if (o->storage != c->opts.storage || o->filter != c->opts.filter) c->tex_dirty = true;
  c->opts = *o;
  return PSC_OK;
}

int psc_get_options(psc_ctx* c, PscMarchOptions* out) {
  if (!c || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  *out = c->opts;
  return PSC_OK;
}

int psc_bake_noise(psc_ctx* c) {
  if (!c) return fail(PSC_ERR_INVALID_ARGUMENT, "null context");
  int rc = ensure_device(c);
  if (rc) return rc;
  if (!c->d_base_u8) PSC_CUDA(cudaMalloc(&c->d_base_u8, 128u * 128u * 128u * 4u), "cudaMalloc base");
  if (!c->d_detail_u8) PSC_CUDA(cudaMalloc(&c->d_detail_u8, 32u * 32u * 32u * 4u), "cudaMalloc detail");
  if (!c->d_curl) PSC_CUDA(cudaMalloc(&c->d_curl, 128u * 128u * 2u), "cudaMalloc curl");
  if (psc::launch_noise_bakes(c->d_base_u8, c->d_detail_u8, c->d_curl, 0))
    return fail(PSC_ERR_CUDA, "noise bake failed: %s", cudaGetErrorString(cudaGetLastError()));
  c->have_base = c->have_detail = c->have_curl = true;
  std::vector<uint8_t> blue(64 * 64);
  psc_generate_blue_noise(blue.data());
  rc = psc_upload_noise(c, PSC_NOISE_BLUE, blue.data(), blue.size());
  if (rc) return rc;
  c->store_form = -1;
  c->tex_dirty = true;
  return build_storage(c);
}

int psc_upload_noise(psc_ctx* c, int kind, const void* texels, size_t bytes) {
  if (!c || !texels) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  const size_t need[] = {128u * 128u * 128u * 4u, 32u * 32u * 32u * 4u, 128u * 128u * 2u, 64u * 64u};
  if (kind < 0 || kind > 3) return fail(PSC_ERR_INVALID_ARGUMENT, "bad noise kind %d", kind);
  if (bytes != need[kind]) return fail(PSC_ERR_INVALID_ARGUMENT, "noise kind %d needs %zu bytes, got %zu", kind, need[kind], bytes);
  int rc = ensure_device(c);
  if (rc) return rc;
  if (kind == PSC_NOISE_BLUE) {
    std::vector<float> f(64 * 64);
    const uint8_t* b = static_cast<const uint8_t*>(texels);
    for (int i = 0; i < 64 * 64; ++i) f[i] = (float)b[i] / 255.0f;
    if (!c->d_blue) PSC_CUDA(cudaMalloc(&c->d_blue, f.size() * 4), "cudaMalloc blue");
    PSC_CUDA(cudaMemcpy(c->d_blue, f.data(), f.size() * 4, cudaMemcpyHostToDevice), "blue upload");
    c->h_blue.assign(b, b + 64 * 64);
    c->have_blue = true;
    return PSC_OK;
  }
  uint8_t** dst = kind == PSC_NOISE_BASE ? &c->d_base_u8 : kind == PSC_NOISE_DETAIL ? &c->d_detail_u8 : &c->d_curl;
  if (!*dst) PSC_CUDA(cudaMalloc(dst, bytes), "cudaMalloc noise");
  PSC_CUDA(cudaMemcpy(*dst, texels, bytes, cudaMemcpyHostToDevice), "noise upload");
  if (kind == PSC_NOISE_BASE) c->have_base = true;
  if (kind == PSC_NOISE_DETAIL) c->have_detail = true;
  if (kind == PSC_NOISE_CURL) c->have_curl = true;
  c->store_form = -1;
  c->tex_dirty = true;
  return build_storage(c);
}

int psc_download_noise(psc_ctx* c, int kind, void* texels, size_t bytes) {
  if (!c || !texels) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  const size_t need[] = {128u * 128u * 128u * 4u, 32u * 32u * 32u * 4u, 128u * 128u * 2u, 64u * 64u};
  if (kind < 0 || kind > 3) return fail(PSC_ERR_INVALID_ARGUMENT, "bad noise kind %d", kind);
  if (bytes != need[kind]) return fail(PSC_ERR_INVALID_ARGUMENT, "noise kind %d needs %zu bytes", kind, need[kind]);
  if (kind == PSC_NOISE_BLUE) {
    if (!c->have_blue) return fail(PSC_ERR_MISSING_INPUT, "no blue noise");
    std::memcpy(texels, c->h_blue.data(), bytes);
    return PSC_OK;
  }
  const uint8_t* src = kind == PSC_NOISE_BASE ? c->d_base_u8 : kind == PSC_NOISE_DETAIL ? c->d_detail_u8 : c->d_curl;
  if (!src) return fail(PSC_ERR_MISSING_INPUT, "noise kind %d not present", kind);
  int rc = ensure_device(c);
  if (rc) return rc;
  PSC_CUDA(cudaMemcpy(texels, src, bytes, cudaMemcpyDeviceToHost), "noise download");
  return PSC_OK;
}

int psc_upload_weather(psc_ctx* c, const void* texels, uint32_t w, uint32_t h, int format) {
  if (!c || !texels) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (!w || !h || w > 16384 || h > 16384) return fail(PSC_ERR_INVALID_ARGUMENT, "weather size %ux%u out of range", w, h);
  std::vector<float> r((size_t)w * h);
  for (size_t i = 0; i < r.size(); ++i) {
    switch (format) {
      case PSC_WEATHER_RGBA16F: r[i] = half_bits_to_float(static_cast<const uint16_t*>(texels)[i * 4]); break;
      case PSC_WEATHER_RG8: r[i] = (float)static_cast<const uint8_t*>(texels)[i * 2] / 255.0f; break;
      case PSC_WEATHER_R32F: r[i] = static_cast<const float*>(texels)[i]; break;
      default: return fail(PSC_ERR_INVALID_ARGUMENT, "bad weather format %d", format);
    }
    if (!std::isfinite(r[i])) return fail(PSC_ERR_NOT_FINITE, "weather texel %zu is not finite", i);
  }
  int rc = ensure_device(c);
  if (rc) return rc;
  if (c->d_weather && (c->weather_w != w || c->weather_h != h)) dfree(c->d_weather);
  if (!c->d_weather) PSC_CUDA(cudaMalloc(&c->d_weather, r.size() * 4), "cudaMalloc weather");
  PSC_CUDA(cudaMemcpy(c->d_weather, r.data(), r.size() * 4, cudaMemcpyHostToDevice), "weather upload");
  dfree(c->d_weather_quad);
  // a uniform map (the reference's synthesis writes R = 1 wherever layers
  // exist): lerp(c, c, w) = fma(w, 0, c) = c exactly, so the FAST schedule
  // skips the tap
  c->weather_uniform = std::all_of(r.begin(), r.end(), [&](float v) { return v == r[0]; });
  c->weather_value = r[0];
  const auto mm = std::minmax_element(r.begin(), r.end());
  c->weather_min = *mm.first;
  c->weather_max = *mm.second;
  const bool pow2 = (w & (w - 1)) == 0 && (h & (h - 1)) == 0;
  if (pow2 && (size_t)w * h <= 1024u * 1024u) {
    // 2x2 bilinear footprints, repeat-wrapped: one 16-byte load per tap
    std::vector<float> q(r.size() * 4);
    for (uint32_t y = 0; y < h; ++y)
      for (uint32_t x = 0; x < w; ++x) {
        const uint32_t x1 = (x + 1) & (w - 1), y1 = (y + 1) & (h - 1);
        float* e = &q[((size_t)y * w + x) * 4];
        e[0] = r[(size_t)y * w + x];
        e[1] = r[(size_t)y * w + x1];
        e[2] = r[(size_t)y1 * w + x];
        e[3] = r[(size_t)y1 * w + x1];
      }
    PSC_CUDA(cudaMalloc(&c->d_weather_quad, q.size() * 4), "cudaMalloc weather quads");
    PSC_CUDA(cudaMemcpy(c->d_weather_quad, q.data(), q.size() * 4, cudaMemcpyHostToDevice), "weather quads");
  }
  c->weather_w = w;
  c->weather_h = h;
  return PSC_OK;
}

int psc_upload_type_grid(psc_ctx* c, const uint8_t* texels, uint32_t w, uint32_t h) {
  if (!c) return fail(PSC_ERR_INVALID_ARGUMENT, "null context");
  int rc = ensure_device(c);
  if (rc) return rc;
  if (!texels) {  // no grid: every sample uses its layer's type
    dfree(c->d_type);
    c->type_w = c->type_h = 0;
    return PSC_OK;
  }
  if (!w || !h || w > 16384 || h > 16384) return fail(PSC_ERR_INVALID_ARGUMENT, "type grid size %ux%u out of range", w, h);
  for (size_t i = 0; i < (size_t)w * h; ++i)
    if (texels[i] > 7 && texels[i] != PSC_TYPE_SENTINEL)
      return fail(PSC_ERR_INVALID_ARGUMENT, "type grid texel %zu = %u is neither 0..7 nor 255", i, texels[i]);
  if (c->d_type && (c->type_w != w || c->type_h != h)) dfree(c->d_type);
  if (!c->d_type) PSC_CUDA(cudaMalloc(&c->d_type, (size_t)w * h), "cudaMalloc type grid");
  PSC_CUDA(cudaMemcpy(c->d_type, texels, (size_t)w * h, cudaMemcpyHostToDevice), "type grid upload");
  c->type_w = w;
  c->type_h = h;
  return PSC_OK;
}

int psc_upload_wind(psc_ctx* c, const uint16_t* rgba16f, size_t count) {
  if (!c || !rgba16f) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (count != 32u * 16u * 32u * 4u) return fail(PSC_ERR_INVALID_ARGUMENT, "wind field needs 32x16x32x4 halves");
  c->h_wind.assign(rgba16f, rgba16f + count);
  return PSC_OK;
}

int psc_upload_lut(psc_ctx* c, int kind, const uint16_t* rgba16f, size_t count) {
  if (!c || !rgba16f) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (kind < 0 || kind > 3) return fail(PSC_ERR_INVALID_ARGUMENT, "bad LUT kind %d", kind);
  if (count != lut_texels(kind) * 4) return fail(PSC_ERR_INVALID_ARGUMENT, "LUT %d needs %zu halves", kind, lut_texels(kind) * 4);
  int rc = ensure_device(c);
  if (rc) return rc;
  if (!c->d_lut_h[kind]) PSC_CUDA(cudaMalloc(&c->d_lut_h[kind], count * 2), "cudaMalloc LUT");
  PSC_CUDA(cudaMemcpy(c->d_lut_h[kind], rgba16f, count * 2, cudaMemcpyHostToDevice), "LUT upload");
  if (kind == PSC_LUT_TRANSMITTANCE || kind == PSC_LUT_MULTISCATTER) ++c->lut_generation;
  return upload_lut_float4(c, kind, rgba16f);
}

int psc_bake_luts(psc_ctx* c, void* stream) {
  if (!c) return fail(PSC_ERR_INVALID_ARGUMENT, "null context");
  if (!c->have_frame) return fail(PSC_ERR_MISSING_INPUT, "psc_set_frame must precede psc_bake_luts");
  int rc = ensure_device(c);
  if (rc) return rc;
  for (int k = 0; k < 4; ++k) {
    if (!c->d_lut_h[k]) PSC_CUDA(cudaMalloc(&c->d_lut_h[k], lut_texels(k) * 8), "cudaMalloc LUT");
    rc = ensure_lut_float4(c, k);
    if (rc) return rc;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // transmittance and multi-scatter depend on the world only: baked when it
  // changed, or when either LUT was uploaded, since their last bake
  const bool statics = !(c->static_luts_baked && c->static_luts_generation == c->lut_generation &&
                         std::memcmp(&c->static_luts_world, &c->world, sizeof(c->world)) == 0);
  if (psc::launch_lut_bakes(c->world, c->frame, statics, c->d_lut_h, c->d_lut, s))
    return fail(PSC_ERR_CUDA, "LUT bake launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  c->launches += statics ? 4 : 2;
  const size_t row = PSC_SKYVIEW_W * sizeof(float4);
  PSC_CUDA(cudaMemcpy2DToArrayAsync(c->arr_sky, 0, 0, c->d_lut[PSC_LUT_SKYVIEW], row, row, PSC_SKYVIEW_H,
                                    cudaMemcpyDeviceToDevice, s), "sky-view array copy");
  if (statics) {
    ++c->lut_generation;
    c->static_luts_baked = true;
    c->static_luts_world = c->world;
    c->static_luts_generation = c->lut_generation;
  }
  for (int k = 0; k < 4; ++k) c->have_lut[k] = true;
  if (!s) PSC_CUDA(cudaStreamSynchronize(s), "LUT bake");
  return PSC_OK;
}

int psc_download_lut(psc_ctx* c, int kind, uint16_t* out, size_t count) {
  if (!c || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (kind < 0 || kind > 3) return fail(PSC_ERR_INVALID_ARGUMENT, "bad LUT kind %d", kind);
  if (count != lut_texels(kind) * 4) return fail(PSC_ERR_INVALID_ARGUMENT, "LUT %d needs %zu halves", kind, lut_texels(kind) * 4);
  if (!c->d_lut_h[kind]) return fail(PSC_ERR_MISSING_INPUT, "LUT %d not present", kind);
  int rc = ensure_device(c);
  if (rc) return rc;
  PSC_CUDA(cudaDeviceSynchronize(), "LUT download: device work in flight");  // a bake on any stream
  PSC_CUDA(cudaMemcpy(out, c->d_lut_h[kind], count * 2, cudaMemcpyDeviceToHost), "LUT download");
  return PSC_OK;
}

namespace {

// Input, option and view checks of a march call (psc_render,
// psc_count_fetches); builds the noise storage form and the texture objects
// the march reads.
int prepare_render(psc_ctx* c, const PscView* views, uint32_t n, bool rt_form, bool outputs_required = true) {
  if (!c->have_frame) return fail(PSC_ERR_MISSING_INPUT, "psc_set_frame was not called");
  if (!c->have_base || !c->have_detail || !c->have_curl || !c->have_blue)
    return fail(PSC_ERR_MISSING_INPUT, "noise volumes missing (psc_bake_noise or psc_upload_noise)");
  if (!c->d_weather) return fail(PSC_ERR_MISSING_INPUT, "weather map missing (psc_upload_weather)");
  if (!c->have_lut[PSC_LUT_TRANSMITTANCE] || !c->have_lut[PSC_LUT_SKYVIEW] || !c->have_lut[PSC_LUT_AERIAL])
    return fail(PSC_ERR_MISSING_INPUT, "atmosphere LUTs missing (psc_upload_lut or psc_bake_luts)");
  int rc = validate_params(c->params);
  if (rc) return rc;
  rc = ensure_device(c);
  if (rc) return rc;
  rc = build_storage(c);
  if (rc) return rc;
  rc = build_textures(c);
  if (rc) return rc;
  if (c->opts.filter != PSC_FILTER_EXACT && (!c->tex_base || !c->tex_detail))
    return fail(PSC_ERR_MISSING_INPUT, "texture objects for the noise volumes were not created");
  for (uint32_t i = 0; i < n; ++i) {
    const PscView& v = views[i];
    if (!v.width || !v.height || v.width > 32768 || v.height > 32768)
      return fail(PSC_ERR_INVALID_ARGUMENT, "view %u: size %ux%u out of range", i, v.width, v.height);
    const uint32_t vw = v.viewport_w ? v.viewport_w : v.width, vh = v.viewport_h ? v.viewport_h : v.height;
    if ((!v.viewport_w && v.x_offset) || (!v.viewport_h && v.y_offset) || vw > 32768 || vh > 32768 ||
        (uint64_t)v.x_offset + v.width > vw || (uint64_t)v.y_offset + v.height > vh)
      return fail(PSC_ERR_INVALID_ARGUMENT, "view %u: rectangle %ux%u at (%u,%u) exceeds viewport %ux%u",
                  i, v.width, v.height, v.x_offset, v.y_offset, vw, vh);
    if (outputs_required && !v.out_luminance && !v.out_transmittance && !(c->opts.composite && v.hdr))
      return fail(PSC_ERR_INVALID_ARGUMENT, "view %u has no output buffer", i);
    if (outputs_required && c->opts.composite && !v.hdr)
      return fail(PSC_ERR_INVALID_ARGUMENT, "view %u: composite needs hdr", i);
    if (rt_form && (v.x_offset || v.y_offset || vw != v.width || vh != v.height))
      return fail(PSC_ERR_INVALID_ARGUMENT, "the half-res / TAA forms render whole viewports");
  }
  return PSC_OK;
}

}  // namespace

int psc_render(psc_ctx* c, const PscView* views, uint32_t n, void* stream) {
  if (!c || (n && !views)) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  const bool rt_form = c->opts.half_res || c->opts.taa;
  if (rt_form && n != 1)
    return fail(PSC_ERR_INVALID_ARGUMENT,
                "the half-res / TAA forms render one view per call (its march, TAA and composite)");
  int rc = prepare_render(c, views, n, rt_form);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ++c->taa[c->active_view].marches;  // a resolve of this march keeps the view's history going
  if (rt_form) return render_rt_view(c, views[0], s);
  psc::MarchUniforms u;
  for (uint32_t i = 0; i < n; ++i) {
    const PscView& v = views[i];
    const uint32_t vw = v.viewport_w ? v.viewport_w : v.width, vh = v.viewport_h ? v.viewport_h : v.height;
    build_uniforms(c, vw, vh, u);
    psc::ViewDev vd{v.width, v.height, v.x_offset, v.y_offset, v.depth,
                    reinterpret_cast<float4*>(v.out_luminance),
                    reinterpret_cast<float4*>(v.out_transmittance), reinterpret_cast<float4*>(v.hdr)};
    rc = launch_view_march(c, u, vd, s);
    if (rc) return rc;
  }
  return PSC_OK;
}

int psc_count_fetches(psc_ctx* c, const PscView* view, PscFetchCounts* out, void* stream) {
  if (!c || !view || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (c->opts.schedule != PSC_SCHED_FAST || c->opts.debug_checks || c->opts.half_res || c->opts.taa)
    return fail(PSC_ERR_UNSUPPORTED,
                "fetch counts come from the FAST schedule's full-resolution march (no debug checks, "
                "half-res or TAA)");
  int rc = prepare_render(c, view, 1, false);
  if (rc) return rc;
  const PscView& v = *view;
  const uint32_t vw = v.viewport_w ? v.viewport_w : v.width, vh = v.viewport_h ? v.viewport_h : v.height;
  psc::MarchUniforms u;
  build_uniforms(c, vw, vh, u);
  const psc::ViewDev vd{v.width, v.height, v.x_offset, v.y_offset, v.depth,
                        reinterpret_cast<float4*>(v.out_luminance),
                        reinterpret_cast<float4*>(v.out_transmittance), reinterpret_cast<float4*>(v.hdr)};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  unsigned long long* d = nullptr;
  unsigned long long h[psc::kFetchTallyKinds] = {};
  PSC_CUDA(cudaMalloc(&d, sizeof(h)), "cudaMalloc fetch counters");
  cudaError_t e = cudaMemsetAsync(d, 0, sizeof(h), s);
  if (e == cudaSuccess) {
    rc = psc::launch_march_fast_tally(u, vd, c->opts, d, s);
    if (rc == PSC_OK) {
      ++c->launches;
      e = cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
  }
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "fetch-count march");
  if (rc == PSC_ERR_UNSUPPORTED)
    return fail(rc, "fetch counts cover F16 and U8 storage with exact or hybrid filtering, up to 4 octaves");
  if (rc) return fail(rc, "fetch-count march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  static_assert(sizeof(PscFetchCounts) == sizeof(h), "PscFetchCounts holds one counter per kind");
  std::memcpy(out, h, sizeof(h));
  return PSC_OK;
}

int psc_composite(const float* l, const float* t, float* hdr, uint32_t w, uint32_t h, void* stream) {
  if (!l || !t || !hdr) return fail(PSC_ERR_INVALID_ARGUMENT, "null buffer");
  if (!w || !h) return fail(PSC_ERR_INVALID_ARGUMENT, "zero-size composite");
  if (psc::launch_composite(reinterpret_cast<const float4*>(l), reinterpret_cast<const float4*>(t),
                            reinterpret_cast<float4*>(hdr), w * h, static_cast<cudaStream_t>(stream)))
    return fail(PSC_ERR_CUDA, "composite launch failed");
  return PSC_OK;
}

int psc_cloud_rt_size(uint32_t w, uint32_t h, uint32_t half_res, uint32_t* rw, uint32_t* rh) {
  if (!rw || !rh) return fail(PSC_ERR_INVALID_ARGUMENT, "null output");
  if (!w || !h) return fail(PSC_ERR_INVALID_ARGUMENT, "zero-size target");
  if (half_res) {
    half_res_dims(w, h, rw, rh);
  } else {
    *rw = w;
    *rh = h;
  }
  return PSC_OK;
}

int psc_taa_resolve(psc_ctx* c, const float* cur_l, const float* cur_t, uint32_t w, uint32_t h, float* out_l,
                    float* out_t, void* stream) {
  if (!c || !cur_l || !cur_t) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (!w || !h || w > 32768 || h > 32768) return fail(PSC_ERR_INVALID_ARGUMENT, "cloud RT %ux%u out of range", w, h);
  if (!c->have_frame) return fail(PSC_ERR_MISSING_INPUT, "psc_set_frame was not called");
  int rc = ensure_device(c);
  if (rc) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float4 *res_l = nullptr, *res_t = nullptr;
  rc = taa_step(c, reinterpret_cast<const float4*>(cur_l), reinterpret_cast<const float4*>(cur_t), w, h, s,
                &res_l, &res_t);
  if (rc) return rc;
  const size_t bytes = (size_t)w * h * sizeof(float4);
  if (out_l) PSC_CUDA(cudaMemcpyAsync(out_l, res_l, bytes, cudaMemcpyDeviceToDevice, s), "TAA output copy");
  if (out_t) PSC_CUDA(cudaMemcpyAsync(out_t, res_t, bytes, cudaMemcpyDeviceToDevice, s), "TAA output copy");
  return PSC_OK;
}

int psc_set_active_view(psc_ctx* c, uint32_t view) {  // lib.rs:722
  if (!c) return fail(PSC_ERR_INVALID_ARGUMENT, "null context");
  c->active_view = std::min(view, PSC_MAX_CLOUD_VIEWS - 1u);
  return PSC_OK;
}

int psc_invalidate_taa_history(psc_ctx* c) {  // lib.rs:729
  if (!c) return fail(PSC_ERR_INVALID_ARGUMENT, "null context");
  for (auto& tv : c->taa) tv.valid = false;
  return PSC_OK;
}

int psc_composite_halfres(const float* l, const float* t, uint32_t rw, uint32_t rh, float* hdr, uint32_t w,
                          uint32_t h, void* stream) {
  if (!l || !t || !hdr) return fail(PSC_ERR_INVALID_ARGUMENT, "null buffer");
  if (!w || !h || !rw || !rh) return fail(PSC_ERR_INVALID_ARGUMENT, "zero-size composite");
  if (w > 32768 || h > 32768 || rw > 32768 || rh > 32768)
    return fail(PSC_ERR_INVALID_ARGUMENT, "composite size out of range");
  if (psc::launch_composite_halfres(reinterpret_cast<const float4*>(l), reinterpret_cast<const float4*>(t), rw, rh,
                                    reinterpret_cast<float4*>(hdr), w, h, static_cast<cudaStream_t>(stream)))
    return fail(PSC_ERR_CUDA, "half-res composite launch failed");
  return PSC_OK;
}

int psc_set_batch_tuning(psc_ctx* c, const PscBatchTuning* t) {
  if (!c || !t) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  const int rc = validate_tuning(*t);
  if (rc) return rc;
  c->batch_tuning = *t;
  return PSC_OK;
}

int psc_get_batch_tuning(psc_ctx* c, PscBatchTuning* out) {
  if (!c || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  *out = c->batch_tuning;
  return PSC_OK;
}

int psc_render_batch(psc_ctx* c, const PscBatchView* views, uint32_t n, void* stream) {
  if (!c || (n && !views)) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) return PSC_OK;
  if (n > PSC_MAX_BATCH_VIEWS) return fail(PSC_ERR_INVALID_ARGUMENT, "%u views exceeds %u", n, PSC_MAX_BATCH_VIEWS);
  if (!c->have_base || !c->have_detail || !c->have_curl || !c->have_blue)
    return fail(PSC_ERR_MISSING_INPUT, "noise volumes missing (psc_bake_noise or psc_upload_noise)");
  if (!c->d_weather) return fail(PSC_ERR_MISSING_INPUT, "weather map missing (psc_upload_weather)");
  if (!c->d_lut_h[PSC_LUT_TRANSMITTANCE] || !c->d_lut_h[PSC_LUT_MULTISCATTER] || !c->have_lut[PSC_LUT_TRANSMITTANCE])
    return fail(PSC_ERR_MISSING_INPUT, "transmittance/multi-scatter LUTs missing (psc_bake_luts or psc_upload_lut)");
  if (c->opts.schedule != PSC_SCHED_FAST)
    return fail(PSC_ERR_UNSUPPORTED, "the batched kernel implements the FAST schedule (options.schedule)");
  if (c->opts.half_res || c->opts.taa || c->opts.debug_checks)
    return fail(PSC_ERR_UNSUPPORTED,
                "the batched kernel renders full-resolution views without TAA or debug checks");
  for (uint32_t i = 0; i < n; ++i) {
    const PscBatchView& v = views[i];
    if (!v.width || !v.height || v.width > 32768 || v.height > 32768)
      return fail(PSC_ERR_INVALID_ARGUMENT, "batch view %u: size %ux%u out of range", i, v.width, v.height);
    if (!v.out_luminance && !v.out_transmittance && !(c->opts.composite && v.hdr))
      return fail(PSC_ERR_INVALID_ARGUMENT, "batch view %u has no output buffer", i);
    if (c->opts.composite && !v.hdr) return fail(PSC_ERR_INVALID_ARGUMENT, "batch view %u: composite needs hdr", i);
    int rc = validate_layers(v.layers, v.n_layers);
    if (rc) return fail(rc, "batch view %u: %s", i, g_last_error.c_str());
    PscCloudParamsGpu p = v.params;
    p.cloud_layer_count = v.n_layers;
    rc = validate_params(p);
    if (rc) return fail(rc, "batch view %u: %s", i, g_last_error.c_str());
    if (p.multi_scatter_octaves == 0 || p.multi_scatter_octaves > 4)
      return fail(PSC_ERR_UNSUPPORTED, "batch view %u: the batched kernel handles 1..4 octaves", i);
    const float* ff = reinterpret_cast<const float*>(&v.frame);
    for (size_t k = 0; k < sizeof(v.frame) / 4; ++k)
      if (k != 94 && !std::isfinite(ff[k])) return fail(PSC_ERR_NOT_FINITE, "batch view %u: frame word %zu", i, k);
  }
  int rc = ensure_device(c);
  if (rc) return rc;
  if (!c->sms) PSC_CUDA(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device), "SM count");
  rc = build_storage(c);
  if (rc) return rc;
  rc = build_textures(c);
  if (rc) return rc;
  if (c->opts.filter != PSC_FILTER_EXACT && (!c->tex_base || !c->tex_detail))
    return fail(PSC_ERR_MISSING_INPUT, "texture objects for the noise volumes were not created");
  uint32_t n_tiles = 0;
  rc = stage_batch(c, views, n, &n_tiles);
  if (rc) return rc;
  // which views bake their sky-view / AP LUTs: those whose inputs changed
  // since their slot's last bake
  std::vector<uint64_t> lut_keys(n);
  {
    const uint64_t ptrs[] = {c->lut_generation, (uint64_t)(uintptr_t)c->d_bsky, (uint64_t)(uintptr_t)c->d_bap,
                             (uint64_t)(uintptr_t)c->d_lut_h[PSC_LUT_TRANSMITTANCE],
                             (uint64_t)(uintptr_t)c->d_lut_h[PSC_LUT_MULTISCATTER]};
    const uint64_t seed = fnv1a(ptrs, sizeof(ptrs), fnv1a(&c->world, sizeof(c->world)));
    const size_t fl = psc::frame_lite_size();
    c->batch_bake.assign(n, 1);
    for (uint32_t i = 0; i < n; ++i) {
      lut_keys[i] = fnv1a(static_cast<const char*>(c->h_bframes) + i * fl, fl, seed);
      c->batch_bake[i] = !(i < c->batch_lut_keys.size() && c->batch_lut_keys[i] == lut_keys[i]);
    }
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool per_view = c->batch_tuning.form == PSC_BATCH_PER_VIEW;
  const uint64_t marches = per_view ? n : 1;  // march-kernel launches per call
  auto enqueue = [&](cudaStream_t st, bool capturing) {
    return per_view ? enqueue_batch_per_view(c, n, st, capturing) : enqueue_batch(c, n, n_tiles, st, capturing);
  };
  if (!c->batch_tuning.use_graph) {
    c->batch_lut_keys.clear();  // a failed enqueue may have baked some views and not others
    rc = enqueue(s, false);
    if (rc) return rc;
    c->batch_lut_keys = lut_keys;
    c->launches += marches;
    return PSC_OK;
  }
  // Graph path: the key is everything the captured nodes bake in (buffer
  // pointers, sizes, options, launch shape, the full or lean kernel form).
  // The persistent form reads its uniforms from the pinned staging at launch
  // time, so they may change freely within that form; the per-view form
  // bakes each view's uniforms into its kernel node, so their bytes are part
  // of its key, and a change of them alone updates the instantiated graph in
  // place (cudaGraphExecUpdate) instead of instantiating a new one.
  std::vector<uint64_t> key = {c->batch_tuning.form, n, n_tiles, c->batch_tuning.threads,
                               c->batch_tuning.tile_w, c->opts.storage, c->opts.filter, c->opts.composite,
                               c->opts.light_batch,
                               (uint64_t)(uintptr_t)c->d_bu, (uint64_t)(uintptr_t)c->d_btiles,
                               (uint64_t)(uintptr_t)c->d_bframes,
                               (uint64_t)(uintptr_t)c->d_base_store, (uint64_t)c->tex_base,
                               (uint64_t)psc::needs_full_paths(c->h_bu, n),
                               fnv1a(c->batch_bake.data(), n)};
  if (per_view) {
    key.push_back(fnv1a(c->h_bu, n * sizeof(psc::MarchUniforms)));
    key.push_back(fnv1a(c->h_bv, n * sizeof(psc::ViewDev)));
  }
  if (!c->batch_exec || key != c->batch_key) {
    cudaGraph_t g = nullptr;
    PSC_CUDA(cudaStreamBeginCapture(c->batch_stream, cudaStreamCaptureModeThreadLocal), "begin capture");
    rc = enqueue(c->batch_stream, true);
    const cudaError_t ce = cudaStreamEndCapture(c->batch_stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "end capture");
    const bool same_shape = c->batch_exec && c->batch_key.size() == key.size() &&
                            std::equal(key.begin(), key.end() - (per_view ? 2 : 0), c->batch_key.begin());
    bool updated = false;
    if (same_shape) {
      cudaGraphExecUpdateResultInfo info;
      updated = cudaGraphExecUpdate(c->batch_exec, g, &info) == cudaSuccess;
      if (!updated) cudaGetLastError();  // clear the failed update's error
    }
    if (!updated) {
      if (c->batch_exec) cudaGraphExecDestroy(c->batch_exec);
      c->batch_exec = nullptr;
      const cudaError_t ie = cudaGraphInstantiate(&c->batch_exec, g, 0);
      if (ie != cudaSuccess) {
        cudaGraphDestroy(g);
        return cuda_fail(ie, "graph instantiate");
      }
    }
    cudaGraphDestroy(g);
    c->batch_key = key;
  }
  c->batch_lut_keys.clear();
  PSC_CUDA(cudaGraphLaunch(c->batch_exec, s), "graph launch");
  c->batch_lut_keys = lut_keys;
  c->launches += marches;
  return PSC_OK;
}

int psc_autotune_batch(psc_ctx* c, const PscBatchView* views, uint32_t n, uint32_t reps,
                       PscBatchTuning* best, float* best_ms, void* stream) {
  if (!c || !views || !n) return fail(PSC_ERR_INVALID_ARGUMENT, "null or empty batch");
  if (reps == 0 || reps > 100) return fail(PSC_ERR_INVALID_ARGUMENT, "reps must be 1..100");
  const PscBatchTuning saved = c->batch_tuning;
  const uint32_t saved_lb = c->opts.light_batch;
  // {form, threads, tile_w}: the persistent form at each launch shape, and
  // the per-view form (whose kernels have their own fixed shape)
  static const uint32_t cand[][3] = {{PSC_BATCH_PERSISTENT, 128, 16}, {PSC_BATCH_PERSISTENT, 128, 32},
                                     {PSC_BATCH_PERSISTENT, 128, 8},  {PSC_BATCH_PERSISTENT, 256, 16},
                                     {PSC_BATCH_PERSISTENT, 256, 32}, {PSC_BATCH_PERSISTENT, 256, 64},
                                     {PSC_BATCH_PERSISTENT, 64, 8},   {PSC_BATCH_PERSISTENT, 64, 16},
                                     {PSC_BATCH_PER_VIEW, 128, 16}};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaEvent_t a = nullptr, b = nullptr;
  PSC_CUDA(cudaEventCreate(&a), "event");
  PSC_CUDA(cudaEventCreate(&b), "event");
  // median of `reps` timed runs of the current tuning and options, after one warm-up
  auto time_current = [&](float* med) -> int {
    int rc = psc_render_batch(c, views, n, stream);
    if (rc) return rc;
    std::vector<float> ts;
    for (uint32_t r = 0; r < reps; ++r) {
      cudaEventRecord(a, s);
      rc = psc_render_batch(c, views, n, stream);
      cudaEventRecord(b, s);
      if (rc) return rc;
      if (cudaEventSynchronize(b) != cudaSuccess) return cuda_fail(cudaGetLastError(), "autotune sync");
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, a, b);
      ts.push_back(ms);
    }
    std::sort(ts.begin(), ts.end());
    *med = ts[ts.size() / 2];
    return PSC_OK;
  };
  float best_t = INFINITY;
  PscBatchTuning best_tu = saved;
  uint32_t best_lb = saved_lb;
  int rc = PSC_OK;
  for (const auto& cd : cand) {
    c->batch_tuning = PscBatchTuning{cd[1], cd[2], 0, cd[0]};
    float med = 0.0f;
    rc = time_current(&med);
    if (rc) break;
    if (med < best_t) {
      best_t = med;
      best_tu = c->batch_tuning;
    }
  }
  // the light-march fetch batch in the fastest launch shape (F16 hybrid)
  if (!rc && c->opts.storage == PSC_STORAGE_F16 && c->opts.filter == PSC_FILTER_HYBRID) {
    c->batch_tuning = best_tu;
    for (uint32_t lb : {0u, 3u, 2u}) {
      if (lb == saved_lb) continue;  // timed above
      c->opts.light_batch = lb;
      float med = 0.0f;
      rc = time_current(&med);
      if (rc) break;
      if (med < best_t) {
        best_t = med;
        best_lb = lb;
      }
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  best_tu.use_graph = saved.use_graph;
  c->batch_tuning = rc ? saved : best_tu;
  c->opts.light_batch = rc ? saved_lb : best_lb;
  if (rc) return rc;
  if (best) *best = best_tu;
  if (best_ms) *best_ms = best_t;
  return PSC_OK;
}

int psc_autotune_steps(psc_ctx* c, PscBatchView* views, uint32_t n, float max_rel_err, float max_share,
                       uint32_t reps, float* ms_before, float* ms_after, void* stream) {
  if (!c || !views || !n) return fail(PSC_ERR_INVALID_ARGUMENT, "null or empty batch");
  if (n > PSC_MAX_BATCH_VIEWS) return fail(PSC_ERR_INVALID_ARGUMENT, "%u views exceeds %u", n, PSC_MAX_BATCH_VIEWS);
  if (!(max_rel_err > 0.0f) || !std::isfinite(max_rel_err))
    return fail(PSC_ERR_INVALID_ARGUMENT, "max_rel_err must be positive and finite");
  if (!(max_share >= 0.0f && max_share < 1.0f)) return fail(PSC_ERR_INVALID_ARGUMENT, "max_share must be in [0, 1)");
  if (reps == 0 || reps > 100) return fail(PSC_ERR_INVALID_ARGUMENT, "reps must be 1..100");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // scratch: reference L / T and candidate L / T per view, one count per view
  std::vector<size_t> off(n + 1, 0);
  for (uint32_t i = 0; i < n; ++i) off[i + 1] = off[i] + (size_t)views[i].width * views[i].height;
  const size_t px = off[n];
  float4* buf = nullptr;
  unsigned int* d_count = nullptr;
  PSC_CUDA(cudaMalloc(&buf, 4 * px * sizeof(float4)), "cudaMalloc step-tuner scratch");
  if (cudaMalloc(&d_count, n * sizeof(unsigned int)) != cudaSuccess) {
    cudaFree(buf);
    return cuda_fail(cudaGetLastError(), "cudaMalloc step-tuner counts");
  }
  float4 *Lr = buf, *Tr = buf + px, *Lc = buf + 2 * px, *Tc = buf + 3 * px;
  const uint32_t saved_composite = c->opts.composite;
  c->opts.composite = 0;
  auto with_outputs = [&](uint32_t i, float4* L, float4* T) {
    PscBatchView v = views[i];
    v.out_luminance = reinterpret_cast<float*>(L + off[i]);
    v.out_transmittance = reinterpret_cast<float*>(T + off[i]);
    v.hdr = nullptr;
    return v;
  };
  std::vector<PscBatchView> ref(n), cand;
  for (uint32_t i = 0; i < n; ++i) ref[i] = with_outputs(i, Lr, Tr);
  std::vector<uint32_t> cloud(n), light(n);
  for (uint32_t i = 0; i < n; ++i) {
    cloud[i] = views[i].params.cloud_steps;
    light[i] = views[i].params.light_steps;
  }
  // renders the views `ids` at counts (cl, ll) and reports which stay within
  // the bar against the reference
  auto trial = [&](const std::vector<uint32_t>& ids, const std::vector<uint32_t>& cl,
                   const std::vector<uint32_t>& ll, std::vector<char>& ok) -> int {
    cand.clear();
    for (uint32_t k = 0; k < ids.size(); ++k) {
      PscBatchView v = with_outputs(ids[k], Lc, Tc);
      v.params.cloud_steps = cl[k];
      v.params.light_steps = ll[k];
      cand.push_back(v);
    }
    int rc = psc_render_batch(c, cand.data(), (uint32_t)cand.size(), stream);
    if (rc) return rc;
    if (cudaMemsetAsync(d_count, 0, n * sizeof(unsigned int), s) != cudaSuccess)
      return cuda_fail(cudaGetLastError(), "step-tuner count reset");
    for (uint32_t k = 0; k < ids.size(); ++k) {
      const uint32_t i = ids[k];
      rc = psc::launch_count_rel_err(Lr + off[i], Tr + off[i], Lc + off[i], Tc + off[i],
                                     reinterpret_cast<const float4*>(views[i].hdr), (uint32_t)(off[i + 1] - off[i]),
                                     max_rel_err, d_count + k, s);
      if (rc) return fail(rc, "step-tuner error count launch failed");
    }
    std::vector<unsigned int> h(ids.size());
    if (cudaMemcpyAsync(h.data(), d_count, ids.size() * sizeof(unsigned int), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return cuda_fail(cudaGetLastError(), "step-tuner count read");
    ok.assign(ids.size(), 0);
    for (uint32_t k = 0; k < ids.size(); ++k) {
      const double allowed = (double)max_share * (double)(off[ids[k] + 1] - off[ids[k]]);
      ok[k] = (double)h[k] <= allowed;
    }
    return PSC_OK;
  };
  int rc = psc_render_batch(c, ref.data(), n, stream);
  // light-march length: one step at a time, down to half of the view's own
  std::vector<char> open(n, 1);
  for (uint32_t j = 1; !rc; ++j) {
    std::vector<uint32_t> ids, cl, ll;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t l0 = views[i].params.light_steps;
      if (open[i] && l0 > j && 2 * (l0 - j) >= l0) {
        ids.push_back(i);
        cl.push_back(cloud[i]);
        ll.push_back(l0 - j);
      } else {
        open[i] = 0;
      }
    }
    if (ids.empty()) break;
    std::vector<char> ok;
    rc = trial(ids, cl, ll, ok);
    for (uint32_t k = 0; !rc && k < ids.size(); ++k) {
      if (ok[k]) light[ids[k]] = ll[k];
      else open[ids[k]] = 0;
    }
  }
  // primary step count: 7/8, 3/4, 5/8, 1/2 of the view's own (at least 8)
  open.assign(n, 1);
  for (uint32_t eighths = 7; !rc && eighths >= 4; --eighths) {
    std::vector<uint32_t> ids, cl, ll;
    for (uint32_t i = 0; i < n; ++i) {
      const uint32_t c0 = views[i].params.cloud_steps;
      const uint32_t cn = std::max(8u, (c0 * eighths + 7u) / 8u);
      if (open[i] && cn < cloud[i]) {
        ids.push_back(i);
        cl.push_back(cn);
        ll.push_back(light[i]);
      }
    }
    if (ids.empty()) continue;
    std::vector<char> ok;
    rc = trial(ids, cl, ll, ok);
    for (uint32_t k = 0; !rc && k < ids.size(); ++k) {
      if (ok[k]) cloud[ids[k]] = cl[k];
      else open[ids[k]] = 0;
    }
  }
  // median batch time before and after
  auto time_batch = [&](const std::vector<PscBatchView>& vs, float* med) -> int {
    if (!med) return PSC_OK;
    int r = psc_render_batch(c, vs.data(), n, stream);
    if (r) return r;
    cudaEvent_t a = nullptr, b = nullptr;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
      if (a) cudaEventDestroy(a);
      return cuda_fail(cudaGetLastError(), "event");
    }
    std::vector<float> ts;
    for (uint32_t k = 0; k < reps && !r; ++k) {
      cudaEventRecord(a, s);
      r = psc_render_batch(c, vs.data(), n, stream);
      cudaEventRecord(b, s);
      if (!r && cudaEventSynchronize(b) != cudaSuccess) r = cuda_fail(cudaGetLastError(), "step-tuner sync");
      float ms = 0.0f;
      if (!r) cudaEventElapsedTime(&ms, a, b);
      ts.push_back(ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (r) return r;
    std::sort(ts.begin(), ts.end());
    *med = ts[ts.size() / 2];
    return PSC_OK;
  };
  if (!rc) rc = time_batch(ref, ms_before);
  if (!rc) {
    std::vector<PscBatchView> tuned(ref);
    for (uint32_t i = 0; i < n; ++i) {
      tuned[i].params.cloud_steps = cloud[i];
      tuned[i].params.light_steps = light[i];
    }
    rc = time_batch(tuned, ms_after);
  }
  cudaStreamSynchronize(s);
  cudaFree(buf);
  cudaFree(d_count);
  c->opts.composite = saved_composite;
  if (rc) return rc;
  for (uint32_t i = 0; i < n; ++i) {
    views[i].params.cloud_steps = cloud[i];
    views[i].params.light_steps = light[i];
  }
  return PSC_OK;
}

}  // extern "C"

namespace {

// Inputs, grid description and view checks of the voxel-grid form; fills
// the uniforms, view record and grid record for the launch.
int prepare_grid(psc_ctx* c, const PscDensityGrid* g, const PscView* v, bool adjoint,
                 psc::MarchUniforms& u, psc::ViewDev& vd, psc::GridDev& gd) {
  if (!c || !g || !v) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (!c->have_frame) return fail(PSC_ERR_MISSING_INPUT, "psc_set_frame was not called");
  if (!c->have_blue) return fail(PSC_ERR_MISSING_INPUT, "blue noise missing (psc_bake_noise or psc_upload_noise)");
  if (!c->have_lut[PSC_LUT_TRANSMITTANCE] || !c->have_lut[PSC_LUT_SKYVIEW])
    return fail(PSC_ERR_MISSING_INPUT, "transmittance/sky-view LUTs missing (psc_upload_lut or psc_bake_luts)");
  int rc = validate_params(c->params);
  if (rc) return rc;
  if (c->n_layers != 1) return fail(PSC_ERR_LAYERS, "the grid form takes exactly one layer (got %u)", c->n_layers);
  if (c->params.cone_light_sampling)
    return fail(PSC_ERR_UNSUPPORTED, "the grid form marches the straight light path (cone sampling off)");
  if (c->params.multi_scatter_octaves == 0 || c->params.multi_scatter_octaves > 4)
    return fail(PSC_ERR_UNSUPPORTED, "the grid form handles 1..4 octaves");
  if (!g->values) return fail(PSC_ERR_INVALID_ARGUMENT, "grid values are null");
  if (!g->nx || !g->ny || !g->nz || (uint64_t)g->nx * g->ny * g->nz > 0x7fffffffull)
    return fail(PSC_ERR_INVALID_ARGUMENT, "grid of %ux%ux%u cells out of range", g->nx, g->ny, g->nz);
  const float fields[] = {g->min_x_m, g->min_z_m, g->size_x_m, g->size_z_m, g->density_scale,
                          g->exit_transmittance};
  for (float f : fields)
    if (!std::isfinite(f)) return fail(PSC_ERR_NOT_FINITE, "grid field is not finite");
  if (g->size_x_m <= 0.0f || g->size_z_m <= 0.0f)
    return fail(PSC_ERR_INVALID_ARGUMENT, "grid extent must be positive");
  if (g->exit_transmittance < 0.0f || g->exit_transmittance >= 1.0f)
    return fail(PSC_ERR_INVALID_ARGUMENT, "exit_transmittance must be in [0, 1)");
  if (adjoint) {
    const uint32_t k = g->checkpoint_every;
    if (k == 0 || k > 32)
      return fail(PSC_ERR_INVALID_ARGUMENT, "checkpoint_every must be 1..32 (got %u)", k);
    if ((c->params.cloud_steps + k - 1) / k > PSC_GRID_MAX_CHECKPOINTS)
      return fail(PSC_ERR_INVALID_ARGUMENT, "%u steps need more than %u checkpoints at interval %u",
                  c->params.cloud_steps, PSC_GRID_MAX_CHECKPOINTS, k);
  }
  if (!v->width || !v->height || v->width > 32768 || v->height > 32768)
    return fail(PSC_ERR_INVALID_ARGUMENT, "view size %ux%u out of range", v->width, v->height);
  const uint32_t vw = v->viewport_w ? v->viewport_w : v->width, vh = v->viewport_h ? v->viewport_h : v->height;
  if ((!v->viewport_w && v->x_offset) || (!v->viewport_h && v->y_offset) || vw > 32768 || vh > 32768 ||
      (uint64_t)v->x_offset + v->width > vw || (uint64_t)v->y_offset + v->height > vh)
    return fail(PSC_ERR_INVALID_ARGUMENT, "view rectangle %ux%u at (%u,%u) exceeds viewport %ux%u", v->width,
                v->height, v->x_offset, v->y_offset, vw, vh);
  if (!adjoint && !v->out_luminance && !v->out_transmittance && !(c->opts.composite && v->hdr))
    return fail(PSC_ERR_INVALID_ARGUMENT, "view has no output buffer");
  if (!adjoint && c->opts.composite && !v->hdr) return fail(PSC_ERR_INVALID_ARGUMENT, "composite needs hdr");
  rc = ensure_device(c);
  if (rc) return rc;
  build_uniforms(c, vw, vh, u);
  vd = psc::ViewDev{v->width, v->height, v->x_offset, v->y_offset, v->depth,
                    reinterpret_cast<float4*>(v->out_luminance), reinterpret_cast<float4*>(v->out_transmittance),
                    reinterpret_cast<float4*>(v->hdr)};
  const psc::LayerConst& L = u.layers[0];
  const float sig = L.sigma_t[0] + L.sigma_t[1] + L.sigma_t[2];
  if (!(sig > 0.0f)) return fail(PSC_ERR_INVALID_ARGUMENT, "layer extinction must be positive");
  gd = psc::GridDev{};
  gd.values = g->values;
  gd.nx = g->nx;
  gd.ny = g->ny;
  gd.nz = g->nz;
  gd.k_cp = g->checkpoint_every;
  gd.min_x = g->min_x_m;
  gd.min_z = g->min_z_m;
  gd.base = L.base_m;
  gd.inv_cell_x = (float)g->nx / g->size_x_m;
  gd.inv_cell_z = (float)g->nz / g->size_z_m;
  gd.inv_cell_y = (float)g->ny / std::max(L.top_m - L.base_m, 1.0f);
  gd.inv_sigma_bar = 3.0f / sig;
  gd.k = g->density_scale * gd.inv_sigma_bar;
  gd.exit_t = g->exit_transmittance;
  gd.inv_n = (float)(1.0 / (3.0 * (double)vw * (double)vh));
  return PSC_OK;
}

// The grid values as (x, z) corner quads (GridDev::quads) on `s`, and for the
// adjoint a zeroed gradient in x pairs (GridDev::grad_pairs).
int stage_grid_layout(psc_ctx* c, psc::GridDev& gd, bool adjoint, cudaStream_t s) {
  const size_t nq = (size_t)gd.ny * (gd.nz + 1u) * (gd.nx + 1u);  // quads
  const size_t np = (size_t)gd.ny * gd.nz * (gd.nx + 1u);         // gradient pairs
  if (c->grid_pairs_cap < nq) {
    dfree(c->d_grid_quads);
    dfree(c->d_grad_pairs);
    c->grid_pairs_cap = 0;
    PSC_CUDA(cudaMalloc(&c->d_grid_quads, nq * sizeof(float4)), "cudaMalloc grid quads");
    PSC_CUDA(cudaMalloc(&c->d_grad_pairs, nq * sizeof(float2)), "cudaMalloc gradient pairs");
    c->grid_pairs_cap = nq;
  }
  if (psc::launch_grid_quads(gd.values, c->d_grid_quads, gd.nx, gd.ny, gd.nz, s))
    return fail(PSC_ERR_CUDA, "grid quad launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  gd.quads = c->d_grid_quads;
  if (adjoint) {
    PSC_CUDA(cudaMemsetAsync(c->d_grad_pairs, 0, np * sizeof(float2), s), "gradient pair reset");
    gd.grad_pairs = c->d_grad_pairs;
  }
  return PSC_OK;
}

}  // namespace

extern "C" {

int psc_render_grid(psc_ctx* c, const PscDensityGrid* g, const PscView* v, void* stream) {
  psc::MarchUniforms u;
  psc::ViewDev vd;
  psc::GridDev gd;
  int rc = prepare_grid(c, g, v, false, u, vd, gd);
  if (rc) return rc;
  rc = stage_grid_layout(c, gd, false, static_cast<cudaStream_t>(stream));
  if (rc) return rc;
  rc = psc::launch_grid_march(u, vd, gd, false, static_cast<cudaStream_t>(stream));
  if (rc) return fail(rc, "grid march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  ++c->launches;
  return PSC_OK;
}

int psc_adjoint(psc_ctx* c, const PscDensityGrid* g, const PscView* v, const float* background,
                const float* target, float* grad_values, double* grad_density_scale, double* loss,
                void* stream) {
  if (!background || !target || !grad_values || !grad_density_scale || !loss)
    return fail(PSC_ERR_INVALID_ARGUMENT, "null adjoint buffer");
  psc::MarchUniforms u;
  psc::ViewDev vd;
  psc::GridDev gd;
  int rc = prepare_grid(c, g, v, true, u, vd, gd);
  if (rc) return rc;
  gd.grad = grad_values;
  gd.bg = reinterpret_cast<const float4*>(background);
  gd.target = reinterpret_cast<const float4*>(target);
  gd.loss = loss;
  gd.grad_scale = grad_density_scale;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  rc = stage_grid_layout(c, gd, true, s);
  if (rc) return rc;
  rc = psc::launch_grid_march(u, vd, gd, true, s);
  if (rc) return fail(rc, "adjoint launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  rc = psc::launch_grid_fold(gd.grad_pairs, grad_values, gd.nx, gd.ny * gd.nz, s);
  if (rc) return fail(rc, "gradient fold launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  ++c->launches;
  return PSC_OK;
}

int psc_layer_gradient(psc_ctx* c, const PscDensityGrid* g, const PscView* v, const float* background,
                       const float* target, double* grad_base_top, void* stream) {
  if (!background || !target || !grad_base_top) return fail(PSC_ERR_INVALID_ARGUMENT, "null gradient buffer");
  psc::MarchUniforms u;
  psc::ViewDev vd;
  psc::GridDev gd;
  int rc = prepare_grid(c, g, v, true, u, vd, gd);
  if (rc) return rc;
  const psc::LayerConst& L = u.layers[0];
  if (L.cloud_type == 7u && u.phase_mode == PSC_PHASE_APPROX_MIE)
    return fail(PSC_ERR_UNSUPPORTED,
                "the layer gradient covers height-independent phase (not the Cumulonimbus droplet blend)");
  if (!(L.top_m - L.base_m > 1.0f))
    return fail(PSC_ERR_INVALID_ARGUMENT, "the layer must be more than 1 m thick for its range gradient");
  // the tangent march reads both LUTs with FP32 bilinear weights, the form
  // whose derivatives it carries
  u.tex_trans = 0;
  u.tex_sky = 0;
  gd.bg = reinterpret_cast<const float4*>(background);
  gd.target = reinterpret_cast<const float4*>(target);
  rc = psc::launch_grid_layer_grad(u, vd, gd, grad_base_top, static_cast<cudaStream_t>(stream));
  if (rc) return fail(rc, "layer-gradient launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  ++c->launches;
  return PSC_OK;
}

int psc_layer_param_gradient(psc_ctx* c, const PscView* v, uint32_t layer, const float* background,
                             const float* target, double* grad, double* loss, void* stream) {
  if (!c || !v || !background || !target || !grad)
    return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (layer >= c->n_layers) return fail(PSC_ERR_INVALID_ARGUMENT, "layer %u of %u", layer, c->n_layers);
  int rc = prepare_render(c, v, 1, false, false);
  if (rc) return rc;
  const uint32_t vw = v->viewport_w ? v->viewport_w : v->width, vh = v->viewport_h ? v->viewport_h : v->height;
  psc::MarchUniforms u;
  build_uniforms(c, vw, vh, u);
  const psc::ViewDev vd{v->width, v->height, v->x_offset, v->y_offset, v->depth, nullptr, nullptr, nullptr};
  // diurnal_modulation of the layer (as build_uniforms_for): the shape and
  // detail biases act through it
  const PscCloudLayerGpu& L = c->layers[layer];
  const PscCloudParamsGpu& p = c->params;
  const uint32_t t = L.cloud_type;
  const bool conv = t == 0 || t == 2 || t == 3 || t == 7;
  const float di = (p.diurnal_strength == 0.0f || !conv)
                       ? 0.0f
                       : smoothstep_h(-0.1f, 0.4f, c->frame.sun_direction[1]) * p.diurnal_strength;
  const float ld_raw = p.detail_strength + L.detail_bias * di;
  psc::ParamGradDev g;
  g.bg = reinterpret_cast<const float4*>(background);
  g.target = reinterpret_cast<const float4*>(target);
  g.inv_n = (float)(1.0 / (3.0 * (double)vw * (double)vh));
  g.layer = layer;
  g.dlf_dshape = di * 0.5f;
  g.dld_ddetail = (ld_raw > 0.0f && ld_raw < 1.0f) ? di : 0.0f;
  // base and top move the wind-cache sample (the layer's mid-altitude, d mid
  // = (d base + d top) / 2; the field is trilinear, so a 0.5 m central
  // difference is its slope) and the skew thickness max(top - base, 1) * s
  {
    const double mid = 0.5 * ((double)L.base_m + (double)L.top_m), h = 0.5;
    double wx0, wz0, wxp, wzp, wxm, wzm;
    wind_at_mid(c, mid, wx0, wz0);
    wind_at_mid(c, mid + h, wxp, wzp);
    wind_at_mid(c, mid - h, wxm, wzm);
    const double dwx = (wxp - wxm) / (2.0 * h) * 0.5, dwz = (wzp - wzm) / (2.0 * h) * 0.5;  // per unit base or top
    const double drift = (double)p.wind_drift_strength * (double)c->frame.simulated_seconds;
    g.dwind[0][0] = g.dwind[0][1] = (float)(dwx * drift);
    g.dwind[1][0] = g.dwind[1][1] = (float)(dwz * drift);
    for (int k = 0; k < 3; ++k) g.dskew[k][0] = g.dskew[k][1] = 0.0f;
    const psc::LayerConst& o = u.layers[layer];
    if (o.skew_thickness != 0.0f) {  // skew active (wind_cache)
      const double sp = std::sqrt(wx0 * wx0 + wz0 * wz0);
      const double dsp = (wx0 * dwx + wz0 * dwz) / sp;
      g.dskew[0][0] = g.dskew[0][1] = (float)((dwx * sp - wx0 * dsp) / (sp * sp));
      g.dskew[1][0] = g.dskew[1][1] = (float)((dwz * sp - wz0 * dsp) / (sp * sp));
      if (L.top_m - L.base_m > 1.0f) {
        g.dskew[2][0] = -p.wind_skew_strength;
        g.dskew[2][1] = p.wind_skew_strength;
      }
    }
  }
  if (L.cloud_type == 7u && u.phase_mode == PSC_PHASE_APPROX_MIE)
    return fail(PSC_ERR_UNSUPPORTED,
                "the layer-parameter gradient covers height-independent phase (not the Cumulonimbus droplet "
                "blend under the approx-Mie phase)");
  if (!(L.top_m - L.base_m > 1.0f))
    return fail(PSC_ERR_INVALID_ARGUMENT, "the layer must be more than 1 m thick for its range gradient");
  rc = psc::launch_march_param_grad(u, vd, g, c->opts.storage, grad, loss, static_cast<cudaStream_t>(stream));
  if (rc) return fail(rc, "parameter-gradient launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  ++c->launches;
  return PSC_OK;
}

int psc_launch_count(psc_ctx* c, uint64_t* out) {
  if (!c || !out) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  *out = c->launches;
  return PSC_OK;
}

}  // extern "C"

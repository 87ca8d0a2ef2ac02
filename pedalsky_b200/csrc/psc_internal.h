// Internal layout shared by the host library and the CUDA kernels.
//
// The host flattens the reference's uniforms (CloudParams, FrameUniforms,
// WorldUniforms, the 8-entry layer array) plus everything that is constant
// per layer or per frame into one `MarchUniforms` block, passed to the march
// kernel by value as a __grid_constant__ parameter (it lives in the constant
// bank; every lane reads the same address, so these loads broadcast).
#pragma once

#include <cstdint>

#include "../../include/psclouds.h"

#ifndef __CUDACC__
#include <cuda_runtime_api.h>
#else
#include <cuda_runtime.h>
#endif

namespace psc {

constexpr uint32_t kFetchTallyKinds = 14;  // counters of PscFetchCounts
constexpr float kPi = 3.14159265358979f;  // HG_PI, cloud_march.wgsl:71

// Per-layer constants.  Everything here is a pure function of the layer,
// CloudParams, the wind field and the sun direction, so the host computes
// it once per frame instead of every pixel re-deriving it.
struct LayerConst {
  float base_m, top_m;
  float inv_thickness;     // 1 / max(top - base, 1)
  float coverage;
  float density_scale;
  uint32_t cloud_type;
  float lf_bias;           // shape_bias * diurnal(layer.type) * 0.5
  float layer_detail;      // clamp(detail_strength + detail_bias * diurnal, 0, 1)
  float anvil_bias;
  float droplet_um;
  float sigma_t[3];        // (sigma_s + sigma_a) * chromatic_mie_modulation(d)
  float wind_off_x, wind_off_z;   // LayerWindCache.wind_offset
  float skew_x, skew_z, skew_thickness;
  // Approx-Mie constants (cloud_phase_constants); exact for every layer
  // type except Cumulonimbus, whose diameter depends on height.
  float g_hg, g_d, alpha, w_d, ice;
  // ndf of types 0..6 as ssr(0, ndf_inv_a, h) * g with g the smoothstep of
  // clamp01(h * ndf_inv_w1 + ndf_b1); a falling second factor 1 - S(t) is
  // stored as S(1 - t) (negated slope, offset 1 - b), so g needs no flip.
  // ndf_mode 0: evaluate by type (Cumulonimbus, unknown types)
  float ndf_inv_a, ndf_b1, ndf_inv_w1;
  uint32_t ndf_mode;
  float lf_c;              // 1 - lf_bias: 1 - clamp01(fbm + lf_bias) = clamp01(lf_c - fbm)
  // Lower bound of 1 - eff over the weather map (eff = clamp01(weather *
  // coverage)) less 1e-6 for rounding; 4 (above every profile) when eff
  // never reaches the 0.01 coverage gate.  A primary step whose profile
  // value nd has (nd - skip_k) * density_scale <= 1e-3 cannot be dense.
  float skip_k;
  float skew_kx, skew_kz;  // skew_x * skew_thickness, skew_z * skew_thickness
  // Altitude band (m) outside which no primary step can pass the profile
  // test above (no type grid): the host's hull of the heights where it can,
  // widened; live_lo > live_hi when no height can.  The FAST march turns it
  // into the range of step indices it runs.
  float live_lo, live_hi;
  // Normalised height above which a light-march tap's density is exactly 0
  // (its profile value is at or below skip_k), widened; above 1 when no such
  // height lies in the layer.  Used by the lean FAST form's light march.
  float light_h_dead;
  double r_bottom, r_top;  // planet_radius + base/top, FP64
};

struct alignas(16) MarchUniforms {
  // frame
  float inv_vp[4][4];      // inv_view_proj, [col][row]
  double inv_vp_d[4][4];   // the same matrix widened to double
  float cam[3];
  float sun[3];
  float sun_illum[3];
  float lightning_rgb[3];
  float lightning_radius;
  float lightning_origin_x, lightning_origin_z;
  float vp_w, vp_h;        // viewport used for NDC and AP uv
  uint32_t temporal_jitter;
  uint32_t frame_index;
  float fwd_factor_unused;
  // world
  float planet_r, atmo_top;
  double planet_r_d;
  // params
  float sigma_s[3];
  float droplet_bias;
  float forward_bias;
  float detail_strength, curl_strength, powder;
  float ms_a, ms_b, ms_c;
  float ambient;
  float base_scale, detail_scale, weather_scale;  // already max(., 1)
  uint32_t light_steps, cloud_steps, octaves, layer_count;
  uint32_t cone;
  // options
  uint32_t phase_mode;
  float hg_f, hg_b, hg_w;
  uint32_t kahan;
  uint32_t composite;
  uint32_t debug_checks;
  // derived per frame, for the FAST schedule
  float base_texel_scale;    // 128 / base_scale  (texel units per metre)
  float detail_texel_scale;  // 32 / detail_scale
  float curl_texel_scale;    // 128 / detail_scale
  float inv_base_scale, inv_detail_scale, inv_weather_scale;
  float curl_offset_scale;   // curl_strength * detail_scale
  float sun_az;              // atan2(sun.x, sun.z)
  float top_minus_r_sq_unused;
  float big_h;               // sqrt(atmo_top^2 - planet_r^2)
  float inv_big_h;           // 1 / max(big_h, 1)
  float inv_planet_r;        // 1 / planet_r
  float rho_1m;              // sqrt(2 planet_r + 1): rho at 1 m altitude
  float inv_cos_sun;         // 1 / max(sun.y, 0.05)
  uint32_t b_half;           // multi_scatter_b == 0.5 exactly
  float apow[8], bpow[8], cpow[8];  // a^n, b^n, c^n
  LayerConst layers[8];

  // inputs (device pointers)
  const void* noise_base;      // layout depends on storage
  const void* noise_detail;
  float noise_scale;           // value = stored * scale (F16/BF16/FP8)
  const uint8_t* curl;         // 128^2 RG8
  const float* blue;           // 64^2, already v/255
  const float* weather;        // R channel as float, weather_w x weather_h
  uint32_t weather_w, weather_h;
  const float4* weather_quad;  // power-of-two maps up to 1024^2: 2x2 footprints, else null
  uint32_t weather_uniform;    // every texel equal: bilinear sampling returns weather_value
  float weather_value;
  const uint8_t* type_grid;    // may be null (all sentinel)
  uint32_t type_w, type_h;
  const float4* lut_trans;     // 256x64
  const float4* lut_sky;       // 192x108
  const float4* lut_ap;        // 32x32x64
  cudaTextureObject_t tex_base, tex_detail;  // PSC_FILTER_TEXTURE only
  // F16 storage in the FAST schedule: channel-folded volumes (R, fbm) and
  // (detail fbm) as 2x2 quads per entry (noise_bake.cu:k_fold_*)
  const uint4* base_quad;
  const uint2* detail_quad;
  const uint4* curl_quad;      // FAST schedule: curl tile as 2x2 (R, G) half quads
  // transmittance / sky-view LUTs through the texture unit; 0 = plain loads
  cudaTextureObject_t tex_trans, tex_sky;
  int* error_word;             // device, debug checks
};

// One view of a launch.
struct ViewDev {
  uint32_t width, height;
  uint32_t x_off, y_off;   // rectangle origin in the viewport
  const float* depth;
  float4* out_l;
  float4* out_t;
  float4* hdr;
};

// Voxel-grid density source of the differentiable form (grid_march.cu).
struct GridDev {
  const float* values;     // ny x nz x nx, x fastest
  float* grad;             // adjoint: d loss / d values (accumulated)
  uint32_t nx, ny, nz;
  uint32_t k_cp;           // adjoint checkpoint interval (steps)
  float min_x, min_z, base;
  float inv_cell_x, inv_cell_y, inv_cell_z;
  float k;                 // density = k * value (density_scale * inv_sigma_bar)
  float inv_sigma_bar;     // 3 / (sigma_t.r + sigma_t.g + sigma_t.b) of layer 0
  float exit_t;            // early exit once max(T) < exit_t
  float inv_n;             // 1 / (3 * viewport pixels)
  const float4* bg;        // adjoint: background per pixel of the view
  const float4* target;    // adjoint: target image per pixel of the view
  double* loss;            // adjoint: accumulated loss
  double* grad_scale;      // adjoint: accumulated d loss / d density_scale
  // the values as (x, z) corner quads: entry (y, zk, xk) holds
  // v[y][zk-1][xk-1], v[y][zk-1][xk], v[y][zk][xk-1], v[y][zk][xk], zero
  // outside the grid, zk = 0..nz, xk = 0..nx (launch_grid_quads); the adjoint
  // adds its gradient into x pairs, entry xk of a (y, z) row for
  // (x = xk - 1, xk) (grad_pairs), and folds them into grad afterwards
  // (launch_grid_fold)
  const float4* quads;
  float2* grad_pairs;
};
int launch_grid_march(const MarchUniforms& u, const ViewDev& v, const GridDev& g, bool adjoint,
                      cudaStream_t stream);
// quads[(y (nz + 1) + zk) (nx + 1) + xk] as GridDev::quads from the ny x nz x
// nx values
// grad[r nx + x] += gp[r (nx + 1) + x + 1].x + gp[r (nx + 1) + x].y
int launch_grid_quads(const float* values, float4* quads, uint32_t nx, uint32_t ny, uint32_t nz, cudaStream_t stream);
int launch_grid_fold(const float2* grad_pairs, float* grad, uint32_t nx, uint32_t rows, cudaStream_t stream);
// d loss / d (base_m, top_m) of layer 0 in the grid form, added to out[0..1]
// (grid_layer_grad.cu); g.bg / g.target / g.inv_n as for the adjoint.
int launch_grid_layer_grad(const MarchUniforms& u, const ViewDev& v, const GridDev& g, double* out,
                           cudaStream_t stream);

// Adds to *count the pixels (of n) whose composited image L + bg T (bg = 1
// when null) differs from the reference's by more than thr relative, max
// over RGB (post.cu; the step autotuner's image-error test).
int launch_count_rel_err(const float4* lr, const float4* tr, const float4* l, const float4* t, const float4* bg,
                         uint32_t n, float thr, unsigned int* count, cudaStream_t stream);

// Tangent inputs of the procedural march's layer-parameter gradient
// (march_param_grad.cu).
struct ParamGradDev {
  const float4* bg;        // background per pixel of the view
  const float4* target;    // target image per pixel of the view
  float inv_n;             // 1 / (3 * viewport pixels)
  uint32_t layer;          // the differentiated layer
  float dlf_dshape;        // d lf_bias / d shape_bias = diurnal / 2
  float dld_ddetail;       // d layer_detail / d detail_bias (diurnal inside the clamp, else 0)
  // derivatives with respect to (base_m, top_m) of the layer's wind offset
  // (x, z) and of its skew direction (x, z) and skew thickness
  float dwind[2][2];
  float dskew[3][2];
};
// out[0..5] += d loss / d (coverage, shape_bias, detail_bias, density_scale,
// base_m, top_m) of layer g.layer; *loss += the loss when loss is not null.
int launch_march_param_grad(const MarchUniforms& u, const ViewDev& v, const ParamGradDev& g, uint32_t storage,
                            double* out, double* loss, cudaStream_t stream);

// TAA resolve of one cloud RT (post.cu, shaders/clouds/cloud_taa.wgsl).
struct TaaParams {
  float inv_vp[4][4];      // current inv_view_proj, [col][row]
  float prev_vp[4][4];     // previous frame's view_proj, [col][row]
  float cam[3];
  float blend_weight;      // weight of the current sample (1/8, 1 on bootstrap)
  float history_valid;     // 0: output = current sample
  uint32_t w, h;
  const float4* cur_l;
  const float4* cur_t;
  const float4* hist_l;
  const float4* hist_t;
  float4* out_l;
  float4* out_t;
};
int launch_taa_resolve(const TaaParams& p, cudaStream_t stream);
int launch_depth_halfres(const float* depth, uint32_t W, uint32_t H, float* out, uint32_t rw,
                         uint32_t rh, cudaStream_t stream);
int launch_composite_halfres(const float4* l, const float4* t, uint32_t rw, uint32_t rh, float4* hdr,
                             uint32_t W, uint32_t H, cudaStream_t stream);

// Launchers (march.cu).
int launch_march(const MarchUniforms& u, const ViewDev& v, const PscMarchOptions& o,
                 cudaStream_t stream);
// FAST schedule (march_fast.cu); returns PSC_ERR_UNSUPPORTED for settings it
// does not cover (more than 4 octaves), which the caller serves with PLAIN.
int launch_march_fast(const MarchUniforms& u, const ViewDev& v, const PscMarchOptions& o,
                      cudaStream_t stream);
// Instrumented FAST march (psc_count_fetches): the kernel of
// launch_march_fast built to count the fetches it issues into `counts`
// (kFetchTallyKinds 64-bit counters in PscFetchCounts order, added to).  F16 and U8 storage, exact or
// hybrid filtering; PSC_ERR_UNSUPPORTED otherwise.
int launch_march_fast_tally(const MarchUniforms& u, const ViewDev& v, const PscMarchOptions& o,
                            unsigned long long* counts, cudaStream_t stream);
int launch_composite(const float4* l, const float4* t, float4* hdr, uint32_t n,
                     cudaStream_t stream);
// Noise bakes (noise_bake.cu), synchronous on `stream`.
int launch_noise_bakes(uint8_t* base, uint8_t* detail, uint8_t* curl, cudaStream_t stream);
// True when a march over these n uniform blocks needs the FAST kernels' full
// form: a layer of type 7 (Cumulonimbus), a cloud-type grid (its cells may
// hold any type), Kahan sums, cone light sampling or lightning.  Otherwise
// the lean form, built without those paths, computes the same values.  The
// batched kernel also evaluates it per view on the device.
inline __host__ __device__ bool needs_full_paths(const MarchUniforms* u, uint32_t n) {
  for (uint32_t v = 0; v < n; ++v) {
    if (u[v].type_grid || u[v].kahan || u[v].cone || u[v].lightning_radius > 0.0f) return true;
    for (uint32_t i = 0; i < u[v].layer_count && i < 8u; ++i)
      if (u[v].layers[i].cloud_type == 7u) return true;
  }
  return false;
}
// Persistent batched march (march_batch.cu); `full` as needs_full_paths.
int launch_march_batch(const PscMarchOptions& o, int threads, uint32_t tile_w,
                       const MarchUniforms* u, const ViewDev* v, const uint32_t* tiles,
                       uint32_t n_tiles, uint32_t* counter, int sms, bool full, cudaStream_t stream);
// Per-view sky-view + aerial-perspective LUTs for a batch (atmosphere.cu):
// `d_frames` holds n frame records built by frame_lite_from; outputs are
// float4 (RGBA16F-rounded), sky 192x108 and AP 32x32x64 per view.
void frame_lite_from(const PscFrameUniformsGpu& f, void* out);
size_t frame_lite_size();
int launch_view_lut_bakes(const PscWorldUniformsGpu& world, const void* d_frames, uint32_t n,
                          const uint16_t* trans_f16, const uint16_t* ms_f16, float4* sky,
                          float4* ap, cudaStream_t stream);
// Atmosphere LUT bakes (atmosphere.cu): the sky-view and aerial LUTs, and
// with `statics` first the transmittance and multi-scatter LUTs, each
// written as RGBA16F (lut_f16[kind]) and as float4 of the same rounded
// values (lut_f32[kind]), kinds in PSC_LUT_* order.
int launch_lut_bakes(const PscWorldUniformsGpu& world, const PscFrameUniformsGpu& frame, bool statics,
                     uint16_t* const lut_f16[4], float4* const lut_f32[4], cudaStream_t stream);

}  // namespace psc

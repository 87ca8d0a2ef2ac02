// The context object behind the C ABI, shared by the host translation
// units (psc_host.cpp and the allocation-free batch path in
// march_noalloc.cu), and the host helpers both use.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/psclouds.h"
#include "psc_internal.h"

struct psc_ctx {
  int device = 0;
  PscCloudParamsGpu params{};
  PscCloudLayerGpu layers[8]{};
  uint32_t n_layers = 0;
  PscFrameUniformsGpu frame{};
  PscWorldUniformsGpu world{};
  bool have_frame = false;
  PscMarchOptions opts{};

  uint8_t* d_base_u8 = nullptr;    // 128^3 RGBA8 (canonical)
  uint8_t* d_detail_u8 = nullptr;  // 32^3 RGBA8
  void* d_base_store = nullptr;    // storage form
  void* d_detail_store = nullptr;
  int store_form = -1;
  float fp8_scale = 448.0f;
  uint8_t* d_curl = nullptr;       // 128^2 RG8
  float* d_blue = nullptr;         // 64^2 floats
  std::vector<uint8_t> h_blue;
  bool have_base = false, have_detail = false, have_curl = false, have_blue = false;

  float* d_weather = nullptr;
  uint32_t weather_w = 0, weather_h = 0;
  float4* d_weather_quad = nullptr;  // FAST schedule: 2x2 footprints (power-of-two maps <= 1024^2)
  bool weather_uniform = false;      // every texel holds weather_value
  float weather_value = 0.0f;
  float weather_min = 0.0f, weather_max = 0.0f;  // extremes of the R channel
  uint8_t* d_type = nullptr;
  uint32_t type_w = 0, type_h = 0;
  std::vector<uint16_t> h_wind;    // 32x16x32 RGBA16F

  float4* d_lut[4] = {nullptr, nullptr, nullptr, nullptr};  // float4 copies
  uint16_t* d_lut_h[4] = {nullptr, nullptr, nullptr, nullptr};  // RGBA16F bake outputs
  bool have_lut[4] = {false, false, false, false};

  // F16 storage, FAST schedule: channel-folded volumes (k_fold_* in
  // noise_bake.cu), one texel per entry and 2x2 quads per entry
  uint32_t* d_base_fold = nullptr;   // 128^3 half2 (R, 5G+2B+A)
  uint4* d_base_quad = nullptr;      // 128^3 x 4 half2
  uint16_t* d_detail_fold = nullptr; // 32^3 half (5R+2G+B)
  uint2* d_detail_quad = nullptr;    // 32^3 x 4 half
  uint4* d_curl_quad = nullptr;      // 128^2 x 4 half2 (R, G), FAST schedule

  // texture-unit path: RGBA8 volumes for U8 storage, the folded volumes for
  // F16 storage
  cudaArray_t arr_base = nullptr, arr_detail = nullptr;
  cudaTextureObject_t tex_base = 0, tex_detail = 0;
  bool tex_dirty = true;
  // transmittance and sky-view LUTs read through the texture unit (bilinear,
  // clamp): transmittance bound to its float4 copy in d_lut, sky-view to the
  // array arr_sky (copied from d_lut on upload); 0 until created
  cudaTextureObject_t tex_lut[4] = {0, 0, 0, 0};
  cudaArray_t arr_sky = nullptr;

  uint64_t launches = 0;
  int* d_check = nullptr;  // options.debug_checks: first out-of-range index site

  // cloud RT of the half-res / TAA forms of psc_render (grow-only scratch)
  float4* d_rt_l = nullptr;
  float4* d_rt_t = nullptr;
  size_t rt_cap = 0;          // texels
  float* d_rt_depth = nullptr;
  size_t rt_depth_cap = 0;
  // per-view TAA history (crates/ps-clouds/src/lib.rs:776-825): ping-pong
  // resolved pairs at the cloud-RT size
  struct TaaView {
    float4* l[2] = {nullptr, nullptr};
    float4* t[2] = {nullptr, nullptr};
    uint32_t w = 0, h = 0;
    uint32_t write_slot = 0;
    bool valid = false;                 // history holds a previous resolve
    uint64_t marches = 0;               // psc_render calls while this view was active
    uint64_t resolved_at = UINT64_MAX;  // `marches` at the last resolve
  } taa[PSC_MAX_CLOUD_VIEWS];
  uint32_t active_view = 0;

  // batching (psc_render_batch)
  PscBatchTuning batch_tuning{128, 16, 0, 0};
  uint32_t batch_cap_views = 0, batch_cap_tiles = 0;
  psc::MarchUniforms* d_bu = nullptr;   // per-view uniform blocks
  psc::ViewDev* d_bv = nullptr;
  void* d_bframes = nullptr;            // per-view frame records for the LUT bakes
  float4* d_bsky = nullptr;             // per-view sky-view LUTs
  std::vector<cudaTextureObject_t> batch_sky_tex;  // per-view sky-view LUTs through the texture unit
  float4* d_bap = nullptr;              // per-view aerial-perspective LUTs
  // voxel-grid form: the grid values as corner quads and the adjoint's
  // gradient as x pairs (GridDev::quads / grad_pairs), grown to the largest
  // grid seen
  float4* d_grid_quads = nullptr;
  float2* d_grad_pairs = nullptr;
  size_t grid_pairs_cap = 0;  // entries of the quad array (the pair array holds as many)
  uint32_t* d_btiles = nullptr;
  uint32_t* d_bcounter = nullptr;
  psc::MarchUniforms* h_bu = nullptr;   // pinned staging
  psc::ViewDev* h_bv = nullptr;
  void* h_bframes = nullptr;
  uint32_t* h_btiles = nullptr;
  cudaEvent_t batch_staged = nullptr;   // staging consumed by the last enqueue
  cudaStream_t batch_stream = nullptr;  // capture stream
  cudaGraphExec_t batch_exec = nullptr;
  std::vector<uint64_t> batch_key;
  // per-view LUT bakes: what each view slot's sky-view / AP LUTs were last
  // baked from (its frame record, the world, the transmittance and
  // multi-scatter LUTs' generation, the LUT buffers); a view whose inputs
  // are unchanged skips its bake (batch_bake: this call's choice per view)
  std::vector<uint64_t> batch_lut_keys;
  std::vector<uint8_t> batch_bake;
  // bumped whenever the transmittance or multi-scatter LUT changes (an
  // upload of either, a bake of both); the per-view sky-view / AP bakes of
  // the batched march read those two
  uint64_t lut_generation = 0;
  // the world uniforms and lut_generation the last bake of the transmittance
  // and multi-scatter LUTs produced: psc_bake_luts re-bakes them only when
  // either differs (the reference's static_dirty latch,
  // crates/ps-atmosphere/src/lib.rs:494-560)
  bool static_luts_baked = false;
  PscWorldUniformsGpu static_luts_world{};
  uint64_t static_luts_generation = 0;
  // per-view form (PscBatchTuning.form = 1): the views in descending
  // estimated cost, and the branch streams and fork/join events the views'
  // kernels are enqueued on (parallel branches of the captured graph)
  std::vector<uint32_t> batch_order;
  static constexpr int kBranches = 8;
  cudaStream_t batch_branch[kBranches] = {};
  cudaEvent_t batch_fork = nullptr;
  cudaEvent_t batch_join[kBranches] = {};
  int sms = 0;
};

namespace psc {
namespace host {

// Thread-local error message + status code (psc_last_error).
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
// Bind the context's device (checks the ordinal).
int ensure_device(psc_ctx* c);
// Context inputs, options and per-view checks shared by the batch entry
// points (the same rules as psc_render_batch).
int validate_batch(psc_ctx* c, const PscBatchView* views, uint32_t n);
// Tiles the batch needs under the launch shape `tu`; UINT64_MAX when a view
// has more than 4096 tiles along one axis (the tile word's 12-bit fields).
uint64_t count_batch_tiles(const PscBatchView* views, uint32_t n, const PscBatchTuning& tu);
// Host records of one batch (per-view uniform blocks pointing at the
// per-view LUTs `sky` + i*192*108 and `ap` + i*32*32*64, view records,
// frame records for the LUT bakes) and the cost-sorted tile list.  Uses no
// heap.  Fails if the tiles would exceed `max_tiles`.
int fill_batch(const psc_ctx* c, const PscBatchView* views, uint32_t n, const PscBatchTuning& tu,
               psc::MarchUniforms* hu, psc::ViewDev* hv, void* hframes, uint32_t* htiles, uint32_t max_tiles,
               float4* sky, float4* ap, uint32_t* n_tiles_out);
// True when the noise storage form (and, for texture filtering, the texture
// objects) for the current options exist, i.e. rendering would not allocate.
bool storage_ready(const psc_ctx* c);

}  // namespace host
}  // namespace psc

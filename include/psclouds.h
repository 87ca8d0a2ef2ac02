/*
 * psclouds.h — C ABI of the B200-native volumetric cloud march.
 *
 * This library is a drop-in for PedalSky's `ps-clouds` march + composite
 * pass.  In the reference that pass sits behind the `RenderSubsystem` trait
 * (crates/ps-core/src/subsystem.rs:66-118) and is implemented by
 * `CloudsSubsystem` (crates/ps-clouds/src/lib.rs:95); its device side is the
 * WGSL fragment shader `fs_main` (shaders/clouds/cloud_march.wgsl:731-1054)
 * plus the composite (shaders/clouds/cloud_composite.wgsl:48-57).
 *
 * Conventions
 *   - Every entry point returns an `int` status: PSC_OK (0) or a negative
 *     PSC_ERR_* code.  `psc_last_error()` returns a thread-local message for
 *     the last failure on the calling thread.  Nothing throws or aborts
 *     across this boundary.
 *   - A `psc_ctx` is single-threaded: one caller thread drives it, like the
 *     reference's `&mut self` subsystem.  Work is enqueued on the caller's
 *     `cudaStream_t`, passed as `void*` (NULL = legacy default stream).
 *   - Device output buffers are caller-owned device pointers.  Host inputs
 *     are copied into context-owned device memory by the upload calls.
 *   - The uniform structs below are byte-identical to the reference's
 *     std140 layouts (sizes and offsets pinned by static asserts here and by
 *     the reference's tests crates/ps-clouds/src/params.rs:220-231,
 *     crates/ps-core/src/weather.rs:537-555, crates/ps-app/tests/wgsl_layout.rs).
 */
#ifndef PSCLOUDS_H
#define PSCLOUDS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSC_ABI_VERSION 2u

/* ---------------------------------------------------------------- status */
enum {
  PSC_OK = 0,
  PSC_ERR_INVALID_ARGUMENT = -1, /* null pointer, zero size, bad enum      */
  PSC_ERR_NOT_FINITE = -2,       /* NaN / Inf in a parameter or uniform    */
  PSC_ERR_LAYERS = -3,           /* >8 layers, top <= base, overlapping    */
  PSC_ERR_MISSING_INPUT = -4,    /* render before noise / LUTs / weather   */
  PSC_ERR_CUDA = -5,             /* a CUDA runtime call failed             */
  PSC_ERR_OUT_OF_MEMORY = -6,
  PSC_ERR_TIMEOUT = -7,          /* a bounded device wait gave up          */
  PSC_ERR_UNSUPPORTED = -8,      /* mode not built / not available         */
  PSC_ERR_DEVICE_CHECK = -9      /* device-side bounds check tripped       */
};

/* --------------------------------------------------- reference constants */
#define PSC_MAX_CLOUD_LAYERS 8u          /* cloud_uniforms.wgsl:8           */
#define PSC_BASE_NOISE_SIZE 128u         /* noise.rs BASE_SIZE              */
#define PSC_DETAIL_NOISE_SIZE 32u        /* noise.rs DETAIL_SIZE            */
#define PSC_CURL_NOISE_SIZE 128u         /* noise.rs CURL_SIZE              */
#define PSC_BLUE_NOISE_SIZE 64u          /* noise.rs BLUE_NOISE_SIZE        */
#define PSC_TRANSMITTANCE_W 256u         /* atmosphere_luts.rs:16           */
#define PSC_TRANSMITTANCE_H 64u
#define PSC_MULTISCATTER_W 32u
#define PSC_MULTISCATTER_H 32u
#define PSC_SKYVIEW_W 192u
#define PSC_SKYVIEW_H 108u
#define PSC_AP_W 32u
#define PSC_AP_H 32u
#define PSC_AP_D 64u
#define PSC_WIND_X 32u                   /* wind_field.rs:36-41             */
#define PSC_WIND_Y 16u
#define PSC_WIND_Z 32u
#define PSC_TYPE_SENTINEL 255u           /* cloud_type_grid.rs SENTINEL     */
#define PSC_MAX_CLOUD_VIEWS 2u           /* lib.rs:69, TAA history slots    */

/* ------------------------------------------------- byte-exact uniforms */

/* Mirrors `CloudParamsGpu` (crates/ps-clouds/src/params.rs:33-140) and WGSL
 * `CloudParams` (shaders/clouds/cloud_uniforms.wgsl:23-83). 112 bytes. */
typedef struct PscCloudParamsGpu {
  float sigma_s[3];
  float _pad_after_sigma_s;
  float sigma_a[3];
  float droplet_diameter_bias;
  uint32_t cone_light_sampling;
  float forward_bias;
  float detail_strength;
  float curl_strength;
  float powder_strength;
  float multi_scatter_a;
  float multi_scatter_b;
  float multi_scatter_c;
  float ambient_strength;
  float base_scale_m;
  float detail_scale_m;
  float weather_scale_m;
  uint32_t light_steps;
  uint32_t cloud_steps;
  uint32_t multi_scatter_octaves;
  uint32_t cloud_layer_count;
  uint32_t temporal_jitter;
  float wind_drift_strength;
  float wind_skew_strength;
  float diurnal_strength;
} PscCloudParamsGpu;

/* Mirrors `CloudLayerGpu` (crates/ps-core/src/weather.rs:100-134) and WGSL
 * `CloudLayerGpu` (shaders/clouds/cloud_uniforms.wgsl:85-106). 48 bytes. */
typedef struct PscCloudLayerGpu {
  float base_m;
  float top_m;
  float coverage;
  float density_scale;
  uint32_t cloud_type;
  float shape_bias;
  float detail_bias;
  float anvil_bias;
  float droplet_diameter_um;
  float _pad_after_droplets_0;
  float _pad_after_droplets_1;
  float _pad_after_droplets_2;
} PscCloudLayerGpu;

/* Mirrors `FrameUniformsGpu` (crates/ps-core/src/frame_uniforms.rs:121-160)
 * and WGSL `FrameUniforms` (shaders/common/uniforms.wgsl:11-33).  Matrices
 * are column-major (`m[col][row]`).  448 bytes. */
typedef struct PscFrameUniformsGpu {
  float view[4][4];
  float proj[4][4];
  float view_proj[4][4];
  float inv_view_proj[4][4];
  float camera_position_world[4];
  float camera_velocity_world[4];
  float sun_direction[4];          /* xyz dir, w angular radius (rad)   */
  float sun_illuminance[4];        /* rgb illuminance, w TOA lux         */
  float lightning_illuminance[4];  /* rgb emission, w falloff radius (m) */
  float lightning_origin_world[4];
  float viewport_size[4];          /* w, h, 1/w, 1/h                     */
  float time_seconds;
  float simulated_seconds;
  uint32_t frame_index;
  float ev100;
  float prev_view_proj[4][4];
} PscFrameUniformsGpu;

/* Mirrors `AtmosphereParams` / `WorldUniformsGpu`
 * (crates/ps-core/src/weather.rs:23-58, defaults :60-84) and WGSL
 * `WorldUniforms` (shaders/common/uniforms.wgsl:39-58).  144 bytes. */
typedef struct PscWorldUniformsGpu {
  float planet_radius_m;
  float atmosphere_top_m;
  float rayleigh_scale_height_m;
  float mie_scale_height_m;
  float rayleigh_scattering[4];
  float mie_scattering[4];
  float mie_absorption[4];
  float mie_g;
  float _pad_after_mie_g[3];
  float ozone_absorption[4];
  float ozone_center_m;
  float ozone_thickness_m;
  float _pad_after_ozone[2];
  float ground_albedo[4];
  float haze_extinction_per_m[4];
} PscWorldUniformsGpu;

/* ------------------------------------------------ extension settings */

/* Phase function used by the multi-scatter octave loop. */
enum {
  PSC_PHASE_APPROX_MIE = 0, /* reference: Jendersie & d'Eon 2023 fit,
                               cloud_march.wgsl:256-296                    */
  PSC_PHASE_DUAL_LOBE_HG = 1 /* mix(HG(gf*c^n), HG(gb*c^n), blend)        */
};

/* Storage form of the base/detail noise volumes on the device. */
enum {
  PSC_STORAGE_U8 = 0,   /* RGBA8 unorm, the reference's own format (exact) */
  PSC_STORAGE_F32 = 1,  /* float4 per texel (the plain FP32 drop-in)      */
  PSC_STORAGE_F16 = 2,  /* half4, per-volume scale 1/255 (exact)          */
  PSC_STORAGE_BF16 = 3, /* bf16x4, per-volume scale 1/255 (exact)         */
  PSC_STORAGE_FP8 = 4   /* e4m3x4, per-volume scale (lossy experiment)    */
};

/* How the noise volumes are filtered. */
enum {
  PSC_FILTER_EXACT = 0,   /* FP32 trilinear weights from point loads      */
  PSC_FILTER_TEXTURE = 1, /* texture-unit trilinear (8-bit fixed weights) */
  PSC_FILTER_HYBRID = 2   /* texture unit for the light-march taps only,
                             exact filtering for the primary density      */
};

/* Kernel schedule. */
enum {
  PSC_SCHED_PLAIN = 0,     /* straight restatement, one thread per ray      */
  PSC_SCHED_FAST = 1       /* hoisted per-ray and per-layer constants,
                              folded FP16 volumes, batched light-march
                              fetches, a profile bound that skips the
                              fetches of steps that cannot be dense, fast
                              transcendentals                              */
};

/* Settings the reference does not expose in `CloudParamsGpu`.  Zero-filled
 * means "reference behaviour" except where a default is stated. */
typedef struct PscMarchOptions {
  uint32_t phase_mode;      /* PSC_PHASE_*                                */
  float hg_g_forward;       /* dual-lobe HG only (default 0.8)            */
  float hg_g_backward;      /* dual-lobe HG only (default -0.2)           */
  float hg_blend;           /* dual-lobe HG only (default 0.5)            */
  uint32_t storage;         /* PSC_STORAGE_*                              */
  uint32_t filter;          /* PSC_FILTER_*                               */
  uint32_t schedule;        /* PSC_SCHED_*                                */
  uint32_t kahan;           /* 1: compensated optical-depth sums          */
  uint32_t composite;       /* 1: fuse `hdr = L + hdr*T` into the march   */
  uint32_t debug_checks;    /* 1: debug march — the PLAIN schedule (exact
                               filtering unless U8 texture) with every
                               texel, LUT, blue-noise, layer and pixel
                               index compared with its buffer; a bad index
                               is skipped and psc_render returns
                               PSC_ERR_DEVICE_CHECK naming it (the call
                               waits for the kernel); batches reject it  */
  uint32_t tile_w;          /* CTA tile width in pixels (0 = default)     */
  uint32_t tile_h;          /* CTA tile height in pixels (0 = default)    */
  uint32_t half_res;        /* 1: half-res march + Catmull-Rom composite
                               (CloudsTuning::half_res_render)            */
  uint32_t taa;             /* 1: TAA resolve of the cloud RT
                               (temporal_taa && !freeze_time)             */
  uint32_t light_batch;     /* light-march taps each thread fetches before
                               combining them, FAST F16 hybrid form: 0 =
                               all six of the reference default in one
                               batch (other counts in 4s), 3 or 2 = batches
                               of that many; the same sums in the same
                               order.  Chosen by psc_autotune_batch.     */
  uint32_t _reserved;
} PscMarchOptions;

/* One view to render: a width x height rectangle of pixels.  By default
 * the rectangle is the whole image; a non-zero `viewport_w/h` makes it the
 * sub-rectangle at (`x_offset`, `y_offset`) of a viewport_w x viewport_h
 * image (row bands of one frame rendered on several GPUs).  `depth` is an
 * optional D32F reverse-Z buffer of the rectangle (width*height floats,
 * device, 0 = sky); NULL means "sky everywhere", a headless render with no
 * opaque geometry.  Outputs are indexed within the rectangle. */
typedef struct PscView {
  uint32_t width;
  uint32_t height;
  const float* depth;          /* device, nullable                       */
  float* out_luminance;        /* device, width*height*4 floats (RGBA)   */
  float* out_transmittance;    /* device, width*height*4 floats (RGBA)   */
  float* hdr;                  /* device, RGBA, read-modify-write when
                                  options.composite = 1; else unused     */
  uint32_t viewport_w;         /* 0 = width                              */
  uint32_t viewport_h;         /* 0 = height                             */
  uint32_t x_offset;
  uint32_t y_offset;
} PscView;

/* Noise volume kinds for upload/download. */
enum {
  PSC_NOISE_BASE = 0,    /* 128^3 RGBA8                                  */
  PSC_NOISE_DETAIL = 1,  /* 32^3 RGBA8                                   */
  PSC_NOISE_CURL = 2,    /* 128^2 RG8                                    */
  PSC_NOISE_BLUE = 3     /* 64^2 R8                                      */
};

/* LUT kinds for upload. */
enum {
  PSC_LUT_TRANSMITTANCE = 0, /* 256x64 RGBA16F                           */
  PSC_LUT_MULTISCATTER = 1,  /* 32x32 RGBA16F                            */
  PSC_LUT_SKYVIEW = 2,       /* 192x108 RGBA16F                          */
  PSC_LUT_AERIAL = 3         /* 32x32x64 RGBA16F                         */
};

/* Weather-map texel formats (only the R channel is read by the march). */
enum {
  PSC_WEATHER_RGBA16F = 0,   /* reference: 128^2 RGBA16F (weather_map.rs)*/
  PSC_WEATHER_RG8 = 1,       /* 2 x unorm8 per texel                     */
  PSC_WEATHER_R32F = 2       /* 1 float per texel                        */
};

/* ------------------------------------------------------- diagnostics */
const char* psc_last_error(void);
uint32_t psc_abi_version(void);

/* No counterpart in the reference: the SHA-256 (hex) of the sources and
 * compile flags this library was built from (pedalsky_b200/build.py),
 * so a caller can check that the binary it loaded matches its sources. */
const char* psc_build_id(void);
size_t psc_sizeof_params(void);     /* 112 */
size_t psc_sizeof_layer(void);      /* 48  */
size_t psc_sizeof_frame(void);      /* 448 */
size_t psc_sizeof_world(void);      /* 144 */

/* ----------------------------------------------- defaults and helpers */

/* `CloudParamsGpu::default()` (crates/ps-clouds/src/params.rs:142-212). */
int psc_params_default(PscCloudParamsGpu* out);
/* `AtmosphereParams::default()` (crates/ps-core/src/weather.rs:60-84). */
int psc_world_default(PscWorldUniformsGpu* out);
/* Reference-behaviour options: approx-Mie, U8 storage, exact filtering,
 * plain schedule, no composite fusion. */
int psc_options_default(PscMarchOptions* out);

/* Scene-side cloud layer (`CloudLayer`, crates/ps-core/src/scene.rs:410-480).
 * Negative `density_scale` / `anvil_bias` / `droplet_diameter_um` select
 * the per-type defaults (the reference's `None`). */
typedef struct PscCloudLayerDesc {
  uint32_t cloud_type;        /* 0..7: Cu St Sc Ac As Ci Cs Cb           */
  float base_m;
  float top_m;
  float coverage;
  float density_scale;
  float shape_octave_bias;
  float detail_octave_bias;
  float anvil_bias;
  float droplet_diameter_um;
} PscCloudLayerDesc;

/* `synthesise_cloud_layers` + `check_non_overlap`
 * (crates/ps-synthesis/src/cloud_layers.rs:44-74,136-150). */
int psc_synthesise_layers(const PscCloudLayerDesc* layers, uint32_t n,
                          PscCloudLayerGpu* out);

/* `FlyCamera` (crates/ps-core/src/camera.rs:11-71) plus
 * `FrameUniforms::{set_matrices,set_sun}` as used by the headless render
 * (crates/ps-app/src/test_harness.rs:335-390). */
typedef struct PscFlyCamera {
  float position[3];
  float pitch_rad;
  float yaw_rad;
  float roll_rad;
  float fov_y_rad;
  float near_m;
} PscFlyCamera;

int psc_frame_from_camera(const PscFlyCamera* cam, uint32_t width,
                          uint32_t height, float sun_altitude_rad,
                          float sun_azimuth_rad, float sun_angular_radius_rad,
                          float toa_illuminance_lux,
                          PscFrameUniformsGpu* out);

/* CPU void-and-cluster blue noise (crates/ps-clouds/src/noise.rs:646-704),
 * 64*64 bytes. */
int psc_generate_blue_noise(uint8_t* out_4096);

/* Reference weather map: 128^2 RGBA16F, R = spatial gate
 * (crates/ps-synthesis/src/weather_map.rs:46-101).  `coverage_grid` may be
 * NULL; otherwise it is a row-major `grid_w*grid_h` f32 grid spanning
 * `grid_extent_m` (coverage_grid.rs:34-60). */
int psc_synthesise_weather_map(uint32_t n_layers, float precip_mm_per_h,
                               float ground_wetness,
                               const float* coverage_grid, uint32_t grid_w,
                               uint32_t grid_h, float grid_extent_m,
                               uint16_t* out_rgba16f /* 128*128*4 */);

/* Procedural wind field, u/v channels (wind_field.rs:71-116,150-170);
 * 32x16x32 RGBA16F, w and turbulence channels zero. */
int psc_synthesise_wind_field(float surface_speed_mps, float wind_dir_deg,
                              uint16_t* out_rgba16f);

/* ------------------------------------------------------ context life */
typedef struct psc_ctx psc_ctx;

int psc_create(int cuda_device, psc_ctx** out);
int psc_destroy(psc_ctx* ctx);

/* `CloudsSubsystem::set_march_steps` (crates/ps-clouds/src/lib.rs:709-712):
 * clamps cloud steps to [8,256] and light steps to [1,16]. */
int psc_set_march_steps(psc_ctx* ctx, uint32_t cloud_steps,
                        uint32_t light_steps);
int psc_set_params(psc_ctx* ctx, const PscCloudParamsGpu* params);
int psc_get_params(psc_ctx* ctx, PscCloudParamsGpu* out);
/* Validates n <= 8, finite fields, top > base, disjoint half-open
 * intervals.  Also sets params.cloud_layer_count = n. */
int psc_set_layers(psc_ctx* ctx, const PscCloudLayerGpu* layers, uint32_t n);
int psc_set_frame(psc_ctx* ctx, const PscFrameUniformsGpu* frame,
                  const PscWorldUniformsGpu* world);
int psc_set_options(psc_ctx* ctx, const PscMarchOptions* options);
int psc_get_options(psc_ctx* ctx, PscMarchOptions* out);

/* ----------------------------------------------------------- inputs */

/* Bake base/detail/curl noise on the device (shaders/clouds/noise_*.comp.wgsl)
 * and generate the blue-noise tile on the host.  Byte-identical to the
 * oracle's CPU bake.  Synchronous. */
int psc_bake_noise(psc_ctx* ctx);
/* Upload one noise volume from host memory (RGBA8 / RG8 / R8 texels). */
int psc_upload_noise(psc_ctx* ctx, int kind, const void* texels,
                     size_t bytes);
/* Copy a noise volume back to the host in its RGBA8/RG8/R8 form. */
int psc_download_noise(psc_ctx* ctx, int kind, void* texels, size_t bytes);

int psc_upload_weather(psc_ctx* ctx, const void* texels, uint32_t width,
                       uint32_t height, int format);
/* Cloud-type grid: row-major u8, 255 = use the layer's type. */
int psc_upload_type_grid(psc_ctx* ctx, const uint8_t* texels, uint32_t width,
                         uint32_t height);
/* Wind field 32x16x32 RGBA16F (wind_field.rs layout). */
int psc_upload_wind(psc_ctx* ctx, const uint16_t* rgba16f, size_t count);
/* One atmosphere LUT, RGBA16F texels in x-fastest order. */
int psc_upload_lut(psc_ctx* ctx, int kind, const uint16_t* rgba16f,
                   size_t count);
/* Bake the atmosphere LUTs on the device from the current frame and world
 * uniforms (shaders/atmosphere/{transmittance,multiscatter,skyview,
 * aerialperspective}.comp.wgsl): the sky-view and aerial-perspective LUTs
 * every call, the transmittance and multi-scatter LUTs only when the world
 * uniforms differ from their last bake's or either was uploaded since (the
 * reference re-bakes those two only when its static inputs are dirty,
 * crates/ps-atmosphere/src/lib.rs:494-560).  Device work only, queued on
 * `stream` (later renders on the same stream see the new LUTs); with a NULL
 * stream the call returns once the bake has finished. */
int psc_bake_luts(psc_ctx* ctx, void* stream);
/* Copy one LUT back to the host as RGBA16F (waits for the device's work in
 * flight first, a bake on any stream included). */
int psc_download_lut(psc_ctx* ctx, int kind, uint16_t* rgba16f, size_t count);

/* ----------------------------------------------------------- render */

/* March `n` views (each with the context's frame uniforms rescaled to the
 * view size) and write L/T per pixel — the `clouds::march` pass
 * (crates/ps-clouds/src/lib.rs:736-994).  With options.composite = 1 the
 * `clouds::composite` blend is fused into the same kernel.
 *
 * With options.half_res or options.taa the call runs the reference's three
 * passes for ONE view (n = 1) covering its whole viewport: the march into
 * the context's cloud RT (psc_cloud_rt_size: floor(w/2) x floor(h/2) at
 * half res, the depth read at the scaled position as the patched march
 * does, crates/ps-clouds/src/pipeline.rs:277-319), the TAA resolve of the
 * active view (psc_taa_resolve) when options.taa, and, with
 * options.composite = 1, the composite into hdr (width x height): the
 * 9-tap Catmull-Rom reconstruction at half res
 * (cloud_composite_halfres.wgsl:60-126), the plain blend otherwise.
 * out_luminance / out_transmittance, when not null, receive the resolved
 * cloud RT (cloud-RT size, RGBA32F). */
int psc_render(psc_ctx* ctx, const PscView* views, uint32_t n, void* stream);

/* Cloud-RT size for a width x height target: ((w as f32 * 0.5) as u32).max(1)
 * per axis with half_res (crates/ps-clouds/src/lib.rs:751-758), else w x h. */
int psc_cloud_rt_size(uint32_t width, uint32_t height, uint32_t half_res, uint32_t* rt_width,
                      uint32_t* rt_height);

/* `clouds::taa` (shaders/clouds/cloud_taa.wgsl:81-197) of the active view:
 * reprojects each pixel at infinite depth through the frame's
 * prev_view_proj, samples the view's history bilinearly, clamps it into the
 * 3x3 neighbourhood AABB of the current RT and blends 1/8 current (the
 * first frame after enabling, a resize or psc_invalidate_taa_history
 * outputs the current sample).  Ping-pong history lives in the context
 * (per view, lib.rs:776-825); the resolve is also copied to out_l / out_t
 * when not null.  Buffers are w x h RGBA32F on the device. */
int psc_taa_resolve(psc_ctx* ctx, const float* cur_luminance, const float* cur_transmittance,
                    uint32_t width, uint32_t height, float* out_luminance,
                    float* out_transmittance, void* stream);

/* Select the view whose TAA history later calls use, clamped to
 * PSC_MAX_CLOUD_VIEWS - 1 (set_active_view, lib.rs:722). */
int psc_set_active_view(psc_ctx* ctx, uint32_t view);

/* Discard every view's TAA history (invalidate_taa_history, lib.rs:729). */
int psc_invalidate_taa_history(psc_ctx* ctx);

/* Half-res `clouds::composite` (cloud_composite_halfres.wgsl:110-126):
 * Catmull-Rom reconstruction of an rt_width x rt_height cloud RT at every
 * pixel of the width x height hdr target, L >= 0, T in [0, 1], then
 * hdr.rgba = L.rgba + hdr.rgba * T.rgba. */
int psc_composite_halfres(const float* luminance, const float* transmittance, uint32_t rt_width,
                          uint32_t rt_height, float* hdr, uint32_t width, uint32_t height,
                          void* stream);

/* `clouds::composite` (cloud_composite.wgsl:48-57, blend One/Src1,
 * pipeline.rs:469-484): hdr.rgba = L.rgba + hdr.rgba * T.rgba. */
int psc_composite(const float* luminance, const float* transmittance,
                  float* hdr, uint32_t width, uint32_t height, void* stream);

/* No counterpart in the reference.  Counts of the fetches the FAST march
 * issues for one view, by kind: the measured side of the fetch roofline
 * (the algorithmic side counts the reference algorithm's fetches, which
 * include taps the FAST kernel proves unnecessary and skips: a uniform
 * weather map is not sampled, and steps whose profile bound keeps them
 * below the density threshold fetch nothing).  Produced by an instrumented
 * build of the FAST kernel that computes the same image (outputs as
 * psc_render for this view) and counts as it goes; the timed kernels carry
 * no counters.  Options: FAST schedule, F16 or U8 storage, exact or hybrid
 * filtering, no debug checks, half-res or TAA; else PSC_ERR_UNSUPPORTED.
 * Synchronous; allocates and frees a 112-byte counter buffer. */
typedef struct PscFetchCounts {
  uint64_t rays;                /* pixels marched                          */
  uint64_t primary_steps;       /* primary steps executed (the steps of a
                                   layer outside the altitude band where the
                                   profile test can pass are not run)      */
  uint64_t live_steps;          /* steps past the profile bound: one base-
                                   shape tap and one curl tap each          */
  uint64_t weather_taps;        /* bilinear weather taps (0: uniform map)  */
  uint64_t type_loads;          /* cloud-type grid loads                   */
  uint64_t detail_taps;         /* trilinear detail taps                   */
  uint64_t dense_samples;       /* samples with density > 1e-3             */
  uint64_t light_taps;          /* light-march base taps                   */
  uint64_t transmittance_taps;  /* transmittance-LUT taps (sunlit samples) */
  uint64_t skyview_taps;        /* sky-view LUT taps                       */
  uint64_t ap_taps;             /* aerial-perspective taps                 */
  uint64_t depth_loads;         /* depth-buffer loads                      */
  uint64_t dense_warp_passes;   /* warp passes through the dense-sample
                                   body (LUTs, light march, octaves)        */
  uint64_t dense_warp_lanes;    /* lanes active in those passes: / (32 x
                                   passes) is the body's SIMT efficiency    */
} PscFetchCounts;
int psc_count_fetches(psc_ctx* ctx, const PscView* view, PscFetchCounts* out, void* stream);

/* Number of march-kernel launches issued by this context so far. */
int psc_launch_count(psc_ctx* ctx, uint64_t* out);

/* --------------------------------------------------------- batching */

#define PSC_MAX_BATCH_VIEWS 256u

/* One view of a batch: its own scene (CloudParams, layers, frame uniforms,
 * i.e. camera and sun) and its own outputs.  World uniforms, noise, weather,
 * wind and the transmittance/multi-scatter LUTs are the context's.  The
 * sky-view and aerial-perspective LUTs are baked per view.  New in this
 * library: the reference draws one view per pass
 * (crates/ps-clouds/src/lib.rs:714-724). */
typedef struct PscBatchView {
  PscFrameUniformsGpu frame;
  PscCloudParamsGpu params;     /* cloud_layer_count is taken from n_layers */
  PscCloudLayerGpu layers[8];
  uint32_t n_layers;
  uint32_t width;
  uint32_t height;
  uint32_t _pad0;
  const float* depth;           /* device, nullable                        */
  float* out_luminance;         /* device, nullable                        */
  float* out_transmittance;     /* device, nullable                        */
  float* hdr;                   /* device; composited when options.composite */
} PscBatchView;

/* Launch shape of the batched march. */
typedef struct PscBatchTuning {
  uint32_t threads;    /* CTA size: 64, 128 or 256 (form 0)                 */
  uint32_t tile_w;     /* tile width in pixels, a multiple of 8 dividing
                          threads/4; tile height = threads/32/(tile_w/8)*4
                          (form 0)                                          */
  uint32_t use_graph;  /* 1: capture the batch once as a CUDA graph and
                          relaunch it while the batch is unchanged          */
  uint32_t form;       /* PSC_BATCH_PERSISTENT or PSC_BATCH_PER_VIEW        */
} PscBatchTuning;

enum {
  /* One persistent kernel for the whole batch: CTAs sized to the SMs'
   * resident capacity pull pixel tiles of all views, in descending cost,
   * from one atomic counter; each view's uniform block is copied to shared
   * memory when a CTA moves to that view. */
  PSC_BATCH_PERSISTENT = 0,
  /* One single-view FAST kernel per view with its uniforms as constant-bank
   * kernel parameters, enqueued in descending cost on parallel branch
   * streams, so the views run concurrently and the block scheduler balances
   * them; with use_graph the branches are one captured CUDA graph. */
  PSC_BATCH_PER_VIEW = 1
};

int psc_set_batch_tuning(psc_ctx* ctx, const PscBatchTuning* tuning);
int psc_get_batch_tuning(psc_ctx* ctx, PscBatchTuning* out);

/* March every view of the batch in one persistent kernel (FAST schedule;
 * storage/filter from the context's options: F16, U8 or F32 exact, F16 or
 * U8 hybrid, U8 texture).  Requires the transmittance and multi-scatter LUTs
 * (psc_bake_luts or psc_upload_lut).  Enqueued on `stream`. */
int psc_render_batch(psc_ctx* ctx, const PscBatchView* views, uint32_t n, void* stream);

/* Time every candidate launch shape on this batch (`reps` timed runs each,
 * after one warm-up): the persistent form at each CTA size and tile width,
 * and the per-view form; then, for the FAST F16 hybrid form, the light-march
 * fetch batch (options.light_batch 0, 3, 2) in the fastest of those.  Keeps
 * the fastest in the context (the light batch in its options,
 * psc_get_options) and returns the launch shape with its median time in
 * milliseconds.  Synchronous. */
int psc_autotune_batch(psc_ctx* ctx, const PscBatchView* views, uint32_t n, uint32_t reps,
                       PscBatchTuning* best, float* best_ms, void* stream);

/* Lower each view's march step counts as far as its image allows: renders
 * the batch at the views' own counts (params.cloud_steps / light_steps) as
 * the reference, then, per view, the light-march length one step at a time
 * (down to half) and then the primary step count (7/8, 3/4, 5/8, 1/2 of
 * it, at least 8), keeping each reduction while at most `max_share` of the
 * view's pixels differ from its reference by more than `max_rel_err`
 * (relative, max over RGB, of the composited image L + B T with B the
 * view's hdr contents at the call, or 1 without hdr); the first reduction
 * that fails ends that view's search.  Writes the chosen counts into
 * views[i].params and the median of `reps` timed runs of the batch before
 * and after into *ms_before / *ms_after (nullable).  Renders into its own
 * scratch outputs with compositing off (64 bytes per pixel of the batch,
 * allocated and freed by the call), so the views' buffers are not written.
 * 1e-3 / 1e-3 is the parity bar of this library's tests (p99.9 within
 * 1e-3).  Synchronous. */
int psc_autotune_steps(psc_ctx* ctx, PscBatchView* views, uint32_t n, float max_rel_err,
                       float max_share, uint32_t reps, float* ms_before, float* ms_after,
                       void* stream);

/* ------------------------------------------ voxel-grid density, adjoint */

/* A voxel density source for the differentiable form of the march.  New in
 * this library: the reference's clouds are procedural only (sample_density,
 * shaders/clouds/cloud_march.wgsl:432-530).  The grid replaces the density of
 * the context's single layer (layer 0 gives the altitude range base_m..top_m,
 * droplet size and type; CloudParams give scattering, phase, octaves,
 * powder, ambient and the step counts), and the march differs from the
 * procedural one in three stated ways: every primary step contributes (no
 * density > 1e-3 gate, so the image is a smooth function of the grid), the
 * step integral is (1 - exp(-x)) / x without the 1e-6 floor, and no aerial
 * perspective is applied.  Cells are trilinearly interpolated between cell
 * centres and read as zero outside the grid.  Values are mean extinction
 * coefficients in 1/m: density = density_scale * value * 3 / (sigma_t.r +
 * sigma_t.g + sigma_t.b) with sigma_t the layer's (sigma_s + sigma_a) x
 * chromatic modulation, so the RGB-mean extinction equals
 * density_scale * value. */
typedef struct PscDensityGrid {
  const float* values;          /* ny x nz x nx FP32, x fastest, then z, then altitude */
  uint32_t nx, ny, nz;          /* cells along world x (east), altitude, world z (south) */
  uint32_t checkpoint_every;    /* psc_adjoint: transmittance checkpoint interval, 1..32 steps */
  float min_x_m, min_z_m;       /* world x / z of the grid's low corner */
  float size_x_m, size_z_m;     /* horizontal extent (altitude extent: layer 0 base..top) */
  float density_scale;          /* multiplies every value */
  float exit_transmittance;     /* stop once max(T) < this; 0.01 as the march, 0 = never */
} PscDensityGrid;

#define PSC_GRID_MAX_CHECKPOINTS 32u

/* Forward march of the grid form for each view (device `values`);
 * outputs as psc_render (luminance, transmittance, optional composite).
 * Needs the frame, blue noise and the transmittance and sky-view LUTs. */
int psc_render_grid(psc_ctx* ctx, const PscDensityGrid* grid, const PscView* view, void* stream);

/* Gradient of an image loss with respect to the grid values and
 * density_scale.  The image is I = L + background * T per pixel and channel
 * (the composite over `background`), the loss is
 * sum((I - target)^2) / (3 * viewport_w * viewport_h), summed over the
 * view's rectangle, so row bands of one viewport add up to the whole
 * image's loss and gradient.  `background` and `target` are device float4
 * per pixel of the rectangle.  The march keeps transmittance at every
 * `checkpoint_every`-th step and recomputes the steps between checkpoints
 * in the reverse sweep.  Results are ADDED to `grad_values` (device, same
 * shape as the grid), `*grad_density_scale` and `*loss` (device doubles),
 * so callers zero them first; view outputs, if given, receive L and T. */
int psc_adjoint(psc_ctx* ctx, const PscDensityGrid* grid, const PscView* view,
                const float* background, const float* target, float* grad_values,
                double* grad_density_scale, double* loss, void* stream);

/* Gradient of the same loss as psc_adjoint with respect to the layer's
 * altitude range: grad_base_top[0] += d loss / d base_m and
 * grad_base_top[1] += d loss / d top_m of layer 0 (device doubles).  No
 * counterpart in the reference.  In the grid form the layer's base and top
 * place the ray's entry and exit (the spheres at planet radius + base and +
 * top), spread the primary samples over that interval, stretch the grid's
 * altitude axis over base..top, end the light path at the top and set the
 * ambient height gradient; the derivative follows all of them (forward
 * mode, FP32, per ray, summed in double).  The layer's other parameters do
 * not enter the grid form, whose grid replaces the procedural density they
 * shape; d loss / d density_scale comes from psc_adjoint.  LUTs are read
 * with FP32 bilinear weights here whatever the filtering option.  Not for a
 * Cumulonimbus layer under the approx-Mie phase (its droplet size varies
 * with height): PSC_ERR_UNSUPPORTED.  Rows of one viewport add up as in
 * psc_adjoint. */
int psc_layer_gradient(psc_ctx* ctx, const PscDensityGrid* grid, const PscView* view,
                       const float* background, const float* target, double* grad_base_top,
                       void* stream);

/* Gradient of the procedural march's image loss with respect to the
 * parameters of scene layer `layer`: grad[0..5] += d loss / d coverage,
 * shape_bias, detail_bias, density_scale (what sample_density,
 * cloud_march.wgsl:432-530, consumes), base_m and top_m (the layer's shell
 * radii, its normalised height, skew thickness, mid-altitude wind sample
 * and light-path end) as device doubles; *loss += the loss when `loss` is
 * not null.  Same loss as psc_adjoint: I = L + background * T per pixel and
 * channel, sum((I - target)^2) / (3 * viewport_w * viewport_h) over the
 * view's rectangle (`background`, `target`: device float4 per pixel), so
 * row bands of one viewport add up.  No counterpart in the reference.
 * Forward mode through the whole march (sample positions, the weather,
 * noise and LUT taps through their filter weights, density, light march,
 * octaves, step integral, transmittance, aerial perspective), FP32 per ray
 * in the PLAIN schedule's arithmetic with exact filtering of the context's
 * noise storage, summed in double; branch decisions (the 1e-3 density
 * threshold, the coverage gate, the early exits, the layer hits) are held
 * at their values.  The shape and detail biases act through the diurnal
 * modulation, so their derivatives are 0 for non-convective layer types or
 * diurnal_strength 0.  Not for a Cumulonimbus layer under the approx-Mie
 * phase (its droplet size varies with height) nor a layer 1 m thick or
 * less: PSC_ERR_UNSUPPORTED / PSC_ERR_INVALID_ARGUMENT.  The view's output
 * pointers are not used. */
int psc_layer_param_gradient(psc_ctx* ctx, const PscView* view, uint32_t layer,
                             const float* background, const float* target, double* grad,
                             double* loss, void* stream);

/* ------------------------------------------------ allocation-free batch */

#define PSC_NOALLOC_MAX_VIEWS 64u
#define PSC_NOALLOC_MAX_TILES (1u << 20)

/* No counterpart in the reference.  Calibration of the fetch roofline the
 * march is measured against (its working set is L2-resident, so its ceilings
 * are on-chip): L2 read bandwidth (16-byte L2-only loads streaming a 64 MiB
 * resident buffer), L1 read bandwidth (16-byte loads that hit in L1) and the
 * trilinear fetch rate of a two-channel FP16 3D texture (the light march's
 * fetch), each saturated from every SM.  Allocates and frees its own
 * buffers; takes about 0.1 s. */
typedef struct PscFetchPeaks {
  float l2_read_gbs;
  float l1_read_gbs;
  float tex_trilinear_gfetch_s;  /* 10^9 trilinear fetches per second */
  float _reserved;
} PscFetchPeaks;
int psc_measure_fetch_peaks(int cuda_device, PscFetchPeaks* out, void* stream);

/* No counterpart in the reference (which allocates its GPU resources through
 * wgpu at set-up).  psc_render_batch with no allocation at call time, for
 * callers that cannot call cudaMalloc while rendering: a real-time frame loop
 * where an allocation or free would synchronise the device, an engine that
 * owns a fixed device-memory budget and must not see it grow, or code that
 * runs in a host callback where the CUDA allocator may not be called.
 *
 * The batch's work list (tile counter, tile list, per-view uniform and frame
 * records) lives in one fixed array of device memory of about 4.1 MiB,
 * reserved in every GPU that loads this library and held until the process
 * exits.  Limits: at most PSC_NOALLOC_MAX_VIEWS views and
 * PSC_NOALLOC_MAX_TILES tiles under the context's launch shape (a tile is
 * tile_w x threads/32/(tile_w/8)*4 pixels, 16x8 by default, so about 134 M
 * pixels); larger batches are rejected with PSC_ERR_INVALID_ARGUMENT.
 *
 * The caller passes the views (inputs and outputs as for psc_render_batch)
 * and two device buffers, 16-byte aligned, that the call fills with each
 * view's LUTs before marching: `sky_luts`, n x 192 x 108 RGBA32F texels, and
 * `ap_luts`, n x 32 x 32 x 64 RGBA32F texels (view i at i x one LUT).
 *
 * Set-up: everything psc_render_batch needs, plus one psc_render or
 * psc_render_batch call after the last change of noise inputs or storage /
 * filter options, which builds the noise storage form and texture objects
 * (those calls allocate); otherwise PSC_ERR_MISSING_INPUT.  The first call
 * on each device looks up the array's device address (and may load the
 * library's GPU code on that device); make that first call before any stream
 * capture.  The address is kept for the life of the device's primary
 * context: do not cudaDeviceReset a device while rendering on it with this
 * entry point.
 *
 * The work list is staged through host arrays shared by all calls and
 * copied with cudaMemcpyAsync from that pageable memory, which the driver
 * stages itself: the calling thread may block until the driver has taken the
 * bytes (about 2 KB per view plus 4 bytes per tile).  Because the staging
 * is shared, a stream that is being captured into a CUDA graph is refused
 * with PSC_ERR_UNSUPPORTED; psc_render_batch with use_graph = 1 is the
 * graph-replayed form.
 *
 * Every call shares the one array, whose contents persist from the previous
 * call (the counter is cleared on each call).  Calls whose work overlaps on
 * the GPU, on different streams or from different contexts on the same
 * device, race on it: order them on one stream or synchronise between them.
 * Calls from several host threads are serialised while they stage. */
int psc_render_batch_noalloc(psc_ctx* ctx, const PscBatchView* views, uint32_t n, float* sky_luts,
                             float* ap_luts, void* stream);

#ifdef __cplusplus
} /* extern "C" */

static_assert(sizeof(PscCloudParamsGpu) == 112, "CloudParamsGpu is 112 B");
static_assert(sizeof(PscDensityGrid) == 48, "PscDensityGrid layout");
static_assert(sizeof(PscBatchView) == 448 + 112 + 384 + 16 + 32, "PscBatchView layout");
static_assert(sizeof(PscCloudLayerGpu) == 48, "CloudLayerGpu is 48 B");
static_assert(sizeof(PscFrameUniformsGpu) == 448, "FrameUniformsGpu is 448 B");
static_assert(sizeof(PscWorldUniformsGpu) == 144, "WorldUniformsGpu is 144 B");
static_assert(offsetof(PscCloudParamsGpu, sigma_a) == 16, "std140 sigma_a");
static_assert(offsetof(PscCloudParamsGpu, droplet_diameter_bias) == 28, "");
static_assert(offsetof(PscCloudParamsGpu, cone_light_sampling) == 32, "");
static_assert(offsetof(PscCloudParamsGpu, powder_strength) == 48, "");
static_assert(offsetof(PscCloudParamsGpu, ambient_strength) == 64, "");
static_assert(offsetof(PscCloudParamsGpu, light_steps) == 80, "");
static_assert(offsetof(PscCloudParamsGpu, temporal_jitter) == 96, "");
static_assert(offsetof(PscCloudLayerGpu, cloud_type) == 16, "");
static_assert(offsetof(PscCloudLayerGpu, droplet_diameter_um) == 32, "");
static_assert(offsetof(PscFrameUniformsGpu, camera_position_world) == 256, "");
static_assert(offsetof(PscFrameUniformsGpu, viewport_size) == 352, "");
static_assert(offsetof(PscFrameUniformsGpu, time_seconds) == 368, "");
static_assert(offsetof(PscFrameUniformsGpu, prev_view_proj) == 384, "");
static_assert(offsetof(PscWorldUniformsGpu, rayleigh_scattering) == 16, "");
static_assert(offsetof(PscWorldUniformsGpu, mie_g) == 64, "");
static_assert(offsetof(PscWorldUniformsGpu, ozone_absorption) == 80, "");
static_assert(offsetof(PscWorldUniformsGpu, ozone_center_m) == 96, "");
static_assert(offsetof(PscWorldUniformsGpu, ground_albedo) == 112, "");
static_assert(offsetof(PscWorldUniformsGpu, haze_extinction_per_m) == 128, "");
#endif

#endif /* PSCLOUDS_H */

/*
 * ORACLE — test infrastructure, not product code.
 *
 * A CPU restatement of PedalSky's volumetric-cloud march path, used only as
 * the checker for the CUDA implementation: by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
 * library (pedalsky_b200/libpsclouds.so) never links or calls it.
 *
 * Parity status: the reference publishes no numeric HDR goldens for this
 * path and its WGSL cannot execute here (no graphics stack), so radiance
 * parity of this restatement is UNPINNED.  What IS pinned against the
 * reference's own tests: struct layouts, the coverage remap endpoints,
 * per-type density/droplet defaults, the weather-map gate, the type-grid
 * sentinel, the blue-noise histogram and the noise channel statistics
 * (see tests/test_oracle_pins.py for the file:line of each).
 *
 * Every function cites the reference file:line it restates.
 */
#ifndef PSC_ORACLE_H
#define PSC_ORACLE_H

#include <stdint.h>
#include "../include/psclouds.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- noise bakes (shaders/clouds/noise_*.comp.wgsl), FP32 as in WGSL ---- */
int oracle_bake_noise_base(uint8_t* out_rgba8);    /* 128^3 * 4 */
int oracle_bake_noise_detail(uint8_t* out_rgba8);  /* 32^3 * 4  */
int oracle_bake_noise_curl(uint8_t* out_rg8);      /* 128^2 * 2 */
int oracle_blue_noise(uint8_t* out_r8);            /* 64^2      */

/* ---- defaults: CloudParamsGpu::default() (crates/ps-clouds/src/params.rs:142-212),
 *      AtmosphereParams::default() (crates/ps-core/src/weather.rs:60-84) ---- */
int oracle_params_default(PscCloudParamsGpu* out);
int oracle_world_default(PscWorldUniformsGpu* out);

/* ---- synthesis (crates/ps-synthesis) ---- */
float oracle_remap_coverage(float scene_coverage);
int oracle_synthesise_layers(const PscCloudLayerDesc* in, uint32_t n,
                             PscCloudLayerGpu* out);
int oracle_weather_map(uint32_t n_layers, float precip_mm_per_h,
                       float ground_wetness, const float* grid, uint32_t gw,
                       uint32_t gh, float grid_extent_m, uint16_t* out);
float oracle_value_noise_2d(float x, float y);
int oracle_wind_field(float surface_speed, float wind_dir_deg, uint16_t* out);
int oracle_frame_from_camera(const PscFlyCamera* cam, uint32_t width,
                             uint32_t height, float sun_alt, float sun_az,
                             float sun_ang_radius, float toa_lux,
                             PscFrameUniformsGpu* out);

/* ---- f16 helpers (IEEE binary16, round-to-nearest-even) ---- */
uint16_t oracle_f32_to_f16(float f);
float oracle_f16_to_f32(uint16_t h);

/* ---- atmosphere LUT bakes (shaders/atmosphere/...), FP32, f16 output ---- */
int oracle_bake_transmittance(const PscWorldUniformsGpu* world, uint16_t* out);
int oracle_bake_multiscatter(const PscWorldUniformsGpu* world,
                             const uint16_t* trans, uint16_t* out);
int oracle_bake_skyview(const PscFrameUniformsGpu* frame,
                        const PscWorldUniformsGpu* world,
                        const uint16_t* trans, const uint16_t* ms,
                        uint16_t* out);
int oracle_bake_aerial(const PscFrameUniformsGpu* frame,
                       const PscWorldUniformsGpu* world, const uint16_t* trans,
                       const uint16_t* ms, uint16_t* out);

/* ---- the march ---- */
typedef struct OracleScene {
  PscCloudParamsGpu params;
  PscCloudLayerGpu layers[8];
  PscFrameUniformsGpu frame;
  PscWorldUniformsGpu world;
  PscMarchOptions options;           /* phase_mode + HG lobes read here    */
  const uint8_t* noise_base;         /* 128^3 RGBA8                       */
  const uint8_t* noise_detail;       /* 32^3 RGBA8                        */
  const uint8_t* noise_curl;         /* 128^2 RG8                         */
  const uint8_t* blue_noise;         /* 64^2 R8                           */
  const void* weather;               /* R channel read                    */
  uint32_t weather_w, weather_h;
  int weather_format;                /* PSC_WEATHER_*                     */
  const uint8_t* type_grid;          /* may be NULL = all sentinel        */
  uint32_t type_w, type_h;
  const uint16_t* wind;              /* 32x16x32 RGBA16F                  */
  const uint16_t* lut_transmittance; /* 256x64 RGBA16F                    */
  const uint16_t* lut_skyview;       /* 192x108 RGBA16F                   */
  const uint16_t* lut_aerial;        /* 32x32x64 RGBA16F                  */
  const float* depth;                /* width*height, may be NULL         */
} OracleScene;

enum { ORACLE_FP32 = 32, ORACLE_FP64 = 64 };
enum { ORACLE_FILTER_EXACT = 0, ORACLE_FILTER_Q8 = 1 };

/* Fetch counters accumulated over the image (executed fetches). */
enum {
  ORACLE_CNT_WEATHER = 0,  /* bilinear weather tap per primary step       */
  ORACLE_CNT_TYPE,         /* type-grid load per primary step             */
  ORACLE_CNT_BASE,         /* primary base-noise trilinear taps           */
  ORACLE_CNT_CURL,         /* curl bilinear taps                          */
  ORACLE_CNT_DETAIL,       /* detail trilinear taps                       */
  ORACLE_CNT_LIGHT,        /* light-march base trilinear taps             */
  ORACLE_CNT_TRANS,        /* transmittance LUT bilinear taps             */
  ORACLE_CNT_SKY,          /* sky-view LUT bilinear taps                  */
  ORACLE_CNT_WIND,         /* per-layer wind-field trilinear taps         */
  ORACLE_CNT_AP,           /* aerial-perspective trilinear taps           */
  ORACLE_CNT_BLUE,         /* blue-noise loads                            */
  ORACLE_CNT_DEPTH,        /* depth loads                                 */
  ORACLE_CNT_STEPS,        /* primary steps executed                      */
  ORACLE_CNT_DENSE,        /* dense (density > 1e-3) primary steps        */
  ORACLE_CNT_PIXELS,
  ORACLE_CNT__COUNT
};

/* Render width x height pixels of the view described by `scene`.
 * out_lum / out_trans: width*height*4 floats (RGBA) each.  `counters` may
 * be NULL, else ORACLE_CNT__COUNT entries.  `threads` <= 0 = all cores.
 * Rows [row0, row1) only (row1 = 0 means all rows); other rows untouched. */
int oracle_render(const OracleScene* scene, uint32_t width, uint32_t height,
                  int precision, int filter, int threads, uint32_t row0,
                  uint32_t row1, float* out_lum, float* out_trans,
                  uint64_t* counters);

/* Same march, one pixel, both outputs in double (for spot checks). */
int oracle_render_pixel(const OracleScene* scene, uint32_t width,
                        uint32_t height, uint32_t x, uint32_t y,
                        int precision, int filter, double* lum4,
                        double* trans4);

/* The FP64 march of rows [row0, row1) (row1 = 0: all rows) recording per
 * pixel how close it came to its two data-dependent branches
 * (cloud_march.wgsl:833,885,996): out_t the smallest |max3(T) - 0.01| / 0.01
 * of its early-exit tests, out_d the smallest |density - 1e-3| / 1e-3 of its
 * primary samples (width*height doubles each; 1e30 where never tested). */
int oracle_branch_margins(const OracleScene* scene, uint32_t width, uint32_t height,
                          int threads, uint32_t row0, uint32_t row1, double* out_t,
                          double* out_d);

/* The FP64 march of `scene` with the outcomes of its discontinuous tests
 * (the layer hits and their order, the early exits, the 1e-3 density
 * threshold, the aerial-perspective opacity test) replayed from the FP64
 * march of `ref` at each pixel: the image as a
 * smooth function of whatever parameters differ between the two scenes,
 * written in double.
 * Returns the number of outcomes a replay needed beyond its record (0 when
 * the two march the same path; -1 on bad arguments). */
long long oracle_render_frozen(const OracleScene* ref, const OracleScene* scene, uint32_t width,
                               uint32_t height, int threads, double* lum, double* tr);

/* One FP64 primary density sample at world point p3 / altitude alt in layer
 * li with weather R value weather_r, and the layer profile ndf(h) there
 * (test support for the density bound of the GPU march's step skip). */
int oracle_density_sample(const OracleScene* scene, uint32_t li, const double* p3,
                          double alt, double weather_r, double* density,
                          double* profile);

/* ---- voxel-grid form (no reference counterpart; see oracle_grid.cpp) ----
 * Images are width x height = the scene's viewport; bg / target are
 * width*height*4 floats; the loss is sum((L + bg*T - target)^2) / (3*w*h). */
int oracle_grid_render(const OracleScene* scene, const PscDensityGrid* grid,
                       uint32_t width, uint32_t height, int precision,
                       int threads, float* out_lum, float* out_trans);
/* FP64 loss over the listed pixel indices (y*width + x); NULL = all. */
int oracle_grid_loss(const OracleScene* scene, const PscDensityGrid* grid,
                     uint32_t width, uint32_t height, const float* bg,
                     const float* target, const uint32_t* pixels,
                     uint32_t n_pixels, int threads, double* loss);
/* FP64 reverse-mode gradient (all steps stored, no checkpoints) of the
 * loss terms of rows [row0, row1) (row1 = 0: all rows); the normalisation
 * stays the whole image's, so row bands add up. */
int oracle_grid_adjoint(const OracleScene* scene, const PscDensityGrid* grid,
                        uint32_t width, uint32_t height, const float* bg,
                        const float* target, uint32_t row0, uint32_t row1,
                        int threads, double* grad, double* grad_density_scale,
                        double* loss);
/* Executed work of the forward march: out[0] pixels, [1] pixels whose ray
 * meets the grid layer, [2] primary steps, [3] in-grid texels read by the
 * primary samples, [4] in-grid texels read by the light taps. */
int oracle_grid_counts(const OracleScene* scene, const PscDensityGrid* grid,
                       uint32_t width, uint32_t height, int threads,
                       uint64_t* out);
/* Central differences of the FP64 loss for each listed voxel index, over
 * the pixels whose samples touch that voxel (their count per voxel goes to
 * n_pixels_out if not NULL). */
int oracle_grid_fd(const OracleScene* scene, const PscDensityGrid* grid,
                   uint32_t width, uint32_t height, const float* bg,
                   const float* target, const uint64_t* voxels, uint32_t n_vox,
                   double eps, int threads, double* out, uint32_t* n_pixels_out);

/* `dst = L + dst*T` per channel (cloud_composite.wgsl + blend One/Src1). */
int oracle_composite(const float* lum, const float* trans, float* hdr,
                     uint32_t n_pixels);

#ifdef __cplusplus
}
#endif
#endif

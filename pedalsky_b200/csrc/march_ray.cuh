// Per-ray set-up shared by the march schedules: the view ray
// (compute_view_ray, shaders/common/math.wgsl:23-33), the depth clip
// (cloud_march.wgsl:764-775), the per-layer shell intersection
// (ray_layer_intersect, cloud_march.wgsl:370-416) and the stable sort of the
// hit layers by entry distance (:796-806).  All in FP64: at planet radius
// (6.36e6 m) the FP32 form |oc|^2 - r^2 cancels catastrophically and moves
// the layer entry by metres, which the detail noise (25 m texels) resolves.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "psc_internal.h"

namespace psc {
namespace {

struct RaySetup {
  float dir[3];
  double dird[3];
  float r0, cos_view, h0;
  float t0[8], t1[8];
  uint32_t hit_mask;
  uint32_t order;  // 4 bits per slot: layer index at sorted position k
};

__device__ __forceinline__ bool sphere_hit(const double oc[3], const double d[3], double r,
                                           double& ta, double& tb) {
  const double b = oc[0] * d[0] + oc[1] * d[1] + oc[2] * d[2];
  const double c = (oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2]) - r * r;
  const double disc = b * b - c;
  if (disc < 0.0) return false;
  const double sq = sqrt(disc);
  ta = -b - sq;
  tb = -b + sq;
  return true;
}

__device__ void setup_ray(const MarchUniforms& u, const ViewDev& v, uint32_t px, uint32_t py,
                          RaySetup& rs) {
  const double fx = (double)(px + v.x_off) + 0.5, fy = (double)(py + v.y_off) + 0.5;
  const double nx = (fx / (double)u.vp_w) * 2.0 - 1.0;
  const double ny = 1.0 - (fy / (double)u.vp_h) * 2.0;
  double nh[4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
    nh[r] = ((u.inv_vp_d[0][r] * nx + u.inv_vp_d[1][r] * ny) + u.inv_vp_d[2][r]) + u.inv_vp_d[3][r];
  double d[3] = {nh[0] / nh[3] - (double)u.cam[0], nh[1] / nh[3] - (double)u.cam[1],
                 nh[2] / nh[3] - (double)u.cam[2]};
  const double inv_l = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    rs.dird[k] = d[k] * inv_l;
    rs.dir[k] = (float)rs.dird[k];
  }
  const double oc[3] = {(double)u.cam[0], (double)u.cam[1] + u.planet_r_d, (double)u.cam[2]};
  const double r0 = sqrt(oc[0] * oc[0] + oc[1] * oc[1] + oc[2] * oc[2]);
  rs.r0 = (float)r0;
  const double rr = fmax(r0, 1.0);
  rs.cos_view = (float)((oc[0] * rs.dird[0] + oc[1] * rs.dird[1] + oc[2] * rs.dird[2]) / rr);
  rs.h0 = (float)(r0 - u.planet_r_d);

  // depth clip (cloud_march.wgsl:764-775)
  double depth_t_max = 1.0e30;
  if (v.depth) {
    const float dn = __ldg(v.depth + (size_t)py * v.width + px);
    if (dn > 0.0f) {
      double hh[4];
#pragma unroll
      for (int r = 0; r < 4; ++r)
        hh[r] = ((u.inv_vp_d[0][r] * nx + u.inv_vp_d[1][r] * ny) + u.inv_vp_d[2][r] * (double)dn) +
                u.inv_vp_d[3][r];
      const double wx = hh[0] / hh[3] - (double)u.cam[0];
      const double wy = hh[1] / hh[3] - (double)u.cam[1];
      const double wz = hh[2] / hh[3] - (double)u.cam[2];
      depth_t_max = fmax(sqrt(wx * wx + wy * wy + wz * wz), 0.0);
    }
  }

  // per-layer intervals (cloud_march.wgsl:370-416, 778-793)
  rs.hit_mask = 0;
  const uint32_t n = u.layer_count;
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    rs.t0[l] = 3.0e38f;
    rs.t1[l] = 0.0f;
    if (l < (int)n) {
      const LayerConst& L = u.layers[l];
      double tt0, tt1, tb0 = 0.0, tb1 = 0.0;
      const bool hit_top = sphere_hit(oc, rs.dird, L.r_top, tt0, tt1);
      const bool hit_bot = sphere_hit(oc, rs.dird, L.r_bottom, tb0, tb1);
      bool ok = hit_top;
      double ta = 0.0, tb = 0.0;
      if (ok) {
        if (r0 < L.r_bottom) {
          ok = hit_bot;
          ta = fmax(tb1, 0.0);
          tb = fmax(tt1, 0.0);
        } else if (r0 > L.r_top) {
          ta = fmax(tt0, 0.0);
          tb = (hit_bot && tb0 > 0.0) ? fmax(tb0, 0.0) : fmax(tt1, 0.0);
        } else {
          ta = 0.0;
          tb = (hit_bot && tb0 > 0.0) ? fmin(fmax(tt1, 0.0), tb0) : fmax(tt1, 0.0);
        }
        ok = ok && (tb > ta);
      }
      // t0 is the sort key even for missed layers (the reference sorts
      // every slot; missed slots carry their computed or zero t0).
      rs.t0[l] = ok ? (float)ta : (hit_top ? (float)ta : 0.0f);
      if (ok) {
        const double t1c = fmin(tb, depth_t_max);
        if (t1c > ta) {
          rs.hit_mask |= 1u << l;
          rs.t1[l] = (float)t1c;
          rs.t0[l] = (float)ta;
        }
      }
    }
  }
  // stable ascending order by t0 (the insertion sort at :796-806)
  rs.order = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (i < (int)n) {
      uint32_t rank = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j)
        if (j < (int)n && j != i)
          rank += (rs.t0[j] < rs.t0[i] || (rs.t0[j] == rs.t0[i] && j < i)) ? 1u : 0u;
      rs.order |= (uint32_t)i << (4 * rank);
    }
  }
}

}  // namespace
}  // namespace psc

// Passes between the cloud march and the HDR target (the reference's
// clouds::taa and clouds::composite passes, crates/ps-clouds/src/lib.rs:
// 1000-1097):
//   * k_depth_halfres: the depth a half-res cloud-RT pixel (x, y) sees, the
//     full-res texel at ivec2(vec2(x, y) * viewport / rt) (the half-res march
//     patch, crates/ps-clouds/src/pipeline.rs:296-305);
//   * k_taa_resolve: shaders/clouds/cloud_taa.wgsl:81-197 — reprojection at
//     infinite depth through prev_view_proj (FP64), bilinear history, 3x3
//     neighbourhood AABB clamp, blend, L >= 0 and T in [0, 1];
//   * k_composite_halfres: shaders/clouds/cloud_composite_halfres.wgsl:60-126
//     — Catmull-Rom (B = 0, C = 0.5) reconstruction of the half-res RT at each
//     full-res pixel, evaluated as the 4x4 kernel on clamped texel indices
//     (the reference's 9 offset-bilinear taps are an exact rewriting of it),
//     then L >= 0, T in [0, 1] and dst = L + dst * T on all four channels.
// All three are one thread per output pixel, 16x16 CTAs; every index is
// clamped into its image.  The composite stages its RT footprint in shared
// memory (k_composite_halfres_tiled) whenever the RT is no larger than the
// target.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "psc_internal.h"

namespace psc {
namespace {

__device__ __forceinline__ int clampi(int i, int n) { return min(max(i, 0), n - 1); }
__device__ __forceinline__ float4 f4(float a) { return make_float4(a, a, a, a); }
__device__ __forceinline__ float4 add4(float4 a, float4 b) {
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
__device__ __forceinline__ float4 mul4(float4 a, float s) {
  return make_float4(a.x * s, a.y * s, a.z * s, a.w * s);
}
__device__ __forceinline__ float4 fma4(float4 a, float s, float4 c) {
  return make_float4(fmaf(a.x, s, c.x), fmaf(a.y, s, c.y), fmaf(a.z, s, c.z), fmaf(a.w, s, c.w));
}
__device__ __forceinline__ float4 min4(float4 a, float4 b) {
  return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w));
}
__device__ __forceinline__ float4 max4(float4 a, float4 b) {
  return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w));
}
__device__ __forceinline__ float4 clamp4(float4 v, float4 lo, float4 hi) { return min4(max4(v, lo), hi); }

__global__ void k_depth_halfres(const float* __restrict__ depth, uint32_t W, uint32_t H,
                                float* __restrict__ out, uint32_t rw, uint32_t rh) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= rw || y >= rh) return;
  const float sx = (float)W / (float)rw, sy = (float)H / (float)rh;
  const uint32_t dx = min((uint32_t)((float)x * sx), W - 1u);
  const uint32_t dy = min((uint32_t)((float)y * sy), H - 1u);
  out[(size_t)y * rw + x] = __ldg(depth + (size_t)dy * W + dx);
}

// Bilinear, clamp-to-edge, FP32 weights, at normalised (u, v).
__device__ __forceinline__ float4 bilinear_clamp(const float4* __restrict__ t, int w, int h, float u,
                                                 float v) {
  const float x = u * (float)w - 0.5f, y = v * (float)h - 0.5f;
  const float fx = floorf(x), fy = floorf(y);
  const float ax = x - fx, ay = y - fy;
  const int x0 = clampi((int)fx, w), x1 = clampi((int)fx + 1, w);
  const int y0 = clampi((int)fy, h), y1 = clampi((int)fy + 1, h);
  const float4 a00 = __ldg(t + y0 * w + x0), a10 = __ldg(t + y0 * w + x1);
  const float4 a01 = __ldg(t + y1 * w + x0), a11 = __ldg(t + y1 * w + x1);
  const float4 a = add4(mul4(a00, 1.0f - ax), mul4(a10, ax));
  const float4 b = add4(mul4(a01, 1.0f - ax), mul4(a11, ax));
  return add4(mul4(a, 1.0f - ay), mul4(b, ay));
}

__global__ void k_taa_resolve(const TaaParams p) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= p.w || y >= p.h) return;
  const int w = (int)p.w, h = (int)p.h;
  const size_t i = (size_t)y * p.w + x;
  const float4 cl = __ldg(p.cur_l + i), ct = __ldg(p.cur_t + i);
  const float bw = fminf(fmaxf(p.blend_weight, 0.0f), 1.0f);
  if (p.history_valid < 0.5f || bw >= 1.0f) {  // bootstrap: the current sample as is
    p.out_l[i] = cl;
    p.out_t[i] = ct;
    return;
  }
  // reproject_uv (cloud_taa.wgsl:84-110): view direction of this pixel,
  // projected with w = 0 (infinite depth) into the previous frame.  In FP64,
  // as the march's ray set-up: the direction is the near-plane point (0.1 m
  // ahead) minus the camera position, which cancels in FP32 and would move
  // the history sample by hundredths of a pixel.
  const double u = ((double)x + 0.5) / (double)w, v = ((double)y + 0.5) / (double)h;
  const double nx = u * 2.0 - 1.0, ny = 1.0 - v * 2.0;
  double nh[4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
    nh[r] = (((double)p.inv_vp[0][r] * nx + (double)p.inv_vp[1][r] * ny) + (double)p.inv_vp[2][r]) +
            (double)p.inv_vp[3][r];
  double d[3] = {nh[0] / nh[3] - (double)p.cam[0], nh[1] / nh[3] - (double)p.cam[1],
                 nh[2] / nh[3] - (double)p.cam[2]};
  const double il = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  d[0] *= il;
  d[1] *= il;
  d[2] *= il;
  double pc[4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
    pc[r] = ((double)p.prev_vp[0][r] * d[0] + (double)p.prev_vp[1][r] * d[1]) + (double)p.prev_vp[2][r] * d[2];
  float pu = 0.0f, pv = 0.0f, inside = 0.0f;
  if (pc[3] > 1e-4) {
    const double du = (pc[0] / pc[3]) * 0.5 + 0.5, dv = 1.0 - ((pc[1] / pc[3]) * 0.5 + 0.5);
    inside = (du >= 0.0 && dv >= 0.0 && du <= 1.0 && dv <= 1.0) ? 1.0f : 0.0f;
    pu = (float)du;
    pv = (float)dv;
  }
  float4 hl = bilinear_clamp(p.hist_l, w, h, pu, pv);
  float4 ht = bilinear_clamp(p.hist_t, w, h, pu, pv);
  // 3x3 neighbourhood AABB of the current frame (clamp_to_neighbourhood)
  float4 mnl = f4(1e10f), mxl = f4(-1e10f), mnt = f4(1e10f), mxt = f4(-1e10f);
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
    for (int dx = -1; dx <= 1; ++dx) {
      const int j = clampi((int)y + dy, h) * w + clampi((int)x + dx, w);
      const float4 sl = __ldg(p.cur_l + j), st = __ldg(p.cur_t + j);
      mnl = min4(mnl, sl);
      mxl = max4(mxl, sl);
      mnt = min4(mnt, st);
      mxt = max4(mxt, st);
    }
  hl = clamp4(hl, mnl, mxl);
  ht = clamp4(ht, mnt, mxt);
  const float eb = 1.0f * (1.0f - inside) + bw * inside;  // mix(1, w, inside)
  const float4 rl = add4(mul4(hl, 1.0f - eb), mul4(cl, eb));
  const float4 rt = add4(mul4(ht, 1.0f - eb), mul4(ct, eb));
  p.out_l[i] = max4(rl, f4(0.0f));
  p.out_t[i] = clamp4(rt, f4(0.0f), f4(1.0f));
}

// Catmull-Rom weights of one axis at fraction f in [0, 1).
__device__ __forceinline__ void cr_weights(float f, float w[4]) {
  w[0] = f * (-0.5f + f * (1.0f - 0.5f * f));
  w[1] = 1.0f + f * f * (-2.5f + 1.5f * f);
  w[2] = f * (0.5f + f * (2.0f - 1.5f * f));
  w[3] = f * f * (-0.5f + 0.5f * f);
}

// First Catmull-Rom tap + 1 of target pixel x (W wide) over an RT rw wide
// (the texel left of the sample point), and the fraction f in [0, 1), with
// every rounding explicit (no contraction into FMAs), so the two composite
// kernels and the tiled kernel's footprint bounds agree exactly.
__device__ __forceinline__ int cr_base(uint32_t x, uint32_t W, uint32_t rw, float& f) {
  const float sp = __fmul_rn(__fdiv_rn(__fadd_rn((float)x, 0.5f), (float)W), (float)rw);
  const float b = floorf(__fsub_rn(sp, 0.5f));
  f = __fsub_rn(sp, __fadd_rn(b, 0.5f));
  return (int)b;
}

__global__ void k_composite_halfres(const float4* __restrict__ l, const float4* __restrict__ t,
                                    uint32_t rw, uint32_t rh, float4* __restrict__ hdr, uint32_t W,
                                    uint32_t H) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  float fx, fy;
  const int bx = cr_base(x, W, rw, fx), by = cr_base(y, H, rh, fy);
  float wx[4], wy[4];
  cr_weights(fx, wx);
  cr_weights(fy, wy);
  int ix[4], iy[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    ix[k] = clampi(bx - 1 + k, (int)rw);
    iy[k] = clampi(by - 1 + k, (int)rh);
  }
  float4 sl = f4(0.0f), st = f4(0.0f);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float4 rl = f4(0.0f), rt = f4(0.0f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int idx = iy[j] * (int)rw + ix[k];
      rl = fma4(__ldg(l + idx), wx[k], rl);
      rt = fma4(__ldg(t + idx), wx[k], rt);
    }
    sl = fma4(rl, wy[j], sl);
    st = fma4(rt, wy[j], st);
  }
  const float4 L = max4(sl, f4(0.0f)), T = clamp4(st, f4(0.0f), f4(1.0f));
  const size_t o = (size_t)y * W + x;
  const float4 d = hdr[o];
  hdr[o] = make_float4(fmaf(d.x, T.x, L.x), fmaf(d.y, T.y, L.y), fmaf(d.z, T.z, L.z), fmaf(d.w, T.w, L.w));
}

constexpr int kCrTile = 24;  // RT texels per axis staged by one CTA

// k_composite_halfres with the RT footprint of the CTA's 16 x 16 target
// pixels staged once in shared memory: every RT texel is read from L2 about
// (footprint / 8)^2 = 2.25 times instead of 16 times per target pixel from
// L1.  Used while the RT is no larger than the target, where the footprint
// is at most 20 x 20 texels.  The same taps, weights and order as
// k_composite_halfres: the same image bit for bit.
__global__ void __launch_bounds__(256) k_composite_halfres_tiled(const float4* __restrict__ l,
                                                                 const float4* __restrict__ t, uint32_t rw,
                                                                 uint32_t rh, float4* __restrict__ hdr,
                                                                 uint32_t W, uint32_t H) {
  __shared__ float4 sl[kCrTile][kCrTile], st[kCrTile][kCrTile];
  const uint32_t x0 = blockIdx.x * 16u, y0 = blockIdx.y * 16u;
  float f;
  const int sx0 = cr_base(x0, W, rw, f) - 1, sy0 = cr_base(y0, H, rh, f) - 1;
  const int sx1 = cr_base(min(x0 + 15u, W - 1u), W, rw, f) + 2;
  const int sy1 = cr_base(min(y0 + 15u, H - 1u), H, rh, f) + 2;
  const int nx = min(sx1 - sx0 + 1, kCrTile), ny = min(sy1 - sy0 + 1, kCrTile);
  for (int i = (int)(threadIdx.y * 16u + threadIdx.x); i < nx * ny; i += 256) {
    const int jy = i / nx, jx = i - jy * nx;
    const int idx = clampi(sy0 + jy, (int)rh) * (int)rw + clampi(sx0 + jx, (int)rw);
    sl[jy][jx] = __ldg(l + idx);
    st[jy][jx] = __ldg(t + idx);
  }
  __syncthreads();
  const uint32_t x = x0 + threadIdx.x, y = y0 + threadIdx.y;
  if (x >= W || y >= H) return;
  float fx, fy;
  const int bx = cr_base(x, W, rw, fx), by = cr_base(y, H, rh, fy);
  float wx[4], wy[4];
  cr_weights(fx, wx);
  cr_weights(fy, wy);
  int jx[4], jy[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {  // tile slot (sx0 + j) holds RT texel clamp(sx0 + j)
    jx[k] = min(max(bx - 1 + k - sx0, 0), nx - 1);
    jy[k] = min(max(by - 1 + k - sy0, 0), ny - 1);
  }
  float4 acl = f4(0.0f), act = f4(0.0f);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    float4 rl = f4(0.0f), rt = f4(0.0f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      rl = fma4(sl[jy[j]][jx[k]], wx[k], rl);
      rt = fma4(st[jy[j]][jx[k]], wx[k], rt);
    }
    acl = fma4(rl, wy[j], acl);
    act = fma4(rt, wy[j], act);
  }
  const float4 L = max4(acl, f4(0.0f)), T = clamp4(act, f4(0.0f), f4(1.0f));
  const size_t o = (size_t)y * W + x;
  const float4 d = hdr[o];
  hdr[o] = make_float4(fmaf(d.x, T.x, L.x), fmaf(d.y, T.y, L.y), fmaf(d.z, T.z, L.z), fmaf(d.w, T.w, L.w));
}

dim3 grid16(uint32_t w, uint32_t h) { return dim3((w + 15u) / 16u, (h + 15u) / 16u); }

// Pixels whose composited image I = L + B T (B = bg, or 1 without one)
// differs from the reference's by more than `thr` relative, max over RGB;
// one atomic add per warp.
__global__ void k_count_rel_err(const float4* __restrict__ lr, const float4* __restrict__ tr,
                                const float4* __restrict__ l, const float4* __restrict__ t,
                                const float4* __restrict__ bg, uint32_t n, float thr,
                                unsigned int* __restrict__ count) {
  const uint32_t stride = gridDim.x * blockDim.x;
  uint32_t over = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const float4 b = bg ? __ldg(bg + i) : f4(1.0f);
    const float4 a = __ldg(lr + i), at = __ldg(tr + i), c = __ldg(l + i), ct = __ldg(t + i);
    const float r0 = fmaf(b.x, at.x, a.x), r1 = fmaf(b.y, at.y, a.y), r2 = fmaf(b.z, at.z, a.z);
    const float d0 = fabsf(fmaf(b.x, ct.x, c.x) - r0), d1 = fabsf(fmaf(b.y, ct.y, c.y) - r1),
                d2 = fabsf(fmaf(b.z, ct.z, c.z) - r2);
    const bool bad = d0 > thr * fabsf(r0) || d1 > thr * fabsf(r1) || d2 > thr * fabsf(r2) ||
                     !(d0 == d0 && d1 == d1 && d2 == d2);
    over += bad ? 1u : 0u;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) over += __shfl_xor_sync(0xffffffffu, over, o);
  if ((threadIdx.x & 31u) == 0 && over) atomicAdd(count, over);
}

}  // namespace

int launch_depth_halfres(const float* depth, uint32_t W, uint32_t H, float* out, uint32_t rw,
                         uint32_t rh, cudaStream_t s) {
  k_depth_halfres<<<grid16(rw, rh), dim3(16, 16), 0, s>>>(depth, W, H, out, rw, rh);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_taa_resolve(const TaaParams& p, cudaStream_t s) {
  k_taa_resolve<<<grid16(p.w, p.h), dim3(16, 16), 0, s>>>(p);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_composite_halfres(const float4* l, const float4* t, uint32_t rw, uint32_t rh, float4* hdr,
                             uint32_t W, uint32_t H, cudaStream_t s) {
  if (W == 0 || H == 0 || rw == 0 || rh == 0) return PSC_OK;
  if (rw <= W && rh <= H)
    k_composite_halfres_tiled<<<grid16(W, H), dim3(16, 16), 0, s>>>(l, t, rw, rh, hdr, W, H);
  else
    k_composite_halfres<<<grid16(W, H), dim3(16, 16), 0, s>>>(l, t, rw, rh, hdr, W, H);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_count_rel_err(const float4* lr, const float4* tr, const float4* l, const float4* t, const float4* bg,
                         uint32_t n, float thr, unsigned int* count, cudaStream_t s) {
  if (n == 0) return PSC_OK;
  const uint32_t blocks = std::min((n + 255u) / 256u, 148u * 8u);
  k_count_rel_err<<<blocks, 256, 0, s>>>(lr, tr, l, t, bg, n, thr, count);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

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
// clamped into its image.  Whenever the RT is at most half the target per
// axis (the half-res RT), the composite runs a 2x2 quad of target pixels per
// thread from one 5x5 RT window (k_composite_halfres_quad).
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
// kernels agree exactly.
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

// The Catmull-Rom sums of one RT array for a 2x2 quad of target pixels
// (k_composite_halfres_quad): rows r = 0..4 of the 5x5 window starting at
// texel (col[0], by0 - 1), each row's horizontal sums serving both pixel
// rows; a<y><x> receive the quad's four sums.
__device__ __forceinline__ void cr_quad_sums(const float4* __restrict__ src, const int col[5], int by0,
                                             uint32_t rw, uint32_t rh, bool dx, bool dy, const float wx0[4],
                                             const float wx1[4], const float wy0[4], const float wy1[4],
                                             float4& a00, float4& a01, float4& a10, float4& a11) {
  a00 = a01 = a10 = a11 = f4(0.0f);
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    const int row = clampi(by0 - 1 + r, (int)rh) * (int)rw;
    float4 cv[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) cv[c] = __ldg(src + row + col[c]);
    float4 h0 = f4(0.0f), h1 = f4(0.0f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      h0 = fma4(cv[k], wx0[k], h0);
      h1 = fma4(dx ? cv[k + 1] : cv[k], wx1[k], h1);
    }
    if (r < 4) {  // row r is tap row r of the upper pixels
      a00 = fma4(h0, wy0[r], a00);
      a01 = fma4(h1, wy0[r], a01);
    }
    // and tap row r - dy of the lower ones
    if (dy ? r >= 1 : r < 4) {
      const float wl = dy ? wy1[r >= 1 ? r - 1 : 0] : wy1[r < 4 ? r : 3];
      a10 = fma4(h0, wl, a10);
      a11 = fma4(h1, wl, a11);
    }
  }
}

// k_composite_halfres for a 2x2 quad of target pixels per thread, while the
// RT is at most half the target per axis: the quad's taps then lie in one
// 5x5 window of RT texels (neighbouring pixels' first taps differ by at most
// one), read once per thread a row at a time, the luminance window and then
// the transmittance window (so one array's row is live at a time).  Each
// row's horizontal 4-tap sums serve both pixel rows of the quad, so a pixel
// costs 12.5 RT loads instead of 32.  Every pixel sums the same taps with
// the same weights in the same order as k_composite_halfres: the same image
// bit for bit.
__global__ void __launch_bounds__(256) k_composite_halfres_quad(const float4* __restrict__ l,
                                                                const float4* __restrict__ t, uint32_t rw,
                                                                uint32_t rh, float4* __restrict__ hdr,
                                                                uint32_t W, uint32_t H) {
  const uint32_t x0 = 2u * (blockIdx.x * blockDim.x + threadIdx.x);
  const uint32_t y0 = 2u * (blockIdx.y * blockDim.y + threadIdx.y);
  if (x0 >= W || y0 >= H) return;
  const uint32_t x1 = min(x0 + 1u, W - 1u), y1 = min(y0 + 1u, H - 1u);
  float fx0, fx1, fy0, fy1;
  const int bx0 = cr_base(x0, W, rw, fx0), bx1 = cr_base(x1, W, rw, fx1);
  const int by0 = cr_base(y0, H, rh, fy0), by1 = cr_base(y1, H, rh, fy1);
  const bool dx = bx1 != bx0, dy = by1 != by0;  // 0 or 1 texel further on
  float wx0[4], wx1[4], wy0[4], wy1[4];
  cr_weights(fx0, wx0);
  cr_weights(fx1, wx1);
  cr_weights(fy0, wy0);
  cr_weights(fy1, wy1);
  int col[5];
#pragma unroll
  for (int c = 0; c < 5; ++c) col[c] = clampi(bx0 - 1 + c, (int)rw);
  float4 a00l, a01l, a10l, a11l, a00t, a01t, a10t, a11t;  // a<y><x>
  cr_quad_sums(l, col, by0, rw, rh, dx, dy, wx0, wx1, wy0, wy1, a00l, a01l, a10l, a11l);
  cr_quad_sums(t, col, by0, rw, rh, dx, dy, wx0, wx1, wy0, wy1, a00t, a01t, a10t, a11t);
  auto put = [&](uint32_t x, uint32_t y, float4 sl, float4 st) {
    const float4 L = max4(sl, f4(0.0f)), T = clamp4(st, f4(0.0f), f4(1.0f));
    const size_t o = (size_t)y * W + x;
    const float4 d = hdr[o];
    hdr[o] = make_float4(fmaf(d.x, T.x, L.x), fmaf(d.y, T.y, L.y), fmaf(d.z, T.z, L.z), fmaf(d.w, T.w, L.w));
  };
  put(x0, y0, a00l, a00t);
  if (x0 + 1u < W) put(x0 + 1u, y0, a01l, a01t);
  if (y0 + 1u < H) {
    put(x0, y0 + 1u, a10l, a10t);
    if (x0 + 1u < W) put(x0 + 1u, y0 + 1u, a11l, a11t);
  }
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
  if (2u * rw <= W && 2u * rh <= H)  // the half-res RT: quads' first taps differ by at most one
    k_composite_halfres_quad<<<grid16((W + 1u) / 2u, (H + 1u) / 2u), dim3(16, 16), 0, s>>>(l, t, rw, rh, hdr,
                                                                                         W, H);
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

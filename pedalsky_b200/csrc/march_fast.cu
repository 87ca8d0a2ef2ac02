// Single-view FAST march kernel: one thread per ray, CTA tile 16x8 pixels,
// warps as 8x4 pixel tiles, 8 CTAs per SM for the lean form (64 registers:
// more resident warps hide more fetch latency than the few spilled values
// cost) and 7 for the full form (72 registers: its extra paths spill more,
// and 7 CTAs measured 2.3 % faster on the Cumulonimbus frames).  The per-ray
// body is march_fast_body.cuh.
#include <cuda_runtime.h>
#include <stdint.h>

#include "march_fast_body.cuh"

namespace psc {
namespace {

constexpr int kTileW = 16;
constexpr int kTileH = 8;
constexpr int kThreads = 128;

// Shared memory per CTA: the entry/exit distances of each of the view's
// layers and kAuxWords more words, per thread (dynamic, sized at launch).
template <int ST, int FILT, bool FULL, int LB>
__global__ void __launch_bounds__(kThreads, FULL ? 7 : 8) k_march_fast(const __grid_constant__ MarchUniforms u,
                                                            const __grid_constant__ ViewDev v) {
  extern __shared__ float s_dyn[];
  const uint32_t nl = u.layer_count;
  float* const s_t0 = s_dyn;
  float* const s_t1 = s_dyn + nl * kThreads;
  float* const s_aux = s_dyn + 2u * nl * kThreads;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * kTileW + (warp & 1u) * 8u + (lane & 7u);
  const uint32_t py = blockIdx.y * kTileH + (warp >> 1) * 4u + (lane >> 3);
  if (px >= v.width || py >= v.height) return;
  march_pixel_fast<ST, FILT, FULL, false, LB>(u, v, px, py, s_t0, s_t1, s_aux, kThreads, threadIdx.x);
}

// The instrumented build of the same kernel (psc_count_fetches): every
// thread counts the fetches its ray issues, and each warp adds its sums to
// `out` (kTallyKinds 64-bit counters).  Not a timed kernel.
template <int ST, int FILT, bool FULL>
__global__ void __launch_bounds__(kThreads) k_march_fast_tally(const __grid_constant__ MarchUniforms u,
                                                               const __grid_constant__ ViewDev v,
                                                               unsigned long long* out) {
  extern __shared__ float s_dyn[];
  const uint32_t nl = u.layer_count;
  float* const s_t0 = s_dyn;
  float* const s_t1 = s_dyn + nl * kThreads;
  float* const s_aux = s_dyn + 2u * nl * kThreads;
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t px = blockIdx.x * kTileW + (warp & 1u) * 8u + (lane & 7u);
  const uint32_t py = blockIdx.y * kTileH + (warp >> 1) * 4u + (lane >> 3);
  uint32_t tc[kTallyKinds];
#pragma unroll
  for (uint32_t k = 0; k < kTallyKinds; ++k) tc[k] = 0u;
  if (px < v.width && py < v.height)
    march_pixel_fast<ST, FILT, FULL, true>(u, v, px, py, s_t0, s_t1, s_aux, kThreads, threadIdx.x, tc);
#pragma unroll
  for (uint32_t k = 0; k < kTallyKinds; ++k) {
    const uint32_t sum = __reduce_add_sync(0xffffffffu, tc[k]);
    if (lane == 0 && sum) atomicAdd(out + k, (unsigned long long)sum);
  }
}

template <int ST, int FILT>
cudaError_t launch_fast_tally(const MarchUniforms& u, const ViewDev& v, unsigned long long* out,
                              cudaStream_t s) {
  const dim3 grid((v.width + kTileW - 1) / kTileW, (v.height + kTileH - 1) / kTileH);
  const size_t smem = (2u * u.layer_count + kAuxWords) * kThreads * sizeof(float);
  if (needs_full_paths(&u, 1))
    k_march_fast_tally<ST, FILT, true><<<grid, kThreads, smem, s>>>(u, v, out);
  else
    k_march_fast_tally<ST, FILT, false><<<grid, kThreads, smem, s>>>(u, v, out);
  return cudaGetLastError();
}

template <int ST, int FILT, int LB = 0>
cudaError_t launch_fast(const MarchUniforms& u, const ViewDev& v, cudaStream_t s) {
  const dim3 grid((v.width + kTileW - 1) / kTileW, (v.height + kTileH - 1) / kTileH);
  const size_t smem = (2u * u.layer_count + kAuxWords) * kThreads * sizeof(float);
  if (needs_full_paths(&u, 1))
    k_march_fast<ST, FILT, true, LB><<<grid, kThreads, smem, s>>>(u, v);
  else
    k_march_fast<ST, FILT, false, LB><<<grid, kThreads, smem, s>>>(u, v);
  return cudaGetLastError();
}

}  // namespace

int launch_march_fast_tally(const MarchUniforms& u, const ViewDev& v, const PscMarchOptions& o,
                            unsigned long long* counts, cudaStream_t s) {
  if (u.octaves > (uint32_t)kMaxOct || u.octaves == 0) return PSC_ERR_UNSUPPORTED;
  cudaError_t e;
  if (o.storage == PSC_STORAGE_F16 && o.filter == PSC_FILTER_HYBRID)
    e = launch_fast_tally<PSC_STORAGE_F16, PSC_FILTER_HYBRID>(u, v, counts, s);
  else if (o.storage == PSC_STORAGE_F16 && o.filter == PSC_FILTER_EXACT)
    e = launch_fast_tally<PSC_STORAGE_F16, PSC_FILTER_EXACT>(u, v, counts, s);
  else if (o.storage == PSC_STORAGE_U8 && o.filter == PSC_FILTER_HYBRID)
    e = launch_fast_tally<PSC_STORAGE_U8, PSC_FILTER_HYBRID>(u, v, counts, s);
  else if (o.storage == PSC_STORAGE_U8 && o.filter == PSC_FILTER_EXACT)
    e = launch_fast_tally<PSC_STORAGE_U8, PSC_FILTER_EXACT>(u, v, counts, s);
  else
    return PSC_ERR_UNSUPPORTED;
  return e == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

int launch_march_fast(const MarchUniforms& u, const ViewDev& v, const PscMarchOptions& o,
                      cudaStream_t s) {
  if (u.octaves > (uint32_t)kMaxOct || u.octaves == 0) return PSC_ERR_UNSUPPORTED;
  cudaError_t e = cudaErrorInvalidValue;
  if (o.filter == PSC_FILTER_TEXTURE) {
    if (o.storage == PSC_STORAGE_U8) e = launch_fast<PSC_STORAGE_U8, PSC_FILTER_TEXTURE>(u, v, s);
    else if (o.storage == PSC_STORAGE_F16) e = launch_fast<PSC_STORAGE_F16, PSC_FILTER_TEXTURE>(u, v, s);
    else return PSC_ERR_UNSUPPORTED;
  } else if (o.filter == PSC_FILTER_HYBRID) {
    // the light-march fetch batch is chosen for the F16 hybrid form only
    if (o.storage == PSC_STORAGE_U8) e = launch_fast<PSC_STORAGE_U8, PSC_FILTER_HYBRID>(u, v, s);
    else if (o.storage == PSC_STORAGE_F16 && o.light_batch == 2)
      e = launch_fast<PSC_STORAGE_F16, PSC_FILTER_HYBRID, 2>(u, v, s);
    else if (o.storage == PSC_STORAGE_F16 && o.light_batch == 3)
      e = launch_fast<PSC_STORAGE_F16, PSC_FILTER_HYBRID, 3>(u, v, s);
    else if (o.storage == PSC_STORAGE_F16) e = launch_fast<PSC_STORAGE_F16, PSC_FILTER_HYBRID>(u, v, s);
    else return PSC_ERR_UNSUPPORTED;
  } else {
    switch (o.storage) {
      case PSC_STORAGE_U8: e = launch_fast<PSC_STORAGE_U8, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_F32: e = launch_fast<PSC_STORAGE_F32, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_F16: e = launch_fast<PSC_STORAGE_F16, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_BF16: e = launch_fast<PSC_STORAGE_BF16, PSC_FILTER_EXACT>(u, v, s); break;
      case PSC_STORAGE_FP8: e = launch_fast<PSC_STORAGE_FP8, PSC_FILTER_EXACT>(u, v, s); break;
      default: return PSC_ERR_INVALID_ARGUMENT;
    }
  }
  return e == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

}  // namespace psc

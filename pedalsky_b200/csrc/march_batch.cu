// Persistent batched march: many views of uneven size, each with its own
// scene (layers, steps, camera, sun, sky-view/AP LUTs), in one launch.
//
// The grid is sized to the SMs' resident capacity (persistent CTAs).  Work
// items are pixel tiles listed by the host in descending estimated cost
// (primary steps x layers) so the expensive views start first and the tail
// is short; each CTA takes the next tile from an atomic counter, copies that
// view's uniform block into shared memory when the view changes, and marches
// the tile with the same per-ray body as the single-view FAST kernel.  There
// is no inter-CTA waiting: a CTA that finds the counter past the end exits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "march_fast_body.cuh"

namespace psc {
namespace {

// Tile word: view (8 bits) | tile column (12 bits) | tile row (12 bits).
__device__ __forceinline__ void unpack_tile(uint32_t w, uint32_t& view, uint32_t& tx, uint32_t& ty) {
  view = w >> 24;
  tx = (w >> 12) & 0xfffu;
  ty = w & 0xfffu;
}

// 768 threads per SM (6 CTAs of 128): the shared-memory uniform block turns
// every uniform operand into a register, and 80 registers per thread remove
// nearly all spills (measured: 8 CTAs/SM 5.80 ms, 7 5.50, 6 5.35 on a 1080p
// view; 64 uneven views 224.9 -> 209.4 ms).  FULL = false: every view of the
// batch runs the lean form.  FULL = true: each view runs the form it needs
// (needs_full_paths on its uniform block), so the views of a mixed batch that
// need no full-form path still get the lean one (64 uneven views 209.5 ->
// 194.2 ms).
template <int ST, int FILT, int NT, bool FULL, int LB>
__global__ void __launch_bounds__(NT, 768 / NT)
    k_march_batch(const MarchUniforms* __restrict__ views_u, const ViewDev* __restrict__ views_v,
                  const uint32_t* __restrict__ tiles, uint32_t n_tiles, uint32_t* __restrict__ counter,
                  uint32_t tile_w) {
  __shared__ MarchUniforms su;
  __shared__ ViewDev sv;
  __shared__ uint32_t s_tile;
  __shared__ float s_t0[8 * NT], s_t1[8 * NT], s_aux[kAuxWords * NT];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t warps_x = tile_w >> 3;  // 8x4-pixel warp tiles per tile row
  uint32_t cur = 0xffffffffu;
  bool vfull = FULL, changed = false;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    if (t >= n_tiles) break;  // the same value in every thread of the CTA
    uint32_t view, tx, ty;
    unpack_tile(__ldg(tiles + t), view, tx, ty);
    if (view != cur) {
      const uint4* src = reinterpret_cast<const uint4*>(views_u + view);
      uint4* dst = reinterpret_cast<uint4*>(&su);
      for (uint32_t i = threadIdx.x; i < sizeof(MarchUniforms) / 16; i += NT) dst[i] = __ldg(src + i);
      if (threadIdx.x == 0) sv = views_v[view];
      cur = view;
      changed = true;
    }
    __syncthreads();
    if (FULL && changed) vfull = needs_full_paths(&su, 1);  // this view's form
    changed = false;
    const uint32_t tile_h = (NT / 32 / warps_x) * 4u;
    const uint32_t px = tx * tile_w + (warp % warps_x) * 8u + (lane & 7u);
    const uint32_t py = ty * tile_h + (warp / warps_x) * 4u + (lane >> 3);
    if (px < sv.width && py < sv.height) {
      if (FULL && vfull)
        march_pixel_fast<ST, FILT, true, false, LB>(su, sv, px, py, s_t0, s_t1, s_aux, NT, threadIdx.x);
      else
        march_pixel_fast<ST, FILT, false, false, LB>(su, sv, px, py, s_t0, s_t1, s_aux, NT, threadIdx.x);
    }
    __syncthreads();  // su, sv and s_tile are rewritten by the next iteration
  }
}

template <int ST, int FILT, int NT, bool FULL, int LB>
int launch_batch_full(const MarchUniforms* u, const ViewDev* v, const uint32_t* tiles, uint32_t n_tiles,
                    uint32_t* counter, uint32_t tile_w, int sms, cudaStream_t s) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_march_batch<ST, FILT, NT, FULL, LB>, NT, 0) !=
      cudaSuccess)
    return PSC_ERR_CUDA;
  per_sm = per_sm < 1 ? 1 : per_sm;
  uint32_t grid = (uint32_t)(sms * per_sm);
  if (grid > n_tiles) grid = n_tiles ? n_tiles : 1;
  k_march_batch<ST, FILT, NT, FULL, LB><<<grid, NT, 0, s>>>(u, v, tiles, n_tiles, counter, tile_w);
  return cudaGetLastError() == cudaSuccess ? PSC_OK : PSC_ERR_CUDA;
}

template <int ST, int FILT, int NT, int LB>
int launch_batch_t(const MarchUniforms* u, const ViewDev* v, const uint32_t* tiles, uint32_t n_tiles,
                   uint32_t* counter, uint32_t tile_w, int sms, bool full, cudaStream_t s) {
  return full ? launch_batch_full<ST, FILT, NT, true, LB>(u, v, tiles, n_tiles, counter, tile_w, sms, s)
            : launch_batch_full<ST, FILT, NT, false, LB>(u, v, tiles, n_tiles, counter, tile_w, sms, s);
}

template <int ST, int FILT, int LB = 0>
int launch_batch_nt(int nt, const MarchUniforms* u, const ViewDev* v, const uint32_t* tiles,
                    uint32_t n_tiles, uint32_t* counter, uint32_t tile_w, int sms, bool full,
                    cudaStream_t s) {
  switch (nt) {
    case 64: return launch_batch_t<ST, FILT, 64, LB>(u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    case 128: return launch_batch_t<ST, FILT, 128, LB>(u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    case 256: return launch_batch_t<ST, FILT, 256, LB>(u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    default: return PSC_ERR_INVALID_ARGUMENT;
  }
}

}  // namespace

int launch_march_batch(const PscMarchOptions& o, int threads, uint32_t tile_w,
                       const MarchUniforms* u, const ViewDev* v, const uint32_t* tiles,
                       uint32_t n_tiles, uint32_t* counter, int sms, bool full, cudaStream_t s) {
  if (o.filter == PSC_FILTER_HYBRID) {
    // the light-march fetch batch is chosen for the F16 hybrid form only
    if (o.storage == PSC_STORAGE_F16 && o.light_batch == 2)
      return launch_batch_nt<PSC_STORAGE_F16, PSC_FILTER_HYBRID, 2>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    if (o.storage == PSC_STORAGE_F16 && o.light_batch == 3)
      return launch_batch_nt<PSC_STORAGE_F16, PSC_FILTER_HYBRID, 3>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    if (o.storage == PSC_STORAGE_F16)
      return launch_batch_nt<PSC_STORAGE_F16, PSC_FILTER_HYBRID>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    if (o.storage == PSC_STORAGE_U8)
      return launch_batch_nt<PSC_STORAGE_U8, PSC_FILTER_HYBRID>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
  } else if (o.filter == PSC_FILTER_EXACT) {
    if (o.storage == PSC_STORAGE_F16)
      return launch_batch_nt<PSC_STORAGE_F16, PSC_FILTER_EXACT>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    if (o.storage == PSC_STORAGE_U8)
      return launch_batch_nt<PSC_STORAGE_U8, PSC_FILTER_EXACT>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
    if (o.storage == PSC_STORAGE_F32)
      return launch_batch_nt<PSC_STORAGE_F32, PSC_FILTER_EXACT>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
  } else if (o.filter == PSC_FILTER_TEXTURE) {
    if (o.storage == PSC_STORAGE_U8)
      return launch_batch_nt<PSC_STORAGE_U8, PSC_FILTER_TEXTURE>(threads, u, v, tiles, n_tiles, counter, tile_w, sms, full, s);
  }
  return PSC_ERR_UNSUPPORTED;
}

}  // namespace psc

// Allocation-free entry point for the persistent batched march.
//
// psc_render_batch keeps its work list (tile counter, cost-sorted tile
// words, per-view uniform blocks, view and frame records) in device buffers
// that the context allocates and grows on demand, staged through pinned host
// buffers.  Some callers cannot allow an allocation at render time:
// allocation and free calls can synchronise the device and stall a real-time
// frame loop, a caller that hands this library a fixed memory budget at
// start-up (an engine with its own pool, an embedded renderer) must not see
// device memory grow behind its back, and code running in a host callback
// may not call the CUDA allocator at all.  psc_render_batch_noalloc serves
// them: the work list lives in one file-scope __device__ array of fixed size,
// reserved once per GPU when the library's module loads and held until the
// process exits; the host staging is a file-scope host array.  Inputs,
// outputs and the per-view sky-view / aerial-perspective LUT buffers are the
// caller's.  The kernel is the same persistent march as psc_render_batch's.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "psc_ctx.h"

namespace {

using psc::host::fail;

constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

constexpr uint32_t kMaxViews = PSC_NOALLOC_MAX_VIEWS;
constexpr uint32_t kMaxTiles = PSC_NOALLOC_MAX_TILES;
constexpr size_t kFrameSlot = 128;  // >= the LUT bakes' per-view frame record (checked per call)

// Scratch layout (byte offsets, each region 256-byte aligned).
constexpr size_t kOffCounter = 0;
constexpr size_t kOffUniforms = align_up(kOffCounter + sizeof(uint32_t));
constexpr size_t kOffViews = align_up(kOffUniforms + kMaxViews * sizeof(psc::MarchUniforms));
constexpr size_t kOffFrames = align_up(kOffViews + kMaxViews * sizeof(psc::ViewDev));
constexpr size_t kOffTiles = align_up(kOffFrames + kMaxViews * kFrameSlot);
constexpr size_t kScratchBytes = align_up(kOffTiles + (size_t)kMaxTiles * sizeof(uint32_t));
static_assert(kScratchBytes <= (size_t)5 << 20, "scratch stays a few MiB per GPU");

// The device copy of the work list.  In host code this name is only a
// host-side stand-in for the symbol, not a device address: host code passes
// the address cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_batch_scratch[kScratchBytes];

// Host staging for the same records.  A pageable H2D cudaMemcpyAsync
// returns once the source bytes have been taken, so the next call may
// overwrite these.
struct HostStaging {
  psc::MarchUniforms u[kMaxViews];
  psc::ViewDev v[kMaxViews];
  alignas(16) unsigned char frames[kMaxViews * kFrameSlot];
  uint32_t tiles[kMaxTiles];
};
HostStaging g_host;

constexpr int kMaxDevices = 64;
unsigned char* g_scratch_dev[kMaxDevices];  // per-device address of g_batch_scratch
std::mutex g_mutex;                         // serialises host staging across threads

// Device address of the scratch array on `device`, which must be current.
// Resolved once per device; the first lookup also loads this library's
// module on that device if it is not loaded yet.  The address stays valid
// for the life of the device's primary context: a cudaDeviceReset while the
// library is in use would leave it stale, so callers must not reset a
// device they render on with this entry point.
int scratch_on(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices)
    return fail(PSC_ERR_INVALID_ARGUMENT, "device %d beyond the allocation-free path's %d devices", device,
                kMaxDevices);
  if (!g_scratch_dev[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_batch_scratch);
    if (e != cudaSuccess || !p) return psc::host::cuda_fail(e, "cudaGetSymbolAddress(batch scratch)");
    g_scratch_dev[device] = static_cast<unsigned char*>(p);
  }
  *out = g_scratch_dev[device];
  return PSC_OK;
}

}  // namespace

extern "C" int psc_render_batch_noalloc(psc_ctx* c, const PscBatchView* views, uint32_t n,
                                        float* sky_luts, float* ap_luts, void* stream) {
  if (!c || (n && !views)) return fail(PSC_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) return PSC_OK;
  if (n > kMaxViews)
    return fail(PSC_ERR_INVALID_ARGUMENT, "%u views exceeds the allocation-free limit of %u", n, kMaxViews);
  if (!sky_luts || !ap_luts) return fail(PSC_ERR_INVALID_ARGUMENT, "null per-view LUT buffer");
  if (reinterpret_cast<uintptr_t>(sky_luts) % 16 || reinterpret_cast<uintptr_t>(ap_luts) % 16)
    return fail(PSC_ERR_INVALID_ARGUMENT, "per-view LUT buffers must be 16-byte aligned");
  int rc = psc::host::validate_batch(c, views, n);
  if (rc) return rc;
  const uint64_t need = psc::host::count_batch_tiles(views, n, c->batch_tuning);
  if (need == UINT64_MAX)
    return fail(PSC_ERR_INVALID_ARGUMENT, "a view has more than 4096 tiles along one axis");
  if (need > kMaxTiles)
    return fail(PSC_ERR_INVALID_ARGUMENT,
                "batch needs %llu tiles of %ux%u pixels; the allocation-free limit is %u tiles "
                "(split the batch or use psc_render_batch)",
                (unsigned long long)need, c->batch_tuning.tile_w,
                (c->batch_tuning.threads / 32 / (c->batch_tuning.tile_w / 8)) * 4, kMaxTiles);
  const size_t fl = psc::frame_lite_size();
  if (fl > kFrameSlot) return fail(PSC_ERR_UNSUPPORTED, "frame record of %zu bytes exceeds its slot", fl);
  rc = psc::host::ensure_device(c);
  if (rc) return rc;
  // The work list is staged through host arrays that every call reuses, so
  // a graph recorded from this call would replay whatever the latest call
  // staged, not the views it was recorded with: a capturing stream is
  // refused before anything is enqueued on it.
  {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    const cudaError_t e = cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap);
    if (e != cudaSuccess) return psc::host::cuda_fail(e, "cudaStreamIsCapturing");
    if (cap != cudaStreamCaptureStatusNone)
      return fail(PSC_ERR_UNSUPPORTED,
                  "the allocation-free batch cannot be recorded into a CUDA graph (its staging is "
                  "shared by all calls); use psc_render_batch with use_graph = 1");
  }
  if (!psc::host::storage_ready(c))
    return fail(PSC_ERR_MISSING_INPUT,
                "noise storage for the current options is not built; render once with psc_render or "
                "psc_render_batch after setting inputs and options (those calls allocate it)");
  if (!c->sms) {
    const cudaError_t e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
    if (e != cudaSuccess) return psc::host::cuda_fail(e, "SM count");
  }

  std::lock_guard<std::mutex> lock(g_mutex);
  unsigned char* scratch = nullptr;
  rc = scratch_on(c->device, &scratch);
  if (rc) return rc;
  float4* sky = reinterpret_cast<float4*>(sky_luts);
  float4* ap = reinterpret_cast<float4*>(ap_luts);
  uint32_t n_tiles = 0;
  rc = psc::host::fill_batch(c, views, n, c->batch_tuning, g_host.u, g_host.v, g_host.frames, g_host.tiles,
                             kMaxTiles, sky, ap, &n_tiles);
  if (rc) return rc;

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto* d_counter = reinterpret_cast<uint32_t*>(scratch + kOffCounter);
  auto* d_u = reinterpret_cast<psc::MarchUniforms*>(scratch + kOffUniforms);
  auto* d_v = reinterpret_cast<psc::ViewDev*>(scratch + kOffViews);
  void* d_frames = scratch + kOffFrames;
  auto* d_tiles = reinterpret_cast<uint32_t*>(scratch + kOffTiles);
  const struct {
    void* dst;
    const void* src;
    size_t bytes;
    const char* what;
  } copies[] = {{d_u, g_host.u, n * sizeof(psc::MarchUniforms), "batch uniforms H2D"},
                {d_v, g_host.v, n * sizeof(psc::ViewDev), "batch views H2D"},
                {d_frames, g_host.frames, n * fl, "batch frames H2D"},
                {d_tiles, g_host.tiles, n_tiles * sizeof(uint32_t), "batch tiles H2D"}};
  for (const auto& cp : copies) {
    const cudaError_t e = cudaMemcpyAsync(cp.dst, cp.src, cp.bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return psc::host::cuda_fail(e, cp.what);
  }
  if (psc::launch_view_lut_bakes(c->world, d_frames, n, c->d_lut_h[PSC_LUT_TRANSMITTANCE],
                                 c->d_lut_h[PSC_LUT_MULTISCATTER], sky, ap, s))
    return fail(PSC_ERR_CUDA, "per-view LUT bake launch failed");
  // The array keeps the previous call's contents: the work counter must
  // start at zero.
  const cudaError_t e = cudaMemsetAsync(d_counter, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess) return psc::host::cuda_fail(e, "batch counter reset");
  rc = psc::launch_march_batch(c->opts, (int)c->batch_tuning.threads, c->batch_tuning.tile_w, d_u, d_v,
                               d_tiles, n_tiles, d_counter, c->sms, psc::needs_full_paths(g_host.u, n), s);
  if (rc == PSC_ERR_UNSUPPORTED)
    return fail(rc, "batched march supports F16/U8/F32 exact, F16/U8 hybrid and U8 texture storage");
  if (rc) return fail(rc, "batched march launch failed: %s", cudaGetErrorString(cudaGetLastError()));
  ++c->launches;
  return PSC_OK;
}

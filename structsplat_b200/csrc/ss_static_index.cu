// Tile index build that allocates nothing: its scratch lives in a device array compiled into
// this library.
//
// Who needs it: callers that cannot allocate device memory when they build the index.  A host
// application that hands every byte of device memory to its own pool up front and forbids
// allocation inside its frame loop; a plugin that runs inside another framework and may only
// use the buffers it was given; code that must not call cudaMalloc because the implicit device
// synchronisation would stall other work on the GPU.  ss_build_tile_index needs a caller-sized
// workspace (packed records, per-tile counters, int64 offsets and the scan's temporary storage);
// ss_build_tile_index_static keeps all of that in g_static_scratch instead, so the caller passes
// only its inputs and the two outputs.
//
// Limits: at most kStaticMaxGaussians Gaussians and kStaticMaxTiles tiles per call, checked
// before any work is queued.  The array (kStaticScratchBytes, a little over 5 MiB) is held on
// every GPU that loads the library, for the life of the process.
//
// Sharing: every call uses the same array and leaves the previous call's contents in it.  The
// per-tile counters are cleared by every call before use; the other regions are fully rewritten.
// Two calls whose work overlaps on the GPU (different streams, or different host threads using
// one device) race on the array and corrupt each other's index: serialise them.
//
// Set-up: the first call on each device, with that device current, resolves the array's device
// address with cudaGetSymbolAddress (and checks it).  That first call on a device should come
// before any stream capture on that device.
#include <mutex>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int64_t kStaticMaxGaussians = 65536;
constexpr int64_t kStaticMaxTiles = 16384;
constexpr size_t kRecordBytes = kStaticMaxGaussians * sizeof(Splat);  // 4 MiB
constexpr size_t kIndexBytes = 1u << 20;                              // 1 MiB
constexpr size_t kStaticScratchBytes = kRecordBytes + kIndexBytes;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_static_scratch on the current device (resolved once per device).
int scratch_for_current_device(void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices)
    return fail(SS_ERR_UNSUPPORTED, "device %d beyond the static scratch table", dev);
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return fail(SS_ERR_CUDA, "cudaGetSymbolAddress(static scratch): %s",
                  cudaGetErrorString(e));
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return SS_OK;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_build_tile_index_static(const float* means, const float* conics, const int64_t* radii,
                               int64_t n, int height, int width, int tile_size,
                               int ellipse_cull, float sigma_cutoff, int32_t* tile_gids,
                               int64_t gid_capacity, int32_t* tile_offsets, uint32_t* status,
                               ss_stream_t stream) {
  if (n < 0 || height < 0 || width < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (tile_size <= 0 || tile_size > 32)  // tile_size^2 <= 1024, without overflow
    return fail(SS_ERR_INVALID_ARGUMENT, "tile_size must be positive with tile_size^2 <= 1024");
  if (n > kStaticMaxGaussians)
    return fail(SS_ERR_CAPACITY, "static tile index takes at most %lld Gaussians, got %lld",
                (long long)kStaticMaxGaussians, (long long)n);
  // in int64: width or height near INT_MAX must not overflow before the limit check
  const int64_t tiles = (((int64_t)width + tile_size - 1) / tile_size) *
                        (((int64_t)height + tile_size - 1) / tile_size);
  if (tiles > kStaticMaxTiles)
    return fail(SS_ERR_CAPACITY, "static tile index takes at most %lld tiles, got %lld",
                (long long)kStaticMaxTiles, (long long)tiles);
  size_t index_bytes = 0;
  int rc = ss_tile_index_workspace_bytes(n, height, width, tile_size, &index_bytes);
  if (rc) return rc;
  if (index_bytes > kIndexBytes)
    return fail(SS_ERR_CAPACITY, "static tile index scratch too small (%zu > %zu bytes)",
                index_bytes, kIndexBytes);
  void* scratch = nullptr;
  if ((rc = scratch_for_current_device(&scratch))) return rc;
  void* records = scratch;
  void* index_ws = static_cast<char*>(scratch) + kRecordBytes;
  // The conic stands in for the colours: binning reads only means, conics and rectangles.
  if (n > 0 && (rc = ss_pack_splats(means, conics, conics, radii, nullptr, n, height, width,
                                    records, stream)))
    return rc;
  if ((rc = ss_tile_index_count(records, n, height, width, tile_size, ellipse_cull,
                                sigma_cutoff, tile_offsets, index_ws, index_bytes, status,
                                stream)))
    return rc;
  return ss_tile_index_fill(records, n, height, width, tile_size, ellipse_cull, sigma_cutoff,
                            tile_offsets, tile_gids, gid_capacity, index_ws, index_bytes,
                            status, stream);
}

}  // extern "C"

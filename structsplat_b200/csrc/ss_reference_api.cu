// One-call entry points shaped like the reference extension's build_tile_index /
// forward_tiled / backward_tiled (render_ext.cpp:89-317): they take the reference tensor
// contract, pack the splat records into the caller's workspace and run the staged calls.
#include <cmath>

#include "ss_common.cuh"

namespace ss {
namespace {

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Workspace: [records n*64 B][tile-index workspace][backward moments]
struct RefWorkspace {
  void* records;
  void* index_ws;
  size_t index_bytes;
  void* backward_ws;
  size_t backward_bytes;
};

size_t backward_bytes(int64_t n, int H, int W) {
  size_t b = 0;
  ss_render_backward_workspace_bytes(n, 0, H, W, 0, &b);
  return b;
}

int carve_ref(void* ws, size_t ws_bytes, int64_t n, int H, int W, int ts, RefWorkspace* out) {
  size_t idx = 0;
  int rc = ss_tile_index_workspace_bytes(n, H, W, ts, &idx);
  if (rc) return rc;
  size_t need = align256((size_t)n * sizeof(Splat)) + align256(idx) + backward_bytes(n, H, W);
  if (!ws || ws_bytes < need)
    return fail(SS_ERR_INVALID_ARGUMENT, "workspace too small (%zu < %zu)", ws_bytes, need);
  if (reinterpret_cast<uintptr_t>(ws) % 256)
    return fail(SS_ERR_INVALID_ARGUMENT, "workspace must be 256-byte aligned");
  out->records = ws;
  out->index_ws = static_cast<char*>(ws) + align256((size_t)n * sizeof(Splat));
  out->index_bytes = idx;
  out->backward_ws = static_cast<char*>(out->index_ws) + align256(idx);
  out->backward_bytes = backward_bytes(n, H, W);
  return SS_OK;
}

// The reference evaluates the tail as expf(-0.5f * cutoff^2) in float (render_ext.cu:976).
float tail_of(int support_fade, float sigma_cutoff) {
  return support_fade ? expf(-0.5f * (float)((double)sigma_cutoff * sigma_cutoff)) : 0.0f;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_reference_workspace_bytes(int64_t n, int height, int width, int tile_size,
                                 int64_t gid_capacity, size_t* bytes) {
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  size_t idx = 0;
  int rc = ss_tile_index_workspace_bytes(n, height, width, tile_size, &idx);
  if (rc) return rc;
  (void)gid_capacity;
  *bytes = align256((size_t)n * sizeof(Splat)) + align256(idx) + backward_bytes(n, height, width);
  return SS_OK;
}

int ss_build_tile_index(const float* means, const float* conics, const int64_t* radii,
                        int64_t n, int height, int width, int tile_size, int ellipse_cull,
                        float sigma_cutoff, int32_t* tile_gids, int64_t gid_capacity,
                        int32_t* tile_offsets, void* workspace, size_t workspace_bytes,
                        uint32_t* status, ss_stream_t stream) {
  RefWorkspace w;
  int rc = carve_ref(workspace, workspace_bytes, n, height, width, tile_size, &w);
  if (rc) return rc;
  // Colours are not needed for binning; the conic stands in so the record is well formed.
  if (n > 0 && (rc = ss_pack_splats(means, conics, conics, radii, nullptr, n, height, width,
                                    w.records, stream)))
    return rc;
  if ((rc = ss_tile_index_count(w.records, n, height, width, tile_size, ellipse_cull,
                                sigma_cutoff, tile_offsets, w.index_ws, w.index_bytes, status,
                                stream)))
    return rc;
  return ss_tile_index_fill(w.records, n, height, width, tile_size, ellipse_cull, sigma_cutoff,
                            tile_offsets, tile_gids, gid_capacity, w.index_ws, w.index_bytes,
                            status, stream);
}

int ss_forward_tiled(const float* means, const float* conics, const float* colors,
                     const int64_t* radii, const float* opacities, int64_t n,
                     const int32_t* tile_gids, int64_t gid_capacity,
                     const int32_t* tile_offsets, int height, int width, int normalize,
                     float eps, int tile_size, int support_fade, float sigma_cutoff, float* out,
                     float* den, void* workspace, size_t workspace_bytes, uint32_t* status,
                     ss_stream_t stream) {
  RefWorkspace w;
  int rc = carve_ref(workspace, workspace_bytes, n, height, width, tile_size, &w);
  if (rc) return rc;
  if (n > 0 && (rc = ss_pack_splats(means, conics, colors, radii, opacities, n, height, width,
                                    w.records, stream)))
    return rc;
  return ss_render_forward(w.records, n, tile_gids, gid_capacity, tile_offsets, height, width,
                           tile_size, normalize, eps, tail_of(support_fade, sigma_cutoff), out,
                           den, status, stream);
}

int ss_backward_tiled(const float* grad_out, const float* means, const float* conics,
                      const float* colors, const int64_t* radii, const float* opacities,
                      int64_t n, const float* den, const float* out, const int32_t* tile_gids,
                      int64_t gid_capacity, const int32_t* tile_offsets, int height, int width,
                      int normalize, float eps, int tile_size, int support_fade,
                      float sigma_cutoff, float* grad_means, float* grad_conics,
                      float* grad_colors, float* grad_opacities, void* workspace,
                      size_t workspace_bytes, uint32_t* status, ss_stream_t stream) {
  RefWorkspace w;
  int rc = carve_ref(workspace, workspace_bytes, n, height, width, tile_size, &w);
  if (rc) return rc;
  if (n > 0 && (rc = ss_pack_splats(means, conics, colors, radii, opacities, n, height, width,
                                    w.records, stream)))
    return rc;
  return ss_render_backward(grad_out, w.records, n, den, out, tile_gids, gid_capacity,
                            tile_offsets, height, width, tile_size, normalize, eps,
                            tail_of(support_fade, sigma_cutoff), opacities != nullptr,
                            grad_means, grad_conics, grad_colors, grad_opacities, 0,
                            w.backward_ws, w.backward_bytes, status, stream);
}

}  // extern "C"

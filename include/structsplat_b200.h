/*
 * structsplat_b200 — B200 (sm_100a) tiled 2D Gaussian rasterizer, C ABI.
 *
 * Plain pointers and sizes only.  Every pointer argument named *_dev or documented as
 * "device" must point to CUDA device memory; the caller allocates every buffer (outputs and
 * workspaces, sized by the *_workspace_bytes queries) and the library only borrows them.
 * Every call is asynchronous on the given stream (a cudaStream_t; 0 = legacy default stream),
 * performs no host synchronisation and no allocation, and is safe to capture in a CUDA graph.
 *
 * Return value: SS_OK (0) or an SS_ERR_* code; ss_last_error() gives a thread-local message.
 * In-kernel conditions the host cannot see are OR-ed into a caller-provided device status
 * word (SS_STATUS_* bits) that the caller reads whenever it chooses.
 *
 * Reference correspondence (intrinsicD/structsplat, src/structsplat/):
 *   ss_build_tile_index  <- cuda/render_ext.cpp:139-167 build_tile_index / render_ext.cu:858-952
 *   ss_forward_tiled     <- cuda/render_ext.cpp:188-211 forward_tiled / render_ext.cu:1011-1063
 *   ss_backward_tiled    <- cuda/render_ext.cpp:269-301 backward_tiled / render_ext.cu:1169-1231
 *   ss_render_*          <- the same three, split into pack / index / render stages
 *   ss_structure_tensor  <- structure_tensor.py:137-186 (NumPy in the reference)
 *   ss_project_rs*       <- gaussians.py:270-321 (conics, radii, opacity) and their autograd
 */
#ifndef STRUCTSPLAT_B200_H
#define STRUCTSPLAT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* ss_stream_t;

enum {
  SS_OK = 0,
  SS_ERR_INVALID_ARGUMENT = 1,
  SS_ERR_CAPACITY = 2,
  SS_ERR_CUDA = 3,
  SS_ERR_UNSUPPORTED = 4
};

/* Device status word bits. */
#define SS_STATUS_INDEX_OVERFLOW 0x1u  /* tile index needed more than gid_capacity entries */
#define SS_STATUS_INDEX_INT32 0x2u     /* entry total exceeded INT32_MAX */
#define SS_STATUS_DETERMINISTIC_TRUNCATED 0x4u /* deterministic backward met a truncated index */

/* ---------------------------------------------------------------- batches
 * A batch renders B images of any sizes as one tile set, so every stage is one launch for the
 * whole batch.  Image b has tiles_x_b = ceil(W_b/ts) by ceil(H_b/ts) tiles numbered row-major
 * from first_tile_b (images in order, first_tile_0 = 0); its Gaussians are the ids
 * [gaussian_base[b], gaussian_base[b+1]) of the concatenated field; its pixels are rows
 * [pixel_base[b], pixel_base[b] + H_b W_b) of the concatenated (P,3) images and (P) weight sums.
 * Means and support rectangles are image-local.  Every image renders exactly as it would alone
 * (the same entries in the same ascending order), so a batch of one image is the plain call.
 * All tables are device arrays built once per batch shape; the struct itself is read on the
 * host at each call and may be a stack variable. */
typedef struct ss_batch {
  int images;                    /* B >= 1 */
  int tile_size;                 /* 16 or 32 for the render calls */
  int64_t tiles;                 /* total tiles T */
  int64_t pixels;                /* total pixels P */
  const int32_t* image_table;    /* device (B,4): height, width, tiles_x, first_tile */
  const int64_t* pixel_base;     /* device (B) */
  const int32_t* gaussian_base;  /* device (B+1); gaussian_base[B] = n */
  const int32_t* gaussian_image; /* device (n): image of each Gaussian */
  const int32_t* tile_image;     /* device (T): image of each tile */
} ss_batch;

/* ---------------------------------------------------------------- library */
const char* ss_last_error(void);
/* Programmatic dependent launch of the library's kernels (no counterpart in the reference):
 * with 1 (the default) a kernel may become resident while its predecessor in the stream
 * drains and waits on the device for that predecessor's results; 0 launches plainly.  Results
 * do not depend on it.  Process-wide. */
int ss_set_dependent_launch(int enable);
int ss_get_dependent_launch(void);
int ss_version(void);
/* Bytes of one packed splat record (64). */
size_t ss_splat_record_bytes(void);

/* ---------------------------------------------------------------- splat records
 * Packs one 64-byte record per Gaussian: mean, exponent-domain conic, opacity, colour, conic,
 * and the clipped support rectangle of render.py:62-78 (torch.round half-to-even centre,
 * clip to the image; a non-finite centre has empty support as in render_ext.cu:25-34).
 * means (n,2) f32, conics (n,3) f32 [a,b,c] with q = a dx^2 + 2b dx dy + c dy^2,
 * colors (n,3) f32, radii (n,2) int64, opacities (n) f32 or NULL (opacity 1). */
int ss_pack_splats(const float* means, const float* conics, const float* colors,
                   const int64_t* radii, const float* opacities, int64_t n, int height,
                   int width, void* records, ss_stream_t stream);

/* Fused RS projection (gaussians.py:270-321): from means (n,2), log_scales (n,2),
 * rotations (n), colors (n,3), opacity_logits (n or NULL) computes the conic with isotropic
 * `dilation`, the radii ceil(cutoff*sqrt(Sigma_axis)) >= 1, the opacity sigmoid, and writes the
 * packed records.  conics_out (n,3) and radii_out (n,2) are optional (NULL skips them). */
int ss_project_rs(const float* means, const float* log_scales, const float* rotations,
                  const float* colors, const float* opacity_logits, int64_t n, float dilation,
                  float sigma_cutoff, int height, int width, void* records, float* conics_out,
                  int64_t* radii_out, ss_stream_t stream);

/* Chain rule of ss_project_rs: conic and opacity gradients -> log_scale, rotation and
 * opacity-logit gradients (written, not accumulated).  grad_opacities / grad_opacity_logits
 * may be NULL together. */
int ss_project_rs_backward(const float* log_scales, const float* rotations,
                           const float* opacity_logits, int64_t n, float dilation,
                           const float* grad_conics, const float* grad_opacities,
                           float* grad_log_scales, float* grad_rotations,
                           float* grad_opacity_logits, ss_stream_t stream);

/* ss_project_rs followed by ss_tile_index_count in one kernel: each thread projects its
 * Gaussian into `records` (bitwise the records ss_project_rs writes) and counts the tiles of
 * its rectangle from them, so the count reads no record back from DRAM; the offsets, status
 * and workspace are ss_tile_index_count's.  Continue with ss_tile_index_fill.  `clear` (NULL
 * when clear_bytes is 0) is a device region the same kernel zeroes, 16-byte aligned, a multiple
 * of 16 bytes and disjoint from every other buffer of the call: a step's scratch that must start
 * at zero (the fast-mode backward moments, a status word), cleared without a memset of its
 * own.  No counterpart in the reference, which projects in torch and bins in its own kernel
 * (gaussians.py:275-321, render_ext.cu:858-952). */
int ss_project_rs_index_count(const float* means, const float* log_scales,
                              const float* rotations, const float* colors,
                              const float* opacity_logits, int64_t n, float dilation,
                              float sigma_cutoff, int height, int width, int tile_size,
                              int ellipse_cull, void* records, int32_t* tile_offsets,
                              void* workspace, size_t workspace_bytes, void* clear,
                              size_t clear_bytes, uint32_t* status, ss_stream_t stream);

/* The same over a batch (ss_batch_project_rs, then ss_batch_tile_index_count). */
int ss_batch_project_rs_index_count(const ss_batch* batch, const float* means,
                                    const float* log_scales, const float* rotations,
                                    const float* colors, const float* opacity_logits, int64_t n,
                                    float dilation, float sigma_cutoff, int ellipse_cull,
                                    void* records, int32_t* tile_offsets, void* workspace,
                                    size_t workspace_bytes, void* clear, size_t clear_bytes,
                                    uint32_t* status, ss_stream_t stream);

/* ---------------------------------------------------------------- tile index
 * Tiles are tile_size x tile_size pixels, tiles_x = ceil(W/ts), T = tiles_x * ceil(H/ts);
 * 1 <= tile_size and tile_size^2 <= 1024 (render_ext.cpp:163-164).  Entries of tile t are
 * tile_gids[tile_offsets[t] .. tile_offsets[t+1]) in ascending Gaussian id.
 * ellipse_cull drops (tile, Gaussian) pairs whose faded weight is zero on the whole tile
 * (render_ext.cu:101-133,178-191); callers enable it only together with the support fade. */
int ss_tile_index_workspace_bytes(int64_t n, int height, int width, int tile_size,
                                  size_t* bytes);
/* Stage 1: per-tile counts and offsets.  tile_offsets (T+1) int32 receives the offsets;
 * tile_offsets[T] is the entry total.  workspace must be kept for stage 2. */
int ss_tile_index_count(const void* records, int64_t n, int height, int width, int tile_size,
                        int ellipse_cull, float sigma_cutoff, int32_t* tile_offsets,
                        void* workspace, size_t workspace_bytes, uint32_t* status,
                        ss_stream_t stream);
/* Stage 2: fill tile_gids (capacity gid_capacity) and sort every tile ascending.  Entries
 * beyond the capacity are dropped and SS_STATUS_INDEX_OVERFLOW is raised; the render calls
 * then render the affected tiles exactly by scanning all Gaussians. */
int ss_tile_index_fill(const void* records, int64_t n, int height, int width, int tile_size,
                       int ellipse_cull, float sigma_cutoff, const int32_t* tile_offsets,
                       int32_t* tile_gids, int64_t gid_capacity, void* workspace,
                       size_t workspace_bytes, uint32_t* status, ss_stream_t stream);

/* Allocation-free variant of ss_build_tile_index, for callers that cannot allocate device
 * memory while building an index (an engine that owns all device memory through its own pool,
 * a plugin limited to the buffers it is handed, code that must not trigger the device
 * synchronisation an allocation implies).  It takes no workspace: its scratch is a 5 MiB
 * device array compiled into the library and held on every GPU that loads it.  Limits:
 * n <= 65536 Gaussians and at most 16384 tiles (SS_ERR_CAPACITY beyond).  All calls share the
 * array: calls that overlap on the GPU race and must be serialised.  The first call on each
 * device resolves the array's address (cudaGetSymbolAddress) with that device current and
 * should come before any stream capture on it.  That address is cached per device for the
 * life of the process and does not survive cudaDeviceReset: do not call this entry point after
 * resetting a device it has already run on.  No counterpart in the reference. */
int ss_build_tile_index_static(const float* means, const float* conics, const int64_t* radii,
                               int64_t n, int height, int width, int tile_size,
                               int ellipse_cull, float sigma_cutoff, int32_t* tile_gids,
                               int64_t gid_capacity, int32_t* tile_offsets, uint32_t* status,
                               ss_stream_t stream);

/* Batched forms of ss_project_rs / ss_tile_index_* (see ss_batch).  height/width/tile_size
 * come from the batch; the index workspace depends only on batch->tiles. */
int ss_batch_project_rs(const ss_batch* batch, const float* means, const float* log_scales,
                        const float* rotations, const float* colors,
                        const float* opacity_logits, int64_t n, float dilation,
                        float sigma_cutoff, void* records, ss_stream_t stream);
int ss_batch_tile_index_workspace_bytes(const ss_batch* batch, int64_t n, size_t* bytes);
int ss_batch_tile_index_count(const ss_batch* batch, const void* records, int64_t n,
                              int ellipse_cull, float sigma_cutoff, int32_t* tile_offsets,
                              void* workspace, size_t workspace_bytes, uint32_t* status,
                              ss_stream_t stream);
int ss_batch_tile_index_fill(const ss_batch* batch, const void* records, int64_t n,
                             int ellipse_cull, float sigma_cutoff, const int32_t* tile_offsets,
                             int32_t* tile_gids, int64_t gid_capacity, void* workspace,
                             size_t workspace_bytes, uint32_t* status, ss_stream_t stream);

/* ---------------------------------------------------------------- render
 * Supported render tile sizes: 16 (the reference default) and 32.  fade_tail is
 * alpha*exp(-cutoff^2/2) rounded to float (0 = no fade); eps > 0 and finite.
 * out (H,W,3) f32 image; den (H,W) f32 raw weight sum without eps. */
int ss_render_forward(const void* records, int64_t n, const int32_t* tile_gids,
                      int64_t gid_capacity, const int32_t* tile_offsets, int height, int width,
                      int tile_size, int normalize, float eps, float fade_tail, float* out,
                      float* den, uint32_t* status, ss_stream_t stream);

/* Launch tuning (process-wide, used by the autotuner): warps per backward CTA for a render
 * tile size — 4 or 8 for tile 16, 8 or 16 for tile 32, 0 restores the default (8 for both).
 * Results do not depend on it.  ss_get_backward_warps returns the value in effect (-1 for an
 * unsupported tile size). */
int ss_set_backward_warps(int tile_size, int warps);
int ss_get_backward_warps(int tile_size);

/* Launch tuning (process-wide): records per streamed chunk of the forward for a render tile
 * size — 64, 128 or 256, 0 restores the default (256).  Only tile lists longer than the
 * forward's 512-record stage stream; images do not depend on it.  ss_get_forward_chunk returns
 * the value in effect (-1 for an unsupported tile size). */
int ss_set_forward_chunk(int tile_size, int records);
int ss_get_forward_chunk(int tile_size);

/* Workspace of ss_render_backward: per-Gaussian moment accumulators (36 B per Gaussian) or,
 * deterministic, per-entry partials (48 B per entry of capacity); height and width are unused. */
int ss_render_backward_workspace_bytes(int64_t n, int64_t gid_capacity, int height, int width,
                                       int deterministic, size_t* bytes);
/* Gradients of sum(out * grad_out) w.r.t. means (n,2), conics (n,3), colors (n,3) and, when
 * has_opacity, opacities (n).  Outputs are overwritten.  Each warp reduces one Gaussian's part
 * inside one tile; deterministic=0 adds it with one atomic per moment, deterministic=1 stores
 * it and sums a Gaussian's parts in ascending tile order, which is bitwise reproducible. */
int ss_render_backward(const float* grad_out, const void* records, int64_t n, const float* den,
                       const float* out, const int32_t* tile_gids, int64_t gid_capacity,
                       const int32_t* tile_offsets, int height, int width, int tile_size,
                       int normalize, float eps, float fade_tail, int has_opacity,
                       float* grad_means, float* grad_conics, float* grad_colors,
                       float* grad_opacities, int deterministic, void* workspace,
                       size_t workspace_bytes, uint32_t* status, ss_stream_t stream);

/* Batched forms of the two render calls: out (P,3), den (P), grad_out (P,3). */
int ss_batch_render_forward(const ss_batch* batch, const void* records, int64_t n,
                            const int32_t* tile_gids, int64_t gid_capacity,
                            const int32_t* tile_offsets, int normalize, float eps,
                            float fade_tail, float* out, float* den, uint32_t* status,
                            ss_stream_t stream);
int ss_batch_render_backward(const ss_batch* batch, const float* grad_out, const void* records,
                             int64_t n, const float* den, const float* out,
                             const int32_t* tile_gids, int64_t gid_capacity,
                             const int32_t* tile_offsets, int normalize, float eps,
                             float fade_tail, int has_opacity, float* grad_means,
                             float* grad_conics, float* grad_colors, float* grad_opacities,
                             int deterministic, void* workspace, size_t workspace_bytes,
                             uint32_t* status, ss_stream_t stream);

/* ---------------------------------------------------------------- fit iteration
 * The reference's plain fit iteration (fit.py:3182-3366: render -> pixel loss -> backward ->
 * torch.optim.Adam step over the five parameter groups of gaussians.py:203-214 -> log-scale
 * clamp) as three launches after the index build, for a batch of independent fits.
 *
 * ss_fit_forward_loss renders, evaluates the per-image pixel loss of fit.py:800-814
 * (loss_kind 0 l1, 1 l2, 2 charbonnier with charbonnier_eps; the loss of image b is the mean
 * over its pixels of the channel mean) and writes, per pixel, the backward's input
 * pixel_grad (P,4) = (dL/dnum_r, dL/dnum_g, dL/dnum_b, dL/dden).  image (P,3) and den (P) are
 * optional outputs (NULL skips them); loss (B,2), optional, receives per image the loss and
 * the mean squared error added atomically (zero it first).  target is (P,3). */
int ss_fit_forward_loss(const ss_batch* batch, const void* records, int64_t n,
                        const int32_t* tile_gids, int64_t gid_capacity,
                        const int32_t* tile_offsets, int normalize, float eps, float fade_tail,
                        const float* target, int loss_kind, float charbonnier_eps,
                        float* pixel_grad, float* image, float* den, float* loss,
                        uint32_t* status, ss_stream_t stream);
/* Workspace of ss_fit_backward and ss_fit_adam_update: moments (36 B per Gaussian) or,
 * deterministic, per-entry partials and their by-Gaussian order (64 B per entry of capacity,
 * 8 B per Gaussian and the radix sort's scratch), followed by the parameter gradients of the
 * Adam step (36 B per Gaussian). */
int ss_fit_backward_workspace_bytes(int64_t n, int64_t gid_capacity, int deterministic,
                                    size_t* bytes);
/* Render backward from pixel_grad into the workspace.  Fast mode adds into per-Gaussian
 * moments that must be zero on entry: zero them once, ss_fit_adam_update re-zeroes them. */
int ss_fit_backward(const ss_batch* batch, const void* records, int64_t n,
                    const int32_t* tile_gids, int64_t gid_capacity, const int32_t* tile_offsets,
                    float fade_tail, const float* pixel_grad, int deterministic,
                    void* workspace, size_t workspace_bytes, uint32_t* status,
                    ss_stream_t stream);
/* ss_fit_forward_loss followed by ss_fit_backward in one kernel launch: each tile's CTA stages
 * its records once, renders its pixels, evaluates the pixel loss and keeps the loss gradient in
 * shared memory for the tile's backward, so pixel_grad never goes through global memory.  The
 * image, the loss (B,2) and the workspace's moments or partials are those of the two calls
 * (the loss sums are float atomics in either form).  image (P,3), den (P) and loss are
 * optional (NULL skips them; zero loss first).  The workspace is ss_fit_backward's (size
 * ss_fit_backward_workspace_bytes); fast mode: moments zero on entry.  Deterministic mode: a
 * tile whose list the capacity truncated raises SS_STATUS_DETERMINISTIC_TRUNCATED and renders
 * nothing (re-plan with more capacity and redo the step).  No counterpart in the reference,
 * whose fit loop runs its renderer and torch autograd as separate passes. */
int ss_fit_forward_backward(const ss_batch* batch, const void* records, int64_t n,
                            const int32_t* tile_gids, int64_t gid_capacity,
                            const int32_t* tile_offsets, int normalize, float eps,
                            float fade_tail, const float* target, int loss_kind,
                            float charbonnier_eps, float* image, float* den, float* loss,
                            int deterministic, void* workspace, size_t workspace_bytes,
                            uint32_t* status, ss_stream_t stream);
/* SSIM term of the fit loss (metrics.py:130-150, builtin backend: 11-tap Gaussian window,
 * sigma 1.5, zero padding, C1 = 0.01^2, C2 = 0.03^2, mean over channels and pixels of each
 * image), mixed as fit.py:3244 mixes it: loss = (1 - w) pixel_loss + w (1 - SSIM).
 * ss_ssim_workspace_bytes: scratch of both calls (72 B per pixel).
 * ss_ssim_target_stats: the target's window statistics (6P floats: mu_t per channel, then
 * sig_t), constant over a fit (metrics.py:85-118, SSIMTargetStats); target (P,3).
 * ss_fit_ssim: after ss_fit_forward_loss has written image (P,3), den (P) and the pixel loss's
 * pixel_grad (P,4), scales pixel_grad by (1 - w) and adds -w dSSIM/dimage mapped to the
 * backward's per-pixel input (normalized: (g, -(g . image)) / (den + eps); additive: (g, 0)).
 * ssim (B), optional, receives each image's SSIM added atomically (zero it first).  With w = 1,
 * normalize = 0 and a zero pixel_grad, pixel_grad[:, :3] is -dSSIM/dimage. */
int ss_ssim_workspace_bytes(int64_t pixels, size_t* bytes);
int ss_ssim_target_stats(const ss_batch* batch, const float* target, float* stats,
                         void* workspace, size_t workspace_bytes, ss_stream_t stream);
int ss_fit_ssim(const ss_batch* batch, const float* image, const float* den, const float* target,
                const float* stats, int normalize, float eps, float ssim_weight,
                float* pixel_grad, float* ssim, void* workspace, size_t workspace_bytes,
                ss_stream_t stream);
/* ss_render_forward followed by ss_render_backward_moments in one kernel launch, for a caller
 * that holds grad_out (H,W,3) before the forward (a fixed image-space gradient, as the
 * reference's fwd+bwd benchmark uses): each tile's CTA stages its records once, renders out and
 * den (written as ss_render_forward writes them) and forms the backward's pixel inputs from
 * grad_out and its own accumulators in shared memory.  The workspace is
 * ss_render_backward_moments's (fast mode: moments zero on entry); finish with
 * ss_render_backward_finalize or ss_render_backward_finalize_rs.  Deterministic mode: a tile
 * whose list the capacity truncated raises SS_STATUS_DETERMINISTIC_TRUNCATED and renders
 * nothing.  No counterpart in the reference, whose renderer and autograd run as separate
 * passes. */
int ss_render_forward_backward(const void* records, int64_t n, const int32_t* tile_gids,
                               int64_t gid_capacity, const int32_t* tile_offsets, int height,
                               int width, int tile_size, int normalize, float eps,
                               float fade_tail, const float* grad_out, float* out, float* den,
                               int deterministic, void* workspace, size_t workspace_bytes,
                               uint32_t* status, ss_stream_t stream);
/* Gradients of the five parameter groups from the backward's workspace, then one Adam step
 * (torch.optim.Adam's multi-tensor step: lerp first moment, step factors formed in double, no
 * weight decay), then the clamp of log_scales to [log_scale_lo, log_scale_hi[image]] that the
 * reference's loop applies after the step.  params / exp_avg / exp_avg_sq: 5 device pointers
 * each, in the order means (n,2), log_scales (n,2), rotations (n), colors (n,3),
 * opacity_logits (n) (the last may be NULL in all three); lrs: 5 host doubles (the parameter
 * groups' learning rates); log_scale_hi: device (B) floats.  step_state: device int[2], zero
 * before the first step; it holds the step count, so the call can be replayed from a CUDA
 * graph.  In fast mode the moments are zeroed for the next ss_fit_backward. */
int ss_fit_adam_update(const ss_batch* batch, const void* records, int64_t n,
                       const int32_t* tile_gids, int64_t gid_capacity,
                       const int32_t* tile_offsets, int deterministic, void* workspace,
                       float dilation, float* const* params, float* const* exp_avg,
                       float* const* exp_avg_sq, const double* lrs, double beta1, double beta2,
                       double adam_eps, float log_scale_lo, const float* log_scale_hi,
                       int* step_state, ss_stream_t stream);

/* ---------------------------------------------------------------- placement
 * Density-weighted placement of a field from the structure tensor (density.py, init.py).
 * All images are (H,W) row-major; the workspace (ss_placement_workspace_bytes) holds a copy of
 * the cdf and CUB's temporary storage.
 *
 * ss_density_from_energy: density.py:16-29.  energy (H,W) f32 -> density (H,W) f64 pmf;
 * ref_dev points to the energy reference (a device double, e.g. stats_dev[0] of
 * ss_structure_tensor). */
int ss_placement_workspace_bytes(int height, int width, size_t* bytes);
int ss_density_from_energy(const float* energy, int height, int width, double base,
                           double power, const double* ref_dev, double* density, void* workspace,
                           size_t workspace_bytes, ss_stream_t stream);
/* sample_candidates (density.py:133-153) for given uniforms: uniforms (3n) f64 hold the n draws
 * of rng.choice followed by the (n,2) jitter block, exactly as the reference's numpy Generator
 * draws them.  points (n,2) f64 (x, y); pixel_index (n) int64 optional. */
int ss_sample_candidates(const double* density, int height, int width, const double* uniforms,
                         int64_t n, double* points, int64_t* pixel_index, void* workspace,
                         size_t workspace_bytes, ss_stream_t stream);
/* Field initialisation at the sampled points for the density_random sampler (init.py:626-631,
 * 778-847 with scale_mode spacing, orientation tensor, colour bilinear, no scale cap, no
 * opacity): writes means (n,2), log_scales (n,2), rotations (n), colors (n,3) f32.
 * density_points is the n of _radius_map (the requested Gaussian count). */
int ss_place_gaussians(const double* points, int64_t n, const double* density,
                       const float* across_edge_angle, const float* coherence,
                       const float* image, int height, int width, int anisotropic,
                       double max_axis_ratio, double coherence_power, double init_scale_mult,
                       int64_t density_points, float* means, float* log_scales,
                       float* rotations, float* colors, ss_stream_t stream);

/* ---------------------------------------------------------------- render backward, staged
 * ss_render_backward split in two, for callers that accumulate several renders' moments before
 * finalising (or time the tile kernel alone).  _moments runs only the tile kernel: in fast mode
 * it ADDS into per-Gaussian moments (zero the workspace first), in deterministic mode it writes
 * the per-entry partials.  Its per-pixel input is either grad_out with out and den (the plain
 * render's gradient), or, when pixel_grad is given, (P,4) f32 per-pixel gradients with respect
 * to the accumulated colour numerator and weight sum (grad_out, out, den, normalize and eps are
 * then unused): (0, 0, 0, g) differentiates sum(g * den), the raw weight map.
 * _finalize turns them into the four gradient outputs. */
int ss_render_backward_moments(const float* grad_out, const float* pixel_grad,
                               const void* records, int64_t n, const float* den,
                               const float* out, const int32_t* tile_gids,
                               int64_t gid_capacity, const int32_t* tile_offsets, int height,
                               int width, int tile_size, int normalize, float eps,
                               float fade_tail, int deterministic, void* workspace,
                               size_t workspace_bytes, uint32_t* status, ss_stream_t stream);
int ss_render_backward_finalize(const void* records, int64_t n, const int32_t* tile_gids,
                                int64_t gid_capacity, const int32_t* tile_offsets, int height,
                                int width, int tile_size, int has_opacity, int deterministic,
                                const void* workspace, float* grad_means, float* grad_conics,
                                float* grad_colors, float* grad_opacities, ss_stream_t stream);

/* _finalize straight to the RS field parameters (the epilogue followed by
 * ss_project_rs_backward, in one pass): grad_means (n,2), grad_log_scales (n,2),
 * grad_rotations (n), grad_colors (n,3) and, with opacity logits, grad_opacity_logits (n). */
int ss_render_backward_finalize_rs(const void* records, int64_t n, const int32_t* tile_gids,
                                   int64_t gid_capacity, const int32_t* tile_offsets, int height,
                                   int width, int tile_size, int deterministic,
                                   const void* workspace, const float* log_scales,
                                   const float* rotations, const float* opacity_logits,
                                   float dilation, float* grad_means, float* grad_log_scales,
                                   float* grad_rotations, float* grad_colors,
                                   float* grad_opacity_logits, ss_stream_t stream);

/* ---------------------------------------------------------------- per-Gaussian passes
 * gaussian_activity (render.py:417-442): activity[g] = sum over the pixels of g's clipped
 * support rectangle of max(exp(-q/2) - fade_tail, 0) (opacity-free), from packed records.
 * lanes_per_gaussian: 8 (fields of small Gaussians) or 32.  Deterministic. */
int ss_gaussian_activity(const void* records, int64_t n, float fade_tail, int lanes_per_gaussian,
                         float* activity, ss_stream_t stream);

/* ---------------------------------------------------------------- SSPL1 field decode
 * The integer streams of an SSPL1 container (codec.py:235-391), inflated on the host (zlib /
 * PNG), in device memory; the header's JSON fields are copied into this struct.  Values are
 * 1, 2 or 4 bytes each by bit depth, little-endian; means may be byte-planar.  Layout: means
 * (x for all Gaussians, then y), scales likewise, rotation, colours (r, g, b planes), opacity
 * (optional, probabilities).  Morton-ordered means and delta colours are modular deltas. */
typedef struct ss_sspl1_streams {
  int64_t n;
  const uint8_t* means;
  int means_bits, means_byte_planar, morton;
  double means_lo[2], means_hi[2];
  const uint8_t* scales;
  int scale_bits;
  double scale_lo[2], scale_hi[2];
  const uint8_t* rotations;
  int rot_bits, rot_circular;
  const uint8_t* colors;
  int color_bits, color_delta;
  double color_lo[3], color_hi[3];
  const uint8_t* opacities;  /* NULL: the container has no opacity stream */
  int opacity_bits;
} ss_sspl1_streams;
int ss_sspl1_workspace_bytes(int64_t n, size_t* bytes);
/* Writes means (n,2), log_scales (n,2), rotations (n), colors (n,3) and, with an opacity
 * stream, opacity logits (n), all f32, bit-identical to the reference's decode except the
 * logit (log of a float32 ratio, within 2 ulp). */
int ss_sspl1_dequantize(const ss_sspl1_streams* streams, float* means, float* log_scales,
                        float* rotations, float* colors, float* opacity_logits, void* workspace,
                        size_t workspace_bytes, ss_stream_t stream);

/* ---------------------------------------------------------------- reference-shaped calls
 * One-call equivalents of the reference extension's entry points, taking its tensor
 * contract (render_ext.cpp:89-137).  They pack records into `workspace` (size from
 * ss_reference_workspace_bytes) and then run the staged calls above. */
int ss_reference_workspace_bytes(int64_t n, int height, int width, int tile_size,
                                 int64_t gid_capacity, size_t* bytes);
int ss_build_tile_index(const float* means, const float* conics, const int64_t* radii,
                        int64_t n, int height, int width, int tile_size, int ellipse_cull,
                        float sigma_cutoff, int32_t* tile_gids, int64_t gid_capacity,
                        int32_t* tile_offsets, void* workspace, size_t workspace_bytes,
                        uint32_t* status, ss_stream_t stream);
int ss_forward_tiled(const float* means, const float* conics, const float* colors,
                     const int64_t* radii, const float* opacities, int64_t n,
                     const int32_t* tile_gids, int64_t gid_capacity,
                     const int32_t* tile_offsets, int height, int width, int normalize,
                     float eps, int tile_size, int support_fade, float sigma_cutoff, float* out,
                     float* den, void* workspace, size_t workspace_bytes, uint32_t* status,
                     ss_stream_t stream);
int ss_backward_tiled(const float* grad_out, const float* means, const float* conics,
                      const float* colors, const int64_t* radii, const float* opacities,
                      int64_t n, const float* den, const float* out, const int32_t* tile_gids,
                      int64_t gid_capacity, const int32_t* tile_offsets, int height, int width,
                      int normalize, float eps, int tile_size, int support_fade,
                      float sigma_cutoff, float* grad_means, float* grad_conics,
                      float* grad_colors, float* grad_opacities, void* workspace,
                      size_t workspace_bytes, uint32_t* status, ss_stream_t stream);

/* ---------------------------------------------------------------- structure tensor
 * J = G_rho * (grad I grad I^T) of an (H,W,C) f32 image, C in {1,3} (structure_tensor.py).
 * taps_grad / taps_tensor are HOST arrays of 2r+1 normalised Gaussian taps (r <= 31) for the
 * pre-smoothing and tensor smoothing (a radius of 0 disables that blur).  gradient_operator:
 * 0 central (np.gradient), 1 sobel, 2 scharr.  color_space: 0 luma (Rec.709), 1 rgb
 * (Di Zenzo sum).  Outputs (H,W) f32 maps and u8 labels; stats_dev receives four doubles:
 * energy_ref, flat threshold, median, 99th percentile. */
int ss_structure_tensor_workspace_bytes(int height, int width, int channels, size_t* bytes);
int ss_structure_tensor(const float* image, int height, int width, int channels,
                        const float* taps_grad, int radius_grad, const float* taps_tensor,
                        int radius_tensor, int gradient_operator, int color_space,
                        double flat_frac, double corner_frac, float* lam1, float* lam2,
                        float* angle, float* coherence, float* energy, uint8_t* label,
                        double* stats_dev, void* workspace, size_t workspace_bytes,
                        ss_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* STRUCTSPLAT_B200_H */

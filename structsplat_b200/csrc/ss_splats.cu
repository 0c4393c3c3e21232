// Library plumbing (errors, version) and the per-Gaussian kernels: record packing and the
// fused RS projection with its chain rule.
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <utility>
#include <vector>

#include "ss_common.cuh"

namespace ss {

static thread_local char g_error[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_error, sizeof(g_error), fmt, ap);
  va_end(ap);
  return code;
}

namespace {
thread_local cudaError_t t_launch_error = cudaSuccess;  // a failed cudaLaunchKernelEx
std::atomic<int> g_dependent_launch{1};
}  // namespace

void note_launch_error(cudaError_t e) { t_launch_error = e; }

bool dependent_launch_enabled() {
  return g_dependent_launch.load(std::memory_order_relaxed) != 0;
}

int check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = t_launch_error;
  t_launch_error = cudaSuccess;
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return SS_OK;
}

int allow_dynamic_smem(const void* kern, size_t bytes) {
  // (kernel, device) pairs already opted in; a handful of kernels use more than 48 KB
  static std::mutex mu;
  static std::vector<std::pair<const void*, int>> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("cudaGetDevice");
  std::lock_guard<std::mutex> lock(mu);
  for (const auto& d : done)
    if (d.first == kern && d.second == dev) return SS_OK;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
      cudaSuccess)
    return check_launch("dynamic shared memory attribute");
  done.emplace_back(kern, dev);
  return SS_OK;
}

int frames_of_batch(const ss_batch* batch, int64_t n, Frames* out) {
  if (!batch) return fail(SS_ERR_INVALID_ARGUMENT, "null batch");
  if (batch->images < 1) return fail(SS_ERR_INVALID_ARGUMENT, "batch needs at least one image");
  if (batch->tile_size <= 0 || batch->tile_size > 32)  // ts^2 <= 1024, without overflow
    return fail(SS_ERR_INVALID_ARGUMENT, "batch tile_size must be positive with ts^2 <= 1024");
  if (batch->tiles < 0 || batch->tiles + 1 > (int64_t)INT32_MAX || batch->pixels < 0)
    return fail(SS_ERR_INVALID_ARGUMENT, "batch tile or pixel total out of range");
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "bad Gaussian count");
  if (!batch->image_table || !batch->pixel_base || !batch->gaussian_base ||
      (n > 0 && !batch->gaussian_image) || (batch->tiles > 0 && !batch->tile_image))
    return fail(SS_ERR_INVALID_ARGUMENT, "batch table pointer is null");
  Frames f{};
  f.image = reinterpret_cast<const int4*>(batch->image_table);
  f.pixel_base = reinterpret_cast<const long long*>(batch->pixel_base);
  f.gauss_base = batch->gaussian_base;
  f.gauss_image = batch->gaussian_image;
  f.tile_image = batch->tile_image;
  *out = f;
  return SS_OK;
}

namespace {

constexpr int kThreads = 256;

inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

__global__ void pack_splats_kernel(const float* __restrict__ means,
                                   const float* __restrict__ conics,
                                   const float* __restrict__ colors,
                                   const int64_t* __restrict__ radii,
                                   const float* __restrict__ opacities, int64_t n, int H, int W,
                                   Splat* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float mx = means[2 * i], my = means[2 * i + 1];
  int x0, y0, x1, y1;
  support_rect(mx, my, radii[2 * i], radii[2 * i + 1], H, W, x0, y0, x1, y1);
  float op = opacities ? opacities[i] : 1.0f;
  store_splat(out + i, make_splat(mx, my, conics[3 * i], conics[3 * i + 1], conics[3 * i + 2],
                                  op, colors[3 * i], colors[3 * i + 1], colors[3 * i + 2], x0,
                                  y0, x1, y1));
}

// RS -> splat record (rs_project_one), plus the conic and radii where asked for.
__global__ void project_rs_kernel(const float* __restrict__ means,
                                  const float* __restrict__ log_scales,
                                  const float* __restrict__ rotations,
                                  const float* __restrict__ colors,
                                  const float* __restrict__ logits, int64_t n, float dilation,
                                  float cutoff, Frames frames, Splat* __restrict__ out,
                                  float* __restrict__ conics_out,
                                  int64_t* __restrict__ radii_out) {
  pdl_wait();
  pdl_trigger();
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const RSField f{means, log_scales, rotations, colors, logits, dilation, cutoff};
  long long rx, ry;
  const Splat sp = rs_project_one(f, i, frame_of_gaussian(frames, i, n), rx, ry);
  store_splat(out + i, sp);
  if (conics_out) {
    conics_out[3 * i] = sp.a;
    conics_out[3 * i + 1] = sp.b;
    conics_out[3 * i + 2] = sp.c;
  }
  if (radii_out) {
    radii_out[2 * i] = rx;
    radii_out[2 * i + 1] = ry;
  }
}

// d(conic)/d(log_scale, rotation) and d(opacity)/d(logit).  With u = 1/(sx^2+d),
// v = 1/(sy^2+d): a = C^2 u + S^2 v, b = CS (u - v), c = S^2 u + C^2 v, so
//   dL/du = ga C^2 + gb CS + gc S^2,   dL/dv = ga S^2 - gb CS + gc C^2,
//   du/dlx = -2 sx^2 u^2,              dv/dly = -2 sy^2 v^2,
//   dL/dθ = (u - v) (-2CS ga + (C^2 - S^2) gb + 2CS gc),   dσ/dl = σ (1 - σ).
__global__ void project_rs_backward_kernel(const float* __restrict__ log_scales,
                                           const float* __restrict__ rotations,
                                           const float* __restrict__ logits, int64_t n,
                                           float dilation, const float* __restrict__ g_conics,
                                           const float* __restrict__ g_opac,
                                           float* __restrict__ g_log_scales,
                                           float* __restrict__ g_rot,
                                           float* __restrict__ g_logits) {
  pdl_wait();
  pdl_trigger();
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rs_conic_chain(log_scales[2 * i], log_scales[2 * i + 1], rotations[i], dilation,
                 g_conics[3 * i], g_conics[3 * i + 1], g_conics[3 * i + 2], g_log_scales[2 * i],
                 g_log_scales[2 * i + 1], g_rot[i]);
  if (logits && g_opac && g_logits) g_logits[i] = logit_chain(logits[i], g_opac[i]);
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

const char* ss_last_error(void) { return ss::g_error; }

int ss_set_dependent_launch(int enable) {
  if (enable != 0 && enable != 1)
    return fail(SS_ERR_INVALID_ARGUMENT, "dependent launch switch must be 0 or 1");
  ss::g_dependent_launch.store(enable, std::memory_order_relaxed);
  return SS_OK;
}

int ss_get_dependent_launch(void) { return ss::dependent_launch_enabled() ? 1 : 0; }

int ss_version(void) { return 1; }

size_t ss_splat_record_bytes(void) { return sizeof(Splat); }

int ss_pack_splats(const float* means, const float* conics, const float* colors,
                   const int64_t* radii, const float* opacities, int64_t n, int height,
                   int width, void* records, ss_stream_t stream) {
  if (n < 0 || height < 0 || width < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "n exceeds int32 ids");
  if (n == 0) return SS_OK;
  if (!means || !conics || !colors || !radii || !records)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (reinterpret_cast<uintptr_t>(records) % 16)
    return fail(SS_ERR_INVALID_ARGUMENT, "records must be 16-byte aligned");
  launch("pack_splats_kernel", pack_splats_kernel, blocks_for(n), kThreads, 0, as_stream(stream), 
      means, conics, colors, radii, opacities, n, height, width,
      reinterpret_cast<Splat*>(records));
  return check_launch("pack_splats");
}

static int project_rs(const Frames& frames, const float* means, const float* log_scales,
                      const float* rotations, const float* colors, const float* opacity_logits,
                      int64_t n, float dilation, float sigma_cutoff, void* records,
                      float* conics_out, int64_t* radii_out, ss_stream_t stream) {
  if (n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "n exceeds int32 ids");
  if (!(dilation >= 0.0f)) return fail(SS_ERR_INVALID_ARGUMENT, "dilation must be >= 0");
  if (n == 0) return SS_OK;
  if (!means || !log_scales || !rotations || !colors || !records)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (reinterpret_cast<uintptr_t>(records) % 16)
    return fail(SS_ERR_INVALID_ARGUMENT, "records must be 16-byte aligned");
  launch("project_rs_kernel", project_rs_kernel, blocks_for(n), kThreads, 0, as_stream(stream), 
      means, log_scales, rotations, colors, opacity_logits, n, dilation, sigma_cutoff, frames,
      reinterpret_cast<Splat*>(records), conics_out, radii_out);
  return check_launch("project_rs");
}

int ss_project_rs(const float* means, const float* log_scales, const float* rotations,
                  const float* colors, const float* opacity_logits, int64_t n, float dilation,
                  float sigma_cutoff, int height, int width, void* records, float* conics_out,
                  int64_t* radii_out, ss_stream_t stream) {
  if (n < 0 || height < 0 || width < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  return project_rs(single_frame(height, width, 1), means, log_scales, rotations, colors,
                    opacity_logits, n, dilation, sigma_cutoff, records, conics_out, radii_out,
                    stream);
}

int ss_batch_project_rs(const ss_batch* batch, const float* means, const float* log_scales,
                        const float* rotations, const float* colors,
                        const float* opacity_logits, int64_t n, float dilation,
                        float sigma_cutoff, void* records, ss_stream_t stream) {
  Frames f;
  int rc = frames_of_batch(batch, n, &f);
  if (rc) return rc;
  return project_rs(f, means, log_scales, rotations, colors, opacity_logits, n, dilation,
                    sigma_cutoff, records, nullptr, nullptr, stream);
}

int ss_project_rs_backward(const float* log_scales, const float* rotations,
                           const float* opacity_logits, int64_t n, float dilation,
                           const float* grad_conics, const float* grad_opacities,
                           float* grad_log_scales, float* grad_rotations,
                           float* grad_opacity_logits, ss_stream_t stream) {
  if (n < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (n == 0) return SS_OK;
  if (!log_scales || !rotations || !grad_conics || !grad_log_scales || !grad_rotations)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  launch("project_rs_backward_kernel", project_rs_backward_kernel, blocks_for(n), kThreads, 0, as_stream(stream), 
      log_scales, rotations, opacity_logits, n, dilation, grad_conics, grad_opacities,
      grad_log_scales, grad_rotations, grad_opacity_logits);
  return check_launch("project_rs_backward");
}

}  // extern "C"

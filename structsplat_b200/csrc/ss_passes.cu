// Per-Gaussian passes that reuse the renderer's pair loop.
//
// Activity (render.py:417-442, gaussian_activity): each Gaussian's summed raw weight
// visible_weight(q) = max(exp(-q/2) - tail, 0) over the pixels of its clipped support
// rectangle — opacity-free, the pruning diagnostic of the reference fitter.  Every pixel of the
// rectangle is one in-rectangle pair, so the work is P pairs with no image data: a warp walks
// one Gaussian's rectangle row-major (lane l takes pixels l, l+32, …) and reduces its 32 partial
// sums in a fixed xor-butterfly order, so the result is deterministic.  Fields of small
// Gaussians would leave most of a warp idle, so the caller may give each Gaussian 8 lanes
// instead of 32.
#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

template <bool FADE>
__device__ __forceinline__ float visible(const Splat& s, int x, int y, float tail) {
  const float dx = (float)x - s.mx, dy = (float)y - s.my;
  const float raw = fast_exp2(fmaf(dy, fmaf(s.qc, dy, s.qb * dx), s.qa * dx * dx));
  return FADE ? fmaxf(raw - tail, 0.0f) : raw;
}

// One group of G lanes per Gaussian: lanes stride the rectangle's pixels row-major.
template <int G, bool FADE>
__global__ void __launch_bounds__(kThreads)
    activity_kernel(const Splat* __restrict__ rec, int64_t n, float tail,
                    float* __restrict__ activity) {
  pdl_wait();
  pdl_trigger();
  const int64_t gid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const int sub = threadIdx.x % G;
  float acc = 0.f;
  if (gid < n) {
    Splat s;
    const float4* src = reinterpret_cast<const float4*>(rec + gid);
    float4* d = reinterpret_cast<float4*>(&s);
    d[0] = src[0];
    d[1] = src[1];
    d[2] = src[2];
    d[3] = src[3];
    const int w = s.x1 - s.x0, h = s.y1 - s.y0;
    if (w > 0 && h > 0) {
      const int64_t area = (int64_t)w * h;
      // lane sub visits pixels sub, sub + G, …: (row, col) advanced incrementally
      int row = sub / w, col = sub - (sub / w) * w;
      const int step_r = G / w, step_c = G - (G / w) * w;
      for (int64_t k = sub; k < area; k += G) {
        acc += visible<FADE>(s, s.x0 + col, s.y0 + row, tail);
        col += step_c;
        row += step_r;
        if (col >= w) {
          col -= w;
          ++row;
        }
      }
    }
  }
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, G);
  if (gid < n && sub == 0) activity[gid] = acc;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_gaussian_activity(const void* records, int64_t n, float fade_tail, int lanes_per_gaussian,
                         float* activity, ss_stream_t stream) {
  if (n < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (n == 0) return SS_OK;
  if (!records || !activity) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (lanes_per_gaussian != 8 && lanes_per_gaussian != 32)
    return fail(SS_ERR_INVALID_ARGUMENT, "lanes_per_gaussian must be 8 or 32");
  const Splat* rec = static_cast<const Splat*>(records);
  const int64_t threads = n * lanes_per_gaussian;
  const unsigned blocks = (unsigned)((threads + kThreads - 1) / kThreads);
  cudaStream_t s = as_stream(stream);
  const bool fade = fade_tail > 0.0f;
#define SS_ACT(G, F) activity_kernel<G, F><<<blocks, kThreads, 0, s>>>(rec, n, fade_tail, activity)
  if (lanes_per_gaussian == 8) {
    if (fade) SS_ACT(8, true); else SS_ACT(8, false);
  } else {
    if (fade) SS_ACT(32, true); else SS_ACT(32, false);
  }
#undef SS_ACT
  return check_launch("gaussian_activity");
}

}  // extern "C"

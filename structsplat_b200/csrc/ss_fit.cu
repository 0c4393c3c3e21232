// Update of a fit iteration, in two passes.  Per Gaussian (fit_grad_kernel): the render
// backward's summed moments become conic / mean / colour / opacity gradients and the chain rule
// carries them to the RS field parameters (gaussians.py:270-300); the moment accumulators are
// zeroed for the next iteration.  Per parameter element (adam_kernel): one Adam step over the
// five parameter tensors as flat arrays, then the clamp of the log-scales that the reference's
// fit loop applies after opt.step() (fit.py:3033, 3359-3366).  The gradients pass through the
// fit workspace so the Adam pass streams four aligned arrays per tensor at full occupancy,
// as torch's multi-tensor Adam does.
//
// Adam is torch.optim.Adam's multi-tensor step (no weight decay, no amsgrad), element by element:
//   m <- lerp(m, g, 1 - beta1)            = m + (1 - beta1)(g - m)
//   v <- v beta2 + (1 - beta2) g^2
//   p <- p - lr / (1 - beta1^t) * m / (sqrt(v) / sqrt(1 - beta2^t) + eps)
// with the step-dependent factors formed in double and rounded to float as torch's Python-side
// scalars are, so the update reproduces the eager optimizer.
//
// The step count lives on the device (step_state[0]) so the update can be replayed from a CUDA
// graph: every thread of the Adam pass uses t = step_state[0] + 1 and its last CTA to finish
// stores t back (step_state[1] counts finished CTAs and is reset by that CTA).
#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

struct AdamHyper {
  double lr[5];  // means, log_scales, rotations, colors, opacity logits
  double beta1, beta2;
  float eps;
  float log_lo;
  float dilation;
};

struct FieldPtrs {
  float *means, *log_scales, *rotations, *colors, *logits;
};

struct AdamStep {
  float w1, b2, s2, bc2s, eps;  // lerp weight, beta2, 1 - beta2, sqrt(1 - beta2^t), eps
  double bc1;                    // 1 - beta1^t
};

__device__ __forceinline__ float adam(float p, float g, float& m, float& v, float step,
                                      const AdamStep& a) {
  m = fmaf(a.w1, g - m, m);
  v = fmaf(a.s2, g * g, v * a.b2);
  const float denom = sqrtf(v) / a.bc2s + a.eps;
  return fmaf(-step, m / denom, p);
}

// Inputs of one Gaussian's gradients: its nine summed moments, the record's opacity and conic,
// and the current log-scales, rotation and opacity logit.
struct GradIn {
  float m[kMoments];
  float op, a, b, c, ls0, ls1, th, lg;
};

__device__ __forceinline__ void load_grad_in(const Splat* __restrict__ rec,
                                             const float* __restrict__ log_scales,
                                             const float* __restrict__ rotations,
                                             const float* __restrict__ logits, int64_t g,
                                             GradIn& in) {
  const float4 p1 = reinterpret_cast<const float4*>(rec + g)[1];
  const float4 p2 = reinterpret_cast<const float4*>(rec + g)[2];
  in.op = p1.y;
  in.a = p2.y;
  in.b = p2.z;
  in.c = p2.w;
  in.ls0 = log_scales[2 * g];
  in.ls1 = log_scales[2 * g + 1];
  in.th = rotations[g];
  in.lg = logits ? logits[g] : 0.f;
}

// The same arithmetic as the plain backward epilogue, then the RS chain rule.
__device__ __forceinline__ void store_grads(const GradIn& in, int64_t g, float dilation,
                                            bool has_logits, const FieldPtrs& grad) {
  const float* m = in.m;
  float gls0, gls1, grot;
  rs_conic_chain(in.ls0, in.ls1, in.th, dilation, -0.5f * in.op * m[6], -in.op * m[7],
                 -0.5f * in.op * m[8], gls0, gls1, grot);
  grad.means[2 * g] = in.op * (in.a * m[4] + in.b * m[5]);
  grad.means[2 * g + 1] = in.op * (in.b * m[4] + in.c * m[5]);
  grad.log_scales[2 * g] = gls0;
  grad.log_scales[2 * g + 1] = gls1;
  grad.rotations[g] = grot;
  grad.colors[3 * g] = in.op * m[0];
  grad.colors[3 * g + 1] = in.op * m[1];
  grad.colors[3 * g + 2] = in.op * m[2];
  if (has_logits) grad.logits[g] = logit_chain(in.lg, m[3]);
}

// Per-Gaussian gradients of the five parameter groups: the summed moments (fast: the atomic
// accumulators, read and zeroed; deterministic: the entry partials in their fixed order) become
// render-input gradients, and the chain rule carries them to the RS parameters at their current
// values.  Grid-stride, a warp's 32 consecutive Gaussians per round (the deterministic sum is
// warp-collective); fast mode takes two rounds at a time with every load issued before the first
// store, so each thread keeps two Gaussians' loads in flight.  The gradients go to tensors shaped
// like the parameters.
template <bool DETERMINISTIC>
__global__ void __launch_bounds__(kThreads)
    fit_grad_kernel(const Splat* __restrict__ rec, int64_t n, float* __restrict__ moments,
                    const float* __restrict__ partials, const int32_t* __restrict__ order,
                    const int32_t* __restrict__ seg, const float* __restrict__ log_scales,
                    const float* __restrict__ rotations, const float* __restrict__ logits,
                    float dilation, FieldPtrs grad) {
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t first = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x - lane);
  if constexpr (DETERMINISTIC) {
    for (int64_t base = first; base < n; base += stride) {
      const int64_t g = base + lane;
      const bool active = g < n;
      GradIn in;
      sum_entry_partials(partials, order, seg, n, g, active, in.m);
      if (!active) continue;
      load_grad_in(rec, log_scales, rotations, logits, g, in);
      store_grads(in, g, dilation, logits != nullptr, grad);
    }
  } else {
  for (int64_t base = first; base < n; base += 2 * stride) {
    const int64_t g[2] = {base + lane, base + stride + lane};
    GradIn in[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (g[u] >= n) continue;
#pragma unroll
      for (int k = 0; k < kMoments; ++k) in[u].m[k] = moments[k * n + g[u]];
      load_grad_in(rec, log_scales, rotations, logits, g[u], in[u]);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      if (g[u] >= n) continue;
#pragma unroll
      for (int k = 0; k < kMoments; ++k) moments[k * n + g[u]] = 0.0f;
      store_grads(in[u], g[u], dilation, logits != nullptr, grad);
    }
  }
  }
}

// One parameter tensor of the Adam step: parameters, both moments, gradient and length; its
// position in AdamTensors is its learning-rate group.
struct AdamTensor {
  float *p, *m, *v;
  const float* g;
  int64_t len;
};
struct AdamTensors {
  AdamTensor t[5];  // means, log_scales, rotations, colors, opacity logits (len 0 if absent)
};

__device__ __forceinline__ float clamp_log_scale(float x, float hi, float lo) {
  x = x > hi ? hi : x;  // clamp_(max=hi) then clamp_(min=lo), NaN passing through as in torch
  return x < lo ? lo : x;
}

// The Adam step over the five tensors as flat arrays (four elements per access where every
// pointer allows it), each block taking a grid-stride share of every tensor; log-scales are
// clamped to [log_lo, log_hi[image]] after the step.  The step-dependent factors are formed
// once per thread; the last block to finish advances the device step count.
__global__ void __launch_bounds__(kThreads)
    adam_kernel(AdamTensors ts, AdamHyper h, Frames frames, const float* __restrict__ log_hi,
                int* __restrict__ step_state) {
  pdl_wait();
  pdl_trigger();
  const int t = step_state[0] + 1;
  AdamStep st;
  st.w1 = (float)(1.0 - h.beta1);
  st.b2 = (float)h.beta2;
  st.s2 = (float)(1.0 - h.beta2);
  st.bc2s = (float)sqrt(1.0 - pow(h.beta2, (double)t));
  st.eps = h.eps;
  st.bc1 = 1.0 - pow(h.beta1, (double)t);
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  auto hi_of = [&](int64_t e) {  // log-scale element e belongs to Gaussian e / 2
    return log_hi[frames.image ? frames.gauss_image[e >> 1] : 0];
  };
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const AdamTensor T = ts.t[k];
    const float step = (float)(h.lr[k] / st.bc1);
    const bool vec = ((reinterpret_cast<uintptr_t>(T.p) | reinterpret_cast<uintptr_t>(T.m) |
                       reinterpret_cast<uintptr_t>(T.v) | reinterpret_cast<uintptr_t>(T.g)) &
                      15) == 0;
    const int64_t n4 = vec ? T.len / 4 : 0;
    for (int64_t i = tid; i < n4; i += stride) {
      float4 p = reinterpret_cast<float4*>(T.p)[i];
      float4 m = reinterpret_cast<float4*>(T.m)[i];
      float4 v = reinterpret_cast<float4*>(T.v)[i];
      const float4 g = reinterpret_cast<const float4*>(T.g)[i];
      p.x = adam(p.x, g.x, m.x, v.x, step, st);
      p.y = adam(p.y, g.y, m.y, v.y, step, st);
      p.z = adam(p.z, g.z, m.z, v.z, step, st);
      p.w = adam(p.w, g.w, m.w, v.w, step, st);
      if (k == 1) {
        const float h0 = hi_of(4 * i), h1 = hi_of(4 * i + 2);
        p.x = clamp_log_scale(p.x, h0, h.log_lo);
        p.y = clamp_log_scale(p.y, h0, h.log_lo);
        p.z = clamp_log_scale(p.z, h1, h.log_lo);
        p.w = clamp_log_scale(p.w, h1, h.log_lo);
      }
      reinterpret_cast<float4*>(T.p)[i] = p;
      reinterpret_cast<float4*>(T.m)[i] = m;
      reinterpret_cast<float4*>(T.v)[i] = v;
    }
    for (int64_t e = 4 * n4 + tid; e < T.len; e += stride) {
      float m = T.m[e], v = T.v[e];
      float p = adam(T.p[e], T.g[e], m, v, step, st);
      if (k == 1) p = clamp_log_scale(p, hi_of(e), h.log_lo);
      T.p[e] = p;
      T.m[e] = m;
      T.v[e] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(step_state + 1, 1) == (int)gridDim.x - 1) {
      step_state[0] = t;
      step_state[1] = 0;
      __threadfence();
    }
  }
}
}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_fit_adam_update(const ss_batch* batch, const void* records, int64_t n,
                       const int32_t* tile_gids, int64_t gid_capacity,
                       const int32_t* tile_offsets, int deterministic, void* workspace,
                       float dilation, float* const* params, float* const* exp_avg,
                       float* const* exp_avg_sq, const double* lrs, double beta1, double beta2,
                       double adam_eps, float log_scale_lo, const float* log_scale_hi,
                       int* step_state, ss_stream_t stream) {
  Frames f;
  int rc = frames_of_batch(batch, n, &f);
  if (rc) return rc;
  if (!params || !exp_avg || !exp_avg_sq || !lrs || !step_state || !log_scale_hi)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (n == 0) return SS_OK;
  if (!records || !workspace) return fail(SS_ERR_INVALID_ARGUMENT, "null records or workspace");
  if (deterministic && (!tile_gids || !tile_offsets))
    return fail(SS_ERR_INVALID_ARGUMENT, "deterministic update needs the tile index");
  for (int k = 0; k < 4; ++k)
    if (!params[k] || !exp_avg[k] || !exp_avg_sq[k])
      return fail(SS_ERR_INVALID_ARGUMENT, "null field tensor %d", k);
  if ((params[4] != nullptr) != (exp_avg[4] != nullptr) ||
      (params[4] != nullptr) != (exp_avg_sq[4] != nullptr))
    return fail(SS_ERR_INVALID_ARGUMENT, "opacity logits and their Adam state go together");
  if (!(beta1 >= 0.0 && beta1 < 1.0 && beta2 >= 0.0 && beta2 < 1.0))
    return fail(SS_ERR_INVALID_ARGUMENT, "Adam betas must lie in [0, 1)");
  FieldPtrs p{params[0], params[1], params[2], params[3], params[4]};
  AdamHyper h;
  for (int k = 0; k < 5; ++k) h.lr[k] = lrs[k];
  h.beta1 = beta1;
  h.beta2 = beta2;
  h.eps = (float)adam_eps;
  h.log_lo = log_scale_lo;
  h.dilation = dilation;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const Splat* rec = static_cast<const Splat*>(records);
  float* ws = static_cast<float*>(workspace);
  const FitGrads fg = fit_grads_layout(
      static_cast<char*>(workspace) + fit_grads_offset(n, gid_capacity, deterministic), n);
  const FieldPtrs gp{fg.means, fg.log_scales, fg.rotations, fg.colors, p.logits ? fg.logits : nullptr};
  cudaStream_t s = as_stream(stream);
  // gradients: a grid of at most 8 blocks per SM, grid-stride beyond that
  const int64_t want = (n + kThreads - 1) / kThreads, cap_blocks = (int64_t)sms * 8;
  const unsigned blocks = (unsigned)(want < cap_blocks ? want : cap_blocks);
  if (deterministic) {
    const EntryOrder eo = entry_order_layout(workspace, n, gid_capacity);
    launch("fit_grad_kernel", fit_grad_kernel<true>, blocks, kThreads, 0, s, rec, n, nullptr, eo.partials, eo.order,
                                                      eo.seg, p.log_scales, p.rotations,
                                                      p.logits, dilation, gp);
  } else {
    launch("fit_grad_kernel", fit_grad_kernel<false>, blocks, kThreads, 0, s, rec, n, ws, nullptr, nullptr, nullptr,
                                                       p.log_scales, p.rotations, p.logits,
                                                       dilation, gp);
  }
  if ((rc = check_launch("fit gradients"))) return rc;
  // the Adam step over the five tensors as flat arrays
  AdamTensors ts;
  const int64_t lens[5] = {2 * n, 2 * n, n, 3 * n, p.logits ? n : 0};
  float* gptr[5] = {fg.means, fg.log_scales, fg.rotations, fg.colors, fg.logits};
  for (int k = 0; k < 5; ++k) {
    ts.t[k].p = params[k];
    ts.t[k].m = exp_avg[k];
    ts.t[k].v = exp_avg_sq[k];
    ts.t[k].g = gptr[k];
    ts.t[k].len = lens[k];
  }
  const int64_t want4 = (3 * n / 4 + kThreads - 1) / kThreads + 1;
  const unsigned ablocks = (unsigned)(want4 < cap_blocks ? want4 : cap_blocks);
  launch("adam_kernel", adam_kernel, ablocks, kThreads, 0, s, ts, h, f, log_scale_hi, step_state);
  return check_launch("fit adam step");
}

}  // extern "C"

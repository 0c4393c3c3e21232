// Per-Gaussian update of a fit iteration: the render backward's summed moments become conic /
// mean / colour / opacity gradients, the chain rule carries them to the RS field parameters
// (gaussians.py:270-300), one Adam step updates every parameter, and the log-scales are clamped
// as the reference's fit loop does after opt.step() (fit.py:3033, 3359-3366).  The moment
// accumulators are zeroed for the next iteration.
//
// Adam is torch.optim.Adam's multi-tensor step (no weight decay, no amsgrad), element by element:
//   m <- lerp(m, g, 1 - beta1)            = m + (1 - beta1)(g - m)
//   v <- v beta2 + (1 - beta2) g^2
//   p <- p - lr / (1 - beta1^t) * m / (sqrt(v) / sqrt(1 - beta2^t) + eps)
// with the step-dependent factors formed in double and rounded to float as torch's Python-side
// scalars are, so the update reproduces the eager optimizer.
//
// The step count lives on the device (step_state[0]) so the update can be replayed from a CUDA
// graph: every thread uses t = step_state[0] + 1 and the last CTA to finish stores t back
// (step_state[1] counts finished CTAs and is reset by that CTA).
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

template <bool DETERMINISTIC>
__global__ void __launch_bounds__(kThreads)
    fit_update_kernel(const Splat* __restrict__ rec, int64_t n, Frames frames,
                      float* __restrict__ moments, const float* __restrict__ partials,
                      const int32_t* __restrict__ order, const int32_t* __restrict__ seg,
                      FieldPtrs field, FieldPtrs exp_avg, FieldPtrs exp_avg_sq, AdamHyper h,
                      const float* __restrict__ log_hi, int* __restrict__ step_state) {
  const int t = step_state[0] + 1;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float m[kMoments];
  if (DETERMINISTIC) sum_entry_partials(partials, order, seg, n, g, g < n, m);
  if (g < n) {
    if (!DETERMINISTIC) {
#pragma unroll
      for (int k = 0; k < kMoments; ++k) {
        m[k] = moments[k * n + g];
        moments[k * n + g] = 0.0f;
      }
    }
    const float4 p1 = reinterpret_cast<const float4*>(rec + g)[1];
    const float4 p2 = reinterpret_cast<const float4*>(rec + g)[2];
    const float op = p1.y, a = p2.y, b = p2.z, c = p2.w;
    // gradients w.r.t. the render inputs (the same arithmetic as the plain backward epilogue)
    const float gm0 = op * (a * m[4] + b * m[5]), gm1 = op * (b * m[4] + c * m[5]);
    const float ga = -0.5f * op * m[6], gb = -op * m[7], gc = -0.5f * op * m[8];
    const float gcol[3] = {op * m[0], op * m[1], op * m[2]};
    // chain rule to log-scales, rotation and the logit
    float gls0, gls1, grot;
    rs_conic_chain(field.log_scales[2 * g], field.log_scales[2 * g + 1], field.rotations[g],
                   h.dilation, ga, gb, gc, gls0, gls1, grot);
    AdamStep st;
    st.w1 = (float)(1.0 - h.beta1);
    st.b2 = (float)h.beta2;
    st.s2 = (float)(1.0 - h.beta2);
    st.bc2s = (float)sqrt(1.0 - pow(h.beta2, (double)t));
    st.eps = h.eps;
    st.bc1 = 1.0 - pow(h.beta1, (double)t);
    float pm, pv;
#define SS_ADAM(PTR, IDX, GRAD, GROUP)                                                   \
  pm = exp_avg.PTR[IDX];                                                                 \
  pv = exp_avg_sq.PTR[IDX];                                                              \
  field.PTR[IDX] = adam(field.PTR[IDX], GRAD, pm, pv, (float)(h.lr[GROUP] / st.bc1), st); \
  exp_avg.PTR[IDX] = pm;                                                                 \
  exp_avg_sq.PTR[IDX] = pv
    if (field.logits) {  // before the update: the chain rule needs the current logit
      const float glogit = logit_chain(field.logits[g], m[3]);
      SS_ADAM(logits, g, glogit, 4);
    }
    SS_ADAM(means, 2 * g, gm0, 0);
    SS_ADAM(means, 2 * g + 1, gm1, 0);
    SS_ADAM(log_scales, 2 * g, gls0, 1);
    SS_ADAM(log_scales, 2 * g + 1, gls1, 1);
    SS_ADAM(rotations, g, grot, 2);
    SS_ADAM(colors, 3 * g, gcol[0], 3);
    SS_ADAM(colors, 3 * g + 1, gcol[1], 3);
    SS_ADAM(colors, 3 * g + 2, gcol[2], 3);
#undef SS_ADAM
    // clamp_(max=hi) then clamp_(min=lo), NaN passing through as in torch
    const float hi = log_hi[frames.image ? frames.gauss_image[g] : 0];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      float x = field.log_scales[2 * g + k];
      x = x > hi ? hi : x;
      x = x < h.log_lo ? h.log_lo : x;
      field.log_scales[2 * g + k] = x;
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
  FieldPtrs m{exp_avg[0], exp_avg[1], exp_avg[2], exp_avg[3], exp_avg[4]};
  FieldPtrs v{exp_avg_sq[0], exp_avg_sq[1], exp_avg_sq[2], exp_avg_sq[3], exp_avg_sq[4]};
  AdamHyper h;
  for (int k = 0; k < 5; ++k) h.lr[k] = lrs[k];
  h.beta1 = beta1;
  h.beta2 = beta2;
  h.eps = (float)adam_eps;
  h.log_lo = log_scale_lo;
  h.dilation = dilation;
  const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
  const Splat* rec = static_cast<const Splat*>(records);
  float* ws = static_cast<float*>(workspace);
  cudaStream_t s = as_stream(stream);
  if (deterministic) {
    const EntryOrder eo = entry_order_layout(workspace, n, gid_capacity);
    fit_update_kernel<true><<<blocks, kThreads, 0, s>>>(rec, n, f, nullptr, eo.partials,
                                                        eo.order, eo.seg, p, m, v, h,
                                                        log_scale_hi, step_state);
  } else {
    fit_update_kernel<false><<<blocks, kThreads, 0, s>>>(rec, n, f, ws, nullptr, nullptr,
                                                         nullptr, p, m, v, h, log_scale_hi,
                                                         step_state);
  }
  return check_launch("fit_adam_update");
}

}  // extern "C"

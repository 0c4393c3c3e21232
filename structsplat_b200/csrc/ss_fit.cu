// Fused per-Gaussian update of a fit iteration: the render backward's summed moments become
// conic / mean / colour / opacity gradients, the chain rule carries them to the RS field
// parameters (gaussians.py:270-300), and one Adam step (torch.optim.Adam: no weight decay, no
// amsgrad; bias corrections 1 - beta^t) updates every parameter, after which log-scales are
// clamped to [log_lo, log_hi] as the reference's fit loop does after opt.step()
// (fit.py:3033, 3359-3366).  The moment accumulators are zeroed for the next iteration.
//
// The step count lives on the device (step_state[0]) so the update can be replayed from a CUDA
// graph: every thread uses t = step_state[0] + 1 and the last CTA to finish stores t back
// (step_state[1] counts finished CTAs and is reset by that CTA).
#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

struct AdamHyper {
  float lr[5];  // means, log_scales, rotations, colors, opacity logits
  float beta1, beta2, eps;
  float log_lo, log_hi;
  float dilation;
};

struct FieldPtrs {
  float *means, *log_scales, *rotations, *colors, *logits;
};

// torch.optim.Adam's update of one value: m, v moments; bc2s = sqrt(1 - beta2^t).
__device__ __forceinline__ float adam(float p, float g, float& m, float& v, float lr_t,
                                      float bc2s, const AdamHyper& h) {
  m = h.beta1 * m + (1.0f - h.beta1) * g;
  v = h.beta2 * v + (1.0f - h.beta2) * g * g;
  const float denom = sqrtf(v) / bc2s + h.eps;
  return p - lr_t * (m / denom);
}

template <bool DETERMINISTIC>
__global__ void __launch_bounds__(kThreads)
    fit_update_kernel(const Splat* __restrict__ rec, int64_t n, float* __restrict__ moments,
                      const float* __restrict__ partials, const int32_t* __restrict__ gids,
                      int64_t cap, const int32_t* __restrict__ offsets, int tiles_x, int ts,
                      FieldPtrs field, FieldPtrs exp_avg, FieldPtrs exp_avg_sq, AdamHyper h,
                      int* __restrict__ step_state) {
  const int t = step_state[0] + 1;
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n) {
    float m[9];
    if (DETERMINISTIC) {
#pragma unroll
      for (int k = 0; k < 9; ++k) m[k] = 0.f;
      const int4 r = reinterpret_cast<const int4*>(rec + g)[3];
      if (r.z > r.x && r.w > r.y) {
        const int gx0 = r.x / ts, gx1 = (r.z - 1) / ts, gy0 = r.y / ts, gy1 = (r.w - 1) / ts;
        for (int gy = gy0; gy <= gy1; ++gy)
          for (int gx = gx0; gx <= gx1; ++gx) {
            const int tt = gy * tiles_x + gx;
            int64_t lo = offsets[tt], hi = offsets[tt + 1];
            if (hi > cap) continue;
            const int64_t end = hi;
            while (lo < hi) {
              const int64_t mid = (lo + hi) >> 1;
              if (gids[mid] < g) lo = mid + 1; else hi = mid;
            }
            if (lo < end && gids[lo] == g) {
#pragma unroll
              for (int k = 0; k < 9; ++k) m[k] += partials[lo * 12 + k];
            }
          }
      }
    } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) {
        m[k] = moments[k * n + g];
        moments[k * n + g] = 0.0f;
      }
    }
    const float4 p1 = reinterpret_cast<const float4*>(rec + g)[1];
    const float4 p2 = reinterpret_cast<const float4*>(rec + g)[2];
    const float op = p1.y, a = p2.y, b = p2.z, c = p2.w;
    // gradients w.r.t. the render inputs
    const float gm0 = op * (a * m[4] + b * m[5]), gm1 = op * (b * m[4] + c * m[5]);
    const float ga = -0.5f * op * m[6], gb = -op * m[7], gc = -0.5f * op * m[8];
    const float gcol[3] = {op * m[0], op * m[1], op * m[2]};
    const float gop = m[3];
    // chain rule to log-scales, rotation (see project_rs_backward_kernel) and the logit
    const float ls0 = field.log_scales[2 * g], ls1 = field.log_scales[2 * g + 1];
    const float th = field.rotations[g];
    const float sx = expf(ls0), sy = expf(ls1);
    const float sx2 = sx * sx, sy2 = sy * sy;
    const float u = 1.0f / (sx2 + h.dilation), v = 1.0f / (sy2 + h.dilation);
    float sn, cs;
    sincosf(th, &sn, &cs);
    const float cc = cs * cs, s2 = sn * sn, csn = cs * sn;
    const float gu = ga * cc + gb * csn + gc * s2;
    const float gv = ga * s2 - gb * csn + gc * cc;
    const float gls0 = gu * (-2.0f * sx2 * u * u), gls1 = gv * (-2.0f * sy2 * v * v);
    const float grot = (u - v) * (2.0f * csn * (gc - ga) + (cc - s2) * gb);
    // Adam
    const float bc1 = 1.0f - powf(h.beta1, (float)t);
    const float bc2s = sqrtf(1.0f - powf(h.beta2, (float)t));
    float pm, pv;
#define SS_ADAM(PTR, IDX, GRAD, LR)                                                    \
  pm = exp_avg.PTR[IDX];                                                               \
  pv = exp_avg_sq.PTR[IDX];                                                            \
  field.PTR[IDX] = adam(field.PTR[IDX], GRAD, pm, pv, (LR) / bc1, bc2s, h);            \
  exp_avg.PTR[IDX] = pm;                                                               \
  exp_avg_sq.PTR[IDX] = pv
    SS_ADAM(means, 2 * g, gm0, h.lr[0]);
    SS_ADAM(means, 2 * g + 1, gm1, h.lr[0]);
    SS_ADAM(log_scales, 2 * g, gls0, h.lr[1]);
    SS_ADAM(log_scales, 2 * g + 1, gls1, h.lr[1]);
    SS_ADAM(rotations, g, grot, h.lr[2]);
    SS_ADAM(colors, 3 * g, gcol[0], h.lr[3]);
    SS_ADAM(colors, 3 * g + 1, gcol[1], h.lr[3]);
    SS_ADAM(colors, 3 * g + 2, gcol[2], h.lr[3]);
    if (field.logits) {
      const float o = 1.0f / (1.0f + expf(-field.logits[g]));
      SS_ADAM(logits, g, gop * o * (1.0f - o), h.lr[4]);
    }
#undef SS_ADAM
    field.log_scales[2 * g] = fminf(fmaxf(field.log_scales[2 * g], h.log_lo), h.log_hi);
    field.log_scales[2 * g + 1] = fminf(fmaxf(field.log_scales[2 * g + 1], h.log_lo), h.log_hi);
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

int ss_fit_update(const void* records, int64_t n, float* moments, const float* partials,
                  const int32_t* tile_gids, int64_t gid_capacity, const int32_t* tile_offsets,
                  int height, int width, int tile_size, float* const* params,
                  float* const* exp_avg, float* const* exp_avg_sq, const float* lrs,
                  float beta1, float beta2, float adam_eps, float log_scale_lo,
                  float log_scale_hi, float dilation, int* step_state, ss_stream_t stream) {
  if (n < 0 || height < 0 || width < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (!params || !exp_avg || !exp_avg_sq || !lrs || !step_state)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (n == 0) return SS_OK;
  const bool det = partials != nullptr;
  if (!det && !moments) return fail(SS_ERR_INVALID_ARGUMENT, "moments or partials required");
  if (det && (!tile_gids || !tile_offsets || tile_size <= 0))
    return fail(SS_ERR_INVALID_ARGUMENT, "deterministic update needs the tile index");
  for (int k = 0; k < 4; ++k)
    if (!params[k] || !exp_avg[k] || !exp_avg_sq[k])
      return fail(SS_ERR_INVALID_ARGUMENT, "null field tensor %d", k);
  if ((params[4] != nullptr) != (exp_avg[4] != nullptr) ||
      (params[4] != nullptr) != (exp_avg_sq[4] != nullptr))
    return fail(SS_ERR_INVALID_ARGUMENT, "opacity logits and their Adam state go together");
  FieldPtrs f{params[0], params[1], params[2], params[3], params[4]};
  FieldPtrs m{exp_avg[0], exp_avg[1], exp_avg[2], exp_avg[3], exp_avg[4]};
  FieldPtrs v{exp_avg_sq[0], exp_avg_sq[1], exp_avg_sq[2], exp_avg_sq[3], exp_avg_sq[4]};
  AdamHyper h;
  for (int k = 0; k < 5; ++k) h.lr[k] = lrs[k];
  h.beta1 = beta1;
  h.beta2 = beta2;
  h.eps = adam_eps;
  h.log_lo = log_scale_lo;
  h.log_hi = log_scale_hi;
  h.dilation = dilation;
  const int tiles_x = tile_size > 0 ? (width + tile_size - 1) / tile_size : 0;
  const unsigned blocks = (unsigned)((n + kThreads - 1) / kThreads);
  const Splat* rec = static_cast<const Splat*>(records);
  cudaStream_t s = as_stream(stream);
  if (det)
    fit_update_kernel<true><<<blocks, kThreads, 0, s>>>(rec, n, moments, partials, tile_gids,
                                                        gid_capacity, tile_offsets, tiles_x,
                                                        tile_size, f, m, v, h, step_state);
  else
    fit_update_kernel<false><<<blocks, kThreads, 0, s>>>(rec, n, moments, partials, tile_gids,
                                                         gid_capacity, tile_offsets, tiles_x,
                                                         tile_size, f, m, v, h, step_state);
  return check_launch("fit_update");
}

}  // extern "C"

// SSIM term of the fit loss, forward and gradient, over a batch of images: metrics.py:130-150
// (the builtin backend: 11-tap Gaussian window, sigma 1.5, zero padding, C1 = 0.01^2,
// C2 = 0.03^2, mean over channels and pixels) mixed as fit.py:3244 does,
//   loss = (1 - w) pixel_loss + w (1 - SSIM).
//
// Per image and channel, with G the separable window (zero padding) and p / t the rendered and
// target channels:
//   mu_p = G p, E_pp = G p^2, E_pt = G (p t), mu_t = G t, sig_t = G t^2 - mu_t^2 (constant over
//   a fit: ss_ssim_target_stats computes it once, as SSIMTargetStats does, metrics.py:85-118)
//   A1 = 2 mu_p mu_t + C1, A2 = 2 (E_pt - mu_p mu_t) + C2, B1 = mu_p^2 + mu_t^2 + C1,
//   B2 = (E_pp - mu_p^2) + sig_t + C2, S = A1 A2 / (B1 B2).
// The gradient of SSIM = mean S at pixel q is (1/N) (G a + 2 p G b + t G c)(q) with the maps
//   a = dS/dmu_p = (2 mu_t (A2 - A1) - S 2 mu_p (B2 - B1)) / (B1 B2),
//   b = dS/dE_pp = -S / B2,   c = dS/dE_pt = 2 A1 / (B1 B2),
// because the zero-padded symmetric window is its own adjoint.  Four passes over the batch
// (per pixel), or, on the tile grid of a render batch (tile sizes 16 and 32), two tile passes
// and a per-pixel fold: one CTA per tile for the horizontal then vertical window of
// (p, p^2, p t) and the maps of all three channels; one CTA per (tile, channel) for the
// horizontal then vertical window of (a, b, c) and the gradient.
// The last step folds -w dSSIM/dp, with (1 - w) times the pixel loss's part already in
// pixel_grad, through the normalisation into pixel_grad.
#include <cmath>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;
constexpr int kRadius = 5;  // 11 taps
constexpr float kC1 = 0.01f * 0.01f, kC2 = 0.03f * 0.03f;

struct Window {
  float g[2 * kRadius + 1];
};

// The reference's window: x = k - 5, exp(-x^2 / (2 sigma^2)), divided by its sum, in float.
Window ssim_window() {
  Window w;
  float sum = 0.f;
  for (int k = 0; k <= 2 * kRadius; ++k) {
    const float x = (float)(k - kRadius);
    w.g[k] = (float)std::exp((double)(-(x * x) / (2.0f * 1.5f * 1.5f)));
    sum += w.g[k];
  }
  for (int k = 0; k <= 2 * kRadius; ++k) w.g[k] /= sum;
  return w;
}

// Image of pixel p of the concatenated batch: the last image whose first pixel is <= p (an
// empty image shares its first pixel with the next one).
__device__ __forceinline__ int image_of_pixel(const int64_t* __restrict__ pixel_base, int B,
                                              int64_t p) {
  int lo = 0, hi = B - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pixel_base[mid] <= p) lo = mid; else hi = mid - 1;
  }
  return lo;
}

struct Geo {
  const int32_t* table;      // (B,4): H, W, tiles_x, first_tile
  const int64_t* pixel_base;  // (B)
  int B;
  int64_t P;
};

struct PixelAt {
  int b, H, W, x, y;
  int64_t base;
};

__device__ __forceinline__ PixelAt locate(const Geo& g, int64_t p) {
  PixelAt a;
  a.b = image_of_pixel(g.pixel_base, g.B, p);
  a.H = g.table[4 * a.b];
  a.W = g.table[4 * a.b + 1];
  a.base = g.pixel_base[a.b];
  const int64_t local = p - a.base;
  a.y = (int)(local / a.W);
  a.x = (int)(local - (int64_t)a.y * a.W);
  return a;
}

// Horizontal window of the products of one (P,3) image and, optionally, a second one: map m of
// channel c goes to out[(3 c + m) P + p]; MODE 0: (p, p^2, p t) of image and target; MODE 1:
// (t, t^2) of the target only (out[(2 c + m) P + p]).
template <int MODE>
__global__ void __launch_bounds__(kThreads)
    window_products_h_kernel(const float* __restrict__ img, const float* __restrict__ tgt, Geo geo,
                             Window win, float* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= geo.P) return;
  const PixelAt a = locate(geo, p);
  constexpr int kMaps = MODE == 0 ? 3 : 2;
  float acc[3][kMaps];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int m = 0; m < kMaps; ++m) acc[c][m] = 0.f;
#pragma unroll
  for (int k = -kRadius; k <= kRadius; ++k) {
    const int xx = a.x + k;
    if (xx < 0 || xx >= a.W) continue;
    const float g = win.g[k + kRadius];
    const int64_t q = p + k;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (MODE == 0) {
        const float v = img[3 * q + c], t = tgt[3 * q + c];
        acc[c][0] = fmaf(g, v, acc[c][0]);
        acc[c][1] = fmaf(g, v * v, acc[c][1]);
        acc[c][2] = fmaf(g, v * t, acc[c][2]);
      } else {
        const float t = tgt[3 * q + c];
        acc[c][0] = fmaf(g, t, acc[c][0]);
        acc[c][1] = fmaf(g, t * t, acc[c][1]);
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int m = 0; m < kMaps; ++m) out[(int64_t)(kMaps * c + m) * geo.P + p] = acc[c][m];
}

// Vertical window of `maps` SoA maps at pixel p (zero outside the image).
template <int MAPS>
__device__ __forceinline__ void window_v(const float* __restrict__ src, const Geo& geo,
                                         const PixelAt& a, int64_t p, const Window& win,
                                         float (&acc)[MAPS]) {
#pragma unroll
  for (int m = 0; m < MAPS; ++m) acc[m] = 0.f;
#pragma unroll
  for (int k = -kRadius; k <= kRadius; ++k) {
    const int yy = a.y + k;
    if (yy < 0 || yy >= a.H) continue;
    const float g = win.g[k + kRadius];
    const int64_t q = p + (int64_t)k * a.W;
#pragma unroll
    for (int m = 0; m < MAPS; ++m) acc[m] = fmaf(g, src[(int64_t)m * geo.P + q], acc[m]);
  }
}

// The target statistics: mu_t (3 maps) and sig_t (3 maps) from the horizontal pass of (t, t^2).
__global__ void __launch_bounds__(kThreads)
    target_stats_v_kernel(const float* __restrict__ h, Geo geo, Window win,
                          float* __restrict__ stats) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= geo.P) return;
  const PixelAt a = locate(geo, p);
  float acc[6];
  window_v<6>(h, geo, a, p, win, acc);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float mu = acc[2 * c], mu2 = mu * mu;
    stats[(int64_t)c * geo.P + p] = mu;
    stats[(int64_t)(3 + c) * geo.P + p] = acc[2 * c + 1] - mu2;
  }
}

// The SSIM maps: vertical window of (p, p^2, p t) per channel (h: 9 maps), S summed into the
// image's SSIM (mean over its 3 H W values, float atomics), and the maps a, b, c per channel
// into abc[(3 c + m) P + p].
__global__ void __launch_bounds__(kThreads)
    ssim_maps_kernel(const float* __restrict__ h, const float* __restrict__ stats, Geo geo,
                     Window win, float* __restrict__ abc, float* __restrict__ ssim) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = p < geo.P;
  float ssum = 0.f;
  int b = -1;
  float inv_n = 0.f;
  if (in) {
    const PixelAt a = locate(geo, p);
    b = a.b;
    inv_n = 1.0f / (float)(3 * (int64_t)a.H * a.W);
    float acc[9];
    window_v<9>(h, geo, a, p, win, acc);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float mu_p = acc[3 * c], e_pp = acc[3 * c + 1], e_pt = acc[3 * c + 2];
      const float mu_t = stats[(int64_t)c * geo.P + p], sig_t = stats[(int64_t)(3 + c) * geo.P + p];
      const float mu_p2 = mu_p * mu_p, mu_pt = mu_p * mu_t, mu_t2 = mu_t * mu_t;
      const float A1 = 2.0f * mu_pt + kC1, A2 = 2.0f * (e_pt - mu_pt) + kC2;
      const float B1 = mu_p2 + mu_t2 + kC1, B2 = (e_pp - mu_p2) + sig_t + kC2;
      const float D = B1 * B2;
      const float S = (A1 * A2) / D;
      ssum += S;
      abc[(int64_t)(3 * c) * geo.P + p] =
          (2.0f * mu_t * (A2 - A1) - S * 2.0f * mu_p * (B2 - B1)) / D;
      abc[(int64_t)(3 * c + 1) * geo.P + p] = -S / B2;
      abc[(int64_t)(3 * c + 2) * geo.P + p] = 2.0f * A1 / D;
    }
  }
  if (!ssim) return;
  // a warp whose pixels lie in one image adds once, otherwise every lane adds its own
  const int lane = threadIdx.x & 31;
  const int b0 = __shfl_sync(0xffffffffu, b, 0);
  if (__all_sync(0xffffffffu, b == b0 || b < 0)) {
    float v = ssum * inv_n;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0 && b0 >= 0) atomicAdd(ssim + b0, v);
  } else if (in) {
    atomicAdd(ssim + b, ssum * inv_n);
  }
}

// Horizontal window of 9 SoA maps (zero outside the image).
__global__ void __launch_bounds__(kThreads)
    window_h9_kernel(const float* __restrict__ src, Geo geo, Window win, float* __restrict__ dst) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= geo.P) return;
  const PixelAt a = locate(geo, p);
  float acc[9];
#pragma unroll
  for (int m = 0; m < 9; ++m) acc[m] = 0.f;
#pragma unroll
  for (int k = -kRadius; k <= kRadius; ++k) {
    const int xx = a.x + k;
    if (xx < 0 || xx >= a.W) continue;
    const float g = win.g[k + kRadius];
#pragma unroll
    for (int m = 0; m < 9; ++m) acc[m] = fmaf(g, src[(int64_t)m * geo.P + p + k], acc[m]);
  }
#pragma unroll
  for (int m = 0; m < 9; ++m) dst[(int64_t)m * geo.P + p] = acc[m];
}

// dSSIM/dp = (G a + 2 p G b + t G c) / N per channel (vertical window of the horizontal pass
// of a, b, c), then pixel_grad <- (1 - w) pixel_grad + V(-w dSSIM/dp), V the map from an image
// gradient g to the backward's per-pixel input: (g / (den + eps), -(g . image) / (den + eps)) in
// normalized mode, (g, 0) in additive mode.
__global__ void __launch_bounds__(kThreads)
    ssim_grad_kernel(const float* __restrict__ h, const float* __restrict__ img,
                     const float* __restrict__ tgt, const float* __restrict__ den, Geo geo,
                     Window win, int normalize, float eps, float weight,
                     float4* __restrict__ pixel_grad) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= geo.P) return;
  const PixelAt a = locate(geo, p);
  const float inv_n = 1.0f / (float)(3 * (int64_t)a.H * a.W);
  float acc[9];
  window_v<9>(h, geo, a, p, win, acc);
  float g[3], o[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o[c] = img[3 * p + c];
    const float t = tgt[3 * p + c];
    const float ds = (acc[3 * c] + 2.0f * o[c] * acc[3 * c + 1] + t * acc[3 * c + 2]) * inv_n;
    g[c] = -weight * ds;
  }
  float4 v = pixel_grad[p];
  const float keep = 1.0f - weight;
  v.x *= keep;
  v.y *= keep;
  v.z *= keep;
  v.w *= keep;
  if (normalize) {
    const float d = den[p] + eps;
    v.x += g[0] / d;
    v.y += g[1] / d;
    v.z += g[2] / d;
    v.w += -(g[0] * o[0] + g[1] * o[1] + g[2] * o[2]) / d;
  } else {
    v.x += g[0];
    v.y += g[1];
    v.z += g[2];
  }
  pixel_grad[p] = v;
}

// The same two windows per pass, one CTA per tile of the batch's tile grid (TS x TS pixels):
// the tile's inputs with a kRadius halo are staged in shared memory (zeros outside the image,
// the zero padding), the horizontal pass runs over all halo rows, the vertical pass over the
// tile, channel by channel.  The taps are summed in the order of the per-pixel kernels above
// (the same results to float rounding), with one global read of each input instead of eleven.
constexpr int kTileThreads = 256;
constexpr int kRun = 4;  // consecutive outputs per thread in a window pass

// Window of `M` arrays along a line: out[m][o] = sum_k g[k] in[m][(o + k) * stride] for the
// kRun outputs o of one thread, the 10 + kRun inputs loaded once into registers.
template <int M>
__device__ __forceinline__ void window_run(const float* const (&in)[M], int stride,
                                           const Window& win, float (&out)[M][kRun]) {
#pragma unroll
  for (int m = 0; m < M; ++m) {
    float v[2 * kRadius + kRun];
#pragma unroll
    for (int i = 0; i < 2 * kRadius + kRun; ++i) v[i] = in[m][i * stride];
#pragma unroll
    for (int o = 0; o < kRun; ++o) {
      float a = 0.f;
#pragma unroll
      for (int k = 0; k <= 2 * kRadius; ++k) a = fmaf(win.g[k], v[o + k], a);
      out[m][o] = a;
    }
  }
}

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

// The maps of all three channels of a tile in one CTA: the tile and its halo of image and target
// (RGB interleaved) are copied into shared memory once, as whole rows (a CTA per channel would
// fetch the same interleaved rows three times), then each channel runs the horizontal window of
// (p, p^2, p t), formed from the raw values as it goes, and the vertical window and the maps.
template <int TS>
struct Maps3Smem {
  static constexpr int R = TS + 2 * kRadius;
  static constexpr size_t kRaw = (size_t)6 * R * R;  // image then target, channel planes
  static constexpr size_t kHs = (size_t)3 * R * TS;
  static constexpr size_t kBytes = (kRaw + kHs) * sizeof(float);
};

template <int TS>
__global__ void __launch_bounds__(kTileThreads)
    ssim_maps_tile3_kernel(const float* __restrict__ img, const float* __restrict__ tgt,
                           const float* __restrict__ stats, Frames frames, int64_t P, Window win,
                           float* __restrict__ abc, float* __restrict__ ssim) {
  pdl_wait();
  pdl_trigger();
  constexpr int R = TS + 2 * kRadius;
  constexpr int kGroups = TS / kRun;
  extern __shared__ float m3_smem[];
  float* raw = m3_smem;                       // [6][R * R]: image c, then target c
  float* hs = m3_smem + Maps3Smem<TS>::kRaw;  // [3][R * TS]
  __shared__ float red[kTileThreads / 32];
  const Frame fr = frame_of_tile(frames, blockIdx.x, 0);
  const int local = blockIdx.x - fr.first_tile;
  const int tx0 = (local % fr.tiles_x) * TS, ty0 = (local / fr.tiles_x) * TS;
  const int H = fr.H, W = fr.W;
  for (int i = threadIdx.x; i < R * 3 * R; i += kTileThreads) {
    const int row = i / (3 * R), f = i - row * (3 * R);
    const int xi = f / 3, ch = f - 3 * xi;
    const int x = tx0 - kRadius + xi, y = ty0 - kRadius + row;
    float* di = raw + ch * (R * R) + row * R + xi;
    float* dt = di + 3 * (R * R);
    if (x >= 0 && x < W && y >= 0 && y < H) {
      const int64_t q = 3 * (fr.pixel_base + (int64_t)y * W + x) + ch;
      cp_async4(di, img + q);
      cp_async4(dt, tgt + q);
    } else {
      *di = 0.f;
      *dt = 0.f;
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  __syncthreads();
  float ssum = 0.f;
  for (int c = 0; c < 3; ++c) {
    const float* rp = raw + c * (R * R);
    const float* rt = raw + (3 + c) * (R * R);
    for (int w = threadIdx.x; w < R * kGroups; w += kTileThreads) {
      const int r = w / kGroups, x0 = (w % kGroups) * kRun;
      float v[2 * kRadius + kRun], pp[2 * kRadius + kRun], pt[2 * kRadius + kRun];
#pragma unroll
      for (int i = 0; i < 2 * kRadius + kRun; ++i) {
        const float a = rp[r * R + x0 + i], t = rt[r * R + x0 + i];
        v[i] = a;
        pp[i] = a * a;
        pt[i] = a * t;
      }
#pragma unroll
      for (int o = 0; o < kRun; ++o) {
        float a0 = 0.f, a1 = 0.f, a2 = 0.f;
#pragma unroll
        for (int k = 0; k <= 2 * kRadius; ++k) {
          a0 = fmaf(win.g[k], v[o + k], a0);
          a1 = fmaf(win.g[k], pp[o + k], a1);
          a2 = fmaf(win.g[k], pt[o + k], a2);
        }
        hs[0 * R * TS + r * TS + x0 + o] = a0;
        hs[1 * R * TS + r * TS + x0 + o] = a1;
        hs[2 * R * TS + r * TS + x0 + o] = a2;
      }
    }
    __syncthreads();
    for (int w = threadIdx.x; w < TS * kGroups; w += kTileThreads) {
      const int x = w % TS, y0 = (w / TS) * kRun;
      const float* const in[3] = {&hs[0 * R * TS + y0 * TS + x], &hs[1 * R * TS + y0 * TS + x],
                                  &hs[2 * R * TS + y0 * TS + x]};
      float out[3][kRun];
      window_run<3>(in, TS, win, out);
#pragma unroll
      for (int o = 0; o < kRun; ++o) {
        const int y = y0 + o;
        if (tx0 + x >= W || ty0 + y >= H) continue;
        const float mu_p = out[0][o], e_pp = out[1][o], e_pt = out[2][o];
        const int64_t p = fr.pixel_base + (int64_t)(ty0 + y) * W + tx0 + x;
        const float mu_t = stats[(int64_t)c * P + p], sig_t = stats[(int64_t)(3 + c) * P + p];
        const float mu_p2 = mu_p * mu_p, mu_pt = mu_p * mu_t, mu_t2 = mu_t * mu_t;
        const float A1 = 2.0f * mu_pt + kC1, A2 = 2.0f * (e_pt - mu_pt) + kC2;
        const float B1 = mu_p2 + mu_t2 + kC1, B2 = (e_pp - mu_p2) + sig_t + kC2;
        const float D = B1 * B2;
        const float S = (A1 * A2) / D;
        ssum += S;
        abc[(int64_t)(3 * c) * P + p] = (2.0f * mu_t * (A2 - A1) - S * 2.0f * mu_p * (B2 - B1)) / D;
        abc[(int64_t)(3 * c + 1) * P + p] = -S / B2;
        abc[(int64_t)(3 * c + 2) * P + p] = 2.0f * A1 / D;
      }
    }
    __syncthreads();  // hs is rewritten by the next channel
  }
  if (!ssim) return;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) ssum += __shfl_xor_sync(0xffffffffu, ssum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ssum;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < kTileThreads / 32; ++w) t += red[w];
    atomicAdd(ssim + fr.image, t / (float)(3 * (int64_t)H * W));
  }
}

// The adjoint window and the gradient of one channel per CTA (blockIdx.y): thread (x, y0) of
// the tile owns the kRun pixels (x, y0 .. y0 + kRun - 1); their -w dSSIM/dp goes to
// gbuf[c P + p] for ssim_fold_kernel.
template <int TS>
__global__ void __launch_bounds__(kTileThreads)
    ssim_grad_tile_kernel(const float* __restrict__ abc, const float* __restrict__ img,
                          const float* __restrict__ tgt, Frames frames, int64_t P, Window win,
                          float weight, float* __restrict__ gbuf) {
  pdl_wait();
  pdl_trigger();
  constexpr int R = TS + 2 * kRadius;
  constexpr int kGroups = TS / kRun;
  __shared__ float sm[3][R * R];
  __shared__ float hs[3][R * TS];
  const Frame fr = frame_of_tile(frames, blockIdx.x, 0);
  const int local = blockIdx.x - fr.first_tile;
  const int tx0 = (local % fr.tiles_x) * TS, ty0 = (local / fr.tiles_x) * TS;
  const int H = fr.H, W = fr.W;
  const int c = blockIdx.y;
  const float inv_n = 1.0f / (float)(3 * (int64_t)H * W);
  {
    // unrolled like the maps kernel's staging: every load in flight before the first store
    constexpr int kIters = (R * R + kTileThreads - 1) / kTileThreads;
    float a[kIters][3];
#pragma unroll
    for (int k = 0; k < kIters; ++k) {
      const int i = threadIdx.x + k * kTileThreads;
      const int xx = tx0 - kRadius + i % R, yy = ty0 - kRadius + i / R;
      const bool in = i < R * R && xx >= 0 && xx < W && yy >= 0 && yy < H;
      const int64_t q = fr.pixel_base + (int64_t)yy * W + xx;
#pragma unroll
      for (int m = 0; m < 3; ++m) a[k][m] = in ? abc[(int64_t)(3 * c + m) * P + q] : 0.f;
    }
#pragma unroll
    for (int k = 0; k < kIters; ++k) {
      const int i = threadIdx.x + k * kTileThreads;
      if (i < R * R) {
#pragma unroll
        for (int m = 0; m < 3; ++m) sm[m][i] = a[k][m];
      }
    }
  }
  __syncthreads();
  for (int w = threadIdx.x; w < R * kGroups; w += kTileThreads) {
    const int r = w / kGroups, x0 = (w % kGroups) * kRun;
    const float* const in[3] = {&sm[0][r * R + x0], &sm[1][r * R + x0], &sm[2][r * R + x0]};
    float out[3][kRun];
    window_run<3>(in, 1, win, out);
#pragma unroll
    for (int m = 0; m < 3; ++m)
#pragma unroll
      for (int k = 0; k < kRun; ++k) hs[m][r * TS + x0 + k] = out[m][k];
  }
  __syncthreads();
  if (threadIdx.x >= TS * kGroups) return;
  const int x = threadIdx.x % TS, y0 = (threadIdx.x / TS) * kRun;
  const float* const in[3] = {&hs[0][y0 * TS + x], &hs[1][y0 * TS + x], &hs[2][y0 * TS + x]};
  float out[3][kRun];
  window_run<3>(in, TS, win, out);
#pragma unroll
  for (int j = 0; j < kRun; ++j) {
    if (tx0 + x >= W || ty0 + y0 + j >= H) continue;
    const int64_t p = fr.pixel_base + (int64_t)(ty0 + y0 + j) * W + tx0 + x;
    const float o = img[3 * p + c], t = tgt[3 * p + c];
    gbuf[(int64_t)c * P + p] = -weight * ((out[0][j] + 2.0f * o * out[1][j] + t * out[2][j]) *
                                          inv_n);
  }
}

// pixel_grad <- (1 - w) pixel_grad + V(g) with g = gbuf's three channels (see ssim_grad_kernel).
__global__ void __launch_bounds__(kThreads)
    ssim_fold_kernel(const float* __restrict__ gbuf, const float* __restrict__ img,
                     const float* __restrict__ den, int64_t P, int normalize, float eps,
                     float weight, float4* __restrict__ pixel_grad) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float g0 = gbuf[p], g1 = gbuf[P + p], g2 = gbuf[2 * P + p];
  float4 v = pixel_grad[p];
  const float keep = 1.0f - weight;
  v.x *= keep;
  v.y *= keep;
  v.z *= keep;
  v.w *= keep;
  if (normalize) {
    const float d = den[p] + eps;
    v.x += g0 / d;
    v.y += g1 / d;
    v.z += g2 / d;
    v.w += -(g0 * img[3 * p] + g1 * img[3 * p + 1] + g2 * img[3 * p + 2]) / d;
  } else {
    v.x += g0;
    v.y += g1;
    v.z += g2;
  }
  pixel_grad[p] = v;
}

Geo geo_of(const ss_batch* b) {
  Geo g;
  g.table = b->image_table;
  g.pixel_base = b->pixel_base;
  g.B = b->images;
  g.P = b->pixels;
  return g;
}

unsigned blocks_for(int64_t P) { return (unsigned)((P + kThreads - 1) / kThreads); }

int check_ssim_batch(const ss_batch* b) {
  if (!b) return fail(SS_ERR_INVALID_ARGUMENT, "null batch");
  if (b->images < 1) return fail(SS_ERR_INVALID_ARGUMENT, "batch needs at least one image");
  if (b->pixels < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative pixel count");
  if (b->pixels > 0 && (!b->image_table || !b->pixel_base))
    return fail(SS_ERR_INVALID_ARGUMENT, "batch tables missing");
  if (b->pixels > ((int64_t)1 << 40)) return fail(SS_ERR_INVALID_ARGUMENT, "batch too large");
  return SS_OK;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_ssim_workspace_bytes(int64_t pixels, size_t* bytes) {
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  if (pixels < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative pixel count");
  *bytes = (size_t)18 * sizeof(float) * (size_t)(pixels > 0 ? pixels : 1);
  return SS_OK;
}

int ss_ssim_target_stats(const ss_batch* batch, const float* target, float* stats,
                         void* workspace, size_t workspace_bytes, ss_stream_t stream) {
  int rc = check_ssim_batch(batch);
  if (rc) return rc;
  const int64_t P = batch->pixels;
  if (P == 0) return SS_OK;
  if (!target || !stats || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "null target, stats or workspace");
  size_t need = 0;
  ss_ssim_workspace_bytes(P, &need);
  if (workspace_bytes < need) return fail(SS_ERR_INVALID_ARGUMENT, "ssim workspace too small");
  const Geo geo = geo_of(batch);
  const Window win = ssim_window();
  cudaStream_t s = as_stream(stream);
  float* h = static_cast<float*>(workspace);
  launch("ssim target window", window_products_h_kernel<1>, blocks_for(P), kThreads, 0, s,
         nullptr, target, geo, win, h);
  launch("ssim target stats", target_stats_v_kernel, blocks_for(P), kThreads, 0, s, h, geo, win,
         stats);
  return check_launch("ssim target stats");
}

int ss_fit_ssim(const ss_batch* batch, const float* image, const float* den, const float* target,
                const float* stats, int normalize, float eps, float ssim_weight,
                float* pixel_grad, float* ssim, void* workspace, size_t workspace_bytes,
                ss_stream_t stream) {
  int rc = check_ssim_batch(batch);
  if (rc) return rc;
  if (!(ssim_weight >= 0.0f && ssim_weight <= 1.0f))
    return fail(SS_ERR_INVALID_ARGUMENT, "ssim_weight must lie in [0, 1]");
  if (normalize && !(eps > 0.0f && std::isfinite(eps)))
    return fail(SS_ERR_INVALID_ARGUMENT, "normalization_eps must be finite and > 0");
  const int64_t P = batch->pixels;
  if (P == 0) return SS_OK;
  if (!image || !target || !stats || !pixel_grad || !workspace || (normalize && !den))
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (reinterpret_cast<uintptr_t>(pixel_grad) % 16)
    return fail(SS_ERR_INVALID_ARGUMENT, "pixel_grad must be 16-byte aligned");
  size_t need = 0;
  ss_ssim_workspace_bytes(P, &need);
  if (workspace_bytes < need) return fail(SS_ERR_INVALID_ARGUMENT, "ssim workspace too small");
  const Geo geo = geo_of(batch);
  const Window win = ssim_window();
  cudaStream_t s = as_stream(stream);
  float* h = static_cast<float*>(workspace);
  float* abc = h + 9 * P;
  Frames f;
  const int ts = batch->tile_size;
  if ((ts == 16 || ts == 32) && batch->tiles > 0 && batch->tiles <= (int64_t)INT32_MAX &&
      frames_of_batch(batch, 0, &f) == SS_OK) {  // the tile grid of a render batch
    const dim3 grid((unsigned)batch->tiles, 3);  // the gradient: (tile, channel)
    float4* pg = reinterpret_cast<float4*>(pixel_grad);
    float* gbuf = h;  // 3P: each channel's -w dSSIM/dp
    if (ts == 32) {
      launch_smem("ssim maps", ssim_maps_tile3_kernel<32>, dim3((unsigned)batch->tiles, 1),
                  kTileThreads, Maps3Smem<32>::kBytes, s, image, target, stats, f, P, win, abc,
                  ssim);
      launch("ssim gradient", ssim_grad_tile_kernel<32>, grid, kTileThreads, 0, s, abc, image,
             target, f, P, win, ssim_weight, gbuf);
    } else {
      launch_smem("ssim maps", ssim_maps_tile3_kernel<16>, dim3((unsigned)batch->tiles, 1),
                  kTileThreads, Maps3Smem<16>::kBytes, s, image, target, stats, f, P, win, abc,
                  ssim);
      launch("ssim gradient", ssim_grad_tile_kernel<16>, grid, kTileThreads, 0, s, abc, image,
             target, f, P, win, ssim_weight, gbuf);
    }
    launch("ssim fold", ssim_fold_kernel, blocks_for(P), kThreads, 0, s, gbuf, image, den, P,
           normalize, eps, ssim_weight, pg);
    return check_launch("fit ssim");
  }
  const unsigned blocks = blocks_for(P);
  launch("ssim window", window_products_h_kernel<0>, blocks, kThreads, 0, s, image, target, geo,
         win, h);
  launch("ssim maps", ssim_maps_kernel, blocks, kThreads, 0, s, h, stats, geo, win, abc, ssim);
  launch("ssim adjoint window", window_h9_kernel, blocks, kThreads, 0, s, abc, geo, win, h);
  launch("ssim gradient", ssim_grad_kernel, blocks, kThreads, 0, s, h, image, target, den, geo,
         win, normalize, eps, ssim_weight, reinterpret_cast<float4*>(pixel_grad));
  return check_launch("fit ssim");
}

}  // extern "C"

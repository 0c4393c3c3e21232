// Structure tensor J = G_rho * (grad I grad I^T) and its eigen-analysis, on the GPU.
//
// Follows structure_tensor.py:137-186 of the reference (NumPy there): source maps (Rec.709 luma,
// or the colour channels for the Di Zenzo tensor) are blurred separably with reflect padding
// (axis 0 then axis 1, taps accumulated in order with separately rounded products and sums, as
// NumPy's `acc += w * padded_slice` does), differentiated (np.gradient central differences,
// or 3x3 Sobel / Scharr correlation with reflect padding), the outer products are summed over
// channels and blurred again, and the closed-form eigen-analysis gives lam1, lam2, the
// across-edge angle, coherence and energy.  The flat / edge / corner labels need the energy's
// median and 99th percentile (float64, NumPy 'linear' interpolation): the energies are
// radix-sorted on the device and one thread evaluates the statistics.
#include <cub/device/device_radix_sort.cuh>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kMaxRadius = 31;

struct Taps {
  float w[2 * kMaxRadius + 1];
  int r;
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// np.pad(mode="reflect"): mirror about the edge samples without repeating them; repeated
// reflection (period 2(n-1)) for pads longer than the axis.
__device__ __forceinline__ int reflect(int i, int n) {
  if (n == 1) return 0;
  const int period = 2 * (n - 1);
  i %= period;
  if (i < 0) i += period;
  return i < n ? i : period - i;
}

// Source maps: luma (one map) or the first `chans` colour channels.
__global__ void source_maps_kernel(const float* __restrict__ img, int H, int W, int C,
                                   int rgb, float* __restrict__ maps) {
  pdl_wait();
  pdl_trigger();
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const int64_t p = (int64_t)y * W + x, HW = (int64_t)H * W;
  const float* px = img + p * C;
  if (C == 1) {
    maps[p] = px[0];
  } else if (rgb) {
    for (int c = 0; c < 3; ++c) maps[c * HW + p] = px[c];
  } else {
    // `img[..., :3] @ luma` evaluates as a fused multiply-add chain in NumPy's float32 dot.
    maps[p] = __fmaf_rn(px[2], 0.0722f, __fmaf_rn(px[1], 0.7152f, __fmul_rn(px[0], 0.2126f)));
  }
}

// One separable pass over `count` stacked (H,W) maps along y (axis 0) or x (axis 1).
template <bool ALONG_Y>
__global__ void blur_kernel(const float* __restrict__ src, float* __restrict__ dst, int H, int W,
                            Taps taps) {
  pdl_wait();
  pdl_trigger();
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const int64_t HW = (int64_t)H * W;
  const float* m = src + blockIdx.z * HW;
  float acc = 0.0f;
  for (int k = -taps.r; k <= taps.r; ++k) {
    const float v = ALONG_Y ? m[(int64_t)reflect(y + k, H) * W + x] : m[(int64_t)y * W + reflect(x + k, W)];
    acc = __fadd_rn(acc, __fmul_rn(taps.w[k + taps.r], v));
  }
  dst[blockIdx.z * HW + (int64_t)y * W + x] = acc;
}

// Gradients of each smoothed map and the channel-summed outer products (Jxx, Jxy, Jyy).
__global__ void tensor_kernel(const float* __restrict__ maps, int chans, int H, int W,
                              int op, float* __restrict__ J) {
  pdl_wait();
  pdl_trigger();
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const int64_t HW = (int64_t)H * W, p = (int64_t)y * W + x;
  float jxx = 0.f, jxy = 0.f, jyy = 0.f;
  for (int c = 0; c < chans; ++c) {
    const float* g = maps + c * HW;
    float ix, iy;
    if (op == 0) {  // np.gradient: central inside, one-sided at the border
      if (x == 0) ix = __fsub_rn(g[p + 1], g[p]);
      else if (x == W - 1) ix = __fsub_rn(g[p], g[p - 1]);
      else ix = __fsub_rn(g[p + 1], g[p - 1]) * 0.5f;
      if (y == 0) iy = __fsub_rn(g[p + W], g[p]);
      else if (y == H - 1) iy = __fsub_rn(g[p], g[p - W]);
      else iy = __fsub_rn(g[p + W], g[p - W]) * 0.5f;
    } else {  // 3x3 correlation, reflect padding: kx = [-1 0 1; -2 0 2; -1 0 1]/8 or Scharr/32
      const float e = op == 1 ? 0.125f : 0.09375f, m = op == 1 ? 0.25f : 0.3125f;
      const float kx[3][3] = {{-e, 0.f, e}, {-m, 0.f, m}, {-e, 0.f, e}};
      float ax = 0.f, ay = 0.f;
      for (int dy = 0; dy < 3; ++dy) {
        const int yy = reflect(y + dy - 1, H);
        for (int dx = 0; dx < 3; ++dx) {
          const float v = g[(int64_t)yy * W + reflect(x + dx - 1, W)];
          ax = __fadd_rn(ax, __fmul_rn(kx[dy][dx], v));
          ay = __fadd_rn(ay, __fmul_rn(kx[dx][dy], v));
        }
      }
      ix = ax;
      iy = ay;
    }
    jxx = __fadd_rn(jxx, __fmul_rn(ix, ix));
    jxy = __fadd_rn(jxy, __fmul_rn(ix, iy));
    jyy = __fadd_rn(jyy, __fmul_rn(iy, iy));
  }
  J[p] = jxx;
  J[HW + p] = jxy;
  J[2 * HW + p] = jyy;
}

__global__ void eigen_kernel(const float* __restrict__ J, int64_t HW, float* __restrict__ lam1,
                             float* __restrict__ lam2, float* __restrict__ angle,
                             float* __restrict__ coherence, float* __restrict__ energy,
                             float* __restrict__ energy_keys) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  const float jxx = J[p], jxy = J[HW + p], jyy = J[2 * HW + p];
  const float half = __fmul_rn(0.5f, __fadd_rn(jxx, jyy));
  const float diff = __fmul_rn(0.5f, __fsub_rn(jxx, jyy));
  const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(diff, diff), __fmul_rn(jxy, jxy)));
  const float l1 = __fadd_rn(half, r);
  const float l2 = fmaxf(__fsub_rn(half, r), 0.0f);
  const float en = __fadd_rn(l1, l2);
  const float coh = __fdiv_rn(__fsub_rn(l1, l2), __fadd_rn(en, 1e-12f));
  lam1[p] = l1;
  lam2[p] = l2;
  angle[p] = __fmul_rn(0.5f, atan2f(__fmul_rn(2.0f, jxy), __fsub_rn(jxx, jyy)));
  coherence[p] = __fmul_rn(coh, coh);
  energy[p] = en;
  energy_keys[p] = en;
}

// NumPy 'linear' quantile of sorted float32 data, in float64 (index (n-1)q, lerp that switches
// to b - (b-a)(1-t) for t >= 0.5).
__device__ double quantile_sorted(const float* s, int64_t n, double q) {
  const double v = (double)(n - 1) * q;
  int64_t lo = (int64_t)floor(v);
  if (lo < 0) lo = 0;
  if (lo > n - 1) lo = n - 1;
  const int64_t hi = lo + 1 < n ? lo + 1 : n - 1;
  const double t = v - (double)lo;
  const double a = fmax((double)s[lo], 0.0), b = fmax((double)s[hi], 0.0);
  const double d = b - a;
  return t >= 0.5 ? b - d * (1.0 - t) : a + d * t;
}

__global__ void stats_kernel(const float* __restrict__ sorted, int64_t n, double flat_frac,
                             double* stats) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double med = 0.0;
  if (n > 0) {
    const double a = fmax((double)sorted[(n - 1) / 2], 0.0), b = fmax((double)sorted[n / 2], 0.0);
    med = (n & 1) ? b : (a + b) / 2.0;
  }
  const double p99 = n > 0 ? quantile_sorted(sorted, n, 0.99) : 0.0;
  const double ref = fmax(p99, 8.0 * med) + 1e-12;
  stats[0] = ref;
  stats[1] = fmax(flat_frac * ref, 1.5 * med);
  stats[2] = med;
  stats[3] = p99;
}

__global__ void label_kernel(const float* __restrict__ energy, const float* __restrict__ lam2,
                             int64_t HW, const double* __restrict__ stats, double corner_frac,
                             uint8_t* __restrict__ label) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  // The thresholds are Python floats compared against float32 arrays: NumPy casts them to
  // float32 first.
  const float flat_thr = (float)stats[1];
  const float corner_thr = (float)(corner_frac * stats[0]);
  const bool flat = energy[p] < flat_thr;
  const bool corner = lam2[p] > corner_thr && !flat;
  label[p] = flat ? 0 : (corner ? 2 : 1);
}

struct StWorkspace {
  float *src, *tmp, *J, *keys;
  void* sort_temp;
  size_t sort_bytes;
};

size_t sort_temp_bytes(int64_t n) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, bytes, (const float*)nullptr, (float*)nullptr, (int)n);
  return bytes;
}

size_t st_workspace_bytes(int64_t HW) {
  return 3 * align256(3 * HW * sizeof(float)) + align256(HW * sizeof(float)) +
         align256(sort_temp_bytes(HW));
}

StWorkspace carve_st(void* base, int64_t HW) {
  StWorkspace w;
  char* p = static_cast<char*>(base);
  w.src = reinterpret_cast<float*>(p);
  p += align256(3 * HW * sizeof(float));
  w.tmp = reinterpret_cast<float*>(p);
  p += align256(3 * HW * sizeof(float));
  w.J = reinterpret_cast<float*>(p);
  p += align256(3 * HW * sizeof(float));
  w.keys = reinterpret_cast<float*>(p);
  p += align256(HW * sizeof(float));
  w.sort_temp = p;
  w.sort_bytes = align256(sort_temp_bytes(HW));
  return w;
}

int make_taps(const float* host, int r, Taps* t) {
  if (r < 0 || r > kMaxRadius) return fail(SS_ERR_UNSUPPORTED, "blur radius %d exceeds %d", r, kMaxRadius);
  t->r = r;
  for (int k = 0; k < 2 * kMaxRadius + 1; ++k) t->w[k] = 0.f;
  if (r > 0) {
    if (!host) return fail(SS_ERR_INVALID_ARGUMENT, "null taps");
    for (int k = 0; k < 2 * r + 1; ++k) t->w[k] = host[k];
  }
  return SS_OK;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_structure_tensor_workspace_bytes(int height, int width, int channels, size_t* bytes) {
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  if (height < 0 || width < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  (void)channels;
  *bytes = st_workspace_bytes((int64_t)height * width);
  return SS_OK;
}

int ss_structure_tensor(const float* image, int height, int width, int channels,
                        const float* taps_grad, int radius_grad, const float* taps_tensor,
                        int radius_tensor, int gradient_operator, int color_space,
                        double flat_frac, double corner_frac, float* lam1, float* lam2,
                        float* angle, float* coherence, float* energy, uint8_t* label,
                        double* stats_dev, void* workspace, size_t workspace_bytes,
                        ss_stream_t stream) {
  if (height < 0 || width < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (channels != 1 && channels < 3)
    return fail(SS_ERR_INVALID_ARGUMENT, "channels must be 1 or >= 3, got %d", channels);
  if (gradient_operator < 0 || gradient_operator > 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "unknown gradient_operator %d", gradient_operator);
  if (color_space < 0 || color_space > 1)
    return fail(SS_ERR_INVALID_ARGUMENT, "unknown color_space %d", color_space);
  const int64_t HW = (int64_t)height * width;
  if (HW > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "image too large");
  if (gradient_operator == 0 && (height < 2 || width < 2))
    return fail(SS_ERR_INVALID_ARGUMENT,
                "central gradients need at least 2 pixels along each axis");
  if (HW == 0) return SS_OK;
  if (!image || !lam1 || !lam2 || !angle || !coherence || !energy || !label || !stats_dev ||
      !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (workspace_bytes < st_workspace_bytes(HW))
    return fail(SS_ERR_INVALID_ARGUMENT, "structure tensor workspace too small");
  Taps tg, tt;
  int rc = make_taps(taps_grad, radius_grad, &tg);
  if (rc) return rc;
  if ((rc = make_taps(taps_tensor, radius_tensor, &tt))) return rc;
  cudaStream_t s = as_stream(stream);
  StWorkspace w = carve_st(workspace, HW);
  const dim3 blk(32, 8), grd((width + 31) / 32, (height + 7) / 8);
  const int rgb = (color_space == 1 && channels >= 3) ? 1 : 0;
  const int chans = rgb ? 3 : 1;
  source_maps_kernel<<<grd, blk, 0, s>>>(image, height, width, channels, rgb, w.src);
  if ((rc = check_launch("structure source maps"))) return rc;
  const float* smoothed = w.src;
  if (tg.r > 0) {
    blur_kernel<true><<<dim3(grd.x, grd.y, chans), blk, 0, s>>>(w.src, w.tmp, height, width, tg);
    blur_kernel<false><<<dim3(grd.x, grd.y, chans), blk, 0, s>>>(w.tmp, w.src, height, width, tg);
  }
  tensor_kernel<<<grd, blk, 0, s>>>(smoothed, chans, height, width, gradient_operator, w.J);
  if ((rc = check_launch("structure gradients"))) return rc;
  const float* Jb = w.J;
  if (tt.r > 0) {
    blur_kernel<true><<<dim3(grd.x, grd.y, 3), blk, 0, s>>>(w.J, w.tmp, height, width, tt);
    blur_kernel<false><<<dim3(grd.x, grd.y, 3), blk, 0, s>>>(w.tmp, w.J, height, width, tt);
  }
  const int lin = (int)((HW + 255) / 256);
  eigen_kernel<<<lin, 256, 0, s>>>(Jb, HW, lam1, lam2, angle, coherence, energy, w.tmp);
  if ((rc = check_launch("structure eigen"))) return rc;
  size_t sb = w.sort_bytes;
  cudaError_t e = cub::DeviceRadixSort::SortKeys(w.sort_temp, sb, w.tmp, w.keys, (int)HW, 0,
                                                 32, s);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, "energy sort: %s", cudaGetErrorString(e));
  stats_kernel<<<1, 32, 0, s>>>(w.keys, HW, flat_frac, stats_dev);
  label_kernel<<<lin, 256, 0, s>>>(energy, lam2, HW, stats_dev, corner_frac, label);
  return check_launch("structure labels");
}

}  // extern "C"

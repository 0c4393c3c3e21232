// Placement: density pmf from structure-tensor energy, the seeded density-weighted sampler, and
// the anisotropic field initialisation at the sampled points.
//
// density_from_energy (density.py:16-29):
//   d = base + (1 - base) clip(max(e, 0) / ref, 0, 1)^power,  pmf = d / sum(d)
// (a uniform pmf when the sum is not positive).  sample_candidates (density.py:133-153), given
// the uniforms its numpy Generator draws (first n for rng.choice, then an (n, 2) block of jitter):
//   p = pmf / sum(pmf); cdf = cumsum(p); cdf /= cdf[-1]; idx = searchsorted(cdf, u, 'right')
//   (y, x) = divmod(idx, W); x += jx - 0.5, y += jy - 0.5, each folded back into [0, W-1] /
//   [0, H-1] by reflection.
// Field initialisation for the density_random sampler (init.py:626-631, 778-847): orientation
// and coherence read at the nearest pixel, spacing from the local expected point density
// (_radius_map, init.py:76-82), axis ratios from coherence, colours by bilinear lookup, and the
// GaussianField.from_numpy conversion (gaussians.py:32-55).  Every step repeats numpy's
// precision and operation order (no contracted multiply-adds), so the only differences from the
// reference come from the two parallel reductions and the parallel prefix sum, which change the
// last bits of the pmf and the cdf.
#include <climits>

#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

// numpy's float power with its fast paths for the common exponents.
__device__ __forceinline__ double np_power(double x, double p) {
  if (p == 1.0) return x;
  if (p == 2.0) return __dmul_rn(x, x);
  if (p == 0.5) return __dsqrt_rn(x);
  if (p == 0.0) return 1.0;
  if (p == -1.0) return __ddiv_rn(1.0, x);
  return pow(x, p);
}

__device__ __forceinline__ double np_clip(double x, double lo, double hi) {
  // np.clip = minimum(maximum(x, lo), hi), NaN propagating
  if (x != x) return x;
  return x < lo ? lo : (x > hi ? hi : x);
}

__global__ void density_kernel(const float* __restrict__ energy, int64_t n,
                               const double* __restrict__ ref, double base, double power,
                               double* __restrict__ d) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double e = (double)energy[i];
  e = e > 0.0 ? e : (e != e ? e : 0.0);  // np.maximum(e, 0) keeps NaN
  const double t = np_power(np_clip(__ddiv_rn(e, *ref), 0.0, 1.0), power);
  d[i] = __dadd_rn(base, __dmul_rn(1.0 - base, t));
}

__global__ void normalize_kernel(double* __restrict__ d, int64_t n,
                                 const double* __restrict__ sum, int uniform_if_empty) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = *sum;
  if (uniform_if_empty && !(s > 0.0)) {
    d[i] = __ddiv_rn(1.0, (double)n);
  } else {
    d[i] = __ddiv_rn(d[i], s);
  }
}

__device__ __forceinline__ double reflect(double v, double hi) {
  v = fabs(v);
  return __dsub_rn(hi, fabs(__dsub_rn(hi, v)));
}

__global__ void sample_kernel(const double* __restrict__ cdf, int64_t npx, int W, int H,
                              const double* __restrict__ uniforms, int64_t n,
                              double* __restrict__ pts, int64_t* __restrict__ index_out) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double last = cdf[npx - 1];
  const double u = uniforms[i];
  // first j with cdf[j] / last > u (searchsorted side='right' on the normalised cdf)
  int64_t lo = 0, hi = npx;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (__ddiv_rn(cdf[mid], last) > u) hi = mid; else lo = mid + 1;
  }
  const int64_t idx = lo < npx ? lo : npx - 1;  // only reachable for a pmf without mass
  if (index_out) index_out[i] = idx;
  const int64_t ys = idx / W, xs = idx - ys * W;
  const double jx = __dsub_rn(uniforms[n + 2 * i], 0.5);
  const double jy = __dsub_rn(uniforms[n + 2 * i + 1], 0.5);
  pts[2 * i] = reflect(__dadd_rn((double)xs, jx), (double)W - 1.0);
  pts[2 * i + 1] = reflect(__dadd_rn((double)ys, jy), (double)H - 1.0);
}

// np.round (half to even) + clip to [0, n-1], as init.py:_nearest indexes maps.
__device__ __forceinline__ int nearest_index(double v, int n) {
  const double r = rint(v);
  // numpy's int64 cast of NaN / out-of-range values yields the most negative int64
  const long long k = fabs(r) < 9.0e18 ? (long long)r : LLONG_MIN;
  return (int)(k < 0 ? 0 : (k > n - 1 ? n - 1 : k));
}

// numpy's float32 power with its fast paths.
__device__ __forceinline__ float np_powerf(float x, float p) {
  if (p == 1.0f) return x;
  if (p == 2.0f) return __fmul_rn(x, x);
  if (p == 0.5f) return __fsqrt_rn(x);
  if (p == 0.0f) return 1.0f;
  return powf(x, p);
}

struct PlaceParams {
  int anisotropic;
  float ratio_gain;        // max_axis_ratio - 1, as float (a weak Python scalar)
  float coherence_power;
  double init_scale_mult;
  double n_points;         // n in _radius_map
  float quarter_turn;      // float32(pi / 2)
};

__global__ void place_kernel(const double* __restrict__ pts, int64_t n,
                             const double* __restrict__ pmf, const float* __restrict__ across,
                             const float* __restrict__ coherence,
                             const float* __restrict__ image, int H, int W, PlaceParams pp,
                             float* __restrict__ means, float* __restrict__ log_scales,
                             float* __restrict__ rotations, float* __restrict__ colors) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double px = pts[2 * i], py = pts[2 * i + 1];
  const int xi = nearest_index(px, W), yi = nearest_index(py, H);
  const int64_t q = (int64_t)yi * W + xi;
  // orientation along the edge: float32(across + float32(pi/2))
  const float angle = __fadd_rn(across[q], pp.quarter_turn);
  // spacing: sqrt(1 / (pi * max(n * density, 1e-9))) clipped to [0.5, 20], times sqrt(pi)
  double lam = __dmul_rn(pp.n_points, pmf[q]);
  lam = lam > 1e-9 ? lam : (lam != lam ? lam : 1e-9);
  double r = __dsqrt_rn(__ddiv_rn(1.0, __dmul_rn(3.141592653589793, lam)));
  r = np_clip(r, 0.5, 20.0);
  const double spacing = __dmul_rn(r, 1.7724538509055159);  // float(np.sqrt(np.pi))
  double sq_ratio;
  if (pp.anisotropic) {
    float coh = coherence[q];
    coh = coh != coh ? coh : fminf(fmaxf(coh, 0.0f), 1.0f);
    coh = np_powerf(coh, pp.coherence_power);
    float ratio = __fadd_rn(1.0f, __fmul_rn(pp.ratio_gain, coh));
    ratio = ratio >= 1.0f ? ratio : (ratio != ratio ? ratio : 1.0f);
    sq_ratio = (double)__fsqrt_rn(ratio);
  } else {
    sq_ratio = 1.0;  // np.sqrt of float64 ones
  }
  double s_along = __dmul_rn(__dmul_rn(spacing, sq_ratio), pp.init_scale_mult);
  double s_across = __dmul_rn(__ddiv_rn(spacing, sq_ratio), pp.init_scale_mult);
  s_along = s_along >= 1e-3 ? s_along : (s_along != s_along ? s_along : 1e-3);
  s_across = s_across >= 1e-3 ? s_across : (s_across != s_across ? s_across : 1e-3);
  means[2 * i] = (float)px;
  means[2 * i + 1] = (float)py;
  log_scales[2 * i] = logf((float)s_along);
  log_scales[2 * i + 1] = logf((float)s_across);
  rotations[i] = angle;
  // bilinear colour (init.py:39-49) in float64, left to right
  const double x = np_clip(px, 0.0, (double)W - 1.001), y = np_clip(py, 0.0, (double)H - 1.001);
  const int x0 = (int)floor(x), y0 = (int)floor(y);
  const int x1 = x0 + 1, y1 = y0 + 1;
  const double fx = __dsub_rn(x, (double)x0), fy = __dsub_rn(y, (double)y0);
  const double gx = __dsub_rn(1.0, fx), gy = __dsub_rn(1.0, fy);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const double c00 = image[((int64_t)y0 * W + x0) * 3 + ch];
    const double c01 = image[((int64_t)y0 * W + x1) * 3 + ch];
    const double c10 = image[((int64_t)y1 * W + x0) * 3 + ch];
    const double c11 = image[((int64_t)y1 * W + x1) * 3 + ch];
    double c = __dmul_rn(__dmul_rn(c00, gx), gy);
    c = __dadd_rn(c, __dmul_rn(__dmul_rn(c01, fx), gy));
    c = __dadd_rn(c, __dmul_rn(__dmul_rn(c10, gx), fy));
    c = __dadd_rn(c, __dmul_rn(__dmul_rn(c11, fx), fy));
    colors[3 * i + ch] = (float)c;
  }
}

struct PlaceWorkspace {
  double* sum;
  double* cdf;
  void* temp;
  size_t temp_bytes;
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t cub_bytes(int64_t npx) {
  size_t a = 0, b = 0;
  cub::DeviceReduce::Sum(nullptr, a, (const double*)nullptr, (double*)nullptr, (int)npx);
  cub::DeviceScan::InclusiveSum(nullptr, b, (const double*)nullptr, (double*)nullptr, (int)npx);
  return a > b ? a : b;
}

size_t place_ws_bytes(int64_t npx) {
  return align256(sizeof(double)) + align256(sizeof(double) * (npx > 0 ? npx : 1)) +
         align256(cub_bytes(npx));
}

PlaceWorkspace carve(void* base, int64_t npx) {
  PlaceWorkspace w;
  char* p = static_cast<char*>(base);
  w.sum = reinterpret_cast<double*>(p);
  p += align256(sizeof(double));
  w.cdf = reinterpret_cast<double*>(p);
  p += align256(sizeof(double) * (npx > 0 ? npx : 1));
  w.temp = p;
  w.temp_bytes = align256(cub_bytes(npx));
  return w;
}

int check_image(int H, int W) {
  if (H <= 0 || W <= 0) return fail(SS_ERR_INVALID_ARGUMENT, "image must be non-empty");
  if ((int64_t)H * W > (int64_t)INT32_MAX)
    return fail(SS_ERR_INVALID_ARGUMENT, "image exceeds 2^31 pixels");
  return SS_OK;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_placement_workspace_bytes(int height, int width, size_t* bytes) {
  int rc = check_image(height, width);
  if (rc) return rc;
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  *bytes = place_ws_bytes((int64_t)height * width);
  return SS_OK;
}

int ss_density_from_energy(const float* energy, int height, int width, double base,
                           double power, const double* ref_dev, double* density, void* workspace,
                           size_t workspace_bytes, ss_stream_t stream) {
  int rc = check_image(height, width);
  if (rc) return rc;
  if (!energy || !ref_dev || !density || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  const int64_t npx = (int64_t)height * width;
  if (workspace_bytes < place_ws_bytes(npx))
    return fail(SS_ERR_INVALID_ARGUMENT, "placement workspace too small");
  PlaceWorkspace w = carve(workspace, npx);
  cudaStream_t s = as_stream(stream);
  density_kernel<<<blocks_for(npx), kThreads, 0, s>>>(energy, npx, ref_dev, base, power, density);
  if ((rc = check_launch("density"))) return rc;
  size_t tb = w.temp_bytes;
  cudaError_t e = cub::DeviceReduce::Sum(w.temp, tb, density, w.sum, (int)npx, s);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, "density sum: %s", cudaGetErrorString(e));
  normalize_kernel<<<blocks_for(npx), kThreads, 0, s>>>(density, npx, w.sum, 1);
  return check_launch("density normalize");
}

int ss_sample_candidates(const double* density, int height, int width, const double* uniforms,
                         int64_t n, double* points, int64_t* pixel_index, void* workspace,
                         size_t workspace_bytes, ss_stream_t stream) {
  int rc = check_image(height, width);
  if (rc) return rc;
  if (n < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative sample count");
  if (n == 0) return SS_OK;
  if (!density || !uniforms || !points || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  const int64_t npx = (int64_t)height * width;
  if (workspace_bytes < place_ws_bytes(npx))
    return fail(SS_ERR_INVALID_ARGUMENT, "placement workspace too small");
  PlaceWorkspace w = carve(workspace, npx);
  cudaStream_t s = as_stream(stream);
  // p = density / density.sum(); cdf = cumsum(p)
  size_t tb = w.temp_bytes;
  cudaError_t e = cub::DeviceReduce::Sum(w.temp, tb, density, w.sum, (int)npx, s);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, "sampler sum: %s", cudaGetErrorString(e));
  if (cudaMemcpyAsync(w.cdf, density, sizeof(double) * npx, cudaMemcpyDeviceToDevice, s) !=
      cudaSuccess)
    return check_launch("sampler copy");
  normalize_kernel<<<blocks_for(npx), kThreads, 0, s>>>(w.cdf, npx, w.sum, 0);
  if ((rc = check_launch("sampler normalize"))) return rc;
  tb = w.temp_bytes;
  e = cub::DeviceScan::InclusiveSum(w.temp, tb, w.cdf, w.cdf, (int)npx, s);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, "sampler cdf: %s", cudaGetErrorString(e));
  sample_kernel<<<blocks_for(n), kThreads, 0, s>>>(w.cdf, npx, width, height, uniforms, n, points,
                                                   pixel_index);
  return check_launch("sample");
}

int ss_place_gaussians(const double* points, int64_t n, const double* density,
                       const float* across_edge_angle, const float* coherence,
                       const float* image, int height, int width, int anisotropic,
                       double max_axis_ratio, double coherence_power, double init_scale_mult,
                       int64_t density_points, float* means, float* log_scales,
                       float* rotations, float* colors, ss_stream_t stream) {
  int rc = check_image(height, width);
  if (rc) return rc;
  if (n < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative point count");
  if (n == 0) return SS_OK;
  if (!points || !density || !across_edge_angle || !image || !means || !log_scales ||
      !rotations || !colors || (anisotropic && !coherence))
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (width < 2 || height < 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "bilinear colours need an image of at least 2x2");
  PlaceParams pp;
  pp.anisotropic = anisotropic;
  pp.ratio_gain = (float)(max_axis_ratio - 1.0);
  pp.coherence_power = (float)coherence_power;
  pp.init_scale_mult = init_scale_mult;
  pp.n_points = (double)density_points;
  pp.quarter_turn = (float)(3.141592653589793 / 2.0);
  place_kernel<<<blocks_for(n), kThreads, 0, as_stream(stream)>>>(
      points, n, density, across_edge_angle, coherence, image, height, width, pp, means,
      log_scales, rotations, colors);
  return check_launch("place_gaussians");
}

}  // extern "C"

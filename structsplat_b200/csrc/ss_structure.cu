// Structure tensor J = G_rho * (grad I grad I^T) and its eigen-analysis, on the GPU.
//
// Follows structure_tensor.py:137-186 of the reference (NumPy there): source maps (Rec.709 luma,
// or the colour channels for the Di Zenzo tensor) are blurred separably with reflect padding
// (axis 0 then axis 1, taps accumulated in order with separately rounded products and sums, as
// NumPy's `acc += w * padded_slice` does), differentiated (np.gradient central differences,
// or 3x3 Sobel / Scharr correlation with reflect padding), the outer products are summed over
// channels and blurred again, and the closed-form eigen-analysis gives lam1, lam2, the
// across-edge angle, coherence and energy.  The flat / edge / corner labels need the energy's
// median and 99th percentile (float64, NumPy 'linear' interpolation): four order statistics of
// the energies found by an exact radix select, then one thread evaluates the statistics.
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

// ---------------------------------------------------------------------------------------------
// Tile kernels: one CTA per 32 x 32 block of output pixels, every intermediate in shared memory.
//
// st_tensor_tile: the source maps of the block and a halo (radius of the gradient blur plus one
// pixel for the gradient stencil) are read once; the axis-0 blur, the axis-1 blur, the gradients
// and the channel-summed outer products follow in shared memory; J (3 maps) is written.
// st_eigen_tile: J of the block and a halo of the tensor blur's radius is read once, blurred
// along axis 0 then axis 1, and the eigen-analysis writes the five maps.  Every value is the
// same float32 arithmetic, in the same order, as the per-pass kernels above (reflect padding
// per axis, taps accumulated in order with separately rounded products and sums).
constexpr int kStTile = 32;
constexpr int kStThreads = 256;
constexpr int kStTileMaxRadius = 12;  // larger blurs take the per-pass kernels

// Window of a tile along one axis: [lo, hi) of the image covering the tile [t0, t1) and `halo`
// on either side (reflected indices of the halo fall inside it).
struct Span {
  int lo, hi;
  __device__ __forceinline__ int len() const { return hi - lo; }
};
__device__ __forceinline__ Span span_of(int t0, int t1, int halo, int n) {
  return Span{max(t0 - halo, 0), min(t1 + halo, n)};
}

// Blur along axis 0 (ALONG_Y) or axis 1 of a window-resident map: src covers rows sy and
// columns sx, dst covers oy x ox; indices are image coordinates.  Threads are laid out 32 (x)
// by 8 (y); reflection (per tap) only where the taps reach past the image edge.
template <bool ALONG_Y>
__device__ __forceinline__ void blur_window(const float* src, Span sy, Span sx, float* dst,
                                            Span oy, Span ox, const Taps& taps, int H, int W) {
  const int nx = ox.len(), sw = sx.len(), r = taps.r;
  for (int y = oy.lo + threadIdx.y; y < oy.hi; y += blockDim.y) {
    for (int x = ox.lo + threadIdx.x; x < ox.hi; x += blockDim.x) {
      float acc = 0.0f;
      const bool inside = ALONG_Y ? (y - r >= 0 && y + r < H) : (x - r >= 0 && x + r < W);
      if (inside) {
        const float* c = ALONG_Y ? src + (y - r - sy.lo) * sw + (x - sx.lo)
                                 : src + (y - sy.lo) * sw + (x - r - sx.lo);
        const int step = ALONG_Y ? sw : 1;
        for (int k = 0; k <= 2 * r; ++k) acc = __fadd_rn(acc, __fmul_rn(taps.w[k], c[k * step]));
      } else {
        for (int k = -r; k <= r; ++k) {
          const int yy = ALONG_Y ? reflect(y + k, H) : y;
          const int xx = ALONG_Y ? x : reflect(x + k, W);
          acc = __fadd_rn(acc, __fmul_rn(taps.w[k + r], src[(yy - sy.lo) * sw + (xx - sx.lo)]));
        }
      }
      dst[(y - oy.lo) * nx + (x - ox.lo)] = acc;
    }
  }
}

template <int CH>
__global__ void __launch_bounds__(kStThreads)
    st_tensor_tile(const float* __restrict__ img, int H, int W, int C, int rgb, Taps tg, int op,
                   float* __restrict__ J) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ float st_smem[];
  const int x0 = blockIdx.x * kStTile, y0 = blockIdx.y * kStTile;
  const int x1 = min(x0 + kStTile, W), y1 = min(y0 + kStTile, H);
  const int rg = tg.r;
  const Span wy = span_of(y0, y1, rg + 1, H), wx = span_of(x0, x1, rg + 1, W);  // sources
  const Span gy = span_of(y0, y1, 1, H), gx = span_of(x0, x1, 1, W);            // smoothed
  const int wn = wy.len() * wx.len(), bn = gy.len() * wx.len(), gn = gy.len() * gx.len();
  float* S = st_smem;               // CH x window: sources, then the smoothed maps
  float* B = st_smem + CH * wn;     // CH x (gy x wx): the axis-0 blur
  const int64_t HW = (int64_t)H * W;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = tid; i < wn; i += kStThreads) {
    const int y = wy.lo + i / wx.len(), x = wx.lo + i % wx.len();
    const float* px = img + ((int64_t)y * W + x) * C;
    if (CH == 3) {
      S[i] = px[0];
      S[wn + i] = px[1];
      S[2 * wn + i] = px[2];
    } else if (C == 1) {
      S[i] = px[0];
    } else {  // `img[..., :3] @ luma`: NumPy's float32 dot, a fused multiply-add chain
      S[i] = __fmaf_rn(px[2], 0.0722f, __fmaf_rn(px[1], 0.7152f, __fmul_rn(px[0], 0.2126f)));
    }
  }
  __syncthreads();
  const float* G = S;  // the smoothed maps, (gy x gx) each, or the sources when rg == 0
  Span sgy = wy, sgx = wx;
  if (rg > 0) {
#pragma unroll
    for (int c = 0; c < CH; ++c) blur_window<true>(S + c * wn, wy, wx, B + c * bn, gy, wx, tg, H, W);
    __syncthreads();
#pragma unroll
    for (int c = 0; c < CH; ++c) blur_window<false>(B + c * bn, gy, wx, S + c * gn, gy, gx, tg, H, W);
    __syncthreads();
    sgy = gy;
    sgx = gx;
  }
  const int gw = sgx.len(), gsz = sgy.len() * gw;
  auto g = [&](int c, int y, int x) { return G[c * gsz + (y - sgy.lo) * gw + (x - sgx.lo)]; };
  for (int y = y0 + threadIdx.y; y < y1; y += blockDim.y)
  for (int x = x0 + threadIdx.x; x < x1; x += blockDim.x) {
    float jxx = 0.f, jxy = 0.f, jyy = 0.f;
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      float ix, iy;
      if (op == 0) {  // np.gradient: central inside, one-sided at the border
        if (x == 0) ix = __fsub_rn(g(c, y, 1), g(c, y, 0));
        else if (x == W - 1) ix = __fsub_rn(g(c, y, x), g(c, y, x - 1));
        else ix = __fsub_rn(g(c, y, x + 1), g(c, y, x - 1)) * 0.5f;
        if (y == 0) iy = __fsub_rn(g(c, 1, x), g(c, 0, x));
        else if (y == H - 1) iy = __fsub_rn(g(c, y, x), g(c, y - 1, x));
        else iy = __fsub_rn(g(c, y + 1, x), g(c, y - 1, x)) * 0.5f;
      } else {  // 3x3 correlation, reflect padding
        const float e = op == 1 ? 0.125f : 0.09375f, m = op == 1 ? 0.25f : 0.3125f;
        const float kx[3][3] = {{-e, 0.f, e}, {-m, 0.f, m}, {-e, 0.f, e}};
        float ax = 0.f, ay = 0.f;
        for (int dy = 0; dy < 3; ++dy) {
          const int yy = reflect(y + dy - 1, H);
          for (int dx = 0; dx < 3; ++dx) {
            const float v = g(c, yy, reflect(x + dx - 1, W));
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
    const int64_t p = (int64_t)y * W + x;
    J[p] = jxx;
    J[HW + p] = jxy;
    J[2 * HW + p] = jyy;
  }
}

// The eigen-analysis of one pixel's tensor (structure_tensor.py:163-176).
struct Eigen {
  float l1, l2, angle, coherence, energy;
};
__device__ __forceinline__ Eigen eigen_of(float jxx, float jxy, float jyy) {
  const float half = __fmul_rn(0.5f, __fadd_rn(jxx, jyy));
  const float diff = __fmul_rn(0.5f, __fsub_rn(jxx, jyy));
  const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(diff, diff), __fmul_rn(jxy, jxy)));
  Eigen e;
  e.l1 = __fadd_rn(half, r);
  e.l2 = fmaxf(__fsub_rn(half, r), 0.0f);
  e.energy = __fadd_rn(e.l1, e.l2);
  const float coh = __fdiv_rn(__fsub_rn(e.l1, e.l2), __fadd_rn(e.energy, 1e-12f));
  e.angle = __fmul_rn(0.5f, atan2f(__fmul_rn(2.0f, jxy), __fsub_rn(jxx, jyy)));
  e.coherence = __fmul_rn(coh, coh);
  return e;
}

__global__ void eigen_kernel(const float* __restrict__ J, int64_t HW, float* __restrict__ lam1,
                             float* __restrict__ lam2, float* __restrict__ angle,
                             float* __restrict__ coherence, float* __restrict__ energy,
                             float* __restrict__ energy_keys) {
  pdl_wait();
  pdl_trigger();
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= HW) return;
  const Eigen e = eigen_of(J[p], J[HW + p], J[2 * HW + p]);
  lam1[p] = e.l1;
  lam2[p] = e.l2;
  angle[p] = e.angle;
  coherence[p] = e.coherence;
  energy[p] = e.energy;
  energy_keys[p] = e.energy;
}

__global__ void __launch_bounds__(kStThreads)
    st_eigen_tile(const float* __restrict__ J, int H, int W, Taps tt, float* __restrict__ lam1,
                  float* __restrict__ lam2, float* __restrict__ angle,
                  float* __restrict__ coherence, float* __restrict__ energy,
                  uint32_t* __restrict__ energy_keys) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ float st_smem[];
  const int x0 = blockIdx.x * kStTile, y0 = blockIdx.y * kStTile;
  const int x1 = min(x0 + kStTile, W), y1 = min(y0 + kStTile, H);
  const int rt = tt.r;
  const Span wy = span_of(y0, y1, rt, H), wx = span_of(x0, x1, rt, W);
  const Span oy{y0, y1}, ox{x0, x1};
  const int wn = wy.len() * wx.len(), bn = oy.len() * wx.len(), on = oy.len() * ox.len();
  float* S = st_smem;              // 3 x window of J, then the blurred maps
  float* B = st_smem + 3 * wn;     // 3 x (tile rows x window columns)
  const int64_t HW = (int64_t)H * W;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int i = tid; i < wn; i += kStThreads) {
    const int64_t p = (int64_t)(wy.lo + i / wx.len()) * W + wx.lo + i % wx.len();
    S[i] = J[p];
    S[wn + i] = J[HW + p];
    S[2 * wn + i] = J[2 * HW + p];
  }
  __syncthreads();
  const float* T = S;
  Span sy = wy, sx = wx;
  if (rt > 0) {
    for (int c = 0; c < 3; ++c) blur_window<true>(S + c * wn, wy, wx, B + c * bn, oy, wx, tt, H, W);
    __syncthreads();
    for (int c = 0; c < 3; ++c) blur_window<false>(B + c * bn, oy, wx, S + c * on, oy, ox, tt, H, W);
    __syncthreads();
    sy = oy;
    sx = ox;
  }
  const int tw = sx.len(), tsz = sy.len() * tw;
  for (int y = y0 + threadIdx.y; y < y1; y += blockDim.y)
  for (int x = x0 + threadIdx.x; x < x1; x += blockDim.x) {
    const int q = (y - sy.lo) * tw + (x - sx.lo);
    const Eigen e = eigen_of(T[q], T[tsz + q], T[2 * tsz + q]);
    const int64_t p = (int64_t)y * W + x;
    lam1[p] = e.l1;
    lam2[p] = e.l2;
    angle[p] = e.angle;
    coherence[p] = e.coherence;
    energy[p] = e.energy;
    energy_keys[p] = __float_as_uint(e.energy);  // >= 0: the bits order like the values
  }
}

size_t tensor_tile_smem(int rg, int chans) {
  const int wn = (kStTile + 2 * (rg + 1)) * (kStTile + 2 * (rg + 1));
  const int bn = (kStTile + 2) * (kStTile + 2 * (rg + 1));
  return (size_t)chans * (wn + bn) * sizeof(float);
}
size_t eigen_tile_smem(int rt) {
  const int wn = (kStTile + 2 * rt) * (kStTile + 2 * rt);
  const int bn = kStTile * (kStTile + 2 * rt);
  return (size_t)3 * (wn + bn) * sizeof(float);
}

// ---------------------------------------------------------------------------------------------
// Exact order statistics of the energies (all >= 0, so their float bits order like the values)
// by a radix select: four passes over 8-bit digits from the top, each building one 256-bin
// histogram per wanted rank among the keys that share that rank's digits so far, then one
// thread descending into the bin holding the rank.  kRanks ranks: the median's one or two
// middle elements and the two elements the 99th percentile interpolates.
constexpr int kRanks = 4;
struct SelectState {
  uint32_t prefix[kRanks];   // digits found so far (high bits)
  long long rank[kRanks];    // rank still to find among the keys with that prefix
  uint32_t hist[kRanks][256];
  unsigned int done;         // CTAs finished with the current pass
};

// One pass: the histograms of the current digit (keys >> shift & 255) of the keys sharing each
// rank's prefix; identical digits of a warp are counted with one shared-memory atomic (the
// energies cluster, so most keys of a pass share a few bins).  The last CTA to finish descends
// into the bin holding each rank and clears the histograms for the next pass.
__global__ void select_pass_kernel(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                   SelectState* __restrict__ st) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint32_t h[kRanks][256];
  __shared__ uint32_t prefix[kRanks];
  __shared__ bool last;
  const int lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < kRanks * 256; i += blockDim.x) (&h[0][0])[i] = 0u;
  if (threadIdx.x < kRanks) prefix[threadIdx.x] = st->prefix[threadIdx.x];
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
    const int64_t i = base + threadIdx.x;
    const uint32_t k = i < n ? keys[i] : 0u;
    const uint32_t high = shift >= 24 ? 0u : (k >> (shift + 8));
    const uint32_t digit = (k >> shift) & 255u;
#pragma unroll
    for (int r = 0; r < kRanks; ++r) {
      const uint32_t key = (i < n && high == prefix[r]) ? digit : 256u;
      const unsigned same = __match_any_sync(0xffffffffu, key);
      if (key < 256u && lane == __ffs(same) - 1) atomicAdd(&h[r][key], (uint32_t)__popc(same));
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRanks * 256; i += blockDim.x) {
    const uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(&(&st->hist[0][0])[i], v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  // the complete histograms (read past L1: the other CTAs added them in L2)
  for (int i = threadIdx.x; i < kRanks * 256; i += blockDim.x)
    (&h[0][0])[i] = __ldcg(&(&st->hist[0][0])[i]);
  __syncthreads();
  if (threadIdx.x < kRanks) {
    const int r = threadIdx.x;
    long long want = st->rank[r];
    int bin = 0;
    for (; bin < 255; ++bin) {
      const long long c = h[r][bin];
      if (want < c) break;
      want -= c;
    }
    st->prefix[r] = (st->prefix[r] << 8) | (uint32_t)bin;
    st->rank[r] = want;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kRanks * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0u;
  if (threadIdx.x == 0) st->done = 0u;
}

__global__ void select_init_kernel(SelectState* st, int64_t n) {
  pdl_wait();
  pdl_trigger();
  for (int i = threadIdx.x; i < kRanks * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0u;
  if (threadIdx.x == 0) {
    const int64_t lo = (int64_t)floor((double)(n - 1) * 0.99);
    const int64_t lo_c = lo < 0 ? 0 : (lo > n - 1 ? n - 1 : lo);
    const long long want[kRanks] = {(long long)((n - 1) / 2), (long long)(n / 2), lo_c,
                                    lo_c + 1 < n ? lo_c + 1 : n - 1};
    for (int r = 0; r < kRanks; ++r) {
      st->prefix[r] = 0u;
      st->rank[r] = want[r];
    }
    st->done = 0u;
  }
}

// The statistics from the four selected keys (the same float64 formulas as stats_kernel).
__global__ void select_stats_kernel(const SelectState* __restrict__ st, int64_t n,
                                    double flat_frac, double* stats) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double med = 0.0, p99 = 0.0;
  if (n > 0) {
    const double a = fmax((double)__uint_as_float(st->prefix[0]), 0.0);
    const double b = fmax((double)__uint_as_float(st->prefix[1]), 0.0);
    med = (n & 1) ? b : (a + b) / 2.0;
    const double v = (double)(n - 1) * 0.99;
    int64_t lo = (int64_t)floor(v);
    if (lo < 0) lo = 0;
    if (lo > n - 1) lo = n - 1;
    const double t = v - (double)lo;
    const double pa = fmax((double)__uint_as_float(st->prefix[2]), 0.0);
    const double pb = fmax((double)__uint_as_float(st->prefix[3]), 0.0);
    const double d = pb - pa;
    p99 = t >= 0.5 ? pb - d * (1.0 - t) : pa + d * t;
  }
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
  float *src, *tmp, *J;
  uint32_t* keys;
  SelectState* select;
};

size_t st_workspace_bytes(int64_t HW) {
  return 3 * align256(3 * HW * sizeof(float)) + align256(HW * sizeof(float)) +
         align256(sizeof(SelectState));
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
  w.keys = reinterpret_cast<uint32_t*>(p);
  p += align256(HW * sizeof(float));
  w.select = reinterpret_cast<SelectState*>(p);
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
  const int rgb = (color_space == 1 && channels >= 3) ? 1 : 0;
  const int chans = rgb ? 3 : 1;
  const int lin = (int)((HW + 255) / 256);
  if (tg.r <= kStTileMaxRadius && tt.r <= kStTileMaxRadius) {
    // two tile kernels, every intermediate in shared memory
    const dim3 tiles((width + kStTile - 1) / kStTile, (height + kStTile - 1) / kStTile);
    const size_t sm1 = tensor_tile_smem(tg.r, chans), sm2 = eigen_tile_smem(tt.r);
    if (rgb)
      rc = launch_smem("st_tensor_tile", st_tensor_tile<3>, tiles, dim3(32, 8), sm1, s, image,
                       height, width, channels, rgb, tg, gradient_operator, w.J);
    else
      rc = launch_smem("st_tensor_tile", st_tensor_tile<1>, tiles, dim3(32, 8), sm1, s, image,
                       height, width, channels, rgb, tg, gradient_operator, w.J);
    if (rc || (rc = check_launch("structure tensor tiles"))) return rc;
    rc = launch_smem("st_eigen_tile", st_eigen_tile, tiles, dim3(32, 8), sm2, s,
                     (const float*)w.J, height, width, tt, lam1, lam2, angle, coherence, energy,
                     w.keys);
    if (rc || (rc = check_launch("structure eigen tiles"))) return rc;
  } else {  // blurs wider than the tiles' halo: one pass per axis in global memory
    const dim3 blk(32, 8), grd((width + 31) / 32, (height + 7) / 8);
    source_maps_kernel<<<grd, blk, 0, s>>>(image, height, width, channels, rgb, w.src);
    if ((rc = check_launch("structure source maps"))) return rc;
    if (tg.r > 0) {
      blur_kernel<true><<<dim3(grd.x, grd.y, chans), blk, 0, s>>>(w.src, w.tmp, height, width, tg);
      blur_kernel<false><<<dim3(grd.x, grd.y, chans), blk, 0, s>>>(w.tmp, w.src, height, width, tg);
    }
    tensor_kernel<<<grd, blk, 0, s>>>(w.src, chans, height, width, gradient_operator, w.J);
    if ((rc = check_launch("structure gradients"))) return rc;
    if (tt.r > 0) {
      blur_kernel<true><<<dim3(grd.x, grd.y, 3), blk, 0, s>>>(w.J, w.tmp, height, width, tt);
      blur_kernel<false><<<dim3(grd.x, grd.y, 3), blk, 0, s>>>(w.tmp, w.J, height, width, tt);
    }
    eigen_kernel<<<lin, 256, 0, s>>>(w.J, HW, lam1, lam2, angle, coherence, energy,
                                     reinterpret_cast<float*>(w.keys));
    if ((rc = check_launch("structure eigen"))) return rc;
  }
  // the energy's median and 99th percentile by an exact radix select
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (HW + 255) / 256;
  const unsigned hblocks = (unsigned)(want < (int64_t)sms * 4 ? want : (int64_t)sms * 4);
  launch("select_init_kernel", select_init_kernel, 1, 256, 0, s, w.select, HW);
  for (int shift = 24; shift >= 0; shift -= 8)
    launch("select_pass_kernel", select_pass_kernel, hblocks, 256, 0, s,
           (const uint32_t*)w.keys, HW, shift, w.select);
  launch("select_stats_kernel", select_stats_kernel, 1, 32, 0, s,
         (const SelectState*)w.select, HW, flat_frac, stats_dev);
  if ((rc = check_launch("structure statistics"))) return rc;
  label_kernel<<<lin, 256, 0, s>>>(energy, lam2, HW, stats_dev, corner_frac, label);
  return check_launch("structure labels");
}

}  // extern "C"

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
static_assert(kStTile + 2 * (kStTileMaxRadius + 1) <= 64, "a window row fits two columns per lane");

// Window of a tile along one axis: [lo, hi) of the image covering the tile [t0, t1) and `halo`
// on either side (reflected indices of the halo fall inside it).
struct Span {
  int lo, hi;
  __device__ __forceinline__ int len() const { return hi - lo; }
};
__device__ __forceinline__ Span span_of(int t0, int t1, int halo, int n) {
  return Span{max(t0 - halo, 0), min(t1 + halo, n)};
}

// Row pitch of a shared-memory plane whose rows hold n values: odd, so that the lanes of a warp
// walking down different rows at the same column hit different banks.
__host__ __device__ __forceinline__ int plane_pitch(int n) { return n | 1; }

// Calls f(row, column) for every element of a window of at most 64 columns (window-relative
// indices), threads laid out 32 (x) by 8 (y): a warp takes a row, each lane one or two columns.
// Unrolled so that each thread has several rows' global loads in flight at once.
template <typename F>
__device__ __forceinline__ void for_window(Span wy, Span wx, F&& f) {
  const int wxl = wx.len(), wyl = wy.len();
  const int c0 = threadIdx.x, c1 = threadIdx.x + 32;
#pragma unroll 4
  for (int r = threadIdx.y; r < wyl; r += 8) {
    if (c0 < wxl) f(r, c0);
    if (c1 < wxl) f(r, c1);
  }
}

// Blur along axis 0 (ALONG_Y) or axis 1 of a window-resident map: src covers rows sy and
// columns sx (row pitch sw), dst covers oy x ox (row pitch nx); indices are image coordinates.  Threads are laid out 32 (x)
// by 8 (y); reflection (per tap) only where the taps reach past the image edge.
template <bool ALONG_Y>
__device__ __forceinline__ void blur_window(const float* src, Span sy, Span sx, int sw,
                                            float* dst, Span oy, Span ox, int nx,
                                            const Taps& taps, int H, int W) {
  const int r = taps.r;
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

// The same blur for a compile-time radius R over NCH maps at once (map c at src + c * scs and
// dst + c * dcs): each thread takes RO consecutive outputs along the blur axis of one map and
// holds the RO + 2R source values they need in registers (one load per source value instead of
// one per tap); the taps are accumulated in the same order.  A segment whose sources all lie in
// the stored window (every interior tile's) loads them from one base address; one that reaches
// the image edge reflects each index.  The maps share one item loop so that the threads' last
// round is shared by the maps rather than repeated per map.
template <bool ALONG_Y, int R, int RO, int NCH>
__device__ __forceinline__ void blur_window_sliding(const float* src, int scs, Span sy, Span sx,
                                                    int sw, float* dst, int dcs, Span oy,
                                                    Span ox, int nx, const Taps& taps, int H,
                                                    int W) {
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nline = ALONG_Y ? ox.len() : oy.len();
  const int nalong = ALONG_Y ? oy.len() : ox.len();
  const int nseg = (nalong + RO - 1) / RO;
  const int per_map = nline * nseg;
  const Span src_span = ALONG_Y ? sy : sx;
  const int n_axis = ALONG_Y ? H : W;
  for (int item = tid; item < NCH * per_map; item += kStThreads) {
    const int ch = NCH == 1 ? 0 : item / per_map;
    const int it = NCH == 1 ? item : item - ch * per_map;
    const int line = ALONG_Y ? it % nline : it / nseg;
    const int seg = ALONG_Y ? it / nline : it % nseg;
    const int a0 = (ALONG_Y ? oy.lo : ox.lo) + seg * RO;
    const int a_end = (ALONG_Y ? oy.hi : ox.hi);
    const int other = (ALONG_Y ? ox.lo : oy.lo) + line;  // the column (ALONG_Y) or the row
    const float* sc = src + ch * scs;
    float win[RO + 2 * R];
    if (a0 - R >= src_span.lo && a0 + RO + R <= src_span.hi) {
      const float* base = ALONG_Y ? sc + (a0 - R - sy.lo) * sw + (other - sx.lo)
                                  : sc + (other - sy.lo) * sw + (a0 - R - sx.lo);
#pragma unroll
      for (int j = 0; j < RO + 2 * R; ++j) win[j] = base[ALONG_Y ? j * sw : j];
    } else {
#pragma unroll
      for (int j = 0; j < RO + 2 * R; ++j) {
        int c = a0 - R + j;
        if (c < 0 || c >= n_axis) c = reflect(c, n_axis);
        c = min(c, src_span.hi - 1);  // sources only the unstored outputs past a_end would use
        win[j] = ALONG_Y ? sc[(c - sy.lo) * sw + (other - sx.lo)]
                         : sc[(other - sy.lo) * sw + (c - sx.lo)];
      }
    }
    float* dc = dst + ch * dcs;
#pragma unroll
    for (int k = 0; k < RO; ++k) {
      if (a0 + k < a_end) {
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j <= 2 * R; ++j) acc = __fadd_rn(acc, __fmul_rn(taps.w[j], win[k + j]));
        const int y = ALONG_Y ? a0 + k : other, x = ALONG_Y ? other : a0 + k;
        dc[(y - oy.lo) * nx + (x - ox.lo)] = acc;
      }
    }
  }
}

// Blur dispatch for NCH maps (src + c * scs -> dst + c * dcs): the register form for the
// workloads' radii (3: sigma 1; 6: rho 2; 9: rho 3), else the per-tap form map by map.
template <bool ALONG_Y, int NCH>
__device__ __forceinline__ void blur_maps(const float* src, int scs, Span sy, Span sx, int sw,
                                          float* dst, int dcs, Span oy, Span ox, int nx,
                                          const Taps& taps, int H, int W) {
  if (taps.r == 3)
    blur_window_sliding<ALONG_Y, 3, 4, NCH>(src, scs, sy, sx, sw, dst, dcs, oy, ox, nx, taps, H, W);
  else if (taps.r == 6)
    blur_window_sliding<ALONG_Y, 6, 4, NCH>(src, scs, sy, sx, sw, dst, dcs, oy, ox, nx, taps, H, W);
  else if (taps.r == 9)
    blur_window_sliding<ALONG_Y, 9, 4, NCH>(src, scs, sy, sx, sw, dst, dcs, oy, ox, nx, taps, H, W);
  else
    for (int c = 0; c < NCH; ++c)
      blur_window<ALONG_Y>(src + c * scs, sy, sx, sw, dst + c * dcs, oy, ox, nx, taps, H, W);
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
  const int pw = plane_pitch(wx.len()), pg = plane_pitch(gx.len());
  const int wn = wy.len() * pw, bn = gy.len() * pw, gn = gy.len() * pg;
  float* S = st_smem;               // CH x window: sources, then the smoothed maps
  float* B = st_smem + CH * wn;     // CH x (gy x wx): the axis-0 blur
  const int64_t HW = (int64_t)H * W;
  for_window(wy, wx, [&](int r, int c) {
    const int i = r * pw + c;
    const float* px = img + ((int64_t)(wy.lo + r) * W + wx.lo + c) * C;
    if (CH == 3) {
      S[i] = px[0];
      S[wn + i] = px[1];
      S[2 * wn + i] = px[2];
    } else if (C == 1) {
      S[i] = px[0];
    } else {  // `img[..., :3] @ luma`: NumPy's float32 dot, a fused multiply-add chain
      S[i] = __fmaf_rn(px[2], 0.0722f, __fmaf_rn(px[1], 0.7152f, __fmul_rn(px[0], 0.2126f)));
    }
  });
  __syncthreads();
  const float* G = S;  // the smoothed maps, (gy x gx) each, or the sources when rg == 0
  Span sgy = wy, sgx = wx;
  int gw = pw, gsz = wn;
  if (rg > 0) {
    blur_maps<true, CH>(S, wn, wy, wx, pw, B, bn, gy, wx, pw, tg, H, W);
    __syncthreads();
    blur_maps<false, CH>(B, bn, gy, wx, pw, S, gn, gy, gx, pg, tg, H, W);
    __syncthreads();
    sgy = gy;
    sgx = gx;
    gw = pg;
    gsz = gn;
  }
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

// The radix-select key of an energy (>= 0): its float bits, which order like the values, with
// -0 read as +0.
__device__ __forceinline__ uint32_t energy_key(float e) {
  const uint32_t k = __float_as_uint(e);
  return k == 0x80000000u ? 0u : k;
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
                             float* __restrict__ coherence, float* __restrict__ energy) {
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
}

__global__ void __launch_bounds__(kStThreads)
    st_eigen_tile(const float* __restrict__ J, int H, int W, Taps tt, float* __restrict__ lam1,
                  float* __restrict__ lam2, float* __restrict__ angle,
                  float* __restrict__ coherence, float* __restrict__ energy,
                  uint32_t* __restrict__ level0_hist) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ float st_smem[];
  const int x0 = blockIdx.x * kStTile, y0 = blockIdx.y * kStTile;
  const int x1 = min(x0 + kStTile, W), y1 = min(y0 + kStTile, H);
  const int rt = tt.r;
  const Span wy = span_of(y0, y1, rt, H), wx = span_of(x0, x1, rt, W);
  const Span oy{y0, y1}, ox{x0, x1};
  const int pw = plane_pitch(wx.len()), po = plane_pitch(ox.len());
  const int wn = wy.len() * pw, bn = oy.len() * pw, on = oy.len() * po;
  float* S = st_smem;              // 3 x window of J, then the blurred maps
  float* B = st_smem + 3 * wn;     // 3 x (tile rows x window columns)
  const int64_t HW = (int64_t)H * W;
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  for_window(wy, wx, [&](int r, int c) {
    const int i = r * pw + c;
    const int64_t p = (int64_t)(wy.lo + r) * W + wx.lo + c;
    S[i] = J[p];
    S[wn + i] = J[HW + p];
    S[2 * wn + i] = J[2 * HW + p];
  });
  __syncthreads();
  const float* T = S;
  Span sy = wy, sx = wx;
  int tw = pw, tsz = wn;
  if (rt > 0) {
    blur_maps<true, 3>(S, wn, wy, wx, pw, B, bn, oy, wx, pw, tt, H, W);
    __syncthreads();
    blur_maps<false, 3>(B, bn, oy, wx, pw, S, on, oy, ox, po, tt, H, W);
    __syncthreads();
    sy = oy;
    sx = ox;
    tw = po;
    tsz = on;
  }
  __shared__ uint32_t h0[256];  // the energies' top key bytes (level 0 of the radix select)
  for (int i = tid; i < 256; i += kStThreads) h0[i] = 0u;
  __syncthreads();
  const int x = x0 + threadIdx.x;
  for (int y = y0 + threadIdx.y; y < y0 + kStTile; y += blockDim.y) {  // warp-uniform
    const bool in = y < y1 && x < x1;
    uint32_t digit = 256u;
    if (in) {
      const int q = (y - sy.lo) * tw + (x - sx.lo);
      const Eigen e = eigen_of(T[q], T[tsz + q], T[2 * tsz + q]);
      const int64_t p = (int64_t)y * W + x;
      lam1[p] = e.l1;
      lam2[p] = e.l2;
      angle[p] = e.angle;
      coherence[p] = e.coherence;
      energy[p] = e.energy;
      digit = energy_key(e.energy) >> 24;
    }
    // neighbouring energies share their top byte: one shared-memory atomic per distinct byte
    const unsigned same = __match_any_sync(0xffffffffu, digit);
    if (in && (threadIdx.x == __ffs(same) - 1)) atomicAdd(&h0[digit], (uint32_t)__popc(same));
  }
  __syncthreads();
  for (int i = tid; i < 256; i += kStThreads)
    if (h0[i]) atomicAdd(&level0_hist[i], h0[i]);
}

size_t tensor_tile_smem(int rg, int chans) {
  const int side = kStTile + 2 * (rg + 1);
  const int wn = side * plane_pitch(side), bn = (kStTile + 2) * plane_pitch(side);
  return (size_t)chans * (wn + bn) * sizeof(float);
}
size_t eigen_tile_smem(int rt) {
  const int side = kStTile + 2 * rt;
  const int wn = side * plane_pitch(side), bn = kStTile * plane_pitch(side);
  return (size_t)3 * (wn + bn) * sizeof(float);
}

// ---------------------------------------------------------------------------------------------
// Exact order statistics of the energies by a radix select over their float bits (the energies
// are >= 0, so the bits order like the values; -0 is read as +0).  Level l (0..3) is the 8-bit
// digit (key >> (24 - 8 l)) & 255; the histogram of level l counts, for each wanted rank, the
// level-l digits of the keys that share that rank's digits of levels < l (ranks whose prefixes
// agree share one histogram, the one of the lowest such rank).  The level-0 histogram is built
// by the eigen tile kernel as it writes the energies; every later pass and the statistics kernel
// first re-derive the prefixes from the finished lower levels (one warp, a few hundred cycles),
// so no CTA waits on another.  kRanks ranks: the median's one or two middle elements and the two
// elements the 99th percentile interpolates.
constexpr int kRanks = 4;
constexpr int kLevels = 4;
struct SelectState {
  long long want[kRanks];                // rank of each wanted element among all keys
  uint32_t hist[kLevels][kRanks][256];
};

// Copies the finished histograms of levels [0, levels) into shared memory (all threads of the
// CTA; one batch of independent loads instead of a chain of dependent ones in select_descend).
__device__ __forceinline__ void select_load(const SelectState* __restrict__ st, int levels,
                                            uint32_t* hs, int tid, int nthreads) {
  const uint32_t* src = &st->hist[0][0][0];
  for (int i = tid; i < levels * kRanks * 256; i += nthreads) hs[i] = __ldcg(src + i);
}

// The digits of levels [0, levels) of every rank (prefix) and each rank's rank among the keys
// with that prefix, from the histograms select_load copied to hs.  Warp r takes rank r; the
// ranks' prefixes meet in the shared arrays after each level (a rank counted in the histogram
// of the lowest rank sharing its prefix).  Every thread of the CTA calls it (at least kRanks
// warps); results in the caller's shared arrays prefix and rank.
__device__ void select_descend(const SelectState* __restrict__ st, const uint32_t* hs,
                               int levels, uint32_t* prefix, long long* rank) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < kRanks) {
    prefix[threadIdx.x] = 0u;
    rank[threadIdx.x] = st->want[threadIdx.x];
  }
  __syncthreads();
  for (int l = 0; l < levels; ++l) {
    uint32_t next = 0u;
    long long left = 0;
    if (warp < kRanks) {
      const int r = warp;
      const uint32_t pre = prefix[r];
      const long long want = rank[r];
      int hr = r;  // the histogram this rank's keys were counted in (prefixes are monotone)
      for (int q = r - 1; q >= 0; --q)
        if (prefix[q] == pre) hr = q;
      // lane i holds bins [8 i, 8 i + 8)
      const uint32_t* bins = hs + (l * kRanks + hr) * 256 + lane * 8;
      uint32_t c[8];
      long long sum = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        c[j] = bins[j];
        sum += c[j];
      }
      long long incl = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const long long excl = incl - sum;
      // the lane whose bins hold the rank (the last lane when the counts fall short)
      const unsigned hit = __ballot_sync(0xffffffffu, want < incl);
      const int owner = hit ? __ffs(hit) - 1 : 31;
      int bin = 0;
      if (lane == owner) {
        long long w = want - excl;
        int j = 0;
        for (; j < 7; ++j) {
          if (w < (long long)c[j]) break;
          w -= c[j];
        }
        bin = lane * 8 + j;
        left = w;
      }
      bin = __shfl_sync(0xffffffffu, bin, owner);
      left = __shfl_sync(0xffffffffu, left, owner);
      next = (pre << 8) | (uint32_t)bin;
    }
    __syncthreads();  // every rank has read this level's prefixes
    if (warp < kRanks && lane == 0) {
      prefix[warp] = next;
      rank[warp] = left;
    }
    __syncthreads();
  }
}

// Adds one key's level-`level` digit to the shared histograms h of every distinct prefix it
// matches (prefix[] from select_descend; at level 0 every prefix is empty).
__device__ __forceinline__ void select_count(uint32_t (*h)[256], const uint32_t* prefix,
                                             int level, uint32_t k) {
  const int shift = 24 - 8 * level;
  const uint32_t high = level == 0 ? 0u : (k >> (shift + 8));
  const uint32_t digit = (k >> shift) & 255u;
#pragma unroll
  for (int r = 0; r < kRanks; ++r) {
    if (r > 0 && prefix[r] == prefix[r - 1]) continue;  // the same keys as rank r - 1
    if (high == prefix[r]) atomicAdd(&h[r][digit], 1u);
  }
}

// Adds a CTA's shared histograms into level `level` of the global state (non-zero bins only).
__device__ __forceinline__ void select_flush(uint32_t (*h)[256], SelectState* st, int level,
                                             int tid, int nthreads) {
  for (int i = tid; i < kRanks * 256; i += nthreads) {
    const uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(&(&st->hist[level][0][0])[i], v);
  }
}

__global__ void select_pass_kernel(const float* __restrict__ energy, int64_t n, int level,
                                   SelectState* __restrict__ st) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint32_t h[kRanks][256];
  __shared__ uint32_t hs[kLevels - 1][kRanks][256];
  __shared__ uint32_t prefix[kRanks];
  __shared__ long long rank[kRanks];
  for (int i = threadIdx.x; i < kRanks * 256; i += blockDim.x) (&h[0][0])[i] = 0u;
  select_load(st, level, &hs[0][0][0], threadIdx.x, blockDim.x);
  __syncthreads();
  select_descend(st, &hs[0][0][0], level, prefix, rank);
  uint32_t pre[kRanks];
#pragma unroll
  for (int r = 0; r < kRanks; ++r) pre[r] = prefix[r];
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // four keys per load where the energies are 16-byte aligned, two loads in flight
  const int64_t n4 = (reinterpret_cast<uintptr_t>(energy) & 15) ? 0 : n / 4;
  const float4* e4 = reinterpret_cast<const float4*>(energy);
  for (int64_t i = first; i < n4; i += 2 * stride) {
    const float4 a = __ldg(e4 + i);
    const bool two = i + stride < n4;
    const float4 b = two ? __ldg(e4 + i + stride) : make_float4(0.f, 0.f, 0.f, 0.f);
    select_count(h, pre, level, energy_key(a.x));
    select_count(h, pre, level, energy_key(a.y));
    select_count(h, pre, level, energy_key(a.z));
    select_count(h, pre, level, energy_key(a.w));
    if (two) {
      select_count(h, pre, level, energy_key(b.x));
      select_count(h, pre, level, energy_key(b.y));
      select_count(h, pre, level, energy_key(b.z));
      select_count(h, pre, level, energy_key(b.w));
    }
  }
  for (int64_t i = 4 * n4 + first; i < n; i += stride)
    select_count(h, pre, level, energy_key(energy[i]));
  __syncthreads();
  select_flush(h, st, level, threadIdx.x, blockDim.x);
}

__global__ void select_init_kernel(SelectState* st, int64_t n) {
  pdl_wait();
  pdl_trigger();
  for (int i = threadIdx.x; i < kLevels * kRanks * 256; i += blockDim.x)
    (&st->hist[0][0][0])[i] = 0u;
  if (threadIdx.x == 0) {
    const int64_t lo = (int64_t)floor((double)(n - 1) * 0.99);
    const int64_t lo_c = lo < 0 ? 0 : (lo > n - 1 ? n - 1 : lo);
    const long long want[kRanks] = {(long long)((n - 1) / 2), (long long)(n / 2), lo_c,
                                    lo_c + 1 < n ? lo_c + 1 : n - 1};
    for (int r = 0; r < kRanks; ++r) st->want[r] = want[r];
  }
}

// The statistics from the four selected keys (the same float64 formulas as stats_kernel).
__global__ void select_stats_kernel(const SelectState* __restrict__ st, int64_t n,
                                    double flat_frac, double* stats) {
  pdl_wait();
  pdl_trigger();
  __shared__ uint32_t hs[kLevels][kRanks][256];
  __shared__ uint32_t key[kRanks];
  __shared__ long long rank[kRanks];
  select_load(st, kLevels, &hs[0][0][0], threadIdx.x, blockDim.x);
  __syncthreads();
  select_descend(st, &hs[0][0][0], kLevels, key, rank);
  if (threadIdx.x != 0) return;
  double med = 0.0, p99 = 0.0;
  if (n > 0) {
    const double a = fmax((double)__uint_as_float(key[0]), 0.0);
    const double b = fmax((double)__uint_as_float(key[1]), 0.0);
    med = (n & 1) ? b : (a + b) / 2.0;
    const double v = (double)(n - 1) * 0.99;
    int64_t lo = (int64_t)floor(v);
    if (lo < 0) lo = 0;
    if (lo > n - 1) lo = n - 1;
    const double t = v - (double)lo;
    const double pa = fmax((double)__uint_as_float(key[2]), 0.0);
    const double pb = fmax((double)__uint_as_float(key[3]), 0.0);
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
  // The thresholds are Python floats compared against float32 arrays: NumPy casts them to
  // float32 first.
  const float flat_thr = (float)stats[1];
  const float corner_thr = (float)(corner_frac * stats[0]);
  auto lab = [&](float e, float l2) -> uint8_t {
    const bool flat = e < flat_thr;
    const bool corner = l2 > corner_thr && !flat;
    return flat ? 0 : (corner ? 2 : 1);
  };
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t first = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // four pixels per thread where every buffer allows it (16-byte loads, a 4-byte store)
  const bool vec = ((reinterpret_cast<uintptr_t>(energy) | reinterpret_cast<uintptr_t>(lam2)) &
                    15) == 0 && (reinterpret_cast<uintptr_t>(label) & 3) == 0;
  const int64_t n4 = vec ? HW / 4 : 0;
  for (int64_t i = first; i < n4; i += stride) {
    const float4 e = __ldg(reinterpret_cast<const float4*>(energy) + i);
    const float4 l = __ldg(reinterpret_cast<const float4*>(lam2) + i);
    reinterpret_cast<uchar4*>(label)[i] =
        make_uchar4(lab(e.x, l.x), lab(e.y, l.y), lab(e.z, l.z), lab(e.w, l.w));
  }
  for (int64_t p = 4 * n4 + first; p < HW; p += stride) label[p] = lab(energy[p], lam2[p]);
}

struct StWorkspace {
  float *src, *tmp, *J;
  SelectState* select;
};

size_t st_workspace_bytes(int64_t HW) {
  return 3 * align256(3 * HW * sizeof(float)) + align256(sizeof(SelectState));
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
  launch("select_init_kernel", select_init_kernel, 1, 256, 0, s, w.select, HW);
  int first_level = 0;  // the first radix-select level not yet counted
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
                     &w.select->hist[0][0][0]);
    if (rc || (rc = check_launch("structure eigen tiles"))) return rc;
    first_level = 1;
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
    eigen_kernel<<<lin, 256, 0, s>>>(w.J, HW, lam1, lam2, angle, coherence, energy);
    if ((rc = check_launch("structure eigen"))) return rc;
  }
  // the energy's median and 99th percentile by an exact radix select
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t want = (HW + 255) / 256;
  const unsigned hblocks = (unsigned)(want < (int64_t)sms * 4 ? want : (int64_t)sms * 4);
  for (int level = first_level; level < kLevels; ++level)
    launch("select_pass_kernel", select_pass_kernel, hblocks, 256, 0, s, (const float*)energy,
           HW, level, w.select);
  launch("select_stats_kernel", select_stats_kernel, 1, 256, 0, s,
         (const SelectState*)w.select, HW, flat_frac, stats_dev);
  if ((rc = check_launch("structure statistics"))) return rc;
  const unsigned lblocks = (unsigned)((HW / 4 + 255) / 256 < (int64_t)sms * 8
                                          ? (HW / 4 + 255) / 256 + 1 : (int64_t)sms * 8);
  label_kernel<<<lblocks, 256, 0, s>>>(energy, lam2, HW, stats_dev, corner_frac, label);
  return check_launch("structure labels");
}

}  // extern "C"

// Shared definitions of the structsplat_b200 CUDA library (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/structsplat_b200.h"

namespace ss {

// One Gaussian, packed for the render kernels: four 16-byte pieces so a tile stage can pull
// it with four cp.async copies and read it back with vector loads.
//   piece 0: mx, my, qa, qb      mean; log2-domain conic (see below)
//   piece 1: qc, op, cr, cg      log2-domain conic; opacity; colour r, g
//   piece 2: cb, a, b, c         colour b; the conic as given
//   piece 3: x0, y0, x1, y1      clipped support [x0,x1) x [y0,y1); x1 == x0 when empty
// The raw weight exp(-q/2), q = a dx^2 + 2b dx dy + c dy^2, is evaluated as
// 2^(qa dx^2 + qb dx dy + qc dy^2) with qa = -a log2(e)/2, qb = -b log2(e), qc = -c log2(e)/2.
struct __align__(16) Splat {
  float mx, my, qa, qb;
  float qc, op, cr, cg;
  float cb, a, b, c;
  int x0, y0, x1, y1;
};
static_assert(sizeof(Splat) == 64, "splat record must be 64 bytes");

constexpr float kLog2e = 1.4426950408889634f;

// Sets the thread-local error message and returns `code`.
int fail(int code, const char* fmt, ...);
// Converts the last CUDA error (if any) into SS_ERR_CUDA.
int check_launch(const char* what);

inline cudaStream_t as_stream(ss_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// Programmatic dependent launch.  The kernels of a step (projection, binning, forward,
// backward, epilogues, update) are launched with the programmatic-serialization attribute, so a
// kernel's CTAs may become resident while its predecessor in the stream drains.  Every kernel
// of the library therefore begins with pdl_wait(): it returns once the preceding grid has
// completed and its writes are visible (immediately when the launch had no attribute), and
// nothing before it reads another kernel's output.  pdl_trigger() then lets the next grid
// launch.  dependent_launch_enabled() is the process-wide switch (ss_set_dependent_launch).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
bool dependent_launch_enabled();
void note_launch_error(cudaError_t e);

// Launches `kern` on `s` with the programmatic-serialization attribute when enabled; returns
// SS_OK or the launch error, which the next check_launch of the thread also reports.
template <typename... KArgs, typename... Args>
int launch(const char* what, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
           cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = dependent_launch_enabled() ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
  if (e != cudaSuccess) {
    note_launch_error(e);  // the caller's next check_launch reports it too
    return fail(SS_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  return SS_OK;
}

// Lets `kern` take `bytes` of dynamic shared memory (beyond the 48 KB default; the largest
// size a kernel is launched with, set once per kernel and device).
int allow_dynamic_smem(const void* kern, size_t bytes);

// launch() of a kernel whose shared memory is dynamic: `smem` bytes, opted in first.
template <typename... KArgs, typename... Args>
int launch_smem(const char* what, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                cudaStream_t s, Args... args) {
  if (smem > 48 * 1024) {
    const int rc = allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    if (rc) return rc;
  }
  return launch(what, kern, grid, block, smem, s, args...);
}

// 2^x on the SFU (PTX ex2.approx.ftz.f32: one MUFU operation, documented max relative error
// 2^-22; results below 2^-126 flush to zero, which for a weight is an absolute error < 1.2e-38).
__device__ __forceinline__ float fast_exp2(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Support rectangle of one Gaussian clipped to the image, as render.py:62-78 computes it in
// int64 (round half-to-even, clip, empty when either side is <= 0).  Non-finite centres have
// no support (render_ext.cu:25-34); |centre| beyond 1e15 px is treated as off-image, which is
// what the int64 arithmetic yields for any radius below 2^40.
__device__ __forceinline__ void support_rect(float mx, float my, long long rx, long long ry,
                                             int H, int W, int& x0, int& y0, int& x1, int& y1) {
  x0 = y0 = x1 = y1 = 0;
  if (!isfinite(mx) || !isfinite(my)) return;
  float fx = rintf(mx), fy = rintf(my);
  if (fabsf(fx) > 1e15f || fabsf(fy) > 1e15f) return;
  const long long lim = 1LL << 40;
  rx = rx > lim ? lim : (rx < -lim ? -lim : rx);
  ry = ry > lim ? lim : (ry < -lim ? -lim : ry);
  long long ix = (long long)fx, iy = (long long)fy;
  long long xl = ix - rx < 0 ? 0 : ix - rx;
  long long xh = ix + rx > W - 1 ? (long long)W - 1 : ix + rx;
  long long yl = iy - ry < 0 ? 0 : iy - ry;
  long long yh = iy + ry > H - 1 ? (long long)H - 1 : iy + ry;
  if (xh < xl || yh < yl) return;
  x0 = (int)xl;
  x1 = (int)xh + 1;
  y0 = (int)yl;
  y1 = (int)yh + 1;
}

__device__ __forceinline__ Splat make_splat(float mx, float my, float a, float b, float c,
                                            float op, float cr, float cg, float cb, int x0,
                                            int y0, int x1, int y1) {
  Splat s;
  s.mx = mx;
  s.my = my;
  s.qa = -0.5f * kLog2e * a;
  s.qb = -kLog2e * b;
  s.qc = -0.5f * kLog2e * c;
  s.op = op;
  s.cr = cr;
  s.cg = cg;
  s.cb = cb;
  s.a = a;
  s.b = b;
  s.c = c;
  s.x0 = x0;
  s.y0 = y0;
  s.x1 = x1;
  s.y1 = y1;
  return s;
}

__device__ __forceinline__ void store_splat(Splat* dst, const Splat& s) {
  const float4* src = reinterpret_cast<const float4*>(&s);
  float4* d = reinterpret_cast<float4*>(dst);
  d[0] = src[0];
  d[1] = src[1];
  d[2] = src[2];
  d[3] = src[3];
}

// Exact minimum of q(d) = a dx^2 + 2b dx dy + c dy^2 over the rectangle [x_lo,x_hi]x[y_lo,y_hi]
// of pixel centres relative to the mean: zero when the mean is inside, otherwise the minimum
// over the four edges (each a 1-D quadratic minimised at its clamped stationary point).
// A conic that is not positive definite returns -FLT_MAX so the pair is always kept.
// Used only for the ellipse cull, whose contract is render_ext.cu:101-133.
__device__ __forceinline__ float conic_q(float dx, float dy, float a, float b, float c) {
  return a * dx * dx + 2.0f * b * dx * dy + c * dy * dy;
}
__device__ __forceinline__ float rect_min_q(float mx, float my, float a, float b, float c,
                                            float x_lo, float x_hi, float y_lo, float y_hi) {
  if (!(a > 0.0f && c > 0.0f && a * c - b * b > 0.0f)) return -3.402823466e38f;
  if (mx >= x_lo && mx <= x_hi && my >= y_lo && my <= y_hi) return 0.0f;
  float best = 3.402823466e38f;
  float xs[2] = {x_lo - mx, x_hi - mx};
  float ys[2] = {y_lo - my, y_hi - my};
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    float dx = xs[k];
    float dy = fminf(fmaxf(-(b / c) * dx, ys[0]), ys[1]);
    best = fminf(best, conic_q(dx, dy, a, b, c));
  }
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    float dy = ys[k];
    float dx = fminf(fmaxf(-(b / a) * dy, xs[0]), xs[1]);
    best = fminf(best, conic_q(dx, dy, a, b, c));
  }
  return best;
}

// True when the (tile, Gaussian) pair has zero faded weight on every pixel of the tile.
__device__ __forceinline__ bool culled(const Splat& s, int gx, int gy, int ts, float cutoff2) {
  int rx0 = max(s.x0, gx * ts), ry0 = max(s.y0, gy * ts);
  int rx1 = min(s.x1 - 1, (gx + 1) * ts - 1), ry1 = min(s.y1 - 1, (gy + 1) * ts - 1);
  float m = rect_min_q(s.mx, s.my, s.a, s.b, s.c, (float)rx0, (float)rx1, (float)ry0,
                       (float)ry1);
  return m > cutoff2 + 1e-5f * fmaxf(cutoff2, 1.0f);
}

// Chain rule of the RS conic (gaussians.py:275-300): conic gradient (ga, gb, gc) -> log-scale
// and rotation gradients.  With u = 1/(sx^2+d), v = 1/(sy^2+d) the conic is
// a = C^2 u + S^2 v, b = CS (u - v), c = S^2 u + C^2 v.
__device__ __forceinline__ void rs_conic_chain(float ls0, float ls1, float th, float dilation,
                                               float ga, float gb, float gc, float& g_ls0,
                                               float& g_ls1, float& g_rot) {
  const float sx = expf(ls0), sy = expf(ls1);
  const float sx2 = sx * sx, sy2 = sy * sy;
  const float u = 1.0f / (sx2 + dilation), v = 1.0f / (sy2 + dilation);
  float cs, sn;
  sincosf(th, &sn, &cs);
  const float cc = cs * cs, s2 = sn * sn, csn = cs * sn;
  const float gu = ga * cc + gb * csn + gc * s2;
  const float gv = ga * s2 - gb * csn + gc * cc;
  g_ls0 = gu * (-2.0f * sx2 * u * u);
  g_ls1 = gv * (-2.0f * sy2 * v * v);
  g_rot = (u - v) * (2.0f * csn * (gc - ga) + (cc - s2) * gb);
}

// d sigmoid(x) / dx applied to an opacity gradient (gaussians.py:270-273).
__device__ __forceinline__ float logit_chain(float logit, float g_op) {
  const float o = 1.0f / (1.0f + expf(-logit));
  return g_op * o * (1.0f - o);
}

// Where the images of a batch live.  A batch of B images is rendered as one set of tiles: the
// tiles of image b are tiles [first_tile_b, first_tile_b + tiles_b), numbered row-major inside
// the image; its Gaussians are ids [gauss_base[b], gauss_base[b+1]); its pixels are pixels
// [pixel_base[b], pixel_base[b] + H_b W_b) of the concatenated row-major images.  Means, support
// rectangles and pixel coordinates stay image-local, so every image renders exactly as it would
// alone.  A single image is the batch with image == nullptr, described by H, W and tiles_x.
struct Frames {
  const int4* image;           // per image {H, W, tiles_x, first tile}, or nullptr
  const long long* pixel_base;  // per image
  const int* gauss_base;        // per image + 1
  const int* gauss_image;       // per Gaussian
  const int* tile_image;        // per tile
  int H, W, tiles_x;            // the single image (image == nullptr)
};

// One image of a batch, as seen from a tile or a Gaussian.
struct Frame {
  int image, H, W, tiles_x, first_tile;
  long long pixel_base;
  int gauss_first, gauss_count;
};

// Validates a batch description (host side) and converts it to Frames.
int frames_of_batch(const ss_batch* batch, int64_t n, Frames* out);

inline Frames single_frame(int H, int W, int ts) {
  Frames f{};
  f.H = H;
  f.W = W;
  f.tiles_x = ts > 0 ? (W + ts - 1) / ts : 0;
  return f;
}

__device__ __forceinline__ Frame frame_of_image(const Frames& f, int b, int64_t n) {
  Frame r;
  r.image = b;
  if (!f.image) {
    r.H = f.H;
    r.W = f.W;
    r.tiles_x = f.tiles_x;
    r.first_tile = 0;
    r.pixel_base = 0;
    r.gauss_first = 0;
    r.gauss_count = (int)n;
    return r;
  }
  const int4 d = f.image[b];
  r.H = d.x;
  r.W = d.y;
  r.tiles_x = d.z;
  r.first_tile = d.w;
  r.pixel_base = f.pixel_base[b];
  r.gauss_first = f.gauss_base[b];
  r.gauss_count = f.gauss_base[b + 1] - r.gauss_first;
  return r;
}

__device__ __forceinline__ Frame frame_of_tile(const Frames& f, int tile, int64_t n) {
  return frame_of_image(f, f.image ? f.tile_image[tile] : 0, n);
}

__device__ __forceinline__ Frame frame_of_gaussian(const Frames& f, int64_t g, int64_t n) {
  return frame_of_image(f, f.image ? f.gauss_image[g] : 0, n);
}

// An RS field in device memory (means 2n, log-scales 2n, rotations n, colours 3n, opacity
// logits n or NULL) with the projection's dilation and sigma cutoff.
struct RSField {
  const float* means;
  const float* log_scales;
  const float* rotations;
  const float* colors;
  const float* logits;
  float dilation, cutoff;
};

// RS -> splat record of Gaussian i of frame fr, with its radii.  The conic follows
// gaussians.py:275-300 and the radii gaussians.py:302-321; every product and sum is rounded
// separately (no FMA contraction) so the radii's ceil() sees the same float the reference's
// elementwise torch ops produce.
__device__ __forceinline__ Splat rs_project_one(const RSField& f, int64_t i, const Frame& fr,
                                                long long& rx, long long& ry) {
  const float dilation = f.dilation, cutoff = f.cutoff;
  float sx = expf(f.log_scales[2 * i]), sy = expf(f.log_scales[2 * i + 1]);
  float sx2 = __fmul_rn(sx, sx), sy2 = __fmul_rn(sy, sy);
  float th = f.rotations[i];
  float cs = cosf(th), sn = sinf(th);
  float cc = __fmul_rn(cs, cs), ss2 = __fmul_rn(sn, sn);
  // conic
  float ix = __fdiv_rn(1.0f, __fadd_rn(sx2, dilation));
  float iy = __fdiv_rn(1.0f, __fadd_rn(sy2, dilation));
  float a = __fadd_rn(__fmul_rn(cc, ix), __fmul_rn(ss2, iy));
  float b = __fmul_rn(__fmul_rn(cs, sn), __fsub_rn(ix, iy));
  float c = __fadd_rn(__fmul_rn(ss2, ix), __fmul_rn(cc, iy));
  // radii: ceil(cutoff * sqrt(var)) clamped >= 1
  float vx2 = __fadd_rn(sx2, dilation), vy2 = __fadd_rn(sy2, dilation);
  float varx = __fadd_rn(__fmul_rn(cc, vx2), __fmul_rn(ss2, vy2));
  float vary = __fadd_rn(__fmul_rn(ss2, vx2), __fmul_rn(cc, vy2));
  float fr_x = ceilf(__fmul_rn(cutoff, __fsqrt_rn(varx)));
  float fr_y = ceilf(__fmul_rn(cutoff, __fsqrt_rn(vary)));
  rx = isfinite(fr_x) ? (long long)fmaxf(fminf(fr_x, 1e15f), 1.0f) : (1LL << 40);
  ry = isfinite(fr_y) ? (long long)fmaxf(fminf(fr_y, 1e15f), 1.0f) : (1LL << 40);
  float op = f.logits ? 1.0f / (1.0f + expf(-f.logits[i])) : 1.0f;
  float mx = f.means[2 * i], my = f.means[2 * i + 1];
  int x0, y0, x1, y1;
  support_rect(mx, my, rx, ry, fr.H, fr.W, x0, y0, x1, y1);
  return make_splat(mx, my, a, b, c, op, f.colors[3 * i], f.colors[3 * i + 1],
                    f.colors[3 * i + 2], x0, y0, x1, y1);
}

// The backward's per-(tile, Gaussian) record in deterministic mode: nine moments, padded.
constexpr int kMoments = 9;
constexpr int kPartialFloats = 12;

// Deterministic-mode workspace.  The backward writes one partial (nine moments, padded to 12
// floats) per tile-list entry; the entries are then ordered by Gaussian with a stable radix sort
// of their ids, so Gaussian g's entries are order[seg[g] .. seg[n + g]) in ascending tile order
// and its moments are summed in that fixed order, whatever the schedule of the backward.
//   partials  cap x 12 floats       keys_in / keys   cap uint32 (ids; n marks unused slots)
//   order_in / order  cap int32      seg              2n int32 (segment begin, end)
//   temp      the radix sort's scratch
struct EntryOrder {
  float* partials;
  uint32_t* keys_in;
  uint32_t* keys;
  int32_t* order_in;
  int32_t* order;
  int32_t* seg;
  void* temp;
  size_t fixed_bytes;  // bytes before temp
};

__host__ __device__ inline size_t align_up256(size_t x) { return (x + 255) & ~size_t(255); }

__host__ __device__ inline EntryOrder entry_order_layout(void* ws, int64_t n, int64_t cap) {
  size_t off[7];
  const size_t bytes[6] = {(size_t)cap * kPartialFloats * sizeof(float), (size_t)cap * 4,
                           (size_t)cap * 4, (size_t)cap * 4, (size_t)cap * 4, (size_t)2 * n * 4};
  off[0] = 0;
  for (int k = 0; k < 6; ++k) off[k + 1] = off[k] + align_up256(bytes[k]);
  char* p = static_cast<char*>(ws);
  EntryOrder e;
  e.partials = reinterpret_cast<float*>(p + off[0]);
  e.keys_in = reinterpret_cast<uint32_t*>(p + off[1]);
  e.keys = reinterpret_cast<uint32_t*>(p + off[2]);
  e.order_in = reinterpret_cast<int32_t*>(p + off[3]);
  e.order = reinterpret_cast<int32_t*>(p + off[4]);
  e.seg = reinterpret_cast<int32_t*>(p + off[5]);
  e.temp = p + off[6];
  e.fixed_bytes = off[6];
  return e;
}

__host__ __device__ inline size_t entry_order_fixed_bytes(int64_t n, int64_t cap) {
  return align_up256((size_t)cap * kPartialFloats * sizeof(float)) +
         4 * align_up256((size_t)cap * 4) + align_up256((size_t)2 * n * 4);
}

// Fit workspace: the backward's part (above) followed by the parameter gradients of the Adam
// step, five arrays shaped like the parameters (means 2n, log-scales 2n, rotations n, colours 3n,
// opacity logits n), each 256-byte aligned.
struct FitGrads {
  float *means, *log_scales, *rotations, *colors, *logits;
};
__host__ __device__ inline size_t fit_grads_bytes(int64_t n) {
  return 2 * align_up256((size_t)8 * n) + 2 * align_up256((size_t)4 * n) +
         align_up256((size_t)12 * n);
}
__host__ __device__ inline FitGrads fit_grads_layout(void* base, int64_t n) {
  char* p = static_cast<char*>(base);
  FitGrads g;
  g.means = reinterpret_cast<float*>(p);
  p += align_up256((size_t)8 * n);
  g.log_scales = reinterpret_cast<float*>(p);
  p += align_up256((size_t)8 * n);
  g.rotations = reinterpret_cast<float*>(p);
  p += align_up256((size_t)4 * n);
  g.colors = reinterpret_cast<float*>(p);
  p += align_up256((size_t)12 * n);
  g.logits = reinterpret_cast<float*>(p);
  return g;
}
// Offset of the gradients in the fit workspace and its total size (ss_render.cu).
size_t fit_grads_offset(int64_t n, int64_t cap, int deterministic);
size_t fit_ws_bytes(int64_t n, int64_t cap, int deterministic);

// Segments up to this many entries are summed by their own lane; longer ones by the warp.
constexpr int kLaneSegment = 32;

__device__ __forceinline__ void add_partial(const float* partials, int32_t e,
                                            float (&acc)[kMoments]) {
  const float4* pp = reinterpret_cast<const float4*>(partials + (int64_t)e * kPartialFloats);
  const float4 u = pp[0], v = pp[1];
  const float w = partials[(int64_t)e * kPartialFloats + 8];
  acc[0] += u.x; acc[1] += u.y; acc[2] += u.z; acc[3] += u.w;
  acc[4] += v.x; acc[5] += v.y; acc[6] += v.z; acc[7] += v.w;
  acc[8] += w;
}

// Sum of Gaussian g's entry partials in its fixed entry order.  Warp-collective: every lane of
// the warp calls it (active = false for a lane without a Gaussian).  A segment of at most
// kLaneSegment entries is summed serially by its lane; a longer one by the whole warp (lane l
// takes entries l, l + 32, ..., then a butterfly over the lanes), so one huge Gaussian does not
// serialise its warp.  The order depends only on the segment's length.
__device__ __forceinline__ void sum_entry_partials(const float* __restrict__ partials,
                                                   const int32_t* __restrict__ order,
                                                   const int32_t* __restrict__ seg, int64_t n,
                                                   int64_t g, bool active,
                                                   float (&acc)[kMoments]) {
#pragma unroll
  for (int k = 0; k < kMoments; ++k) acc[k] = 0.f;
  int beg = 0, end = 0;
  if (active) {
    beg = seg[g];
    end = seg[n + g];
  }
  if (end - beg <= kLaneSegment)
    for (int i = beg; i < end; ++i) add_partial(partials, order[i], acc);
  const int lane = threadIdx.x & 31;
  unsigned big = __ballot_sync(0xffffffffu, end - beg > kLaneSegment);
  while (big) {
    const int src = __ffs(big) - 1;
    big &= big - 1;
    const int b = __shfl_sync(0xffffffffu, beg, src), e = __shfl_sync(0xffffffffu, end, src);
    float t[kMoments];
#pragma unroll
    for (int k = 0; k < kMoments; ++k) t[k] = 0.f;
    for (int i = b + lane; i < e; i += 32) add_partial(partials, order[i], t);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int k = 0; k < kMoments; ++k) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
    if (lane == src)
#pragma unroll
      for (int k = 0; k < kMoments; ++k) acc[k] = t[k];
  }
}

__device__ __forceinline__ void raise_status(uint32_t* status, uint32_t bits) {
  if (status) atomicOr(status, bits);
}

}  // namespace ss

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

__device__ __forceinline__ void raise_status(uint32_t* status, uint32_t bits) {
  if (status) atomicOr(status, bits);
}

}  // namespace ss

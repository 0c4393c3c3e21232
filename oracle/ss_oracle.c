/*
 * TEST INFRASTRUCTURE ONLY — plain-C restatement of the StructSplat renderer path.
 *
 * Used by the tests as an independent checker and as the float64 error yardstick at full
 * benchmark sizes; never linked into the product library.
 *
 *   ora_support_rect   <- render.py:62-78 (_tile_bounds) / render_ext.cu:13-50 (support_bounds)
 *   ora_tile_index_*   <- cuda_render.py:177-226 (_build_tile_index), ascending ids per tile
 *   ora_render_f64     <- render.py:180-235 (_accumulate), evaluated in float64
 *   ora_backward_f64   <- autograd of render.py:180-235; same formulas as render_ext.cu:785-818
 *
 * Paths are relative to the reference project (intrinsicD/structsplat, src/structsplat/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* Clipped support rectangle of Gaussian i.  Centres round half-to-even (nearbyint under the
 * default rounding mode, like torch.round); a non-finite or astronomically far centre has no
 * in-image support.  Returns the pixel count tx*ty. */
int64_t ora_support_rect(const float* means, const int64_t* radii, int64_t i, int H, int W,
                         int64_t* x0, int64_t* y0, int64_t* tx, int64_t* ty) {
  double mx = means[2 * i], my = means[2 * i + 1];
  *x0 = *y0 = *tx = *ty = 0;
  if (!isfinite(mx) || !isfinite(my)) return 0;
  double cx = nearbyint(mx), cy = nearbyint(my);
  if (fabs(cx) > 1e15 || fabs(cy) > 1e15) return 0;
  int64_t ix = (int64_t)cx, iy = (int64_t)cy;
  int64_t rx = radii[2 * i], ry = radii[2 * i + 1];
  const int64_t lim = (int64_t)1 << 40;
  if (rx > lim) rx = lim;
  if (rx < -lim) rx = -lim;
  if (ry > lim) ry = lim;
  if (ry < -lim) ry = -lim;
  int64_t xl = ix - rx < 0 ? 0 : ix - rx;
  int64_t xh = ix + rx > W - 1 ? W - 1 : ix + rx;
  int64_t yl = iy - ry < 0 ? 0 : iy - ry;
  int64_t yh = iy + ry > H - 1 ? H - 1 : iy + ry;
  int64_t w = xh - xl + 1, h = yh - yl + 1;
  if (w <= 0 || h <= 0) return 0;
  *x0 = xl;
  *y0 = yl;
  *tx = w;
  *ty = h;
  return w * h;
}

int64_t ora_pair_count(const float* means, const int64_t* radii, int64_t n, int H, int W) {
  int64_t total = 0, x0, y0, tx, ty;
  for (int64_t i = 0; i < n; ++i) total += ora_support_rect(means, radii, i, H, W, &x0, &y0, &tx, &ty);
  return total;
}

/* offsets[T+1]: tile t lists offsets[t] .. offsets[t+1]-1.  Returns the entry total. */
int64_t ora_tile_index_offsets(const float* means, const int64_t* radii, int64_t n, int H, int W,
                               int ts, int64_t* offsets) {
  int64_t tiles_x = (W + ts - 1) / ts, tiles_y = (H + ts - 1) / ts;
  int64_t T = tiles_x * tiles_y;
  memset(offsets, 0, sizeof(int64_t) * (size_t)(T + 1));
  int64_t x0, y0, tx, ty;
  for (int64_t i = 0; i < n; ++i) {
    if (ora_support_rect(means, radii, i, H, W, &x0, &y0, &tx, &ty) == 0) continue;
    for (int64_t gy = y0 / ts; gy <= (y0 + ty - 1) / ts; ++gy)
      for (int64_t gx = x0 / ts; gx <= (x0 + tx - 1) / ts; ++gx) offsets[gy * tiles_x + gx + 1] += 1;
  }
  for (int64_t t = 0; t < T; ++t) offsets[t + 1] += offsets[t];
  return offsets[T];
}

/* Fill gids (size offsets[T]) in ascending Gaussian id within every tile. */
void ora_tile_index_fill(const float* means, const int64_t* radii, int64_t n, int H, int W, int ts,
                         const int64_t* offsets, int64_t* gids) {
  int64_t tiles_x = (W + ts - 1) / ts, tiles_y = (H + ts - 1) / ts;
  int64_t T = tiles_x * tiles_y;
  int64_t* cursor = (int64_t*)malloc(sizeof(int64_t) * (size_t)(T > 0 ? T : 1));
  for (int64_t t = 0; t < T; ++t) cursor[t] = offsets[t];
  int64_t x0, y0, tx, ty;
  for (int64_t i = 0; i < n; ++i) {
    if (ora_support_rect(means, radii, i, H, W, &x0, &y0, &tx, &ty) == 0) continue;
    for (int64_t gy = y0 / ts; gy <= (y0 + ty - 1) / ts; ++gy)
      for (int64_t gx = x0 / ts; gx <= (x0 + tx - 1) / ts; ++gx) gids[cursor[gy * tiles_x + gx]++] = i;
  }
  free(cursor);
}

static double visible(double raw, double tail) { return tail > 0.0 ? fmax(raw - tail, 0.0) : raw; }

/* Float64 forward.  out (H*W*3) is the image, den (H*W) the raw weight sum (no eps). */
void ora_render_f64(const float* means, const float* conics, const float* colors,
                    const int64_t* radii, const float* opac, int64_t n, int H, int W, int normalize,
                    double eps, double tail, double* out, double* den) {
  int64_t npx = (int64_t)H * W;
  double* num = (double*)calloc((size_t)(3 * npx > 0 ? 3 * npx : 1), sizeof(double));
  memset(den, 0, sizeof(double) * (size_t)npx);
  int64_t x0, y0, tx, ty;
  for (int64_t i = 0; i < n; ++i) {
    if (ora_support_rect(means, radii, i, H, W, &x0, &y0, &tx, &ty) == 0) continue;
    double mx = means[2 * i], my = means[2 * i + 1];
    double a = conics[3 * i], b = conics[3 * i + 1], c = conics[3 * i + 2];
    double o = opac ? (double)opac[i] : 1.0;
    for (int64_t py = y0; py < y0 + ty; ++py) {
      double dy = (double)py - my;
      for (int64_t px = x0; px < x0 + tx; ++px) {
        double dx = (double)px - mx;
        double q = a * dx * dx + 2.0 * b * dx * dy + c * dy * dy;
        double w = o * visible(exp(-0.5 * q), tail);
        int64_t p = py * W + px;
        num[3 * p] += w * colors[3 * i];
        num[3 * p + 1] += w * colors[3 * i + 1];
        num[3 * p + 2] += w * colors[3 * i + 2];
        den[p] += w;
      }
    }
  }
  for (int64_t p = 0; p < npx; ++p)
    for (int k = 0; k < 3; ++k) out[3 * p + k] = normalize ? num[3 * p + k] / (den[p] + eps) : num[3 * p + k];
  free(num);
}

/* Float64 gradients of sum(image * grad_out) w.r.t. means (N,2), conics (N,3), colors (N,3)
 * and opacities (N; only written when opac != NULL).  den/out come from ora_render_f64. */
void ora_backward_f64(const double* grad_out, const float* means, const float* conics,
                      const float* colors, const int64_t* radii, const float* opac, int64_t n,
                      int H, int W, int normalize, double eps, double tail, const double* den,
                      const double* out, double* g_means, double* g_conics, double* g_colors,
                      double* g_opac) {
  int64_t x0, y0, tx, ty;
  for (int64_t i = 0; i < n; ++i) {
    double gm[2] = {0, 0}, gq[3] = {0, 0, 0}, gc[3] = {0, 0, 0}, go = 0;
    if (ora_support_rect(means, radii, i, H, W, &x0, &y0, &tx, &ty) > 0) {
      double mx = means[2 * i], my = means[2 * i + 1];
      double a = conics[3 * i], b = conics[3 * i + 1], c = conics[3 * i + 2];
      double o = opac ? (double)opac[i] : 1.0;
      double col[3] = {colors[3 * i], colors[3 * i + 1], colors[3 * i + 2]};
      for (int64_t py = y0; py < y0 + ty; ++py) {
        double dy = (double)py - my;
        for (int64_t px = x0; px < x0 + tx; ++px) {
          double dx = (double)px - mx;
          int64_t p = py * W + px;
          double q = a * dx * dx + 2.0 * b * dx * dy + c * dy * dy;
          double raw = exp(-0.5 * q);
          double base = visible(raw, tail);
          double w = base * o;
          double dn[3], dd = 0.0;
          for (int k = 0; k < 3; ++k) {
            double g = grad_out[3 * p + k];
            if (normalize) {
              dn[k] = g / (den[p] + eps);
              dd -= g * out[3 * p + k] / (den[p] + eps);
            } else {
              dn[k] = g;
            }
          }
          double dw = dd;
          for (int k = 0; k < 3; ++k) {
            gc[k] += dn[k] * w;
            dw += dn[k] * col[k];
          }
          go += dw * base;
          double dq = (tail > 0.0 && raw <= tail) ? 0.0 : -0.5 * raw * dw * o;
          gm[0] += dq * (-2.0 * a * dx - 2.0 * b * dy);
          gm[1] += dq * (-2.0 * b * dx - 2.0 * c * dy);
          gq[0] += dq * dx * dx;
          gq[1] += dq * 2.0 * dx * dy;
          gq[2] += dq * dy * dy;
        }
      }
    }
    g_means[2 * i] = gm[0];
    g_means[2 * i + 1] = gm[1];
    for (int k = 0; k < 3; ++k) {
      g_conics[3 * i + k] = gq[k];
      g_colors[3 * i + k] = gc[k];
    }
    if (opac && g_opac) g_opac[i] = go;
  }
}

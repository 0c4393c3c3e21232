// Tiled forward and backward of the clipped-support normalized / additive renderer.
//
// Both kernels run one CTA per TS x TS tile (TS = 16 or 32) and stage the tile's Gaussian list
// into shared memory with cp.async: whole when it fits (one barrier per tile), otherwise 64
// records at a time, double-buffered, so the L2 gather of the next chunk overlaps the math on
// the current one.
//
// Forward (render_ext.cu:349-431 contract): each warp owns an 8x8 pixel block (two pixels per
// lane, rows r and r+4).  For every 32 staged records a warp builds, with one ballot, the mask
// of the Gaussians whose support rectangle touches its block and walks only those, in
// ascending id; a lane masks its own pixels with the in-rectangle test.  The weight is 2^(qa dx^2 + qb dx dy + qc dy^2)
// on the SFU.  The epilogue writes den raw and out = num / (den + eps) or num.
//
// Backward (render_ext.cu:696-847 contract): a prologue turns grad_out, out and den into the
// per-pixel (dnum_r, dnum_g, dnum_b, dden) of the tile in shared memory (the fit path hands
// them over ready-made).  Work is then Gaussian-major: four lanes own one staged Gaussian and
// walk exactly the pixels of its support rectangle inside the tile — lane q takes columns q,
// q+4, … and runs down each column — so a warp works on eight Gaussians at once.  A counting
// sort orders the staged entries by their loop trip counts first, so the eight Gaussians of a
// warp need nearly the same number of iterations.  Each Gaussian accumulates nine moments
//   R_k = Σ base·dnum_k,  G = Σ base·dw,  S1 = Σ t dx,  S2 = Σ t dy,  S3 = Σ t dx²,
//   S4 = Σ t dx dy,  S5 = Σ t dy²,     dw = dnum·c + dden,  t = raw·dw (0 where the fade clamps)
// from which
//   dL/dμx = o(a S1 + b S2),  dL/dμy = o(b S1 + c S2),  dL/da = -o S3/2,  dL/db = -o S4,
//   dL/dc = -o S5/2,  dL/dc_k = o R_k,  dL/do = G,
// i.e. the reference's per-pixel formulas (render_ext.cu:785-818) summed over pixels.  Along a
// column dx is constant, so S1, S3 and S4 fold into per-column products.  The moments are
// reduce-scattered over the four lanes and added with one atomic per moment into per-Gaussian
// accumulators (fast mode), or stored per (tile, Gaussian) entry, the entries ordered by
// Gaussian with a stable radix sort, and summed per Gaussian in ascending tile order by a second
// kernel (deterministic mode: every entry is computed by its own four lanes in a fixed order, so
// the result does not depend on the scheduling).  A per-Gaussian epilogue applies o, a, b, c
// once.
#include <atomic>

#include <cub/device/device_radix_sort.cuh>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kEpilogueThreads = 256;

template <int TS>
struct Tiling {
  // forward: one warp per 8x8 block of the tile
  static constexpr int kFwdThreads = 32 * (TS / 8) * (TS / 8);
  // backward whole-list stage: what fits in 48 KB of static shared memory beside the pixels
  static constexpr int kBwdStageAll = TS == 16 ? 512 : 448;
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_one() {
  asm volatile("cp.async.wait_group 1;\n" ::: "memory");
}

// Source of a tile's Gaussians: its index list, or — when the list was truncated by the
// capacity — every Gaussian of its image in ascending id (the same order, so results are
// identical).
struct TileList {
  const int32_t* gids;
  int64_t first, count;
  bool direct;
  __device__ __forceinline__ int gid(int64_t k) const {
    return direct ? (int)(first + k) : gids[first + k];
  }
};

__device__ __forceinline__ TileList tile_list(const int32_t* gids, const int32_t* offsets,
                                              int64_t cap, const Frame& fr, int tile) {
  TileList L;
  int64_t lo = offsets[tile], hi = offsets[tile + 1];
  L.gids = gids;
  L.direct = hi > cap;
  L.first = L.direct ? fr.gauss_first : lo;
  L.count = L.direct ? fr.gauss_count : hi - lo;
  return L;
}

constexpr int kFarRect = 48;          // rectangle side (px) above which blocks are tested
constexpr float kUnderflowQ = 230.0f;  // q beyond which every weight is +0 (174.7 + 30%)

// Cover of the 8x8 block at (sx0, sy0) by staged record j (rectangle b): bit c (c < 8) for block
// column c inside [x0, x1), bit 8 + k for block row k inside [y0, y1); 0 when the rectangle
// misses the block.  A large rectangle (an elongated or wide Gaussian) may touch the block only
// where every weight underflows: exp(-q/2) < 2^-126, which ex2.approx.ftz returns as +0, when
// q > 174.7.  Such a block is not covered when the exact minimum of q over the covered pixels
// exceeds kUnderflowQ, a margin of 30% for the rounding of q in either evaluation; adding the
// zero weights would leave every sum unchanged.  Only for a finite opacity and colour: an
// infinite one times a zero weight is NaN, which the full evaluation keeps.
__device__ __forceinline__ unsigned block_cover(const float4 (*st)[4], int j, const int4& b,
                                                int sx0, int sy0) {
  const int x0 = min(max(b.x - sx0, 0), 8), x1 = min(max(b.z - sx0, 0), 8);
  const int y0 = min(max(b.y - sy0, 0), 8), y1 = min(max(b.w - sy0, 0), 8);
  const unsigned xm = ((1u << x1) - 1u) & ~((1u << x0) - 1u);
  const unsigned ym = ((1u << y1) - 1u) & ~((1u << y0) - 1u);
  if (!xm || !ym) return 0u;
  if (b.z - b.x > kFarRect || b.w - b.y > kFarRect) {
    // (mx, my, ·, ·), (·, op, r, g), (b, a, b, c)
    const float4 p0 = st[j][0], p1 = st[j][1], p2 = st[j][2];
    const float qmin = rect_min_q(p0.x, p0.y, p2.y, p2.z, p2.w, (float)(sx0 + x0),
                                  (float)(sx0 + x1 - 1), (float)(sy0 + y0),
                                  (float)(sy0 + y1 - 1));
    const bool finite = isfinite(p1.y) && isfinite(p1.z) && isfinite(p1.w) && isfinite(p2.x);
    if (qmin > kUnderflowQ && finite) return 0u;
  }
  return xm | (ym << 8);
}

// Ballot of the staged entries [0, min(m, 32)) covering the block at (sx0, sy0); lane l also
// gets entry l's cover.  The rectangles come from `rects` when given, else from the records.
__device__ __forceinline__ unsigned hit_cover(const float4 (*st)[4], const int4* rects, int m,
                                              int sx0, int sy0, int lane, unsigned& cover) {
  cover = 0u;
  if (lane < m) {
    const int4 b = rects ? rects[lane] : *reinterpret_cast<const int4*>(&st[lane][3]);
    cover = block_cover(st, lane, b, sx0, sy0);
  }
  return __ballot_sync(0xffffffffu, cover != 0u);
}

// Lists up to kStageAll Gaussians are staged whole (one barrier per tile; the warps then run
// independently); longer lists stream through the two halves of the stage, double-buffered.
constexpr int kStageAll = 512;

// Issues the copies of entries [k0, k0+m) into `dst` with NT threads: 16-byte piece (q & 3) of
// entry (q >> 2) for q = threadIdx.x, threadIdx.x + NT, …  With `rect_dst` the rectangles
// (piece 3) go to that packed array instead: the lanes of a warp reading 32 consecutive
// entries' rectangles then hit distinct banks (at the 64-byte record stride every fourth
// entry shares a bank group).
template <int NT>
__device__ __forceinline__ void stage_range(float4 (*dst)[4], const Splat* rec,
                                            const TileList& L, int64_t k0, int m,
                                            int* gid_dst = nullptr, int4* rect_dst = nullptr) {
  for (int q = threadIdx.x; q < 4 * m; q += NT) {
    const int slot = q >> 2, piece = q & 3;
    const int g = L.gid(k0 + slot);
    void* to = (rect_dst && piece == 3) ? static_cast<void*>(&rect_dst[slot])
                                        : static_cast<void*>(&dst[slot][piece]);
    cp_async16(to, reinterpret_cast<const float4*>(rec + g) + piece);
    if (gid_dst && piece == 0) gid_dst[slot] = g;  // the backward's atomics need the id
  }
}

// ---------------------------------------------------------------------------------------------
// Forward evaluation of one 8x8 pixel block by one warp, four Gaussians at a time.
//
// The block's hits (staged entries whose rectangle touches it and is not wholly underflowed, in
// ascending list order) are listed per warp in shared memory; an entry is the staged slot
// (bits 0-14) and its cover of the block (bits 16-23 block columns, 24-31 block rows).  The
// lanes form four groups of eight: group g = lane >> 3 evaluates hit 4i + g, lane (c, g) the
// eight pixels of block column c, so the setup of a Gaussian (record loads, dx terms) serves
// eight pixels, and rows k and k + 4 share packed (f32x2) arithmetic.  Each lane keeps a
// partial sum per pixel and channel; the k-th hit of a block always goes to partial k mod 4,
// however its tile list was staged or chunked, and the partials are combined as
// (p0 + p1) + (p2 + p3).  Every kernel that renders a tile (forward, fused render pass, fused
// fit pass) evaluates its blocks this way, so their images agree bitwise.  A list is padded to
// a multiple of four with the null record (opacity 0, no cover).
constexpr int kQueueLen = 40;   // per-batch queue: ≥ 3 pending + 32 new hits + 3 padding
constexpr int kCarrySlots = 4;  // per warp: staged slots for pending hits across a refill

// Row offsets of the fast evaluation: for row pair k (rows k and k + 4) the row's index when
// the 8-bit row mask covers it, and kRowMasked when not.  Added to dy0, a masked
// row's dy becomes so large that qc dy^2 overflows to -inf and its weight is exactly +0, so
// the pair needs no per-pixel select.  Valid for regular records only (below).
constexpr float kRowMasked = 1e30f;
struct RowOffsets {
  // v[rows][h] = the pairs k = 2h and 2h + 1 as (k, k + 4, k + 1, k + 5): two 16-byte loads
  float4 v[256][2];
};
constexpr float row_offset(int m, int row) { return ((m >> row) & 1) ? (float)row : kRowMasked; }
constexpr RowOffsets make_row_offsets() {
  RowOffsets t{};
  for (int m = 0; m < 256; ++m)
    for (int h = 0; h < 2; ++h) {
      t.v[m][h].x = row_offset(m, 2 * h);
      t.v[m][h].y = row_offset(m, 2 * h + 4);
      t.v[m][h].z = row_offset(m, 2 * h + 1);
      t.v[m][h].w = row_offset(m, 2 * h + 5);
    }
  return t;
}
__device__ const RowOffsets kRowOff = make_row_offsets();

// A record whose masked pixels the fast evaluation zeroes exactly: a positive-definite conic
// (qa, qc < 0 with qb^2 < 4 qa qc, and qc not so small that dy = kRowMasked leaves q finite)
// and a finite opacity and colour.  A tile staging any other record renders by select.
__device__ __forceinline__ bool regular_record(const float4& p0, const float4& p1, float cb) {
  return p0.z < 0.0f && p1.x < -1e-20f && p0.w * p0.w < 4.0f * p0.z * p1.x &&
         fabsf(p1.y) + fabsf(p1.z) + fabsf(p1.w) + fabsf(cb) < 3.0e38f;
}

// Staged slots [0, m): true when every record is regular.  A CTA-wide barrier: every thread
// of the CTA calls it.
template <int NT>
__device__ __forceinline__ bool all_regular(const float4 (*st)[4], int m) {
  bool ok = true;
  for (int t = threadIdx.x; t < m; t += NT) ok = ok && regular_record(st[t][0], st[t][1], st[t][2].x);
  return __syncthreads_and(ok) != 0;
}

// The null record: zero opacity and colour, a unit conic, an empty rectangle.
__device__ __forceinline__ void write_null_record(float4 (*st)[4], int slot) {
  st[slot][0] = make_float4(0.f, 0.f, -1.f, 0.f);
  st[slot][1] = make_float4(-1.f, 0.f, 0.f, 0.f);
  st[slot][2] = make_float4(0.f, 0.f, 0.f, 0.f);
  st[slot][3] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Hits q[0..4) of groups 0-3: lane (c, g) adds its eight pixels of hit q[g].  EXACT: masked
// pixels by select (any record); otherwise by the row offsets (regular records).
template <bool FADE, bool EXACT>
__device__ __forceinline__ void eval4(const float4 (*st)[4], const uint32_t* q, int lane,
                                      float fx, float fy0, float tail, float2 (&acc)[4][4]) {
  const uint32_t e = q[lane >> 3];
  const int j = (int)(e & 0x7fffu);
  const uint32_t rows = (e & (1u << (16 + (lane & 7)))) ? (e >> 24) : 0u;
  const float4 p0 = st[j][0], p1 = st[j][1];
  const float cb = st[j][2].x;
  const float dx = fx - p0.x, dy0 = fy0 - p0.y;
  const float bdx = p0.w * dx, adx2 = p0.z * dx * dx;
  const float2 bdx2 = make_float2(bdx, bdx), adx22 = make_float2(adx2, adx2);
  const float2 qc2 = make_float2(p1.x, p1.x), op2 = make_float2(p1.y, p1.y);
  const float2 dy02 = make_float2(dy0, dy0);
  const float2 cr2 = make_float2(p1.z, p1.z), cg2 = make_float2(p1.w, p1.w);
  const float2 cb2 = make_float2(cb, cb);
  float4 o4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (!EXACT && (k & 1) == 0) o4 = kRowOff.v[rows][k >> 1];
    const float2 off = EXACT ? make_float2((float)k, (float)(k + 4))
                             : ((k & 1) ? make_float2(o4.z, o4.w) : make_float2(o4.x, o4.y));
    const float2 dy = __fadd2_rn(dy02, off);
    const float2 t = __ffma2_rn(qc2, dy, bdx2);
    const float2 qq = __ffma2_rn(dy, t, adx22);
    float2 v = make_float2(fast_exp2(qq.x), fast_exp2(qq.y));
    if (FADE) v = make_float2(fmaxf(v.x - tail, 0.0f), fmaxf(v.y - tail, 0.0f));
    float2 w = __fmul2_rn(v, op2);
    if (EXACT) {
      w.x = (rows & (1u << k)) ? w.x : 0.0f;
      w.y = (rows & (1u << (k + 4))) ? w.y : 0.0f;
    }
    acc[k][0] = __ffma2_rn(w, cr2, acc[k][0]);
    acc[k][1] = __ffma2_rn(w, cg2, acc[k][1]);
    acc[k][2] = __ffma2_rn(w, cb2, acc[k][2]);
    acc[k][3] = __fadd2_rn(acc[k][3], w);
  }
}

// Appends the hits among staged slots [slot0, slot0 + min(cnt, 32)) to the list q[0..qn).
__device__ __forceinline__ int enqueue_hits(const float4 (*st)[4], const int4* rects, int slot0,
                                            int cnt, int sx0, int sy0, int lane, uint32_t* q,
                                            int qn) {
  unsigned cover;
  const unsigned hits = hit_cover(st + slot0, rects ? rects + slot0 : nullptr, cnt, sx0, sy0,
                                  lane, cover);
  if (cover) q[qn + __popc(hits & ((1u << lane) - 1u))] = (uint32_t)(slot0 + lane) | (cover << 16);
  return qn + __popc(hits);
}

// Evaluates the listed hits four at a time.  `all`: the last partial group too, padded with the
// null record (the list ends empty); otherwise the remainder (< 4) moves to the front.  Returns
// the new length.  The list needs room for 3 entries of padding.
template <bool FADE>
__device__ __forceinline__ int drain(const float4 (*st)[4], uint32_t* q, int qn, bool all,
                                     bool exact, int null_slot, int lane, float fx, float fy0,
                                     float tail, float2 (&acc)[4][4]) {
  if (all && (qn & 3)) {
    if (lane < 4 && lane >= (qn & 3)) q[(qn & ~3) + lane] = (uint32_t)null_slot;
    qn = (qn + 3) & ~3;
  }
  __syncwarp();
  const int full = qn & ~3;
  if (exact) {
#pragma unroll 1
    for (int i = 0; i < full; i += 4) eval4<FADE, true>(st, q + i, lane, fx, fy0, tail, acc);
  } else {
#pragma unroll 1
    for (int i = 0; i < full; i += 4) eval4<FADE, false>(st, q + i, lane, fx, fy0, tail, acc);
  }
  const int r = qn - full;
  if (r == 0) return 0;
  const uint32_t keep = lane < r ? q[full + lane] : 0u;
  __syncwarp();
  if (lane < r) q[lane] = keep;
  __syncwarp();
  return r;
}

// Before a staged chunk is refilled: the records of the pending hits q[0..qn) (qn < 4) move to
// the warp's carry slots carry0 + i (a hit already there stays), and the list points at them.
__device__ __forceinline__ void carry_pending(float4 (*st)[4], uint32_t* q, int qn, int carry0,
                                              int lane) {
  if (lane < 3 * qn) {  // pieces 0-2 hold what the evaluation reads
    const int i = lane / 3, piece = lane - 3 * i;
    const int src = (int)(q[i] & 0x7fffu);
    if (src != carry0 + i) st[carry0 + i][piece] = st[src][piece];
  }
  __syncwarp();
  if (lane < qn) q[lane] = (q[lane] & 0xffff0000u) | (uint32_t)(carry0 + lane);
  __syncwarp();
}

// The four group partials of a block combined as (p0 + p1) + (p2 + p3) by a two-level
// reduce-scatter: lane (c, g) ends with block rows first_row(lane) and first_row(lane) + 1 of
// column c.
__device__ __forceinline__ int block_first_row(int lane) {
  return ((lane & 8) ? 4 : 0) + ((lane & 16) ? 2 : 0);
}
__device__ __forceinline__ void combine_groups(const float2 (&acc)[4][4], int lane,
                                               float (&v)[2][4]) {
  // acc[r][ch].x is block row r, .y block row r + 4
  float h[4][4];
  const bool odd = lane & 8;
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      const float send = odd ? acc[r][ch].x : acc[r][ch].y;
      const float keep = odd ? acc[r][ch].y : acc[r][ch].x;
      h[r][ch] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
  const bool hi = lane & 16;
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) {
      const float send = hi ? h[r][ch] : h[r + 2][ch];
      const float keep = hi ? h[r + 2][ch] : h[r][ch];
      v[r][ch] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
}

// Pixel losses of fit.py:800-809 (mean over channels, then over the image's pixels).
enum LossKind { kNoLoss = 0, kL1 = 1, kL2 = 2, kCharbonnier = 3 };

// 1/(H W) then /3: autograd's factors for the mean over the image's pixels of the channel mean.
__device__ __forceinline__ float pixel_loss_scale(int H, int W) {
  const float per_pixel = 1.0f / (float)((int64_t)H * W);
  return per_pixel / 3.0f;
}

// Finishes pixel p of a forward from its accumulators a = (num_r, num_g, num_b, den): writes
// den and the image (LOSS == kNoLoss always, otherwise where the pointers are given) and, for a
// fit iteration, returns the backward's per-pixel input (dL/dnum_rgb, dL/dden) with the pixel's
// loss in lp and squared error in sq.  The loss gradient repeats autograd's arithmetic for the
// mean-of-means, so it is bitwise the eager gradient.
template <bool NORMALIZE, int LOSS>
__device__ __forceinline__ float4 finish_pixel(const float* a, int64_t p, float eps,
                                               float per_value, float charb_eps2, float* out,
                                               float* den, const float* target, float& lp,
                                               float& sq) {
  float o[3];
  const float denom = a[3] + eps, inv = 1.0f / denom;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) o[ch] = NORMALIZE ? a[ch] * inv : a[ch];
  if (LOSS == kNoLoss || den) den[p] = a[3];
  if (LOSS == kNoLoss || out) {
    out[3 * p] = o[0];
    out[3 * p + 1] = o[1];
    out[3 * p + 2] = o[2];
  }
  lp = sq = 0.f;
  if constexpr (LOSS == kNoLoss) {
    return make_float4(0.f, 0.f, 0.f, 0.f);
  } else {
  float g[3];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float d = o[ch] - target[3 * p + ch];
    const float d2 = d * d;
    sq += d2;
    if (LOSS == kL2) {
      g[ch] = per_value * d + per_value * d;
      lp += d2;
    } else if (LOSS == kL1) {
      g[ch] = per_value * (float)((d > 0.f) - (d < 0.f));
      lp += fabsf(d);
    } else {
      const float r = sqrtf(d2 + charb_eps2);
      const float q = per_value / (2.0f * r);
      g[ch] = q * d + q * d;
      lp += r;
    }
  }
  if (NORMALIZE)
    return make_float4(g[0] * inv, g[1] * inv, g[2] * inv,
                       -(g[0] * o[0] + g[1] * o[1] + g[2] * o[2]) * inv);
  return make_float4(g[0], g[1], g[2], 0.f);
  }
}

// Shared memory of the forward kernel (dynamic): the stage (whole lists up to kStageAll
// records, or two halves of it for a streamed list) followed by every warp's carry slots and
// the null record; the staged records' rectangles, packed; and every warp's hit list, which
// after the block's last evaluation holds the block's 8x8 pixels (RGB rows, then den) on their
// way out as whole float4 image rows.  One warp per 8x8 block.
template <int TS>
struct FwdSmem {
  static constexpr int kWarps = (TS / 8) * (TS / 8);
  static constexpr int kNullSlot = kStageAll + kWarps * kCarrySlots;
  static constexpr int kSlots = kNullSlot + 1;
  static constexpr int kListLen = kStageAll + 4;  // a whole stage's hits and padding
  static constexpr size_t kStageBytes = (size_t)kSlots * 4 * sizeof(float4);
  static constexpr size_t kRectBytes = (size_t)kStageAll * sizeof(int4);
  static constexpr size_t kListBytes = (size_t)kWarps * kListLen * sizeof(uint32_t);
  static constexpr size_t kRectOff = kStageBytes;
  static constexpr size_t kListOff = kRectOff + kRectBytes;
  static constexpr size_t kBytes = kListOff + kListBytes;
  static_assert(kListLen * sizeof(uint32_t) >= 8 * 32 * sizeof(float), "a block's pixels fit");
  static_assert(kListLen * sizeof(uint32_t) % 16 == 0 && kListOff % 16 == 0, "float4 rows");
};

// Accumulates one warp's 8x8 block over a tile's list, staged whole by the caller (who also
// passed the barrier after it), or streamed here through two halves of the stage with the
// pending hits carried across each refill (chunk 0 already in flight when `chunk0_issued`; the
// stream ends with a barrier, after which the stage may be refilled).  `qcap` is the capacity
// of the warp's list q: with room for a whole stage (or half) plus padding the hits are listed
// first and evaluated in one run, otherwise batch by batch.  `exact`: the staged records were
// checked (all_regular) and some is not regular.  Every thread of the CTA calls it: it holds
// the CTA's barriers.
template <int NT, bool FADE>
__device__ __forceinline__ void accumulate_block(float4 (*stage)[4], int stage_slots,
                                                 const Splat* __restrict__ rec,
                                                 const TileList& L, uint32_t* q, int qcap,
                                                 int carry0, int null_slot, bool active, int sx0,
                                                 int sy0, int lane, float tail,
                                                 float2 (&acc)[4][4], bool staged_whole,
                                                 bool exact, bool chunk0_issued = false,
                                                 int4* rects = nullptr) {
  const float fx = (float)(sx0 + (lane & 7)), fy0 = (float)sy0;
  int qn = 0;
  if (staged_whole) {  // the caller staged the list and passed the barrier
    const int m = (int)L.count;
    if (active) {
      const bool listed = qcap >= m + 4;
      for (int base = 0; base < m; base += 32) {
        qn = enqueue_hits(stage, rects, base, m - base, sx0, sy0, lane, q, qn);
        if (!listed) qn = drain<FADE>(stage, q, qn, false, exact, null_slot, lane, fx, fy0, tail, acc);
      }
      drain<FADE>(stage, q, qn, true, exact, null_slot, lane, fx, fy0, tail, acc);
    }
    return;
  }
  const int half = stage_slots / 2;
  const bool listed = qcap >= half + 8;
  const int64_t count = L.count;
  const int nchunks = (int)((count + half - 1) / half);
  auto len = [&](int64_t k0) { return (int)(count - k0 < half ? count - k0 : half); };
  if (!chunk0_issued) {
    stage_range<NT>(stage, rec, L, 0, len(0), nullptr, rects);
    cp_async_commit();
  }
  for (int c = 0; c < nchunks; ++c) {
    const int64_t k0 = (int64_t)c * half;
    if (c + 1 < nchunks)
      stage_range<NT>(stage + ((c + 1) & 1) * half, rec, L, k0 + half, len(k0 + half), nullptr,
                      rects ? rects + ((c + 1) & 1) * half : nullptr);
    cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
    const int m = len(k0), s0 = (c & 1) * half;
    exact = exact || !all_regular<NT>(stage + s0, m);
    if (active) {
      for (int base = 0; base < m; base += 32) {
        qn = enqueue_hits(stage, rects, s0 + base, m - base, sx0, sy0, lane, q, qn);
        if (!listed) qn = drain<FADE>(stage, q, qn, false, exact, null_slot, lane, fx, fy0, tail, acc);
      }
      if (listed) qn = drain<FADE>(stage, q, qn, false, exact, null_slot, lane, fx, fy0, tail, acc);
      if (c + 1 < nchunks) carry_pending(stage, q, qn, carry0, lane);
    }
    __syncthreads();
  }
  if (active) drain<FADE>(stage, q, qn, true, exact, null_slot, lane, fx, fy0, tail, acc);
  __syncthreads();
}

// Forward of one tile, one warp per 8x8 block.  LOSS == kNoLoss: writes out and den.
// Otherwise (a fit iteration) it also evaluates the pixel loss against target and writes the
// backward's per-pixel input pixel_grad = (dL/dnum_rgb, dL/dden) (out and den only when given)
// and adds each image's loss and mean squared error into loss[2 b], loss[2 b + 1]
// (finish_pixel).  Each warp lists its block's hits (accumulate_block), per staged chunk when
// the list streams.
template <int TS, bool NORMALIZE, bool FADE, int LOSS>
__global__ void __launch_bounds__(Tiling<TS>::kFwdThreads, 2)
    forward_kernel(const Splat* __restrict__ rec, int64_t n, const int32_t* __restrict__ gids,
                   int64_t cap, const int32_t* __restrict__ offsets, Frames frames, float eps,
                   float tail, float* __restrict__ out, float* __restrict__ den,
                   const float* __restrict__ target, float4* __restrict__ pixel_grad,
                   float* __restrict__ loss, float charb_eps2, int chunk) {
  pdl_wait();
  pdl_trigger();
  using S = FwdSmem<TS>;
  constexpr int NT = Tiling<TS>::kFwdThreads;
  extern __shared__ __align__(16) unsigned char fwd_smem[];
  float4(*stage)[4] = reinterpret_cast<float4(*)[4]>(fwd_smem);
  const int tile = blockIdx.x;
  const Frame fr = frame_of_tile(frames, tile, n);
  const int local = tile - fr.first_tile;
  const int tx0 = (local % fr.tiles_x) * TS, ty0 = (local / fr.tiles_x) * TS;
  const int H = fr.H, W = fr.W;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int sx0 = tx0 + (warp % (TS / 8)) * 8, sy0 = ty0 + (warp / (TS / 8)) * 8;
  uint32_t* q = reinterpret_cast<uint32_t*>(fwd_smem + S::kListOff) + warp * S::kListLen;
  int4* rects = reinterpret_cast<int4*>(fwd_smem + S::kRectOff);
  const TileList L = tile_list(gids, offsets, cap, fr, tile);
  const bool whole = L.count <= kStageAll;
  if (threadIdx.x == 0) write_null_record(stage, S::kNullSlot);
  float2 acc[4][4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int ch = 0; ch < 4; ++ch) acc[k][ch] = make_float2(0.f, 0.f);
  bool exact = false;
  if (whole) {
    stage_range<NT>(stage, rec, L, 0, (int)L.count, nullptr, rects);
    cp_async_commit();
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    exact = !all_regular<NT>(stage, (int)L.count);
  }
  // a streamed list moves through two chunks of `chunk` records (at most half the stage)
  accumulate_block<NT, FADE>(stage, 2 * chunk, rec, L, q, S::kListLen,
                             kStageAll + warp * kCarrySlots, S::kNullSlot, true, sx0, sy0, lane,
                             tail, acc, whole, exact, false, rects);
  float v[2][4];
  combine_groups(acc, lane, v);
  const int cx = lane & 7, r0 = block_first_row(lane);
  const int px = sx0 + cx;
  if constexpr (LOSS == kNoLoss) {
    // whole float4 rows when the block lies inside the image and its rows are 16-B aligned
    const int64_t p_row0 = fr.pixel_base + (int64_t)sy0 * W + sx0;
    const bool vec = sx0 + 8 <= W && sy0 + 8 <= H && (W & 3) == 0 && (p_row0 & 3) == 0 &&
                     ((reinterpret_cast<uintptr_t>(out) | reinterpret_cast<uintptr_t>(den)) & 15) == 0;
    if (vec) {
      // the warp's 8 rows of 32 floats: 24 interleaved RGB, then 8 den, in the warp's list
      // (every lane has read its last hit: the reduce-scatter above is warp-synchronous)
      __syncwarp();
      float* tb = reinterpret_cast<float*>(q);
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const float inv = 1.0f / (v[k][3] + eps);
        float* row = tb + (r0 + k) * 32;
        row[3 * cx] = NORMALIZE ? v[k][0] * inv : v[k][0];
        row[3 * cx + 1] = NORMALIZE ? v[k][1] * inv : v[k][1];
        row[3 * cx + 2] = NORMALIZE ? v[k][2] * inv : v[k][2];
        row[24 + cx] = v[k][3];
      }
      __syncwarp();
#pragma unroll
      for (int it = 0; it < 2; ++it) {
        const int idx = lane + 32 * it;  // 48 RGB float4s (8 rows x 6), then 16 den float4s
        if (idx < 48) {
          const int row = idx / 6, part = idx - 6 * row;
          const float4 vv = reinterpret_cast<const float4*>(tb + row * 32)[part];
          reinterpret_cast<float4*>(out + 3 * (p_row0 + (int64_t)row * W))[part] = vv;
        } else {
          const int d = idx - 48, row = d >> 1, part = d & 1;
          const float4 vv = reinterpret_cast<const float4*>(tb + row * 32 + 24)[part];
          reinterpret_cast<float4*>(den + p_row0 + (int64_t)row * W)[part] = vv;
        }
      }
      return;
    }
  }
  float loss_sum = 0.f, sq_sum = 0.f;
  const float per_value = pixel_loss_scale(H, W);
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int py = sy0 + r0 + k;
    if (px < W && py < H) {
      const int64_t p = fr.pixel_base + (int64_t)py * W + px;
      float lp, sq;
      const float4 pg = finish_pixel<NORMALIZE, LOSS>(v[k], p, eps, per_value, charb_eps2, out,
                                                      den, target, lp, sq);
      if (LOSS != kNoLoss) {
        pixel_grad[p] = pg;
        loss_sum += lp;
        sq_sum += sq;
      }
    }
  }
  if (LOSS != kNoLoss && loss) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      loss_sum += __shfl_xor_sync(0xffffffffu, loss_sum, o);
      sq_sum += __shfl_xor_sync(0xffffffffu, sq_sum, o);
    }
    if (lane == 0) {
      atomicAdd(loss + 2 * fr.image, loss_sum * per_value);
      atomicAdd(loss + 2 * fr.image + 1, sq_sum * per_value);
    }
  }
}

// One level of a reduce-scatter butterfly: lanes whose `bit` is clear keep slots [0, K) of v,
// the others keep slots [K, N) (as their new slots 0..); each side receives the partner's copy
// of the slots it keeps and adds it.  Missing slots count as zero.
template <int N, int K>
__device__ __forceinline__ void scatter_level(const float (&v)[N], float (&w)[K], bool bit,
                                              int lane_mask) {
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const float hi_v = (K + i < N) ? v[K + i] : 0.0f;
    const float send = bit ? v[i] : hi_v;
    const float keep = bit ? hi_v : v[i];
    w[i] = keep + __shfl_xor_sync(0xffffffffu, send, lane_mask);
  }
}

// Inputs and outputs of the fused fit tile pass (FUSED backward): the forward of the tile runs
// first in the same CTA over the staged records and its loss gradient goes straight into the
// backward's shared-memory pixel inputs.  image / den / loss are optional (NULL skips them).
struct FusedFit {
  const float* target;
  float* image;
  float* den;
  float* loss;
  int loss_kind;  // LossKind: kL1, kL2 or kCharbonnier
  float charb_eps2;
  // render mode (target unused): the pixel inputs come from this (P,3) image gradient as in the
  // backward's own prologue, and image / den are always written
  const float* grad_out;
};

// A render forward's outputs at pixel p and the backward's per-pixel input from grad_out: the
// arithmetic of forward_kernel's epilogue and of the backward prologue (out = num / (den + eps)
// in normalized mode).
__device__ __forceinline__ float4 render_pixel_grad(int normalize, const float* a, int64_t p,
                                                    float eps, const float* __restrict__ go,
                                                    float* out, float* den) {
  const float denom = a[3] + eps, inv = 1.0f / denom;
  float o[3];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) o[ch] = normalize ? a[ch] * inv : a[ch];
  den[p] = a[3];
  out[3 * p] = o[0];
  out[3 * p + 1] = o[1];
  out[3 * p + 2] = o[2];
  const float gr = go[3 * p], gg = go[3 * p + 1], gb = go[3 * p + 2];
  if (!normalize) return make_float4(gr, gg, gb, 0.f);
  // the backward prologue's arithmetic (backward_kernel), so the pixel inputs agree bitwise
  return make_float4(gr * inv, gg * inv, gb * inv, -(gr * o[0] + gg * o[1] + gb * o[2]) * inv);
}

// finish_pixel with the loss kind and normalisation chosen at run time (uniform per launch).
__device__ __forceinline__ float4 finish_pixel_rt(int normalize, int loss_kind, const float* a,
                                                  int64_t p, float eps, float per_value,
                                                  float ce2, float* out, float* den,
                                                  const float* target, float& lp, float& sq) {
#define SS_FIN(N, K) finish_pixel<N, K>(a, p, eps, per_value, ce2, out, den, target, lp, sq)
  if (normalize) {
    if (loss_kind == kL1) return SS_FIN(true, kL1);
    if (loss_kind == kL2) return SS_FIN(true, kL2);
    return SS_FIN(true, kCharbonnier);
  }
  if (loss_kind == kL1) return SS_FIN(false, kL1);
  if (loss_kind == kL2) return SS_FIN(false, kL2);
  return SS_FIN(false, kCharbonnier);
#undef SS_FIN
}

// Shared memory of the backward tile kernel (dynamic): the stage (plus, in the fused pass, every
// warp's carry slots for the forward phase), the tile's per-pixel inputs, the staged ids, the
// cost-class order and counters, and in the fused pass the warps' hit queues.
template <int TS, int NT, bool FUSED>
struct BwdSmem {
  static constexpr int kStageMax = Tiling<TS>::kBwdStageAll;
  static constexpr int kWarps = NT / 32;
  // fused pass only: every warp's carry slots, then the null record (slot kSlots - 1)
  static constexpr int kSlots = kStageMax + (FUSED ? kWarps * kCarrySlots + 1 : 0);
  static constexpr size_t kPixOff = (size_t)kSlots * 4 * sizeof(float4);
  static constexpr size_t kGidOff = kPixOff + (size_t)TS * TS * sizeof(float4);
  static constexpr size_t kOrderOff = kGidOff + (size_t)kStageMax * sizeof(int);
  static constexpr size_t kClassOff = kOrderOff + (size_t)kStageMax * sizeof(int);
  static constexpr size_t kNextOff = kClassOff + 256 * sizeof(int);
  static constexpr size_t kQueueOff = kNextOff + 16;
  static constexpr size_t kBytes =
      kQueueOff + (FUSED ? (size_t)kWarps * kQueueLen * sizeof(uint32_t) : 0);
};

template <int TS, int NT>
struct BackwardOccupancy {  // CTAs per SM the register budget is planned for
  static constexpr int kBlocks = TS == 16 ? (NT == 128 ? 6 : 4) : (NT == 256 ? 4 : 2);
};

// FUSED: the pixel inputs come from the tile's own forward (FusedFit) instead of grad_out /
// out / den or pixel_grad.
template <int TS, int NT, bool FADE, bool DETERMINISTIC, bool PIXGRAD, bool FUSED = false>
__global__ void __launch_bounds__(NT, (BackwardOccupancy<TS, NT>::kBlocks))
    backward_kernel(const float* __restrict__ grad_out, const Splat* __restrict__ rec,
                    int64_t n, const float* __restrict__ den, const float* __restrict__ out,
                    const float4* __restrict__ pixel_grad, const int32_t* __restrict__ gids,
                    int64_t cap, const int32_t* __restrict__ offsets, Frames frames,
                    int normalize, float eps, float tail, float* __restrict__ moments,
                    float* __restrict__ partials, uint32_t* status, FusedFit ff) {
  pdl_wait();
  pdl_trigger();
  using S = BwdSmem<TS, NT, FUSED>;
  constexpr int kStageMax = Tiling<TS>::kBwdStageAll;
  constexpr int kHalf = kStageMax / 2;  // entries per chunk when a long list streams through
  extern __shared__ __align__(16) unsigned char bwd_smem[];
  float4(*stage)[4] = reinterpret_cast<float4(*)[4]>(bwd_smem);
  float4* pix = reinterpret_cast<float4*>(bwd_smem + S::kPixOff);
  int* stage_gid = reinterpret_cast<int*>(bwd_smem + S::kGidOff);
  int* order = reinterpret_cast<int*>(bwd_smem + S::kOrderOff);
  int* class_count = reinterpret_cast<int*>(bwd_smem + S::kClassOff);
  int& next_group = *reinterpret_cast<int*>(bwd_smem + S::kNextOff);  // the next group a warp takes
  const int tile = blockIdx.x;
  const Frame fr = frame_of_tile(frames, tile, n);
  const int local = tile - fr.first_tile;
  const int tx0 = (local % fr.tiles_x) * TS, ty0 = (local / fr.tiles_x) * TS;
  const int H = fr.H, W = fr.W;
  const TileList L = tile_list(gids, offsets, cap, fr, tile);
  if (DETERMINISTIC && L.direct) {
    if (threadIdx.x == 0) raise_status(status, SS_STATUS_DETERMINISTIC_TRUNCATED);
    return;
  }
  // the first records' copies are in flight while the pixel inputs load
  if (L.count <= kStageMax)
    stage_range<NT>(stage, rec, L, 0, (int)L.count, stage_gid);
  else
    stage_range<NT>(stage, rec, L, 0, (int)(L.count < kHalf ? L.count : kHalf), stage_gid);
  cp_async_commit();
  // every pixel input this thread wrote is finite (the underflowed-entry skip below needs it)
  bool pix_ok = true;
  // Per-pixel inputs of the tile: every load is issued before the first is used.
  constexpr int kPx = TS * TS / NT;
  static_assert(TS * TS % NT == 0, "pixels per thread");
  if constexpr (!FUSED) {
    float4 va[kPx];
    float dn[kPx], o0[kPx], o1[kPx], o2[kPx];
#pragma unroll
    for (int i = 0; i < kPx; ++i) {
      const int q = threadIdx.x + i * NT;
      const int x = tx0 + (q % TS), y = ty0 + (q / TS);
      va[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      dn[i] = 0.f;
      o0[i] = o1[i] = o2[i] = 0.f;
      if (x < W && y < H) {
        const int64_t p = fr.pixel_base + (int64_t)y * W + x;
        if (PIXGRAD) {
          va[i] = pixel_grad[p];
        } else {
          va[i] = make_float4(grad_out[3 * p], grad_out[3 * p + 1], grad_out[3 * p + 2], 0.f);
          if (normalize) {
            dn[i] = den[p];
            o0[i] = out[3 * p];
            o1[i] = out[3 * p + 1];
            o2[i] = out[3 * p + 2];
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kPx; ++i) {
      const int q = threadIdx.x + i * NT;
      float4 v = va[i];
      if (!PIXGRAD && normalize) {
        const int x = tx0 + (q % TS), y = ty0 + (q / TS);
        if (x < W && y < H) {
          const float inv = 1.0f / (dn[i] + eps);
          const float gr = v.x, gg = v.y, gb = v.z;
          v.x = gr * inv;
          v.y = gg * inv;
          v.z = gb * inv;
          v.w = -(gr * o0[i] + gg * o1[i] + gb * o2[i]) * inv;
        }
      }
      pix_ok = pix_ok && isfinite(v.x) && isfinite(v.y) && isfinite(v.z) && isfinite(v.w);
      pix[q] = v;
    }
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int member = lane >> 2, quad = lane & 3;
  // Order of the staged entries [0, m) by a counting sort into 256 cost classes (loop passes
  // descending, then rows descending), so the eight Gaussians of a warp have nearly the same
  // loop trip counts and the heaviest groups start first.  The order within a class comes
  // from shared-memory atomics and varies from run to run; no result depends on it (every
  // entry's moments are computed by its own four lanes).
  bool tile_finite = false;  // set once the pixel inputs are in shared memory
  auto prepare = [&](float4(*st)[4], int m, int* ord) {
    constexpr int kPer = (kStageMax + NT - 1) / NT;  // entries per thread
    int code[kPer];
    for (int i = threadIdx.x; i < 256; i += NT) class_count[i] = 0;
    if (threadIdx.x == 0) next_group = 0;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
      const int t = threadIdx.x + i * NT;
      code[i] = -1;
      if (t < m) {
        int4 r = *reinterpret_cast<const int4*>(&st[t][3]);
        // An entry whose every pixel in the tile has q > kUnderflowQ adds exactly +0 to every
        // moment (weight +0 times finite inputs): its rectangle is emptied so that its four
        // lanes skip the walk (the forward's block test, at the scale of the entry).
        if (tile_finite && (r.z - r.x > kFarRect || r.w - r.y > kFarRect)) {
          const float4 p0 = st[t][0], p1 = st[t][1], p2 = st[t][2];
          const int rx0 = max(r.x, tx0), rx1 = min(r.z, tx0 + TS) - 1;
          const int ry0 = max(r.y, ty0), ry1 = min(r.w, ty0 + TS) - 1;
          if (rx1 >= rx0 && ry1 >= ry0 && isfinite(p1.y) && isfinite(p1.z) && isfinite(p1.w) &&
              isfinite(p2.x) &&
              rect_min_q(p0.x, p0.y, p2.y, p2.z, p2.w, (float)rx0, (float)rx1, (float)ry0,
                         (float)ry1) > kUnderflowQ) {
            r.z = r.x;
            reinterpret_cast<int4*>(&st[t][3])->z = r.x;
          }
        }
        const int w = min(r.z - tx0, TS) - max(r.x - tx0, 0);
        const int h = min(r.w - ty0, TS) - max(r.y - ty0, 0);
        const int passes = w > 0 && h > 0 ? min((w + 3) >> 2, 8) : 0;
        const int cls = passes > 0 ? (8 - passes) * 32 + (32 - min(h, 32)) : 255;
        code[i] = (cls << 16) | atomicAdd(&class_count[cls], 1);
      }
    }
    __syncthreads();
    if (warp == 0) {  // exclusive scan of the 256 class counts, eight per lane
      int cc[8];
      int x = 0;
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        cc[k] = class_count[8 * lane + k];
        x += cc[k];
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      int run = x;
#pragma unroll
      for (int k = 7; k >= 0; --k) {
        run -= cc[k];
        class_count[8 * lane + k] = run;
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kPer; ++i)
      if (code[i] >= 0) ord[class_count[code[i] >> 16] + (code[i] & 0xffff)] = threadIdx.x + i * NT;
    __syncthreads();
  };
  // Group g of the sorted entries: member k of the warp takes entry ord[8 g + k] with its four
  // lanes; lane (k, q) walks columns q, q+4, … of the rectangle, each over all its rows.
  auto work_group = [&](const float4(*st)[4], const int* ord, const int* gsm, int m, int g,
                        int64_t k0) {
    const int slot = g * 8 + member;
    const bool active = slot < m;
    const int j = active ? ord[slot] : 0;
    float acc[kMoments];
#pragma unroll
    for (int k = 0; k < kMoments; ++k) acc[k] = 0.f;
    bool walked = false;  // an empty walk leaves every moment +0: fast mode adds nothing
    if (active) {
      const float4 p0 = st[j][0], p1 = st[j][1], p2 = st[j][2];
      const int4 r = *reinterpret_cast<const int4*>(&st[j][3]);
      const int cx0 = max(r.x - tx0, 0), cx1 = min(r.z - tx0, TS);
      const int cy0 = max(r.y - ty0, 0), cy1 = min(r.w - ty0, TS);
      const int rows = cy1 - cy0;
      const int passes = (cx1 - cx0 + 3) >> 2;
      walked = passes > 0 && rows > 0;
      const float dy0 = (float)(ty0 + cy0) - p0.y;
      for (int pass = 0; pass < passes; ++pass) {
        const int cx = cx0 + quad + 4 * pass;
        if (cx < cx1 && rows > 0) {
          const float dx = (float)(tx0 + cx) - p0.x;
          const float bdx = p0.w * dx, adx2 = p0.z * dx * dx;
          float tc = 0.f, uc = 0.f;
          float dy = dy0;
          int pidx = cy0 * TS + cx;
#pragma unroll 2
          for (int k = 0; k < rows; ++k, dy += 1.0f, pidx += TS) {
            const float4 gp = pix[pidx];
            const float e = fmaf(dy, fmaf(p1.x, dy, bdx), adx2);
            const float raw = fast_exp2(e);
            const float base_w = FADE ? fmaxf(raw - tail, 0.0f) : raw;
            const float dw = fmaf(gp.x, p1.z, fmaf(gp.y, p1.w, fmaf(gp.z, p2.x, gp.w)));
            acc[0] = fmaf(base_w, gp.x, acc[0]);
            acc[1] = fmaf(base_w, gp.y, acc[1]);
            acc[2] = fmaf(base_w, gp.z, acc[2]);
            if (FADE) acc[3] = fmaf(base_w, dw, acc[3]);
            const float t = (FADE && raw <= tail) ? 0.0f : raw * dw;
            const float u = t * dy;
            tc += t;
            uc += u;
            acc[8] = fmaf(u, dy, acc[8]);
          }
          if (!FADE) acc[3] += tc;  // without the fade base_w = raw, so G's column sum is tc
          acc[4] = fmaf(dx, tc, acc[4]);
          acc[5] += uc;
          acc[6] = fmaf(dx * dx, tc, acc[6]);
          acc[7] = fmaf(dx, uc, acc[7]);
        }
      }
    }
    // reduce-scatter over the member's four lanes: lane q ends with moments
    // (q&2 ? 5 : 0) + (q&1 ? 3 : 0) + s for s < (q&1 ? 2 : 3), those below 9
    float a[5], b[3];
    scatter_level<9, 5>(acc, a, lane & 2, 2);
    scatter_level<5, 3>(a, b, lane & 1, 1);
    if (active && (DETERMINISTIC || walked)) {
      const int base = ((quad & 2) ? 5 : 0) + ((quad & 1) ? 3 : 0);
      const int cnt = (quad & 1) ? 2 : 3;
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int mo = base + s;
        if (s < cnt && mo < kMoments) {
          if (DETERMINISTIC)
            partials[(L.first + k0 + j) * kPartialFloats + mo] = b[s];
          else
            atomicAdd(moments + (int64_t)mo * n + gsm[j], b[s]);
        }
      }
    }
  };
  auto run = [&](float4(*st)[4], int m, int* ord, const int* gsm, int64_t k0) {
    prepare(st, m, ord);
    // Groups go to warps as they become free (heaviest first, by the class order), so the
    // warps of a CTA finish close together instead of idling behind a round-robin share.
    const int groups = (m + 7) >> 3;
    for (;;) {
      int g = 0;
      if (lane == 0) g = atomicAdd(&next_group, 1);
      g = __shfl_sync(0xffffffffu, g, 0);
      if (g >= groups) break;
      work_group(st, ord, gsm, m, g, k0);
    }
  };
  if constexpr (FUSED) {
    // The tile's forward over the staged records, evaluated block by block exactly as
    // forward_kernel evaluates them (so the image, the loss gradient and the moments are bitwise
    // those of the two-kernel step), then each pixel's loss gradient straight into pix.  Warp w
    // takes the 8x8 blocks w, w + NT/32, … one pass each; a list longer than the stage streams
    // through once per pass, and once more for the backward.
    constexpr int kBlocks = (TS / 8) * (TS / 8);
    constexpr int kWarps = NT / 32;
    constexpr int kPer = (kBlocks + kWarps - 1) / kWarps;
    uint32_t* q = reinterpret_cast<uint32_t*>(bwd_smem + S::kQueueOff) + warp * kQueueLen;
    const bool whole = L.count <= kStageMax;
    constexpr int kNullSlot = S::kSlots - 1;
    if (threadIdx.x == 0) write_null_record(stage, kNullSlot);
    bool exact = false;
    if (whole) {
      asm volatile("cp.async.wait_group 0;\n" ::: "memory");
      __syncthreads();
      exact = !all_regular<NT>(stage, (int)L.count);
    }
    const float per_value = pixel_loss_scale(H, W);
    float loss_sum = 0.f, sq_sum = 0.f;
#pragma unroll 1
    for (int i = 0; i < kPer; ++i) {
      const int b = warp + i * kWarps;
      const bool active = b < kBlocks;
      const int bx = active ? (b % (TS / 8)) * 8 : 0, by = active ? (b / (TS / 8)) * 8 : 0;
      float2 acc[4][4];
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int ch = 0; ch < 4; ++ch) acc[k][ch] = make_float2(0.f, 0.f);
      accumulate_block<NT, FADE>(stage, kStageMax, rec, L, q, kQueueLen,
                                 kStageMax + warp * kCarrySlots, kNullSlot, active, tx0 + bx,
                                 ty0 + by, lane, tail, acc, whole, exact, i == 0);
      if (!active) continue;
      float v[2][4];
      combine_groups(acc, lane, v);
      const int lx = bx + (lane & 7), px = tx0 + lx;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int ly = by + block_first_row(lane) + k, py = ty0 + ly;
        float4 pv = make_float4(0.f, 0.f, 0.f, 0.f);
        if (px < W && py < H) {
          const int64_t p = fr.pixel_base + (int64_t)py * W + px;
          if (ff.grad_out) {
            pv = render_pixel_grad(normalize, v[k], p, eps, ff.grad_out, ff.image, ff.den);
          } else {
            float lp, sq;
            pv = finish_pixel_rt(normalize, ff.loss_kind, v[k], p, eps, per_value, ff.charb_eps2,
                                 ff.image, ff.den, ff.target, lp, sq);
            loss_sum += lp;
            sq_sum += sq;
          }
        }
        pix_ok = pix_ok && isfinite(pv.x) && isfinite(pv.y) && isfinite(pv.z) && isfinite(pv.w);
        pix[ly * TS + lx] = pv;
      }
    }
    if (!whole) {  // chunk 0 again, with its ids, for the backward
      stage_range<NT>(stage, rec, L, 0, (int)(L.count < kHalf ? L.count : kHalf), stage_gid);
      cp_async_commit();
    }
    if (ff.loss) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        loss_sum += __shfl_xor_sync(0xffffffffu, loss_sum, o);
        sq_sum += __shfl_xor_sync(0xffffffffu, sq_sum, o);
      }
      if (lane == 0) {
        atomicAdd(ff.loss + 2 * fr.image, loss_sum * per_value);
        atomicAdd(ff.loss + 2 * fr.image + 1, sq_sum * per_value);
      }
    }
    // the barrier before the first group (below) orders these pix writes before their reads
  }
  tile_finite = __syncthreads_and(pix_ok) != 0;
  if (L.count <= kStageMax) {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    run(stage, (int)L.count, order, stage_gid, 0);
  } else {
    float4(*buf)[kHalf][4] = reinterpret_cast<float4(*)[kHalf][4]>(stage);
    const int64_t count = L.count;
    const int nchunks = (int)((count + kHalf - 1) / kHalf);
    auto len = [&](int64_t k0) { return (int)(count - k0 < kHalf ? count - k0 : kHalf); };
    for (int c = 0; c < nchunks; ++c) {
      const int64_t k0 = (int64_t)c * kHalf;
      if (c + 1 < nchunks)
        stage_range<NT>(buf[(c + 1) & 1], rec, L, k0 + kHalf, len(k0 + kHalf),
                        stage_gid + ((c + 1) & 1) * kHalf);
      cp_async_commit();
      cp_async_wait_one();
      __syncthreads();
      run(buf[c & 1], len(k0), order + (c & 1) * kHalf, stage_gid + (c & 1) * kHalf, k0);
      __syncthreads();
    }
  }
}

// Gradients from a Gaussian's nine summed moments m (see the header of this file).
__device__ __forceinline__ void write_gradients(const Splat* rec, int64_t g, const float (&m)[9],
                                                int has_opacity, float* g_means,
                                                float* g_conics, float* g_colors,
                                                float* g_opac) {
  const float4 p1 = reinterpret_cast<const float4*>(rec + g)[1];
  const float4 p2 = reinterpret_cast<const float4*>(rec + g)[2];
  const float op = p1.y, a = p2.y, b = p2.z, c = p2.w;
  g_means[2 * g] = op * (a * m[4] + b * m[5]);
  g_means[2 * g + 1] = op * (b * m[4] + c * m[5]);
  g_conics[3 * g] = -0.5f * op * m[6];
  g_conics[3 * g + 1] = -op * m[7];
  g_conics[3 * g + 2] = -0.5f * op * m[8];
  g_colors[3 * g] = op * m[0];
  g_colors[3 * g + 1] = op * m[1];
  g_colors[3 * g + 2] = op * m[2];
  if (has_opacity) g_opac[g] = m[3];
}

// Fast-mode epilogue: per-Gaussian factors applied once to the atomically summed moments.
__global__ void finalize_moments_kernel(const Splat* __restrict__ rec, int64_t n,
                                        const float* __restrict__ moments, int has_opacity,
                                        float* __restrict__ g_means,
                                        float* __restrict__ g_conics,
                                        float* __restrict__ g_colors,
                                        float* __restrict__ g_opac) {
  pdl_wait();
  pdl_trigger();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  float m[kMoments];
#pragma unroll
  for (int k = 0; k < kMoments; ++k) m[k] = moments[k * n + g];
  write_gradients(rec, g, m, has_opacity, g_means, g_conics, g_colors, g_opac);
}

// Deterministic second pass: per-Gaussian sum of the entry partials in the fixed entry order
// (sum_entry_partials), then the per-Gaussian factors.
__global__ void reduce_partials_kernel(const Splat* __restrict__ rec, int64_t n,
                                       const float* __restrict__ partials,
                                       const int32_t* __restrict__ order,
                                       const int32_t* __restrict__ seg, int has_opacity,
                                       float* __restrict__ g_means,
                                       float* __restrict__ g_conics,
                                       float* __restrict__ g_colors,
                                       float* __restrict__ g_opac) {
  pdl_wait();
  pdl_trigger();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float acc[kMoments];
  sum_entry_partials(partials, order, seg, n, g, g < n, acc);
  if (g >= n) return;
  write_gradients(rec, g, acc, has_opacity, g_means, g_conics, g_colors, g_opac);
}

// Per-Gaussian epilogue straight to the RS field parameters: moments (fast) or the sum of the
// entry partials (deterministic) -> render-input gradients -> the RS chain rule, the same
// arithmetic as the backward epilogue followed by ss_project_rs_backward, in one pass.
template <bool DETERMINISTIC>
__global__ void finalize_rs_kernel(const Splat* __restrict__ rec, int64_t n,
                                   const float* __restrict__ ws,
                                   const int32_t* __restrict__ order,
                                   const int32_t* __restrict__ seg,
                                   const float* __restrict__ log_scales,
                                   const float* __restrict__ rotations,
                                   const float* __restrict__ logits, float dilation,
                                   float* __restrict__ g_means, float* __restrict__ g_ls,
                                   float* __restrict__ g_rot, float* __restrict__ g_colors,
                                   float* __restrict__ g_logits) {
  pdl_wait();
  pdl_trigger();
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float m[kMoments];
  if (DETERMINISTIC) sum_entry_partials(ws, order, seg, n, g, g < n, m);
  if (g >= n) return;
  if (!DETERMINISTIC) {
#pragma unroll
    for (int k = 0; k < kMoments; ++k) m[k] = ws[k * n + g];
  }
  const float4 p1 = reinterpret_cast<const float4*>(rec + g)[1];
  const float4 p2 = reinterpret_cast<const float4*>(rec + g)[2];
  const float op = p1.y, a = p2.y, b = p2.z, c = p2.w;
  g_means[2 * g] = op * (a * m[4] + b * m[5]);
  g_means[2 * g + 1] = op * (b * m[4] + c * m[5]);
  g_colors[3 * g] = op * m[0];
  g_colors[3 * g + 1] = op * m[1];
  g_colors[3 * g + 2] = op * m[2];
  rs_conic_chain(log_scales[2 * g], log_scales[2 * g + 1], rotations[g], dilation,
                 -0.5f * op * m[6], -op * m[7], -0.5f * op * m[8], g_ls[2 * g], g_ls[2 * g + 1],
                 g_rot[g]);
  if (logits && g_logits) g_logits[g] = logit_chain(logits[g], m[3]);
}

// Deterministic mode, after the backward: the entries of the tile lists ordered by Gaussian.
// Keys are the entry ids (n for slots past the filled part of the index); a stable radix sort
// keeps each Gaussian's entries in ascending tile order; the segment kernel records where each
// Gaussian's run begins and ends (Gaussians without entries keep the empty run 0..0).
__global__ void entry_keys_kernel(const int32_t* __restrict__ gids,
                                  const int32_t* __restrict__ offsets, int64_t T, int64_t cap,
                                  int64_t n, uint32_t* __restrict__ keys,
                                  int32_t* __restrict__ order) {
  pdl_wait();
  pdl_trigger();
  // the entries of tiles [0, T): positions [offsets[0], offsets[T]) of the list (offsets[0] > 0
  // for a window of an image's tile rows)
  const int64_t first = offsets[0], last = offsets[T];
  const int64_t total = last < cap ? last : cap;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < cap; e += stride) {
    const int32_t id = e >= first && e < total ? gids[e] : -1;
    keys[e] = (id >= 0 && id < n) ? (uint32_t)id : (uint32_t)n;
    order[e] = (int32_t)e;
  }
}

__global__ void entry_segments_kernel(const uint32_t* __restrict__ keys, int64_t cap, int64_t n,
                                      int32_t* __restrict__ seg) {
  pdl_wait();
  pdl_trigger();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += stride) {
    const uint32_t k = keys[i];
    if (k >= (uint64_t)n) continue;
    if (i == 0 || keys[i - 1] != k) seg[k] = (int32_t)i;
    if (i + 1 == cap || keys[i + 1] != k) seg[n + k] = (int32_t)(i + 1);
  }
}

int key_bits(int64_t n) {
  int b = 1;
  while (b < 32 && ((int64_t)1 << b) <= n) ++b;
  return b;  // keys 0..n fit in b bits
}

size_t sort_temp_bytes(int64_t n, int64_t cap) {
  size_t b = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (const int32_t*)nullptr, (int32_t*)nullptr,
                                  (int)(cap > 0 ? cap : 1), 0, key_bits(n));
  return b;
}

int clear_entry_segments(void* ws, int64_t n, int64_t cap, cudaStream_t s) {
  const EntryOrder eo = entry_order_layout(ws, n, cap);
  cudaMemsetAsync(eo.seg, 0, sizeof(int32_t) * 2 * n, s);
  return check_launch("entry segments zero-fill");
}

int order_entries(const int32_t* gids, const int32_t* offsets, int64_t T, int64_t cap,
                  int64_t n, void* ws, cudaStream_t s) {
  int rc;
  if ((rc = clear_entry_segments(ws, n, cap, s))) return rc;
  if (cap == 0) return SS_OK;
  const EntryOrder eo = entry_order_layout(ws, n, cap);
  const int64_t want = (cap + kEpilogueThreads - 1) / kEpilogueThreads;
  const unsigned blocks = (unsigned)(want < 148 * 16 ? want : 148 * 16);
  launch("entry_keys_kernel", entry_keys_kernel, blocks, kEpilogueThreads, 0, s, gids, offsets, T, cap, n, eo.keys_in,
                                                         eo.order_in);
  if ((rc = check_launch("entry keys"))) return rc;
  size_t tb = sort_temp_bytes(n, cap);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(eo.temp, tb, eo.keys_in, eo.keys, eo.order_in,
                                                  eo.order, (int)cap, 0, key_bits(n), s);
  if (e != cudaSuccess)
    return fail(SS_ERR_CUDA, "entry order sort: %s", cudaGetErrorString(e));
  launch("entry_segments_kernel", entry_segments_kernel, blocks, kEpilogueThreads, 0, s, eo.keys, cap, n, eo.seg);
  return check_launch("entry segments");
}

int check_render_args(int64_t n, int H, int W, int ts, float eps) {
  if (n < 0 || H < 0 || W < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "n exceeds int32 ids");
  if (ts != 16 && ts != 32)
    return fail(SS_ERR_UNSUPPORTED, "render tile_size must be 16 or 32, got %d", ts);
  if (!(eps > 0.0f) || !isfinite(eps))
    return fail(SS_ERR_INVALID_ARGUMENT, "normalization_eps must be finite and > 0");
  return SS_OK;
}

// Records per streamed chunk of the forward (lists longer than the stage): a process-wide
// tuning knob per tile size (0 = half the stage).  Results do not depend on it.
std::atomic<int> g_forward_chunk[2] = {{0}, {0}};

template <int TS, bool NORM, bool FADE>
void launch_forward_loss(int loss_kind, unsigned T, cudaStream_t s, const Splat* rec, int64_t n,
                         const int32_t* gids, int64_t cap, const int32_t* offsets,
                         const Frames& f, float eps, float tail, float* out, float* den,
                         const float* target, float4* pixel_grad, float* loss, float ce2) {
  constexpr int NT = Tiling<TS>::kFwdThreads;
  const int c = g_forward_chunk[TS == 16 ? 0 : 1].load(std::memory_order_relaxed);
  const int chunk = c ? c : kStageAll / 2;
#define SS_FWD(LOSS)                                                                          \
  launch_smem("forward_kernel", forward_kernel<TS, NORM, FADE, LOSS>, T, NT,                  \
              FwdSmem<TS>::kBytes, s, rec, n, gids, cap, offsets, f, eps, tail, out, den,      \
              target, pixel_grad, loss, ce2, chunk)
  switch (loss_kind) {
    case kL1: SS_FWD(kL1); break;
    case kL2: SS_FWD(kL2); break;
    case kCharbonnier: SS_FWD(kCharbonnier); break;
    default: SS_FWD(kNoLoss); break;
  }
#undef SS_FWD
}

template <int TS>
void launch_forward(int loss_kind, unsigned T, cudaStream_t s, const Splat* rec, int64_t n,
                    const int32_t* gids, int64_t cap, const int32_t* offsets, const Frames& f,
                    bool normalize, float eps, float tail, float* out, float* den,
                    const float* target, float4* pixel_grad, float* loss, float ce2) {
  const bool fade = tail > 0.0f;
#define SS_FWD(NORM, FADE)                                                                     \
  launch_forward_loss<TS, NORM, FADE>(loss_kind, T, s, rec, n, gids, cap, offsets, f, eps,     \
                                      tail, out, den, target, pixel_grad, loss, ce2)
  if (normalize) {
    if (fade) SS_FWD(true, true); else SS_FWD(true, false);
  } else {
    if (fade) SS_FWD(false, true); else SS_FWD(false, false);
  }
#undef SS_FWD
}

// Warps per backward CTA: a process-wide tuning knob (0 = the default of the tile size).
std::atomic<int> g_backward_warps[2] = {{0}, {0}};

template <int TS, int NT, bool PIXGRAD>
void launch_backward_nt(unsigned T, cudaStream_t s, bool deterministic, const float* grad_out,
                        const Splat* rec, int64_t n, const float* den, const float* out,
                        const float4* pixel_grad, const int32_t* gids, int64_t cap,
                        const int32_t* offsets, const Frames& f, int normalize, float eps,
                        float tail, float* ws, uint32_t* status) {
  const bool fade = tail > 0.0f;
#define SS_BWD(FADE, DET)                                                                     \
  launch_smem("backward_kernel", backward_kernel<TS, NT, FADE, DET, PIXGRAD>, T, NT,         \
              (BwdSmem<TS, NT, false>::kBytes), s, grad_out, rec, n, den, out, pixel_grad,   \
              gids, cap, offsets, f, normalize, eps, tail, ws, ws, status, FusedFit{})
  if (deterministic) {
    if (fade) SS_BWD(true, true); else SS_BWD(false, true);
  } else {
    if (fade) SS_BWD(true, false); else SS_BWD(false, false);
  }
#undef SS_BWD
}

template <int TS, bool PIXGRAD>
void launch_backward(unsigned T, cudaStream_t s, bool deterministic, const float* grad_out,
                     const Splat* rec, int64_t n, const float* den, const float* out,
                     const float4* pixel_grad, const int32_t* gids, int64_t cap,
                     const int32_t* offsets, const Frames& f, int normalize, float eps,
                     float tail, float* ws, uint32_t* status) {
  const int warps = g_backward_warps[TS == 16 ? 0 : 1].load(std::memory_order_relaxed);
  constexpr int kSmall = TS == 16 ? 128 : 256, kLarge = TS == 16 ? 256 : 512;
  if (warps * 32 == kSmall || (TS == 32 && warps == 0))  // tile 32: 8 warps unless asked
    launch_backward_nt<TS, kSmall, PIXGRAD>(T, s, deterministic, grad_out, rec, n, den, out,
                                            pixel_grad, gids, cap, offsets, f, normalize, eps,
                                            tail, ws, status);
  else
    launch_backward_nt<TS, kLarge, PIXGRAD>(T, s, deterministic, grad_out, rec, n, den, out,
                                            pixel_grad, gids, cap, offsets, f, normalize, eps,
                                            tail, ws, status);
}

// The fused fit tile pass (forward + loss + backward in one CTA per tile).
template <int TS, int NT>
void launch_fused_nt(unsigned T, cudaStream_t s, bool deterministic, const Splat* rec, int64_t n,
                     const int32_t* gids, int64_t cap, const int32_t* offsets, const Frames& f,
                     int normalize, float eps, float tail, float* ws, uint32_t* status,
                     const FusedFit& ff) {
  const bool fade = tail > 0.0f;
#define SS_FUS(FADE, DET)                                                                       \
  launch_smem("fit_tile_kernel", backward_kernel<TS, NT, FADE, DET, false, true>, T, NT,     \
              (BwdSmem<TS, NT, true>::kBytes), s, nullptr, rec, n, nullptr, nullptr, nullptr, \
              gids, cap, offsets, f, normalize, eps, tail, ws, ws, status, ff)
  if (deterministic) {
    if (fade) SS_FUS(true, true); else SS_FUS(false, true);
  } else {
    if (fade) SS_FUS(true, false); else SS_FUS(false, false);
  }
#undef SS_FUS
}

template <int TS>
void launch_fused(unsigned T, cudaStream_t s, bool deterministic, const Splat* rec, int64_t n,
                  const int32_t* gids, int64_t cap, const int32_t* offsets, const Frames& f,
                  int normalize, float eps, float tail, float* ws, uint32_t* status,
                  const FusedFit& ff) {
  const int warps = g_backward_warps[TS == 16 ? 0 : 1].load(std::memory_order_relaxed);
  constexpr int kSmall = TS == 16 ? 128 : 256, kLarge = TS == 16 ? 256 : 512;
  if (warps * 32 == kSmall || (TS == 32 && warps == 0))
    launch_fused_nt<TS, kSmall>(T, s, deterministic, rec, n, gids, cap, offsets, f, normalize,
                                eps, tail, ws, status, ff);
  else
    launch_fused_nt<TS, kLarge>(T, s, deterministic, rec, n, gids, cap, offsets, f, normalize,
                                eps, tail, ws, status, ff);
}

// Forward over any tile set; loss_kind selects the plain render or a fit forward.
int render_forward(const Frames& f, int ts, int64_t T, const void* records, int64_t n,
                   const int32_t* gids, int64_t cap, const int32_t* offsets, int normalize,
                   float eps, float tail, int loss_kind, const float* target, float ce2,
                   float* pixel_grad, float* out, float* den, float* loss, cudaStream_t s) {
  if (T == 0) return SS_OK;
  if (!offsets) return fail(SS_ERR_INVALID_ARGUMENT, "null tile offsets");
  if (n > 0 && !records) return fail(SS_ERR_INVALID_ARGUMENT, "null records");
  if (T > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "too many tiles");
  const Splat* rec = static_cast<const Splat*>(records);
  float4* pg = reinterpret_cast<float4*>(pixel_grad);
  if (ts == 16)
    launch_forward<16>(loss_kind, (unsigned)T, s, rec, n, gids, cap, offsets, f, normalize, eps,
                       tail, out, den, target, pg, loss, ce2);
  else
    launch_forward<32>(loss_kind, (unsigned)T, s, rec, n, gids, cap, offsets, f, normalize, eps,
                       tail, out, den, target, pg, loss, ce2);
  return check_launch("render_forward");
}

// Backward kernel (no epilogue) over any tile set.
int render_backward_tiles(const Frames& f, int ts, int64_t T, const float* grad_out,
                          const void* records, int64_t n, const float* den, const float* out,
                          const float* pixel_grad, const int32_t* gids, int64_t cap,
                          const int32_t* offsets, int normalize, float eps, float tail,
                          int deterministic, float* ws, uint32_t* status, cudaStream_t s) {
  if (n == 0) return SS_OK;
  if (T == 0) return deterministic ? clear_entry_segments(ws, n, cap, s) : SS_OK;
  if (T > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "too many tiles");
  if (deterministic && cap > (int64_t)INT32_MAX)
    return fail(SS_ERR_INVALID_ARGUMENT, "deterministic backward needs capacity < 2^31");
  const Splat* rec = static_cast<const Splat*>(records);
  const float4* pg = reinterpret_cast<const float4*>(pixel_grad);
  if (pixel_grad) {
    if (ts == 16)
      launch_backward<16, true>((unsigned)T, s, deterministic, grad_out, rec, n, den, out, pg,
                                gids, cap, offsets, f, normalize, eps, tail, ws, status);
    else
      launch_backward<32, true>((unsigned)T, s, deterministic, grad_out, rec, n, den, out, pg,
                                gids, cap, offsets, f, normalize, eps, tail, ws, status);
  } else {
    if (ts == 16)
      launch_backward<16, false>((unsigned)T, s, deterministic, grad_out, rec, n, den, out, pg,
                                 gids, cap, offsets, f, normalize, eps, tail, ws, status);
    else
      launch_backward<32, false>((unsigned)T, s, deterministic, grad_out, rec, n, den, out, pg,
                                 gids, cap, offsets, f, normalize, eps, tail, ws, status);
  }
  int rc = check_launch("render_backward");
  if (rc || !deterministic) return rc;
  return order_entries(gids, offsets, T, cap, n, ws, s);
}

size_t backward_ws_bytes(int64_t n, int64_t cap, int deterministic) {
  return deterministic ? entry_order_fixed_bytes(n, cap) + align_up256(sort_temp_bytes(n, cap))
                       : (size_t)n * kMoments * sizeof(float);
}

// Plain backward over any tile set: moments / partials, then the per-Gaussian epilogue.
int render_backward(const Frames& f, int ts, int64_t T, int64_t npx, const float* grad_out,
                    const void* records, int64_t n, const float* den, const float* out,
                    const int32_t* gids, int64_t cap, const int32_t* offsets, int normalize,
                    float eps, float tail, int has_opacity, float* grad_means,
                    float* grad_conics, float* grad_colors, float* grad_opacities,
                    int deterministic, void* workspace, size_t workspace_bytes,
                    uint32_t* status, cudaStream_t s) {
  if (n == 0) return SS_OK;
  if (!grad_means || !grad_conics || !grad_colors || (has_opacity && !grad_opacities))
    return fail(SS_ERR_INVALID_ARGUMENT, "null gradient output");
  if (npx == 0) {  // nothing is rendered: every gradient is zero
    cudaMemsetAsync(grad_means, 0, sizeof(float) * 2 * n, s);
    cudaMemsetAsync(grad_conics, 0, sizeof(float) * 3 * n, s);
    cudaMemsetAsync(grad_colors, 0, sizeof(float) * 3 * n, s);
    if (has_opacity) cudaMemsetAsync(grad_opacities, 0, sizeof(float) * n, s);
    return check_launch("backward zero-fill");
  }
  if (!grad_out || !records || !den || !out || !offsets)
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  const size_t need = backward_ws_bytes(n, cap, deterministic);
  if (workspace_bytes < need || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "backward workspace too small (%zu < %zu)",
                workspace_bytes, need);
  float* ws = static_cast<float*>(workspace);
  int rc;
  if (!deterministic) {
    if (cudaMemsetAsync(ws, 0, sizeof(float) * kMoments * n, s) != cudaSuccess)
      return check_launch("backward moment zero-fill");
  }
  if ((rc = render_backward_tiles(f, ts, T, grad_out, records, n, den, out, nullptr, gids, cap,
                                  offsets, normalize, eps, tail, deterministic, ws, status, s)))
    return rc;
  const Splat* rec = static_cast<const Splat*>(records);
  const unsigned gblocks = (unsigned)((n + kEpilogueThreads - 1) / kEpilogueThreads);
  if (deterministic) {
    const EntryOrder eo = entry_order_layout(ws, n, cap);
    launch("reduce_partials_kernel", reduce_partials_kernel, gblocks, kEpilogueThreads, 0, s, 
        rec, n, eo.partials, eo.order, eo.seg, has_opacity, grad_means, grad_conics,
        grad_colors, grad_opacities);
  } else
    launch("finalize_moments_kernel", finalize_moments_kernel, gblocks, kEpilogueThreads, 0, s, 
        rec, n, ws, has_opacity, grad_means, grad_conics, grad_colors, grad_opacities);
  return check_launch("backward epilogue");
}

int check_batch_render(const ss_batch* batch, int64_t n, float eps, Frames* f) {
  int rc = frames_of_batch(batch, n, f);
  if (rc) return rc;
  return check_render_args(n, 0, 0, batch->tile_size, eps);
}

}  // namespace

size_t fit_grads_offset(int64_t n, int64_t cap, int deterministic) {
  return align_up256(backward_ws_bytes(n, cap, deterministic));
}

size_t fit_ws_bytes(int64_t n, int64_t cap, int deterministic) {
  return fit_grads_offset(n, cap, deterministic) + fit_grads_bytes(n);
}

}  // namespace ss

using namespace ss;

extern "C" {

int ss_render_forward(const void* records, int64_t n, const int32_t* tile_gids,
                      int64_t gid_capacity, const int32_t* tile_offsets, int height, int width,
                      int tile_size, int normalize, float eps, float fade_tail, float* out,
                      float* den, uint32_t* status, ss_stream_t stream) {
  int rc = check_render_args(n, height, width, tile_size, eps);
  if (rc) return rc;
  (void)status;
  if ((int64_t)height * width == 0) return SS_OK;
  if (!out || !den) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  const int64_t T = (int64_t)((width + tile_size - 1) / tile_size) *
                    ((height + tile_size - 1) / tile_size);
  return render_forward(single_frame(height, width, tile_size), tile_size, T, records, n,
                        tile_gids, gid_capacity, tile_offsets, normalize, eps, fade_tail,
                        kNoLoss, nullptr, 0.f, nullptr, out, den, nullptr, as_stream(stream));
}

int ss_batch_render_forward(const ss_batch* batch, const void* records, int64_t n,
                            const int32_t* tile_gids, int64_t gid_capacity,
                            const int32_t* tile_offsets, int normalize, float eps,
                            float fade_tail, float* out, float* den, uint32_t* status,
                            ss_stream_t stream) {
  Frames f;
  int rc = check_batch_render(batch, n, eps, &f);
  if (rc) return rc;
  (void)status;
  if (batch->pixels == 0) return SS_OK;
  if (!out || !den) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  return render_forward(f, batch->tile_size, batch->tiles, records, n, tile_gids, gid_capacity,
                        tile_offsets, normalize, eps, fade_tail, kNoLoss, nullptr, 0.f, nullptr,
                        out, den, nullptr, as_stream(stream));
}

int ss_set_backward_warps(int tile_size, int warps) {
  if (tile_size != 16 && tile_size != 32)
    return fail(SS_ERR_UNSUPPORTED, "render tile_size must be 16 or 32, got %d", tile_size);
  const int small = tile_size == 16 ? 4 : 8, large = tile_size == 16 ? 8 : 16;
  if (warps != 0 && warps != small && warps != large)
    return fail(SS_ERR_INVALID_ARGUMENT, "backward warps for tile %d must be 0, %d or %d",
                tile_size, small, large);
  g_backward_warps[tile_size == 16 ? 0 : 1].store(warps, std::memory_order_relaxed);
  return SS_OK;
}

int ss_get_backward_warps(int tile_size) {
  if (tile_size != 16 && tile_size != 32) return -1;
  const int w = g_backward_warps[tile_size == 16 ? 0 : 1].load(std::memory_order_relaxed);
  return w ? w : 8;
}

int ss_set_forward_chunk(int tile_size, int records) {
  if (tile_size != 16 && tile_size != 32)
    return fail(SS_ERR_UNSUPPORTED, "render tile_size must be 16 or 32, got %d", tile_size);
  if (records != 0 && records != 64 && records != 128 && records != kStageAll / 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "forward chunk must be 0, 64, 128 or %d records, got %d",
                kStageAll / 2, records);
  g_forward_chunk[tile_size == 16 ? 0 : 1].store(records, std::memory_order_relaxed);
  return SS_OK;
}

int ss_get_forward_chunk(int tile_size) {
  if (tile_size != 16 && tile_size != 32) return -1;
  const int c = g_forward_chunk[tile_size == 16 ? 0 : 1].load(std::memory_order_relaxed);
  return c ? c : kStageAll / 2;
}

int ss_render_backward_workspace_bytes(int64_t n, int64_t gid_capacity, int height, int width,
                                       int deterministic, size_t* bytes) {
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  if (n < 0 || gid_capacity < 0 || height < 0 || width < 0)
    return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  *bytes = backward_ws_bytes(n, gid_capacity, deterministic);
  return SS_OK;
}

int ss_render_backward(const float* grad_out, const void* records, int64_t n, const float* den,
                       const float* out, const int32_t* tile_gids, int64_t gid_capacity,
                       const int32_t* tile_offsets, int height, int width, int tile_size,
                       int normalize, float eps, float fade_tail, int has_opacity,
                       float* grad_means, float* grad_conics, float* grad_colors,
                       float* grad_opacities, int deterministic, void* workspace,
                       size_t workspace_bytes, uint32_t* status, ss_stream_t stream) {
  int rc = check_render_args(n, height, width, tile_size, eps);
  if (rc) return rc;
  const int64_t T = (int64_t)((width + tile_size - 1) / tile_size) *
                    ((height + tile_size - 1) / tile_size);
  return render_backward(single_frame(height, width, tile_size), tile_size, T,
                         (int64_t)height * width, grad_out, records, n, den, out, tile_gids,
                         gid_capacity, tile_offsets, normalize, eps, fade_tail, has_opacity,
                         grad_means, grad_conics, grad_colors, grad_opacities, deterministic,
                         workspace, workspace_bytes, status, as_stream(stream));
}

int ss_render_backward_moments(const float* grad_out, const float* pixel_grad,
                               const void* records, int64_t n, const float* den,
                               const float* out, const int32_t* tile_gids,
                               int64_t gid_capacity, const int32_t* tile_offsets, int height,
                               int width, int tile_size, int normalize, float eps,
                               float fade_tail, int deterministic, void* workspace,
                               size_t workspace_bytes, uint32_t* status, ss_stream_t stream) {
  int rc = check_render_args(n, height, width, tile_size, eps);
  if (rc) return rc;
  if (n == 0) return SS_OK;
  const size_t need = backward_ws_bytes(n, gid_capacity, deterministic);
  if ((int64_t)height * width == 0) {  // nothing rendered; the finalize sums no entries
    if (!deterministic) return SS_OK;
    if (workspace_bytes < need || !workspace)
      return fail(SS_ERR_INVALID_ARGUMENT, "backward workspace too small (%zu < %zu)",
                  workspace_bytes, need);
    return clear_entry_segments(workspace, n, gid_capacity, as_stream(stream));
  }
  if (!records || !tile_offsets) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (!pixel_grad && (!grad_out || !den || !out))
    return fail(SS_ERR_INVALID_ARGUMENT, "need grad_out, out and den, or pixel_grad");
  if (pixel_grad && reinterpret_cast<uintptr_t>(pixel_grad) % 16)
    return fail(SS_ERR_INVALID_ARGUMENT, "pixel_grad must be 16-byte aligned");
  if (workspace_bytes < need || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "backward workspace too small (%zu < %zu)",
                workspace_bytes, need);
  const int64_t T = (int64_t)((width + tile_size - 1) / tile_size) *
                    ((height + tile_size - 1) / tile_size);
  return render_backward_tiles(single_frame(height, width, tile_size), tile_size, T,
                               pixel_grad ? nullptr : grad_out, records, n, den, out,
                               pixel_grad, tile_gids, gid_capacity, tile_offsets, normalize, eps,
                               fade_tail, deterministic, static_cast<float*>(workspace), status,
                               as_stream(stream));
}

int ss_render_backward_finalize(const void* records, int64_t n, const int32_t* tile_gids,
                                int64_t gid_capacity, const int32_t* tile_offsets, int height,
                                int width, int tile_size, int has_opacity, int deterministic,
                                const void* workspace, float* grad_means, float* grad_conics,
                                float* grad_colors, float* grad_opacities, ss_stream_t stream) {
  int rc = check_render_args(n, height, width, tile_size, 1.0f);
  if (rc) return rc;
  if (n == 0) return SS_OK;
  if (!records || !workspace || !grad_means || !grad_conics || !grad_colors ||
      (has_opacity && !grad_opacities) || (deterministic && !tile_offsets))
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  const Splat* rec = static_cast<const Splat*>(records);
  const float* ws = static_cast<const float*>(workspace);
  const unsigned gblocks = (unsigned)((n + kEpilogueThreads - 1) / kEpilogueThreads);
  cudaStream_t s = as_stream(stream);
  if (deterministic) {
    const EntryOrder eo = entry_order_layout(const_cast<float*>(ws), n, gid_capacity);
    launch("reduce_partials_kernel", reduce_partials_kernel, gblocks, kEpilogueThreads, 0, s, 
        rec, n, eo.partials, eo.order, eo.seg, has_opacity, grad_means, grad_conics,
        grad_colors, grad_opacities);
  } else
    launch("finalize_moments_kernel", finalize_moments_kernel, gblocks, kEpilogueThreads, 0, s, 
        rec, n, ws, has_opacity, grad_means, grad_conics, grad_colors, grad_opacities);
  return check_launch("backward finalize");
}

int ss_render_backward_finalize_rs(const void* records, int64_t n, const int32_t* tile_gids,
                                   int64_t gid_capacity, const int32_t* tile_offsets, int height,
                                   int width, int tile_size, int deterministic,
                                   const void* workspace, const float* log_scales,
                                   const float* rotations, const float* opacity_logits,
                                   float dilation, float* grad_means, float* grad_log_scales,
                                   float* grad_rotations, float* grad_colors,
                                   float* grad_opacity_logits, ss_stream_t stream) {
  int rc = check_render_args(n, height, width, tile_size, 1.0f);
  if (rc) return rc;
  if (n == 0) return SS_OK;
  if (!records || !workspace || !log_scales || !rotations || !grad_means || !grad_log_scales ||
      !grad_rotations || !grad_colors || (opacity_logits && !grad_opacity_logits) ||
      (deterministic && !tile_offsets))
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  const Splat* rec = static_cast<const Splat*>(records);
  const float* ws = static_cast<const float*>(workspace);
  const unsigned gblocks = (unsigned)((n + kEpilogueThreads - 1) / kEpilogueThreads);
  cudaStream_t s = as_stream(stream);
  if (deterministic) {
    const EntryOrder eo = entry_order_layout(const_cast<float*>(ws), n, gid_capacity);
    launch("finalize_rs_kernel", finalize_rs_kernel<true>, gblocks, kEpilogueThreads, 0, s, 
        rec, n, eo.partials, eo.order, eo.seg, log_scales, rotations, opacity_logits, dilation,
        grad_means, grad_log_scales, grad_rotations, grad_colors, grad_opacity_logits);
  } else {
    launch("finalize_rs_kernel", finalize_rs_kernel<false>, gblocks, kEpilogueThreads, 0, s, 
        rec, n, ws, nullptr, nullptr, log_scales, rotations, opacity_logits, dilation,
        grad_means, grad_log_scales, grad_rotations, grad_colors, grad_opacity_logits);
  }
  return check_launch("backward finalize rs");
}

int ss_batch_render_backward(const ss_batch* batch, const float* grad_out, const void* records,
                             int64_t n, const float* den, const float* out,
                             const int32_t* tile_gids, int64_t gid_capacity,
                             const int32_t* tile_offsets, int normalize, float eps,
                             float fade_tail, int has_opacity, float* grad_means,
                             float* grad_conics, float* grad_colors, float* grad_opacities,
                             int deterministic, void* workspace, size_t workspace_bytes,
                             uint32_t* status, ss_stream_t stream) {
  Frames f;
  int rc = check_batch_render(batch, n, eps, &f);
  if (rc) return rc;
  return render_backward(f, batch->tile_size, batch->tiles, batch->pixels, grad_out, records, n,
                         den, out, tile_gids, gid_capacity, tile_offsets, normalize, eps,
                         fade_tail, has_opacity, grad_means, grad_conics, grad_colors,
                         grad_opacities, deterministic, workspace, workspace_bytes, status,
                         as_stream(stream));
}

int ss_fit_forward_loss(const ss_batch* batch, const void* records, int64_t n,
                        const int32_t* tile_gids, int64_t gid_capacity,
                        const int32_t* tile_offsets, int normalize, float eps, float fade_tail,
                        const float* target, int loss_kind, float charbonnier_eps,
                        float* pixel_grad, float* image, float* den, float* loss,
                        uint32_t* status, ss_stream_t stream) {
  Frames f;
  int rc = check_batch_render(batch, n, eps, &f);
  if (rc) return rc;
  (void)status;
  if (loss_kind < 0 || loss_kind > 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "loss_kind must be 0 (l1), 1 (l2) or 2 (charbonnier)");
  if (batch->pixels == 0) return SS_OK;
  if (!target || !pixel_grad) return fail(SS_ERR_INVALID_ARGUMENT, "null target or pixel_grad");
  if (reinterpret_cast<uintptr_t>(pixel_grad) % 16)
    return fail(SS_ERR_INVALID_ARGUMENT, "pixel_grad must be 16-byte aligned");
  const int kinds[3] = {kL1, kL2, kCharbonnier};
  const float ce2 = (float)((double)charbonnier_eps * (double)charbonnier_eps);
  return render_forward(f, batch->tile_size, batch->tiles, records, n, tile_gids, gid_capacity,
                        tile_offsets, normalize, eps, fade_tail, kinds[loss_kind], target, ce2,
                        pixel_grad, image, den, loss, as_stream(stream));
}

int ss_fit_backward_workspace_bytes(int64_t n, int64_t gid_capacity, int deterministic,
                                    size_t* bytes) {
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  if (n < 0 || gid_capacity < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  *bytes = fit_ws_bytes(n, gid_capacity, deterministic);
  return SS_OK;
}

int ss_fit_backward(const ss_batch* batch, const void* records, int64_t n,
                    const int32_t* tile_gids, int64_t gid_capacity, const int32_t* tile_offsets,
                    float fade_tail, const float* pixel_grad, int deterministic,
                    void* workspace, size_t workspace_bytes, uint32_t* status,
                    ss_stream_t stream) {
  Frames f;
  int rc = check_batch_render(batch, n, 1.0f, &f);
  if (rc) return rc;
  if (n == 0) return SS_OK;
  const size_t need = fit_ws_bytes(n, gid_capacity, deterministic);
  if (batch->pixels == 0) {  // nothing rendered; the update sums no entries
    if (!deterministic) return SS_OK;
    if (workspace_bytes < need || !workspace)
      return fail(SS_ERR_INVALID_ARGUMENT, "fit backward workspace too small (%zu < %zu)",
                  workspace_bytes, need);
    return clear_entry_segments(workspace, n, gid_capacity, as_stream(stream));
  }
  if (!records || !tile_offsets || !pixel_grad) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (workspace_bytes < need || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "fit backward workspace too small (%zu < %zu)",
                workspace_bytes, need);
  return render_backward_tiles(f, batch->tile_size, batch->tiles, nullptr, records, n, nullptr,
                               nullptr, pixel_grad, tile_gids, gid_capacity, tile_offsets, 1,
                               1.0f, fade_tail, deterministic, static_cast<float*>(workspace),
                               status, as_stream(stream));
}

int ss_fit_forward_backward(const ss_batch* batch, const void* records, int64_t n,
                            const int32_t* tile_gids, int64_t gid_capacity,
                            const int32_t* tile_offsets, int normalize, float eps,
                            float fade_tail, const float* target, int loss_kind,
                            float charbonnier_eps, float* image, float* den, float* loss,
                            int deterministic, void* workspace, size_t workspace_bytes,
                            uint32_t* status, ss_stream_t stream) {
  Frames f;
  int rc = check_batch_render(batch, n, eps, &f);
  if (rc) return rc;
  if (loss_kind < 0 || loss_kind > 2)
    return fail(SS_ERR_INVALID_ARGUMENT, "loss_kind must be 0 (l1), 1 (l2) or 2 (charbonnier)");
  const size_t need = fit_ws_bytes(n, gid_capacity, deterministic);
  if (workspace_bytes < need || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "fit workspace too small (%zu < %zu)", workspace_bytes,
                need);
  cudaStream_t s = as_stream(stream);
  if (batch->pixels == 0)  // nothing rendered; the update sums no entries
    return deterministic && n > 0 ? clear_entry_segments(workspace, n, gid_capacity, s) : SS_OK;
  if (!tile_offsets || !target) return fail(SS_ERR_INVALID_ARGUMENT, "null tile offsets or target");
  if (n > 0 && !records) return fail(SS_ERR_INVALID_ARGUMENT, "null records");
  if (deterministic && gid_capacity > (int64_t)INT32_MAX)
    return fail(SS_ERR_INVALID_ARGUMENT, "deterministic backward needs capacity < 2^31");
  const int64_t T = batch->tiles;
  if (T > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "too many tiles");
  const int kinds[3] = {kL1, kL2, kCharbonnier};
  FusedFit ff;
  ff.target = target;
  ff.image = image;
  ff.den = den;
  ff.loss = loss;
  ff.loss_kind = kinds[loss_kind];
  ff.charb_eps2 = (float)((double)charbonnier_eps * (double)charbonnier_eps);
  ff.grad_out = nullptr;
  const Splat* rec = static_cast<const Splat*>(records);
  float* ws = static_cast<float*>(workspace);
  if (batch->tile_size == 16)
    launch_fused<16>((unsigned)T, s, deterministic, rec, n, tile_gids, gid_capacity,
                     tile_offsets, f, normalize, eps, fade_tail, ws, status, ff);
  else
    launch_fused<32>((unsigned)T, s, deterministic, rec, n, tile_gids, gid_capacity,
                     tile_offsets, f, normalize, eps, fade_tail, ws, status, ff);
  if ((rc = check_launch("fit forward + backward"))) return rc;
  if (!deterministic || n == 0) return SS_OK;
  return order_entries(tile_gids, tile_offsets, T, gid_capacity, n, workspace, s);
}

int ss_render_forward_backward(const void* records, int64_t n, const int32_t* tile_gids,
                               int64_t gid_capacity, const int32_t* tile_offsets, int height,
                               int width, int tile_size, int normalize, float eps,
                               float fade_tail, const float* grad_out, float* out, float* den,
                               int deterministic, void* workspace, size_t workspace_bytes,
                               uint32_t* status, ss_stream_t stream) {
  int rc = check_render_args(n, height, width, tile_size, eps);
  if (rc) return rc;
  const size_t need = backward_ws_bytes(n, gid_capacity, deterministic);
  if (workspace_bytes < need || !workspace)
    return fail(SS_ERR_INVALID_ARGUMENT, "backward workspace too small (%zu < %zu)",
                workspace_bytes, need);
  cudaStream_t s = as_stream(stream);
  if ((int64_t)height * width == 0)
    return deterministic && n > 0 ? clear_entry_segments(workspace, n, gid_capacity, s) : SS_OK;
  if (!tile_offsets || !grad_out || !out || !den)
    return fail(SS_ERR_INVALID_ARGUMENT, "null tile offsets, grad_out, out or den");
  if (n > 0 && !records) return fail(SS_ERR_INVALID_ARGUMENT, "null records");
  if (deterministic && gid_capacity > (int64_t)INT32_MAX)
    return fail(SS_ERR_INVALID_ARGUMENT, "deterministic backward needs capacity < 2^31");
  const int64_t T = (int64_t)((width + tile_size - 1) / tile_size) *
                    ((height + tile_size - 1) / tile_size);
  if (T > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "too many tiles");
  FusedFit ff{};
  ff.image = out;
  ff.den = den;
  ff.grad_out = grad_out;
  const Frames f = single_frame(height, width, tile_size);
  const Splat* rec = static_cast<const Splat*>(records);
  float* ws = static_cast<float*>(workspace);
  if (tile_size == 16)
    launch_fused<16>((unsigned)T, s, deterministic, rec, n, tile_gids, gid_capacity,
                     tile_offsets, f, normalize, eps, fade_tail, ws, status, ff);
  else
    launch_fused<32>((unsigned)T, s, deterministic, rec, n, tile_gids, gid_capacity,
                     tile_offsets, f, normalize, eps, fade_tail, ws, status, ff);
  if ((rc = check_launch("render forward + backward"))) return rc;
  if (!deterministic || n == 0) return SS_OK;
  return order_entries(tile_gids, tile_offsets, T, gid_capacity, n, workspace, s);
}

}  // extern "C"

// SSPL1 field decode on the GPU: the integer streams of a container (already inflated on the
// host: zlib / PNG are serial byte codecs) become the five field tensors, as codec.py:333-391
// decodes them.
//
//   unpack     : 1, 2 or 4 bytes per value (uint8/16/32 by bit depth, codec.py:102-131),
//                little-endian, or byte-planar for the means (plane k holds byte k of every value)
//   undelta    : Morton-ordered means and (optionally) colours are stored as modular deltas along
//                the order; an inclusive prefix sum (CUB, uint32 wrap-around) restores them and
//                the bit mask is applied on use
//   dequantise : lo + (q / (2^bits - 1)) (hi - lo) in float64, then float32 (codec.py:86-99);
//                rotation over [0, pi) circular (q / 2^bits · pi) or linear; opacity
//                p = clip(dequant(q, 0, 1), 1e-4, 1 - 1e-4) in float32, logit = log(p / (1 - p))
//
// The float64 steps are written with explicit round-to-nearest intrinsics in numpy's order, so
// every value but the opacity logit (CUDA logf vs numpy's float32 log) is bit-identical.
#include <cub/device/device_scan.cuh>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(int64_t n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__host__ __device__ inline int item_bytes(int bits) { return bits <= 8 ? 1 : (bits <= 16 ? 2 : 4); }

__global__ void unpack_kernel(const uint8_t* __restrict__ raw, int bits, int planar,
                              int64_t count, uint32_t* __restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int nb = item_bytes(bits);
  uint32_t v = 0;
  if (planar && nb > 1) {
    for (int k = 0; k < nb; ++k) v |= (uint32_t)raw[(int64_t)k * count + i] << (8 * k);
  } else {
    for (int k = 0; k < nb; ++k) v |= (uint32_t)raw[i * nb + k] << (8 * k);
  }
  out[i] = v;
}

__device__ __forceinline__ float dequant(uint32_t q, int bits, double lo, double hi) {
  const double levels = (double)((1u << bits) - 1u);
  return (float)__dadd_rn(lo, __dmul_rn(__ddiv_rn((double)q, levels), __dsub_rn(hi, lo)));
}

struct DequantArgs {
  int64_t n;
  int means_bits, scale_bits, rot_bits, color_bits, opacity_bits;
  int morton, color_delta, rot_circular;
  double means_lo[2], means_hi[2], scale_lo[2], scale_hi[2], color_lo[3], color_hi[3];
};

__global__ void dequant_kernel(const uint32_t* __restrict__ qm, const uint32_t* __restrict__ qs,
                               const uint32_t* __restrict__ qr, const uint32_t* __restrict__ qc,
                               const uint32_t* __restrict__ qo, DequantArgs a,
                               float* __restrict__ means, float* __restrict__ log_scales,
                               float* __restrict__ rotations, float* __restrict__ colors,
                               float* __restrict__ logits) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const int64_t n = a.n;
  const uint32_t mmask = a.morton ? (1u << a.means_bits) - 1u : 0xffffffffu;
  for (int d = 0; d < 2; ++d) {
    means[2 * i + d] = dequant(qm[d * n + i] & mmask, a.means_bits, a.means_lo[d], a.means_hi[d]);
    log_scales[2 * i + d] = dequant(qs[d * n + i], a.scale_bits, a.scale_lo[d], a.scale_hi[d]);
  }
  if (a.rot_circular) {
    const double levels = (double)(1u << a.rot_bits);
    rotations[i] = (float)__dmul_rn(__ddiv_rn((double)qr[i], levels), 3.141592653589793);
  } else {
    rotations[i] = dequant(qr[i], a.rot_bits, 0.0, 3.141592653589793);
  }
  const uint32_t cmask = a.color_delta ? (1u << a.color_bits) - 1u : 0xffffffffu;
  for (int c = 0; c < 3; ++c)
    colors[3 * i + c] = dequant(qc[c * n + i] & cmask, a.color_bits, a.color_lo[c], a.color_hi[c]);
  if (qo) {
    float p = dequant(qo[i], a.opacity_bits, 0.0, 1.0);
    const float lo = 1e-4f, hi = 1.0f - 1e-4f;  // np.clip with float32 bounds
    p = p < lo ? lo : (p > hi ? hi : p);
    logits[i] = logf(__fdiv_rn(p, __fsub_rn(1.0f, p)));
  }
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t scan_bytes(int64_t n) {
  size_t b = 0;
  cub::DeviceScan::InclusiveSum(nullptr, b, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                (int)(n > 0 ? n : 1));
  return b;
}

size_t decode_ws_bytes(int64_t n) {
  // q arrays: means 2n, scales 2n, rotation n, colours 3n, opacity n
  return align256(sizeof(uint32_t) * 9 * (n > 0 ? n : 1)) + align256(scan_bytes(n));
}

int check_bits(int bits, const char* what) {
  if (bits < 1 || bits > 31) return fail(SS_ERR_INVALID_ARGUMENT, "%s bits must be 1..31", what);
  return SS_OK;
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_sspl1_workspace_bytes(int64_t n, size_t* bytes) {
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "bad count");
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  *bytes = decode_ws_bytes(n);
  return SS_OK;
}

int ss_sspl1_dequantize(const ss_sspl1_streams* s, float* means, float* log_scales,
                        float* rotations, float* colors, float* opacity_logits, void* workspace,
                        size_t workspace_bytes, ss_stream_t stream) {
  if (!s) return fail(SS_ERR_INVALID_ARGUMENT, "null stream description");
  const int64_t n = s->n;
  if (n < 0 || n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "bad count");
  int rc;
  if ((rc = check_bits(s->means_bits, "means")) || (rc = check_bits(s->scale_bits, "scale")) ||
      (rc = check_bits(s->rot_bits, "rotation")) || (rc = check_bits(s->color_bits, "colour")))
    return rc;
  if (s->opacities && (rc = check_bits(s->opacity_bits, "opacity"))) return rc;
  if (n == 0) return SS_OK;
  if (!s->means || !s->scales || !s->rotations || !s->colors || !means || !log_scales ||
      !rotations || !colors || !workspace || (s->opacities && !opacity_logits))
    return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (workspace_bytes < decode_ws_bytes(n))
    return fail(SS_ERR_INVALID_ARGUMENT, "decode workspace too small");
  cudaStream_t st = as_stream(stream);
  uint32_t* q = static_cast<uint32_t*>(workspace);
  uint32_t *qm = q, *qs = q + 2 * n, *qr = q + 4 * n, *qc = q + 5 * n, *qo = q + 8 * n;
  void* temp = static_cast<char*>(workspace) + align256(sizeof(uint32_t) * 9 * n);
  unpack_kernel<<<blocks_for(2 * n), kThreads, 0, st>>>(s->means, s->means_bits,
                                                        s->means_byte_planar, 2 * n, qm);
  unpack_kernel<<<blocks_for(2 * n), kThreads, 0, st>>>(s->scales, s->scale_bits, 0, 2 * n, qs);
  unpack_kernel<<<blocks_for(n), kThreads, 0, st>>>(s->rotations, s->rot_bits, 0, n, qr);
  unpack_kernel<<<blocks_for(3 * n), kThreads, 0, st>>>(s->colors, s->color_bits, 0, 3 * n, qc);
  if (s->opacities)
    unpack_kernel<<<blocks_for(n), kThreads, 0, st>>>(s->opacities, s->opacity_bits, 0, n, qo);
  if ((rc = check_launch("sspl1 unpack"))) return rc;
  auto scan = [&](uint32_t* col) -> int {
    size_t tb = scan_bytes(n);
    cudaError_t e = cub::DeviceScan::InclusiveSum(temp, tb, col, col, (int)n, st);
    return e == cudaSuccess ? SS_OK : fail(SS_ERR_CUDA, "sspl1 delta scan: %s",
                                           cudaGetErrorString(e));
  };
  if (s->morton)
    for (int d = 0; d < 2; ++d)
      if ((rc = scan(qm + d * n))) return rc;
  if (s->color_delta)
    for (int c = 0; c < 3; ++c)
      if ((rc = scan(qc + c * n))) return rc;
  DequantArgs a;
  a.n = n;
  a.means_bits = s->means_bits;
  a.scale_bits = s->scale_bits;
  a.rot_bits = s->rot_bits;
  a.color_bits = s->color_bits;
  a.opacity_bits = s->opacity_bits;
  a.morton = s->morton;
  a.color_delta = s->color_delta;
  a.rot_circular = s->rot_circular;
  for (int d = 0; d < 2; ++d) {
    a.means_lo[d] = s->means_lo[d];
    a.means_hi[d] = s->means_hi[d];
    a.scale_lo[d] = s->scale_lo[d];
    a.scale_hi[d] = s->scale_hi[d];
  }
  for (int c = 0; c < 3; ++c) {
    a.color_lo[c] = s->color_lo[c];
    a.color_hi[c] = s->color_hi[c];
  }
  dequant_kernel<<<blocks_for(n), kThreads, 0, st>>>(qm, qs, qr, qc, s->opacities ? qo : nullptr,
                                                     a, means, log_scales, rotations, colors,
                                                     opacity_logits);
  return check_launch("sspl1 dequantize");
}

}  // extern "C"

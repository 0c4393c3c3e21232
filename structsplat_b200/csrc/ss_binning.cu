// Tile binning: count -> exclusive scan -> fill -> per-tile sort.
//
// Result contract (cuda_render.py:177-226, render_ext.cu:858-952): tile t lists every Gaussian
// whose clipped support rectangle touches it, offsets[t]..offsets[t+1]; the lists are sorted by
// ascending Gaussian id, which is the order the reference's stable radix sort leaves and makes
// every downstream sum deterministic.  No sort over all pairs is needed: per-tile counts come
// from atomics, a device-wide scan gives the offsets, the fill claims slots with per-tile atomic
// cursors, and a per-tile bitonic sort in shared memory restores ascending ids.  The scan is one
// single-CTA kernel for up to 16,384 tiles and CUB's device scan beyond.
#include <climits>

#include <cub/block/block_radix_sort.cuh>
#include <cub/block/block_scan.cuh>
#include <cub/device/device_scan.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/iterator/transform_iterator.h>

#include "ss_common.cuh"

namespace ss {
namespace {

constexpr int kThreads = 256;
constexpr int kSmallRect = 8;          // tiles a lane enumerates alone; larger rects use the warp
constexpr int kWarpSortMax = 1024;     // per-warp register sort capacity (ints)
constexpr int kBigSortSmem = 16384;    // per-CTA shared-memory sort capacity (ints)
// Per-tile counters sit one per 32-byte sector: a tile receives one atomic per Gaussian that
// touches it, and packing 8 neighbouring tiles' counters into a sector would serialise their
// atomics in the L2.
constexpr int kCounterStride = 8;

struct CounterLoad {
  const int* base;
  __host__ __device__ int operator()(int64_t t) const { return base[t * kCounterStride]; }
};

inline auto counter_iter(const int* base) {
  return thrust::make_transform_iterator(thrust::make_counting_iterator<int64_t>(0),
                                         CounterLoad{base});
}

struct TileGrid {
  int ts, tiles_x, tiles_y;
  int64_t T;
};

inline TileGrid make_grid(int H, int W, int ts) {
  TileGrid g;
  g.ts = ts;
  g.tiles_x = (W + ts - 1) / ts;
  g.tiles_y = (H + ts - 1) / ts;
  g.T = (int64_t)g.tiles_x * g.tiles_y;
  return g;
}

// Workspace layout (each region 256-byte aligned).
struct IndexWorkspace {
  int* tile_count;        // T+1   per-tile counters (fill consumes them back to zero)
  long long* offsets64;   // T+1   exclusive scan in int64
  int* big_tiles;         // T     tiles whose list is too long for the warp sort
  int* big_count;         // 1
  void* scan_temp;
  size_t scan_bytes;
};

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

size_t scan_temp_bytes(int64_t items) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveScan(nullptr, bytes, counter_iter(nullptr), (long long*)nullptr,
                                 ::cuda::std::plus<long long>(), (long long)0, (int)items);
  return bytes;
}

size_t index_workspace_bytes(int64_t T) {
  return align256(sizeof(int) * kCounterStride * (T + 1)) +
         align256(sizeof(long long) * (T + 1)) +
         align256(sizeof(int) * (T > 0 ? T : 1)) + align256(sizeof(int)) +
         align256(scan_temp_bytes(T + 1));
}

IndexWorkspace carve(void* base, int64_t T) {
  IndexWorkspace w;
  char* p = static_cast<char*>(base);
  w.tile_count = reinterpret_cast<int*>(p);
  p += align256(sizeof(int) * kCounterStride * (T + 1));
  w.offsets64 = reinterpret_cast<long long*>(p);
  p += align256(sizeof(long long) * (T + 1));
  w.big_tiles = reinterpret_cast<int*>(p);
  p += align256(sizeof(int) * (T > 0 ? T : 1));
  w.big_count = reinterpret_cast<int*>(p);
  p += align256(sizeof(int));
  w.scan_temp = p;
  w.scan_bytes = align256(scan_temp_bytes(T + 1));
  return w;
}

struct TileRect {
  int gx0, gy0, gw, gh;
};

__device__ __forceinline__ TileRect tile_rect_of(const Splat* rec, int64_t i, int ts) {
  TileRect r{0, 0, 0, 0};
  int4 b = reinterpret_cast<const int4*>(rec + i)[3];
  if (b.z > b.x && b.w > b.y) {
    r.gx0 = b.x / ts;
    r.gy0 = b.y / ts;
    r.gw = (b.z - 1) / ts - r.gx0 + 1;
    r.gh = (b.w - 1) / ts - r.gy0 + 1;
  }
  return r;
}

__device__ __forceinline__ Splat load_splat(const Splat* rec, int64_t i) {
  Splat s;
  const float4* src = reinterpret_cast<const float4*>(rec + i);
  float4* d = reinterpret_cast<float4*>(&s);
  d[0] = src[0];
  d[1] = src[1];
  d[2] = src[2];
  d[3] = src[3];
  return s;
}

// Calls visit(gaussian, tile) for every (tile, Gaussian) pair of the index, in any order.
// Each lane enumerates a rectangle of up to kSmallRect tiles itself (unrolled, so independent
// atomics are in flight together); a larger rectangle is enumerated by the whole warp so one
// huge Gaussian cannot serialise a lane.  Tile coordinates advance incrementally (no division).
template <bool CULL, typename Visit>
__device__ __forceinline__ void enumerate_pairs(const Splat* rec, int64_t n, int ts,
                                                const Frames& frames, float cutoff2,
                                                Visit visit) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int lane = threadIdx.x & 31;
  TileRect r{0, 0, 0, 0};
  int tiles_x = 0, first_tile = 0;
  if (i < n) {
    r = tile_rect_of(rec, i, ts);
    const Frame fr = frame_of_gaussian(frames, i, n);
    tiles_x = fr.tiles_x;
    first_tile = fr.first_tile;
  }
  int cnt = r.gw * r.gh;
  if (cnt > 0 && cnt <= kSmallRect) {
    Splat s;
    if (CULL) s = load_splat(rec, i);
    int gx = r.gx0, gy = r.gy0;
#pragma unroll
    for (int k = 0; k < kSmallRect; ++k) {
      if (k < cnt) {
        if (!(CULL && culled(s, gx, gy, ts, cutoff2)))
          visit(k, (int)i, first_tile + gy * tiles_x + gx);
        if (++gx == r.gx0 + r.gw) {
          gx = r.gx0;
          ++gy;
        }
      }
    }
  }
  unsigned big = __ballot_sync(0xffffffffu, cnt > kSmallRect);
  while (big) {
    int src = __ffs(big) - 1;
    big &= big - 1;
    int gx0 = __shfl_sync(0xffffffffu, r.gx0, src);
    int gy0 = __shfl_sync(0xffffffffu, r.gy0, src);
    int gw = __shfl_sync(0xffffffffu, r.gw, src);
    int total = __shfl_sync(0xffffffffu, cnt, src);
    const int tx_src = __shfl_sync(0xffffffffu, tiles_x, src);
    const int base_src = __shfl_sync(0xffffffffu, first_tile, src);
    long long gi = __shfl_sync(0xffffffffu, (long long)i, src);
    Splat s;
    if (CULL) s = load_splat(rec, gi);
    const int step_y = 32 / gw, step_x = 32 - step_y * gw;
    int gy = gy0 + lane / gw, gx = gx0 + lane % gw;
    for (int k = lane; k < total; k += 32) {
      if (!(CULL && culled(s, gx, gy, ts, cutoff2)))
        visit(-1, (int)gi, base_src + gy * tx_src + gx);
      gx += step_x;
      gy += step_y;
      if (gx >= gx0 + gw) {
        gx -= gw;
        ++gy;
      }
    }
  }
}

// Exclusive scan of the T+1 counters into int64 and int32 offsets by one CTA of kThreads
// threads, in rounds of kScanItems kThreads items (one round for up to 2,047 tiles); the counters
// are read from L2 (other CTAs' atomics), every load of a round in flight before the scan.
constexpr int kScanItems = 8;
__device__ void block_scan_counts(const int* tile_count, int64_t items, long long* off64,
                                  int32_t* off32) {
  using Scan = cub::BlockScan<long long, kThreads>;
  __shared__ typename Scan::TempStorage tmp;
  long long carry = 0;
  for (int64_t b0 = 0; b0 < items; b0 += kScanItems * kThreads) {
    long long v[kScanItems];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int64_t idx = b0 + kScanItems * threadIdx.x + k;
      v[k] = idx < items ? __ldcg(tile_count + idx * kCounterStride) : 0;
    }
    long long total;
    Scan(tmp).ExclusiveSum(v, v, total);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      const int64_t idx = b0 + kScanItems * threadIdx.x + k;
      if (idx < items) {
        const long long o = carry + v[k];
        off64[idx] = o;
        off32[idx] = (int32_t)(o < 2147483647LL ? o : 2147483647LL);
      }
    }
    carry += total;
    __syncthreads();  // tmp is reused by the next round
  }
}

// Per-tile counts by atomics.  SCAN: the last CTA to finish (a ticket in the padding word after
// counter 0, zeroed with the counters) also scans the counts into the offsets, which saves the
// separate scan launch for small tile sets.
template <bool CULL, bool SCAN>
__global__ void tile_count_kernel(const Splat* __restrict__ rec, int64_t n, int ts, Frames frames,
                                  float cutoff2, int* __restrict__ tile_count, int64_t items,
                                  long long* __restrict__ off64, int32_t* __restrict__ off32) {
  pdl_wait();
  pdl_trigger();
  enumerate_pairs<CULL>(rec, n, ts, frames, cutoff2,
                        [&](int, int, int t) { atomicAdd(tile_count + (int64_t)t * kCounterStride, 1); });
  if constexpr (SCAN) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();  // this CTA's counts before its ticket
      const unsigned ticket = atomicAdd(reinterpret_cast<unsigned*>(tile_count + 1), 1u);
      last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();  // every other CTA's counts are visible after its ticket
    block_scan_counts(tile_count, items, off64, off32);
  }
}

// The RS projection (rs_project_one, as project_rs_kernel) and the per-tile counts in one pass:
// each thread stores its Gaussian's record and counts its tiles from it, so the counts need no
// second read of the records from DRAM.  The record is read back by its own thread (and, for a
// rectangle the warp enumerates together, by the warp after __syncwarp), so `out` carries no
// read-only qualifier.  SCAN as in tile_count_kernel.  The grid also zeroes `clear_vec` 16-byte
// words at `clear` (a caller's per-step scratch, such as the next backward's moments).
template <bool CULL, bool SCAN>
__global__ void project_count_kernel(RSField field, int64_t n, int ts, Frames frames,
                                     float cutoff2, Splat* out, int* __restrict__ tile_count,
                                     int64_t items, long long* __restrict__ off64,
                                     int32_t* __restrict__ off32, uint4* __restrict__ clear,
                                     int64_t clear_vec) {
  pdl_wait();
  pdl_trigger();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t v = i; v < clear_vec; v += (int64_t)gridDim.x * blockDim.x)
    clear[v] = make_uint4(0u, 0u, 0u, 0u);
  if (i < n) {
    long long rx, ry;
    store_splat(out + i, rs_project_one(field, i, frame_of_gaussian(frames, i, n), rx, ry));
  }
  __syncwarp();
  enumerate_pairs<CULL>(out, n, ts, frames, cutoff2,
                        [&](int, int, int t) { atomicAdd(tile_count + (int64_t)t * kCounterStride, 1); });
  if constexpr (SCAN) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const unsigned ticket = atomicAdd(reinterpret_cast<unsigned*>(tile_count + 1), 1u);
      last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    block_scan_counts(tile_count, items, off64, off32);
  }
}

// Writes int32 offsets, checks capacity, then claims one slot per pair.  Slots are claimed by
// counting each tile's counter back down, which leaves the counters at zero.  A lane's own
// (small) rectangle claims all its slots first and stores afterwards, so the atomics overlap.
template <bool CULL>
__global__ void tile_fill_kernel(const Splat* __restrict__ rec, int64_t n, int ts, Frames frames,
                                 float cutoff2, int64_t T, const long long* __restrict__ off64,
                                 int* __restrict__ tile_count, int32_t* __restrict__ offsets32,
                                 int32_t* __restrict__ gids, int64_t cap, int* big_count,
                                 uint32_t* status) {
  pdl_wait();
  pdl_trigger();
  int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  long long total = off64[T];
  for (int64_t t = tid; t <= T; t += stride) offsets32[t] = (int32_t)min(off64[t], 2147483647LL);
  if (tid == 0) {
    *big_count = 0;
    if (total > 2147483647LL) raise_status(status, SS_STATUS_INDEX_INT32);
    if (total > cap) raise_status(status, SS_STATUS_INDEX_OVERFLOW);
  }
  long long pos[kSmallRect];
#pragma unroll
  for (int k = 0; k < kSmallRect; ++k) pos[k] = -1;
  int owner = -1;
  enumerate_pairs<CULL>(rec, n, ts, frames, cutoff2, [&](int k, int g, int t) {
    long long p = off64[t] + (atomicSub(tile_count + (int64_t)t * kCounterStride, 1) - 1);
    if (k < 0) {
      if (p < cap) gids[p] = g;
    } else {
#pragma unroll
      for (int q = 0; q < kSmallRect; ++q)
        if (q == k) pos[q] = p;
      owner = g;
    }
  });
#pragma unroll
  for (int k = 0; k < kSmallRect; ++k)
    if (pos[k] >= 0 && pos[k] < cap) gids[pos[k]] = owner;
}

// Offsets of small tile sets in one launch: a single CTA scans up to kSingleScanMax per-tile
// counts (each thread a contiguous run of kScanPerThread, then a block scan of the run totals)
// and writes the int64 and the int32 offsets.  Larger tile sets use CUB's device scan.
constexpr int kScanThreads = 1024;
constexpr int kScanPerThread = 16;
constexpr int64_t kSingleScanMax = (int64_t)kScanThreads * kScanPerThread;
constexpr int64_t kFusedScanMax = 16 * kThreads;

__global__ void __launch_bounds__(kScanThreads)
    single_scan_kernel(const int* __restrict__ tile_count, int64_t items,
                       long long* __restrict__ off64, int32_t* __restrict__ off32) {
  pdl_wait();
  pdl_trigger();
  __shared__ long long warp_total[kScanThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t base = (int64_t)tid * kScanPerThread;
  long long run[kScanPerThread];
  long long sum = 0;
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    const int64_t idx = base + k;
    run[k] = sum;
    sum += idx < items ? tile_count[idx * kCounterStride] : 0;
  }
  long long incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) warp_total[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const long long v = warp_total[lane];
    long long w = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_total[lane] = w - v;  // exclusive prefix of the warp totals
  }
  __syncthreads();
  const long long prefix = warp_total[warp] + (incl - sum);
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    const int64_t idx = base + k;
    if (idx < items) {
      const long long o = prefix + run[k];
      off64[idx] = o;
      off32[idx] = (int32_t)(o < 2147483647LL ? o : 2147483647LL);
    }
  }
}

// Ascending sort of buf[0..len) using a bitonic network over the next power of two in which
// every comparator puts the smaller key first; positions >= len act as +inf and never move.
template <typename Sync>
__device__ void bitonic_sort(int* buf, int len, int tid, int nthreads, Sync sync) {
  int n2 = 1;
  while (n2 < len) n2 <<= 1;
  for (int lk = 1; (1 << lk) <= n2; ++lk) {
    const int k = 1 << lk;
    for (int lj = lk - 1; lj >= 0; --lj) {
      const int j = 1 << lj;
      for (int p = tid; p < (n2 >> 1); p += nthreads) {
        int blk = p >> lj, r = p & (j - 1), a, b;
        if (j == (k >> 1)) {
          a = blk * k + r;
          b = blk * k + k - 1 - r;
        } else {
          a = blk * 2 * j + r;
          b = a + j;
        }
        if (b < len) {
          int va = buf[a], vb = buf[b];
          if (va > vb) {
            buf[a] = vb;
            buf[b] = va;
          }
        }
      }
      sync();
    }
  }
}

// Ascending sort of up to 32*K keys held in registers across a warp: key k of lane l is element
// 32k + l, missing elements are INT_MAX.  Standard bitonic network: at block size `size` and
// distance j, elements e and e^j are compared and the block (e & size) == 0 sorts upward.
// Distances below 32 exchange through xor shuffles, larger ones swap registers in-lane.
template <int K>
__device__ __forceinline__ void warp_bitonic(int (&v)[K], int lane) {
#pragma unroll
  for (int size = 2; size <= 32 * K; size <<= 1) {
#pragma unroll
    for (int j = size >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int kp = k ^ (j >> 5);
          if (kp > k) {
            const bool up = ((32 * k + lane) & size) == 0;
            const int lo = min(v[k], v[kp]), hi = max(v[k], v[kp]);
            v[k] = up ? lo : hi;
            v[kp] = up ? hi : lo;
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int other = __shfl_xor_sync(0xffffffffu, v[k], j);
          const bool up = ((32 * k + lane) & size) == 0;
          const bool lower = (lane & j) == 0;
          v[k] = (up == lower) ? min(v[k], other) : max(v[k], other);
        }
      }
    }
  }
}

template <int K>
__device__ __forceinline__ void warp_sort_list(int32_t* __restrict__ g, int len, int lane) {
  int v[K];
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = 32 * k + lane < len ? g[32 * k + lane] : INT_MAX;
  warp_bitonic<K>(v, lane);
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (32 * k + lane < len) g[32 * k + lane] = v[k];
}

// One warp per tile: lists up to kWarpSortMax ids sort in registers (32 K keys for the smallest
// power-of-two K that holds the list); longer lists are queued for tile_sort_big_kernel.
__global__ void __launch_bounds__(kThreads) tile_sort_kernel(const int32_t* __restrict__ offsets,
                                                             int32_t* __restrict__ gids,
                                                             int64_t cap, int64_t T,
                                                             int* big_tiles, int* big_count) {
  pdl_wait();
  pdl_trigger();
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t t = (int64_t)blockIdx.x * (kThreads / 32) + warp;
  if (t >= T) return;
  int64_t lo = offsets[t], hi = offsets[t + 1];
  if (hi > cap) return;  // truncated list: the renderers scan all Gaussians for this tile
  int len = (int)(hi - lo);
  if (len <= 1) return;
  int32_t* g = gids + lo;
  if (len <= 32) {
    warp_sort_list<1>(g, len, lane);
  } else if (len <= 64) {
    warp_sort_list<2>(g, len, lane);
  } else if (len <= 128) {
    warp_sort_list<4>(g, len, lane);
  } else if (len <= 256) {
    warp_sort_list<8>(g, len, lane);
  } else if (len <= 512) {
    warp_sort_list<16>(g, len, lane);
  } else if (len <= kWarpSortMax) {
    warp_sort_list<32>(g, len, lane);
  } else if (lane == 0) {
    big_tiles[atomicAdd(big_count, 1)] = (int)t;
  }
}

// Long lists: one CTA per list, in shared memory up to kBigSortSmem ids, else in place.
// Lists of up to kRadixSortMax ids sort with CUB's block radix sort over the bits the ids need
// (key_bits: pad keys 2^bits - 1 sort last), with 2, 3 or 4 keys per thread, the fewest that
// hold the list (a radix sort's work grows with its keys, pads included); longer lists with the
// shared-memory bitonic network (the ids of a list are distinct, so every path gives the one
// ascending order).
constexpr int kRadixItems = 4;
constexpr int kRadixSortMax = 1024 * kRadixItems;
template <int K>
using BigRadixSortK = cub::BlockRadixSort<unsigned, 1024, K>;
union BigRadixTemp {
  typename BigRadixSortK<2>::TempStorage k2;
  typename BigRadixSortK<3>::TempStorage k3;
  typename BigRadixSortK<4>::TempStorage k4;
};

template <int K>
__device__ __forceinline__ void radix_sort_list(int32_t* __restrict__ g, int len, unsigned pad,
                                                int key_bits,
                                                typename BigRadixSortK<K>::TempStorage& tmp) {
  unsigned keys[K];
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const int e = threadIdx.x * K + i;
    keys[i] = e < len ? (unsigned)g[e] : pad;
  }
  BigRadixSortK<K>(tmp).Sort(keys, 0, key_bits);
#pragma unroll
  for (int i = 0; i < K; ++i) {
    const int e = threadIdx.x * K + i;
    if (e < len) g[e] = (int32_t)keys[i];
  }
}

__global__ void __launch_bounds__(1024) tile_sort_big_kernel(const int32_t* __restrict__ offsets,
                                                             int32_t* __restrict__ gids,
                                                             const int* __restrict__ big_tiles,
                                                             const int* __restrict__ big_count,
                                                             int key_bits) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ int sbuf[];
  __shared__ BigRadixTemp radix_temp;
  int count = *big_count;
  const unsigned pad = key_bits >= 32 ? 0xffffffffu : (1u << key_bits) - 1u;
  for (int k = blockIdx.x; k < count; k += gridDim.x) {
    int t = big_tiles[k];
    int64_t lo = offsets[t];
    int len = (int)(offsets[t + 1] - lo);
    auto sync = [] { __syncthreads(); };
    if (len <= 2 * 1024) {  // lists here are longer than the warp sort's 1,024 ids
      radix_sort_list<2>(gids + lo, len, pad, key_bits, radix_temp.k2);
    } else if (len <= 3 * 1024) {
      radix_sort_list<3>(gids + lo, len, pad, key_bits, radix_temp.k3);
    } else if (len <= kRadixSortMax) {
      radix_sort_list<4>(gids + lo, len, pad, key_bits, radix_temp.k4);
    } else if (len <= kBigSortSmem) {
      for (int e = threadIdx.x; e < len; e += blockDim.x) sbuf[e] = gids[lo + e];
      __syncthreads();
      bitonic_sort(sbuf, len, threadIdx.x, blockDim.x, sync);
      for (int e = threadIdx.x; e < len; e += blockDim.x) gids[lo + e] = sbuf[e];
    } else {
      bitonic_sort(gids + lo, len, threadIdx.x, blockDim.x, sync);
    }
    __syncthreads();
  }
}

// Bits that hold every id below n and the pad 2^bits - 1 above them.
int sort_key_bits(int64_t n) {
  int b = 1;
  while (b < 32 && ((int64_t)1 << b) <= n) ++b;
  return b;
}

constexpr int kBigSortCtas = 296;  // 2 per SM: long lists are common under heavy-tailed fields

// Opts tile_sort_big_kernel into its dynamic shared memory once per device.
int allow_big_sort_smem() {
  static bool done[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_launch("cudaGetDevice");
  if (dev >= 0 && dev < 64 && done[dev]) return SS_OK;
  if (cudaFuncSetAttribute(tile_sort_big_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)(kBigSortSmem * sizeof(int))) != cudaSuccess)
    return check_launch("tile_sort_big smem attribute");
  if (dev >= 0 && dev < 64) done[dev] = true;
  return SS_OK;
}

int check_index_args(int64_t n, int H, int W, int ts) {
  if (n < 0 || H < 0 || W < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative size");
  if (n > (int64_t)INT32_MAX) return fail(SS_ERR_INVALID_ARGUMENT, "n exceeds int32 ids");
  if (ts <= 0 || ts > 32)  // ts^2 <= 1024, without overflow
    return fail(SS_ERR_INVALID_ARGUMENT, "tile_size must be positive with tile_size^2 <= 1024");
  TileGrid g = make_grid(H, W, ts);
  if (g.T + 1 > (int64_t)INT32_MAX)
    return fail(SS_ERR_INVALID_ARGUMENT, "tile grid exceeds int32 tile ids");
  return SS_OK;
}


// Stage 1 over any tile set (one image or a batch): counts, scan, int32 offsets.
// With `rs`, the records are first projected from that RS field in the same kernel
// (project_count_kernel) and written to `records`.
int index_count(const Frames& frames, int ts, int64_t T, const void* records, int64_t n,
                int ellipse_cull, float sigma_cutoff, int32_t* tile_offsets, void* workspace,
                size_t workspace_bytes, uint32_t* status, ss_stream_t stream,
                const RSField* rs = nullptr, void* clear = nullptr, size_t clear_bytes = 0) {
  int rc;
  if (!tile_offsets || !workspace) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (n > 0 && !records) return fail(SS_ERR_INVALID_ARGUMENT, "null records");
  if (workspace_bytes < index_workspace_bytes(T))
    return fail(SS_ERR_INVALID_ARGUMENT, "tile index workspace too small (%zu < %zu)",
                workspace_bytes, index_workspace_bytes(T));
  cudaStream_t s = as_stream(stream);
  IndexWorkspace w = carve(workspace, T);
  if (cudaMemsetAsync(w.tile_count, 0, sizeof(int) * kCounterStride * (T + 1), s) !=
      cudaSuccess)
    return check_launch("tile_index_count memset");
  const Splat* rec = static_cast<const Splat*>(records);
  float cutoff2 = sigma_cutoff * sigma_cutoff;
  // the count kernel's last CTA scans up to kFusedScanMax counters (two rounds); larger sets
  // up to kSingleScanMax take the 1024-thread scan kernel, beyond that CUB's device scan
  const bool fused_scan = T + 1 <= kFusedScanMax;
  const bool single_scan = T + 1 <= kSingleScanMax;
  if (clear_bytes && (!clear || reinterpret_cast<uintptr_t>(clear) % 16 || clear_bytes % 16))
    return fail(SS_ERR_INVALID_ARGUMENT,
                "clear region must be 16-byte aligned and a multiple of 16 bytes");
  if (clear_bytes && !(rs && n > 0) && cudaMemsetAsync(clear, 0, clear_bytes, s) != cudaSuccess)
    return check_launch("clear region memset");
  if (rs && n > 0) {  // project even when the tile set is empty: the records are an output
    if (reinterpret_cast<uintptr_t>(records) % 16)
      return fail(SS_ERR_INVALID_ARGUMENT, "records must be 16-byte aligned");
    int blocks = (int)((n + kThreads - 1) / kThreads);
    Splat* out = static_cast<Splat*>(const_cast<void*>(records));
#define SS_PCOUNT(C, S)                                                                       \
  launch("project_count_kernel", project_count_kernel<C, S>, blocks, kThreads, 0, s, *rs, n,   \
         ts, frames, cutoff2, out, w.tile_count, T + 1, w.offsets64, tile_offsets,           \
         static_cast<uint4*>(clear), (int64_t)(clear_bytes / 16))
    if (ellipse_cull) {
      if (fused_scan) SS_PCOUNT(true, true); else SS_PCOUNT(true, false);
    } else {
      if (fused_scan) SS_PCOUNT(false, true); else SS_PCOUNT(false, false);
    }
#undef SS_PCOUNT
    if ((rc = check_launch("project_count"))) return rc;
    if (fused_scan) return SS_OK;
  } else if (n > 0 && T > 0) {
    int blocks = (int)((n + kThreads - 1) / kThreads);
#define SS_COUNT(C, S)                                                                        \
  launch("tile_count_kernel", tile_count_kernel<C, S>, blocks, kThreads, 0, s, rec, n, ts,     \
         frames, cutoff2, w.tile_count, T + 1, w.offsets64, tile_offsets)
    if (ellipse_cull) {
      if (fused_scan) SS_COUNT(true, true); else SS_COUNT(true, false);
    } else {
      if (fused_scan) SS_COUNT(false, true); else SS_COUNT(false, false);
    }
#undef SS_COUNT
    if ((rc = check_launch("tile_count"))) return rc;
    if (fused_scan) return SS_OK;
  }
  (void)status;
  if (single_scan) {
    launch("single_scan_kernel", single_scan_kernel, 1, kScanThreads, 0, s, w.tile_count, T + 1, w.offsets64,
                                                  tile_offsets);
    return check_launch("tile_offsets scan");
  }
  size_t sb = w.scan_bytes;
  cudaError_t e = cub::DeviceScan::ExclusiveScan(w.scan_temp, sb, counter_iter(w.tile_count),
                                                 w.offsets64,
                                                 ::cuda::std::plus<long long>(), (long long)0,
                                                 (int)(T + 1), s);
  if (e != cudaSuccess) return fail(SS_ERR_CUDA, "tile offsets scan: %s", cudaGetErrorString(e));
  // int32 offsets for callers that only run stage 1 (the fill rewrites them identically).
  launch("tile_fill_kernel", tile_fill_kernel<false>, (int)((T + 1 + kThreads - 1) / kThreads), kThreads, 0, s, 
      rec, 0, ts, frames, cutoff2, T, w.offsets64, w.tile_count, tile_offsets, nullptr,
      INT64_MAX, w.big_count, nullptr);
  return check_launch("tile_offsets");
}

// Stage 2 over any tile set: fill, per-tile sort.
int index_fill(const Frames& frames, int ts, int64_t T, const void* records, int64_t n,
               int ellipse_cull, float sigma_cutoff, const int32_t* tile_offsets,
               int32_t* tile_gids, int64_t gid_capacity, void* workspace,
               size_t workspace_bytes, uint32_t* status, ss_stream_t stream) {
  int rc;
  if (!tile_offsets || !workspace) return fail(SS_ERR_INVALID_ARGUMENT, "null pointer");
  if (gid_capacity < 0) return fail(SS_ERR_INVALID_ARGUMENT, "negative gid capacity");
  if (gid_capacity > 0 && !tile_gids) return fail(SS_ERR_INVALID_ARGUMENT, "null tile_gids");
  if (workspace_bytes < index_workspace_bytes(T))
    return fail(SS_ERR_INVALID_ARGUMENT, "tile index workspace too small");
  if (T == 0) return SS_OK;
  cudaStream_t s = as_stream(stream);
  IndexWorkspace w = carve(workspace, T);
  const Splat* rec = static_cast<const Splat*>(records);
  float cutoff2 = sigma_cutoff * sigma_cutoff;
  int64_t threads_needed = n > T + 1 ? n : T + 1;
  int blocks = (int)((threads_needed + kThreads - 1) / kThreads);
  int32_t* offsets32 = const_cast<int32_t*>(tile_offsets);
  if (ellipse_cull)
    launch("tile_fill_kernel", tile_fill_kernel<true>, blocks, kThreads, 0, s, rec, n, ts, frames, cutoff2, T,
                                                       w.offsets64, w.tile_count, offsets32,
                                                       tile_gids, gid_capacity, w.big_count,
                                                       status);
  else
    launch("tile_fill_kernel", tile_fill_kernel<false>, blocks, kThreads, 0, s, rec, n, ts, frames, cutoff2, T,
                                                        w.offsets64, w.tile_count, offsets32,
                                                        tile_gids, gid_capacity, w.big_count,
                                                        status);
  if ((rc = check_launch("tile_fill"))) return rc;
  int sort_blocks = (int)((T + (kThreads / 32) - 1) / (kThreads / 32));
  launch("tile_sort_kernel", tile_sort_kernel, sort_blocks, kThreads, 0, s, tile_offsets, tile_gids, gid_capacity, T,
                                                     w.big_tiles, w.big_count);
  if ((rc = check_launch("tile_sort"))) return rc;
  if ((rc = allow_big_sort_smem())) return rc;
  launch("tile_sort_big_kernel", tile_sort_big_kernel, kBigSortCtas, 1024,
         kBigSortSmem * sizeof(int), s, tile_offsets, tile_gids, w.big_tiles, w.big_count,
         sort_key_bits(n));
  return check_launch("tile_sort_big");
}

}  // namespace
}  // namespace ss

using namespace ss;

extern "C" {

int ss_tile_index_workspace_bytes(int64_t n, int height, int width, int tile_size,
                                  size_t* bytes) {
  int rc = check_index_args(n, height, width, tile_size);
  if (rc) return rc;
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  *bytes = index_workspace_bytes(make_grid(height, width, tile_size).T);
  return SS_OK;
}

int ss_batch_tile_index_workspace_bytes(const ss_batch* batch, int64_t n, size_t* bytes) {
  Frames f;
  int rc = frames_of_batch(batch, n, &f);
  if (rc) return rc;
  if (!bytes) return fail(SS_ERR_INVALID_ARGUMENT, "null bytes pointer");
  *bytes = index_workspace_bytes(batch->tiles);
  return SS_OK;
}

int ss_tile_index_count(const void* records, int64_t n, int height, int width, int tile_size,
                        int ellipse_cull, float sigma_cutoff, int32_t* tile_offsets,
                        void* workspace, size_t workspace_bytes, uint32_t* status,
                        ss_stream_t stream) {
  int rc = check_index_args(n, height, width, tile_size);
  if (rc) return rc;
  return index_count(single_frame(height, width, tile_size), tile_size,
                     make_grid(height, width, tile_size).T, records, n, ellipse_cull,
                     sigma_cutoff, tile_offsets, workspace, workspace_bytes, status, stream);
}

int ss_batch_tile_index_count(const ss_batch* batch, const void* records, int64_t n,
                              int ellipse_cull, float sigma_cutoff, int32_t* tile_offsets,
                              void* workspace, size_t workspace_bytes, uint32_t* status,
                              ss_stream_t stream) {
  Frames f;
  int rc = frames_of_batch(batch, n, &f);
  if (rc) return rc;
  return index_count(f, batch->tile_size, batch->tiles, records, n, ellipse_cull, sigma_cutoff,
                     tile_offsets, workspace, workspace_bytes, status, stream);
}

int ss_project_rs_index_count(const float* means, const float* log_scales,
                              const float* rotations, const float* colors,
                              const float* opacity_logits, int64_t n, float dilation,
                              float sigma_cutoff, int height, int width, int tile_size,
                              int ellipse_cull, void* records, int32_t* tile_offsets,
                              void* workspace, size_t workspace_bytes, void* clear,
                              size_t clear_bytes, uint32_t* status, ss_stream_t stream) {
  int rc = check_index_args(n, height, width, tile_size);
  if (rc) return rc;
  if (n > 0 && (!means || !log_scales || !rotations || !colors))
    return fail(SS_ERR_INVALID_ARGUMENT, "null RS field pointer");
  if (!(dilation >= 0.0f)) return fail(SS_ERR_INVALID_ARGUMENT, "dilation must be >= 0");
  const RSField f{means, log_scales, rotations, colors, opacity_logits, dilation, sigma_cutoff};
  return index_count(single_frame(height, width, tile_size), tile_size,
                     make_grid(height, width, tile_size).T, records, n, ellipse_cull,
                     sigma_cutoff, tile_offsets, workspace, workspace_bytes, status, stream, &f,
                     clear, clear_bytes);
}

int ss_batch_project_rs_index_count(const ss_batch* batch, const float* means,
                                    const float* log_scales, const float* rotations,
                                    const float* colors, const float* opacity_logits, int64_t n,
                                    float dilation, float sigma_cutoff, int ellipse_cull,
                                    void* records, int32_t* tile_offsets, void* workspace,
                                    size_t workspace_bytes, void* clear, size_t clear_bytes,
                                    uint32_t* status, ss_stream_t stream) {
  Frames fr;
  int rc = frames_of_batch(batch, n, &fr);
  if (rc) return rc;
  if (n > 0 && (!means || !log_scales || !rotations || !colors))
    return fail(SS_ERR_INVALID_ARGUMENT, "null RS field pointer");
  if (!(dilation >= 0.0f)) return fail(SS_ERR_INVALID_ARGUMENT, "dilation must be >= 0");
  const RSField f{means, log_scales, rotations, colors, opacity_logits, dilation, sigma_cutoff};
  return index_count(fr, batch->tile_size, batch->tiles, records, n, ellipse_cull, sigma_cutoff,
                     tile_offsets, workspace, workspace_bytes, status, stream, &f, clear,
                     clear_bytes);
}

int ss_tile_index_fill(const void* records, int64_t n, int height, int width, int tile_size,
                       int ellipse_cull, float sigma_cutoff, const int32_t* tile_offsets,
                       int32_t* tile_gids, int64_t gid_capacity, void* workspace,
                       size_t workspace_bytes, uint32_t* status, ss_stream_t stream) {
  int rc = check_index_args(n, height, width, tile_size);
  if (rc) return rc;
  return index_fill(single_frame(height, width, tile_size), tile_size,
                    make_grid(height, width, tile_size).T, records, n, ellipse_cull,
                    sigma_cutoff, tile_offsets, tile_gids, gid_capacity, workspace,
                    workspace_bytes, status, stream);
}

int ss_batch_tile_index_fill(const ss_batch* batch, const void* records, int64_t n,
                             int ellipse_cull, float sigma_cutoff, const int32_t* tile_offsets,
                             int32_t* tile_gids, int64_t gid_capacity, void* workspace,
                             size_t workspace_bytes, uint32_t* status, ss_stream_t stream) {
  Frames f;
  int rc = frames_of_batch(batch, n, &f);
  if (rc) return rc;
  return index_fill(f, batch->tile_size, batch->tiles, records, n, ellipse_cull, sigma_cutoff,
                    tile_offsets, tile_gids, gid_capacity, workspace, workspace_bytes, status,
                    stream);
}

}  // extern "C"

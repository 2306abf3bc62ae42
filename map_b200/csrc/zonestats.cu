// Per-zone statistics of a float32 value raster over an int32 zone raster:
// count, min, max, sum and mean of the values of every zone 0 .. nzones-1.
//
// The reference's zonal skeleton (runtime/skeleton/ZonalSkeleton.cpp:33-292)
// reduces a whole raster to one scalar; a zone raster that splits the
// reduction into bins is a new operation of this library. The per-cell rules
// are those of the reference's reductions (runtime/skeleton/util.cpp:518-540,
// util/ReductionType.cpp): SUM adds in float32, MIN / MAX compare.
//
// Rules of this operation:
//   * a cell counts when its zone id is in [0, nzones) and its value is not NaN;
//     other cells are skipped (zone ids outside the range are "no data");
//   * min / max order floats as IEEE totalOrder does for non-NaN values
//     (-0 before +0), so they are exact and independent of the visiting order;
//   * count is exact (64-bit); sum accumulates in float32 (its rounding depends on
//     the order in which the hardware serves the atomics, so it may differ in the
//     last bits between runs); mean = sum / (float)count;
//   * an empty zone reports count 0, sum 0, min +inf, max -inf, mean NaN.
//
// Kernels (one pass over the rasters, HBM-bound: 8 bytes per cell):
//   1. zs_accumulate: a persistent grid; each CTA owns a contiguous range of
//      128-cell row chunks and keeps the zones' bins in shared memory, and each
//      warp walks a contiguous part of that range, 4 chunks in flight, loading a
//      chunk with 16-byte loads (4 cells per lane). The warp stages its 4 chunks
//      (512 cells) in shared memory in cell order and each lane folds 16
//      consecutive cells into a running aggregate (count, sum, min / max keys);
//      zones come in long runs along rows, so lanes of equal zones are adjacent:
//      a segmented shuffle scan merges them and the last lane of each run adds the
//      aggregate to the shared bins with atomics. At the end the CTA adds its
//      non-empty bins into the global bins with atomics. Zone counts whose bins do
//      not fit in shared memory use the global bins directly.
//   2. zs_finalize: converts the global bins into the caller's output arrays.
// Global bins must start at zero before step 1 (a zero bin is the empty bin:
// min / max are kept as order-preserving integer keys whose empty value is 0).
#include "zonestats.hpp"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

namespace mapb {
namespace {

struct Bin {
  unsigned long long count;
  float sum;
  unsigned nmin;   // ~key(min): atomicMax of ~key is atomicMin of key
  unsigned max;    // key(max)
  unsigned pad;
};
static_assert(sizeof(Bin) == 24, "bin layout");

constexpr int kThreads = 256;
constexpr int kUnroll = 4;           // chunks in flight per warp
constexpr int kChunk = 128;          // cells per warp chunk (32 lanes x 4)
constexpr int kMaxSmemZones = 8192;  // 128 KiB of shared bins

// Order-preserving map of a non-NaN float to an unsigned key in [1, 2^32-1).
__device__ __forceinline__ unsigned fkey(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(unsigned k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

struct SmemBins {
  unsigned *cnt;
  float *sum;
  unsigned *nmin;
  unsigned *max;
};

template <bool SMEM>
__device__ __forceinline__ void bin_add(const SmemBins &s, Bin *g, int z, unsigned c, float sm, unsigned nmn,
                                        unsigned mx) {
  if (SMEM) {
    atomicAdd(&s.cnt[z], c);
    atomicAdd(&s.sum[z], sm);
    atomicMax(&s.nmin[z], nmn);
    atomicMax(&s.max[z], mx);
  } else {
    atomicAdd(&g[z].count, (unsigned long long)c);
    atomicAdd(&g[z].sum, sm);
    atomicMax(&g[z].nmin, nmn);
    atomicMax(&g[z].max, mx);
  }
}

struct Geometry {
  const char *val;
  long long vpitch;
  const char *zone;
  long long zpitch;
  int W, H, nzones;
  long long nchunk_x;      // chunks per row
  long long chunks;        // total chunks
  long long per_cta;       // chunks per CTA (contiguous range)
  int vec;                 // 16-byte loads allowed for full chunks
};

// Running aggregate of one lane over consecutive cells of one zone.
struct LaneAcc {
  int key;
  unsigned cnt, nmn, mx;
  float sm;
};

// Adds every lane's aggregate to the bins, lanes of equal zones merged first by a
// segmented shuffle scan (runs of equal keys, in lane order) so only the last
// lane of each run issues atomics. Called by all 32 lanes; key < 0 lanes skip.
template <bool SMEM>
__device__ __forceinline__ void warp_flush(const SmemBins &sb, Bin *gbins, const LaneAcc &a, int lane, unsigned below) {
  int key = a.cnt ? a.key : -1;
  unsigned cnt = a.cnt, nmn = a.nmn, mx = a.mx;
  float sm = a.sm;
  const int up = __shfl_up_sync(0xffffffffu, key, 1);
  const unsigned heads = __ballot_sync(0xffffffffu, lane == 0 || up != key);
  const int seg_start = 31 - __clz(heads & below);
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const unsigned c2 = __shfl_up_sync(0xffffffffu, cnt, off);
    const float s2 = __shfl_up_sync(0xffffffffu, sm, off);
    const unsigned n2 = __shfl_up_sync(0xffffffffu, nmn, off);
    const unsigned m2 = __shfl_up_sync(0xffffffffu, mx, off);
    if (lane - off >= seg_start) {
      sm = s2 + sm;
      cnt += c2;
      nmn = max(nmn, n2);
      mx = max(mx, m2);
    }
  }
  const int dn = __shfl_down_sync(0xffffffffu, key, 1);
  if ((lane == 31 || dn != key) && key >= 0 && cnt > 0) bin_add<SMEM>(sb, gbins, key, cnt, sm, nmn, mx);
}

constexpr int kStep = kChunk * kUnroll;          // cells a warp stages per step (512)
constexpr int kRun = kStep / 32;                   // consecutive cells a lane folds per step (16)
constexpr int kStage = kStep + kStep / 32;         // staging words per warp and array (one pad word per 32)

__device__ __forceinline__ int stage_idx(int i) { return i + (i >> 5); }   // conflict-free both ways

template <bool SMEM>
__global__ void __launch_bounds__(kThreads, 3) zs_accumulate(const Geometry geo, Bin *gbins) {
  extern __shared__ __align__(16) unsigned char zs_smem[];
  __shared__ float st_v[kThreads / 32][kStage];
  __shared__ int st_z[kThreads / 32][kStage];
  SmemBins sb = {nullptr, nullptr, nullptr, nullptr};
  const int nz = geo.nzones;
  if (SMEM) {
    sb.cnt = (unsigned *)zs_smem;
    sb.sum = (float *)(sb.cnt + nz);
    sb.nmin = (unsigned *)(sb.sum + nz);
    sb.max = sb.nmin + nz;
    for (int i = threadIdx.x; i < 4 * nz; i += blockDim.x) ((unsigned *)zs_smem)[i] = 0u;
    __syncthreads();
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  // the CTA's contiguous chunk range, split into one contiguous sub-range per warp
  const long long c0 = (long long)blockIdx.x * geo.per_cta;
  const long long c1 = min(geo.chunks, c0 + geo.per_cta);
  const long long per_warp = (c1 - c0 + nwarps - 1) / nwarps;
  const long long w0 = min(c1, c0 + (long long)warp * per_warp);
  const long long w1 = min(c1, w0 + per_warp);
  const unsigned below = (lane == 31) ? 0xffffffffu : ((2u << lane) - 1u);   // lanes <= this one
  float *sv = st_v[warp];
  int *sz = st_z[warp];
  const int st_base = lane * 4 + (lane >> 3);       // stage_idx(4 * lane), the lane's 4 cells of a chunk
  const int run_base = lane * kRun + (lane >> 1);   // stage_idx(16 * lane), the lane's run
  // row and chunk column of chunk cb, advanced incrementally (one division per warp)
  long long yb = w0 / geo.nchunk_x;
  long long xb = w0 - yb * geo.nchunk_x;

  // Loads of one step (kUnroll chunks of 128 cells) into registers; cells past
  // the warp's range or the raster edge get zone -1.
  float v[kUnroll][4];
  int z[kUnroll][4];
  auto load_step = [&](long long cb, long long xs, long long ys) {
    // the step's 4 chunks usually lie in one row: one row pointer for all of them
    const bool one_row = xs + kUnroll <= geo.nchunk_x && cb + kUnroll <= w1;
    const float *vrow = (const float *)(geo.val + ys * geo.vpitch);
    const int *zrow = (const int *)(geo.zone + ys * geo.zpitch);
#pragma unroll
    for (int u = 0; u < kUnroll; u++) {
      const long long c = cb + u;
#pragma unroll
      for (int j = 0; j < 4; j++) z[u][j] = -1;
      if (c < w1) {
        const float *vr = vrow;
        const int *zr = zrow;
        int x;
        if (one_row) {
          x = ((int)xs + u) * kChunk + lane * 4;
        } else {
          long long y = ys, cx = xs + u;
          while (cx >= geo.nchunk_x) {
            cx -= geo.nchunk_x;
            y++;
          }
          x = (int)cx * kChunk + lane * 4;
          vr = (const float *)(geo.val + y * geo.vpitch);
          zr = (const int *)(geo.zone + y * geo.zpitch);
        }
        if (geo.vec && x + 3 < geo.W) {
          const float4 a = __ldcs((const float4 *)(vr + x));
          const int4 b = __ldcs((const int4 *)(zr + x));
          v[u][0] = a.x; v[u][1] = a.y; v[u][2] = a.z; v[u][3] = a.w;
          z[u][0] = b.x; z[u][1] = b.y; z[u][2] = b.z; z[u][3] = b.w;
        } else {
#pragma unroll
          for (int j = 0; j < 4; j++)
            if (x + j < geo.W) {
              v[u][j] = __ldcs(vr + x + j);
              z[u][j] = __ldcs(zr + x + j);
            }
        }
      }
    }
  };
  if (w0 < w1) load_step(w0, xb, yb);
  for (long long cb = w0; cb < w1; cb += kUnroll) {
    // stage the step's cells in order, then let each lane fold a run of consecutive cells
    // cell u*128 + 4*lane + j sits at stage_idx() = u*132 + st_base + j
#pragma unroll
    for (int u = 0; u < kUnroll; u++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        sv[st_base + u * (kChunk + kChunk / 32) + j] = v[u][j];
        sz[st_base + u * (kChunk + kChunk / 32) + j] = z[u][j];
      }
    // the next step's loads go out now, into the registers just staged, and are
    // in flight while this step is folded and flushed
    xb += kUnroll;
    while (xb >= geo.nchunk_x) {
      xb -= geo.nchunk_x;
      yb++;
    }
    if (cb + kUnroll < w1) load_step(cb + kUnroll, xb, yb);
    __syncwarp();
    // the lane's run: cells 16*lane + k at stage_idx() = run_base + k
    int key = -1;
    unsigned cnt = 0u, kmin = 0xffffffffu, kmax = 0u;
    float sm = 0.0f;
#pragma unroll
    for (int k = 0; k < kRun; k++) {
      const int zz = sz[run_base + k];
      const float vv = sv[run_base + k];
      if ((unsigned)zz >= (unsigned)nz || vv != vv) continue;
      if (zz != key) {
        // a zone edge inside the lane's run (rare): the finished part goes straight to the bins
        if (cnt) bin_add<SMEM>(sb, gbins, key, cnt, sm, ~kmin, kmax);
        key = zz;
        cnt = 0u;
        kmin = 0xffffffffu;
        kmax = 0u;
        sm = 0.0f;
      }
      const unsigned kk = fkey(vv);
      cnt++;
      sm += vv;
      kmin = min(kmin, kk);
      kmax = max(kmax, kk);
    }
    // lanes are in cell order, so equal zones form runs of lanes: merge and add
    warp_flush<SMEM>(sb, gbins, LaneAcc{key, cnt, ~kmin, kmax, sm}, lane, below);
    __syncwarp();   // the staging area is rewritten by the next step
  }
  if (SMEM) {
    __syncthreads();
    for (int i = threadIdx.x; i < nz; i += blockDim.x) {
      const unsigned c = sb.cnt[i];
      if (c == 0) continue;
      atomicAdd(&gbins[i].count, (unsigned long long)c);
      atomicAdd(&gbins[i].sum, sb.sum[i]);
      atomicMax(&gbins[i].nmin, sb.nmin[i]);
      atomicMax(&gbins[i].max, sb.max[i]);
    }
  }
}

__global__ void zs_finalize(const Bin *gbins, int nz, unsigned long long *count, float *vmin, float *vmax, float *sum,
                            float *mean) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nz) return;
  const Bin b = gbins[i];
  if (count) count[i] = b.count;
  if (sum) sum[i] = b.sum;
  if (vmin) vmin[i] = b.count ? fkey_inv(~b.nmin) : INFINITY;
  if (vmax) vmax[i] = b.count ? fkey_inv(b.max) : -INFINITY;
  if (mean) mean[i] = b.count ? b.sum / (float)b.count : NAN;
}

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw MapError(std::string("zone statistics: ") + what + ": " + cudaGetErrorString(e));
}

struct DevInfo {
  int sms = 0;
  bool ready = false;
};

DevInfo &dev_info() {
  static std::mutex m;
  static DevInfo info[64];
  int d = 0;
  check(cudaGetDevice(&d), "cudaGetDevice");
  if (d < 0 || d >= 64) throw MapError("zone statistics: device ordinal out of range");
  std::lock_guard<std::mutex> lk(m);
  DevInfo &I = info[d];
  if (!I.ready) {
    check(cudaDeviceGetAttribute(&I.sms, cudaDevAttrMultiProcessorCount, d), "cudaDeviceGetAttribute");
    check(cudaFuncSetAttribute(zs_accumulate<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kMaxSmemZones * 16),
          "cudaFuncSetAttribute");
    I.ready = true;
  }
  return I;
}

}  // namespace

static void zone_stats_validate(const ZoneStatsArgs &a) {
  if (a.W < 0 || a.H < 0) throw MapError("zone statistics: negative raster size");
  if (a.nzones < 1) throw MapError("zone statistics: nzones must be at least 1");
  if (a.W > 0 && a.H > 0) {
    if (!a.value || !a.zone) throw MapError("zone statistics: null raster pointer");
    if (a.value_pitch < (long long)a.W * 4 || a.zone_pitch < (long long)a.W * 4)
      throw MapError("zone statistics: pitch smaller than a row");
    if (((uintptr_t)a.value | (uintptr_t)a.zone) % 4 != 0 || a.value_pitch % 4 != 0 || a.zone_pitch % 4 != 0)
      throw MapError("zone statistics: rasters and pitches must be 4-byte aligned");
  }
}

// Enqueues the accumulation and finalisation on `st`; `bins` holds
// zone_stats_bin_bytes(nzones) bytes of zeros.
static void zone_stats_run(const ZoneStatsArgs &a, void *bins, cudaStream_t st) {
  DevInfo &I = dev_info();
  const long long cells = (long long)a.W * a.H;
  if (cells > 0) {
    Geometry g;
    g.val = (const char *)a.value;
    g.vpitch = a.value_pitch;
    g.zone = (const char *)a.zone;
    g.zpitch = a.zone_pitch;
    g.W = a.W;
    g.H = a.H;
    g.nzones = a.nzones;
    g.nchunk_x = (a.W + kChunk - 1) / kChunk;
    g.chunks = g.nchunk_x * a.H;
    g.vec = (((uintptr_t)a.value | (uintptr_t)a.zone) % 16 == 0 && a.value_pitch % 16 == 0 &&
             a.zone_pitch % 16 == 0)
                ? 1
                : 0;
    const bool smem = a.nzones <= kMaxSmemZones;
    const size_t smem_bytes = smem ? (size_t)a.nzones * 16 : 0;
    int occ = 0;
    if (smem)
      check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, zs_accumulate<true>, kThreads, smem_bytes),
            "occupancy");
    else
      check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, zs_accumulate<false>, kThreads, 0), "occupancy");
    occ = std::max(1, occ);
    // enough chunks per CTA that every warp has work; per-CTA counts stay below 2^32
    const long long max_ctas = (long long)I.sms * occ;
    long long ctas = std::min<long long>(max_ctas, (g.chunks + (kThreads / 32) * kUnroll - 1) /
                                                       ((kThreads / 32) * kUnroll));
    // per-CTA shared counts are 32-bit: at most 2^31 cells per CTA
    ctas = std::max<long long>(ctas, (g.chunks + (1LL << 24) - 1) >> 24);
    ctas = std::max<long long>(1, ctas);
    g.per_cta = (g.chunks + ctas - 1) / ctas;
    ctas = (g.chunks + g.per_cta - 1) / g.per_cta;
    if (smem)
      zs_accumulate<true><<<(unsigned)ctas, kThreads, smem_bytes, st>>>(g, (Bin *)bins);
    else
      zs_accumulate<false><<<(unsigned)ctas, kThreads, 0, st>>>(g, (Bin *)bins);
    check(cudaGetLastError(), "accumulate launch");
  }
  zs_finalize<<<(a.nzones + 255) / 256, 256, 0, st>>>((const Bin *)bins, a.nzones, a.count, a.vmin, a.vmax, a.sum,
                                                       a.mean);
  check(cudaGetLastError(), "finalize launch");
}

static size_t zone_stats_bin_bytes(int nzones) { return (size_t)nzones * sizeof(Bin); }

void zone_stats(const ZoneStatsArgs &a, cudaStream_t st) {
  zone_stats_validate(a);
  const size_t bytes = zone_stats_bin_bytes(a.nzones);
  void *bins = nullptr;
  check(cudaMallocAsync(&bins, bytes, st), "cudaMallocAsync(bins)");
  cudaError_t e = cudaMemsetAsync(bins, 0, bytes, st);
  if (e == cudaSuccess) {
    try {
      zone_stats_run(a, bins, st);
    } catch (...) {
      cudaFreeAsync(bins, st);
      throw;
    }
  }
  cudaFreeAsync(bins, st);
  check(e, "cudaMemsetAsync(bins)");
}

// ------------------------------------------------- allocation-free variant
//
// For callers that must not allocate device memory while they run: a server
// that reserved its whole HBM budget up front (an allocation from the stream's
// pool could fail or push it past the budget), or a latency-critical loop in
// which an allocation may stall (cudaMalloc / cudaFree synchronise the device,
// and a pool allocation may have to grow the pool).
//
// Its working bins live in one fixed file-scope array per device instead of the
// stream's memory pool, so it serves at most kStaticZones zones (larger zone
// counts are rejected with an error). The first call on a device does the
// set-up for that device: it looks up the array's address and loads the
// kernels; make it before any stream capture begins. Every call on a device
// shares the one array: calls whose work may overlap on the device (different
// streams, or several host threads) race and corrupt each other's results, so
// issue them in order on one stream. Each call clears the bins it uses
// (cudaMemsetAsync on the caller's stream) before it accumulates into them.

constexpr int kStaticZones = 16384;   // 16384 x 24 B = 384 KiB per device
static __device__ __align__(256) Bin zs_static_bins[kStaticZones];

// Address of the array in the current device's context. The address is looked
// up on every call (a host-side lookup, no allocation), so a device or context
// reset by the application between calls is harmless: the next call finds the
// array in the new context. The kernels are loaded on the first call per device
// so that later calls load nothing; after a reset the runtime loads them again
// on the next call.
static void *static_bins() {
  static std::mutex m;
  static bool loaded[64] = {};
  int d = 0;
  check(cudaGetDevice(&d), "cudaGetDevice");
  if (d < 0 || d >= 64) throw MapError("zone statistics: device ordinal out of range");
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, zs_static_bins);
  if (e != cudaSuccess || !p)
    throw MapError(std::string("zone statistics: cudaGetSymbolAddress of the static bins failed: ") +
                   cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(m);
  if (!loaded[d]) {
    dev_info();   // loads the shared-bin accumulation kernel
    cudaFuncAttributes fa;
    check(cudaFuncGetAttributes(&fa, zs_accumulate<false>), "cudaFuncGetAttributes");
    check(cudaFuncGetAttributes(&fa, zs_finalize), "cudaFuncGetAttributes");
    loaded[d] = true;
  }
  return p;
}

void zone_stats_no_alloc(const ZoneStatsArgs &a, cudaStream_t st) {
  zone_stats_validate(a);
  if (a.nzones > kStaticZones)
    throw MapError("zone statistics without allocation: nzones " + std::to_string(a.nzones) +
                   " exceeds the fixed scratch of " + std::to_string(kStaticZones) +
                   " zones (the allocating entry point has no such limit)");
  void *bins = static_bins();
  check(cudaMemsetAsync(bins, 0, zone_stats_bin_bytes(a.nzones), st), "cudaMemsetAsync(static bins)");
  zone_stats_run(a, bins, st);
}

}  // namespace mapb

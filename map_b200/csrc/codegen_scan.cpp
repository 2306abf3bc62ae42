// Execution of the Radiating (radial scan) and Spreading (flow accumulation)
// skeletons; their kernels are generated in codegen.cpp (gen_radial, gen_spread).
//
// Radiating (runtime/skeleton/RadiatingSkeleton.cpp:32-323): one CTA per octant
// sweeps the octant's fronts d0 = 1, 2, ... in order; the cells of a front are
// independent and are spread over the CTA's threads. A cell's scan value is
// op(LIT(prev front at d1, prev front at d1-1), in) when `in` is finite; the
// start cell holds the neutral value. The previous and current fronts are kept in
// the CTA's shared memory when both fit (radial_front_smem, up to 200 KiB); for
// rasters at least kRadialClusterDim cells across, the octant runs on a cluster of
// kRadialCluster CTAs, each holding one segment of both fronts in its shared
// memory and reading the value left of its segment from its neighbour's
// (distributed shared memory). Fronts too long for either are read back from the
// scan's own output raster (written by this CTA one step earlier; cells on an
// octant boundary are written by both adjacent octants with identical values).
// The group's local nodes before the scan are evaluated per cell to produce
// `in`; those after it are evaluated right after the cell's scan value.
//
// Spreading (runtime/skeleton/SpreadingSkeleton.cpp:288-393): the reference
// relaxes "pending spread" one neighbour per iteration, block by block, until
// stable; the fixed point is, for every cell, the sum of the water of all
// strictly-upstream cells. Here the same fixed point is reached without
// iterating to convergence. In-degrees are counted by pulling from the 8
// neighbours; then either one CTA sweeps frontier by frontier (topological
// order; rasters up to kSpreadKahnCells = 64 K cells) or, for larger rasters, a thread per source
// walks down its flow path pushing (accumulation + water) with atomic adds and
// continues into a cell only when its push was the cell's last pending one, so
// each cell is completed exactly once after all its upstream cells. Integer
// sums are exact and order-independent.
#include "codegen.hpp"
#include "cuda_env.hpp"
#include "executor.hpp"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <unordered_map>

namespace mapb {

// Flow accumulations of at most this many cells run as one CTA's frontier sweep;
// larger ones as the two grid-wide passes (in-degrees, then downstream walks),
// which spread over every SM (measured at 1024²: 1.7 ms against 5.6 ms for one
// CTA). Serving runs one CTA per window instead, many windows side by side.
constexpr size_t kSpreadKahnCells = (size_t)1 << 16;
// Integer flow accumulations of more cells than kSpreadKahnCells and at most this
// many run as pointer jumping over the Euler tour of the D8 forest (a fixed
// number of rounds, independent of the longest flow path; O(N log N) work).
// Whole rasters on an otherwise idle GPU walk faster (measured 0.21 against
// 0.43 ms at 1024^2, 0.61 against 1.82 ms at 2048^2), so the default is 0
// (never); serving windows, which run beside other requests, jump (server.cpp).
// ma_setFlowJumpCells, or MAP_B200_SPREAD_PJ for the default, sets the limit.
size_t spread_pj_cells() {
  static const size_t dflt = [] {
    const char *e = std::getenv("MAP_B200_SPREAD_PJ");
    return e ? (size_t)std::strtoull(e, nullptr, 10) : (size_t)0;
  }();
  const long long v = Runtime::get().flow_jump_cells;
  return v < 0 ? dflt : (size_t)v;
}
// rounds of pointer jumping for N cells: 2^rounds exceeds 2N, the longest tour
int spread_pj_rounds(size_t N) {
  int r = 1;
  while (((size_t)1 << r) <= 2 * N) r++;
  return r;
}
bool spread_pj_type(int dt) { return dt == S32 || dt == U32 || dt == S64 || dt == U64; }
size_t spread_pj_scratch(size_t N, int dt) { return 4 * N * (sizeof(int32_t) + dt_size(dt)); }
// radial scans of rasters at least this wide or tall use CTA clusters per octant
constexpr int kRadialClusterDim = 2048;
constexpr int kRadialCluster = 8;

size_t radial_front_smem(int W, int H, int dtype) {
  const size_t b = 2 * (size_t)std::max(W, H) * dt_size(dtype);   // previous and current front
  return b <= (size_t)200 * 1024 ? b : 0;                          // larger: fronts re-read from the output
}

void run_scan_group(const Group &g, const KernelPlan &P, std::unordered_map<Node *, DevRaster> &bufs,
                    const std::function<DevRaster &(Node *)> &get, const std::function<DevRaster(Node *)> &alloc_out) {
  CudaEnv &env = CudaEnv::get();
  cudaStream_t st = (cudaStream_t)env.stream();
  for (Node *o : P.out_rasters)
    if (!bufs.count(o)) bufs[o] = alloc_out(o);
  Node *scan = P.core;
  KernelHandle kh = env.kernel(P.source, P.kname, 0);
  if (scan->kind == K_RADIALSCAN) {
    int ri = -1;
    for (size_t k = 0; k < P.out_rasters.size(); k++)
      if (P.out_rasters[k] == scan) ri = (int)k;
    if (ri < 0) throw MapError("radial scan output missing");
    long long lim = -1;
    if (scan->radius > 0) {
      lim = (long long)scan->radius;
      for (Node *o : P.out_rasters) {
        DevRaster &r = bufs.at(o);
        cuda_check(cudaMemset2DAsync(r.ptr, r.pitch, 0xFF, (size_t)r.W * dt_size(r.dtype), r.H, st), "memset");
      }
    }
    uint64_t aux[4] = {(uint64_t)scan->coord.arr[0], (uint64_t)scan->coord.arr[1], (uint64_t)lim, (uint64_t)ri};
    auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux);
    // long fronts: a cluster of kRadialCluster CTAs per octant, each holding a
    // segment of the fronts in shared memory
    const int maxdim = std::max(g.W, g.H);
    const size_t seg = ((size_t)maxdim + kRadialCluster - 1) / kRadialCluster;
    const size_t csmem = 2 * seg * dt_size(scan->meta.dtype);
    if (maxdim >= kRadialClusterDim && csmem <= (size_t)200 * 1024) {
      KernelHandle kc = env.kernel(P.source, P.kname + "_cl", csmem);
      env.launch_cluster(kc, 8 * kRadialCluster, 512, kRadialCluster, csmem, (CUstream_st *)st, a.data());
      return;
    }
    const size_t smem = radial_front_smem(g.W, g.H, scan->meta.dtype);
    env.launch(env.kernel(P.source, P.kname, smem), 8, 512, smem, (CUstream_st *)st, a.data(), a.size());
    return;
  }
  const size_t N = (size_t)g.W * g.H;
  if (N >= (size_t)1 << 31) throw MapError("spreadScan: raster too large");
  if (N > kSpreadKahnCells && N <= spread_pj_cells() && spread_pj_type(scan->meta.dtype)) {
    void *work = nullptr;
    cuda_check(cudaMallocAsync(&work, spread_pj_scratch(N, scan->meta.dtype), st), "cudaMallocAsync(spread work)");
    const int rounds = spread_pj_rounds(N);
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((2 * N + 255) / 256, (size_t)env.sm_count() * 8));
    uint64_t aux[4] = {(uint64_t)(uintptr_t)work, 0, 0, 0};
    auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux);
    env.launch(env.kernel(P.source, P.kname + "_pj_init", 0), grid, 256, 0, (CUstream_st *)st, a.data(), a.size());
    KernelHandle ks = env.kernel(P.source, P.kname + "_pj_step", 0);
    for (int r = 0; r < rounds; r++) {
      aux[1] = (uint64_t)r;
      auto ar = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux);
      env.launch(ks, grid, 256, 0, (CUstream_st *)st, ar.data(), ar.size());
    }
    aux[1] = (uint64_t)rounds;
    auto af = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux);
    env.launch(env.kernel(P.source, P.kname + "_pj_final", 0), grid, 256, 0, (CUstream_st *)st, af.data(), af.size());
    cuda_check(cudaFreeAsync(work, st), "cudaFreeAsync");
    return;
  }
  void *work = nullptr;
  cuda_check(cudaMallocAsync(&work, 6 * N * sizeof(int32_t), st), "cudaMallocAsync(spread work)");
  uint64_t aux[4] = {(uint64_t)(uintptr_t)work, (uint64_t)(uintptr_t)((int32_t *)work + 2 * N),
                     (uint64_t)(uintptr_t)((int32_t *)work + 4 * N), (uint64_t)(N + 1)};
  auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux);
  if (N <= kSpreadKahnCells) {
    // one CTA, frontier by frontier: the lowest latency up to 64 K cells
    env.launch(env.kernel(P.source, P.kname + "_kahn", 0), 1, 1024, 0, (CUstream_st *)st, a.data(), a.size());
  } else {
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((N + 255) / 256, (size_t)env.sm_count() * 8));
    KernelHandle ki = env.kernel(P.source, P.kname + "_init", 0);
    env.launch(ki, grid, 256, 0, (CUstream_st *)st, a.data(), a.size());
    env.launch(kh, grid, 256, 0, (CUstream_st *)st, a.data(), a.size());
  }
  cuda_check(cudaFreeAsync(work, st), "cudaFreeAsync");
}

}  // namespace mapb

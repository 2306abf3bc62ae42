// Evaluation engine: runs the groups of one evaluation on the device.
//
// Replaces the reference's Program / Task / Scheduler / Worker / Cache / Block
// runtime (runtime/Program.cpp, runtime/task/*, runtime/Scheduler.cpp,
// runtime/Worker.cpp, runtime/Cache.cpp, runtime/Block.cpp) with an HBM-resident
// design: every raster lives whole in device memory (row-major, 128-byte pitch),
// allocated stream-ordered from the CUDA memory pool, and all work is enqueued on
// one stream. Two launch granularities:
//  * fused: one launch per group over the whole raster;
//  * plain: one launch per group per block, issued in the order of a ready-queue
//    of (group, block) jobs keyed by a Morton interleave of (x, y, group), with the
//    focal 3x3 block dependencies of runtime/task/FocalTask.cpp:36-115.
// Programs from host rasters to host rasters can instead stream through row
// bands (evaluate_streamed), which replaces the reference Cache's spilling of
// blocks between host and device (runtime/Cache.cpp:505-571).
#pragma once

#include "codegen.hpp"
#include "fusion.hpp"

#include <functional>
#include <map>
#include <unordered_map>
#include <memory>
#include <set>
#include <string>
#include <vector>

namespace mapb {

struct DevRaster {
  void *ptr = nullptr;
  long long pitch = 0;   // bytes
  bool owned = false;
  int dtype = 0;
  int W = 0, H = 0;
  // Row band of a raster (streamed evaluation): the buffer holds raster rows
  // org .. org + rows - 1 and `ptr` is the virtual address of raster row 0
  // (buffer - org * pitch, modulo 2^64), so kernels index it with raster rows.
  long long org = 0;
  int rows = 0;          // 0: the whole raster is held
};

// Where a requested raster goes after evaluation.
struct Sink {
  Node *node = nullptr;
  void *host = nullptr;      // dense row-major host destination (or null)
  void *dev = nullptr;       // device destination (or null)
  long long dev_pitch = 0;
};

// One job of the plain-mode schedule.
struct PlainJob {
  int group = 0;
  int bx = -1, by = -1;   // block coordinate, -1 for whole-raster jobs
  int kind = 0;           // 0 block launch, 1 whole-raster launch, 2 zonal finalisation, 3 host scalar step
};

// Plain-mode launch order for the given groups (pure host logic).
std::vector<PlainJob> plain_schedule(const std::vector<std::unique_ptr<Group>> &groups,
                                     const std::vector<KernelPlan> &plans);

// Packs the kernel argument struct of plan K for a launch over region
// [rx0,rx1) x [ry0,ry1); rasters are looked up with `get` (inputs) and in `bufs` (outputs).
// `scalars`, when given, overrides the values of scalar argument nodes.
// `out_maps`: the outputs are whole rasters at their own base addresses, so a
// plan with output tile stores (K.tma_out) gets their tensor maps and aux[2] = 1.
std::vector<unsigned char> pack_args(const Group &g, const KernelPlan &K, const std::function<DevRaster &(Node *)> &get,
                                     std::unordered_map<Node *, DevRaster> &bufs, int rx0, int ry0, int rx1, int ry1,
                                     const uint64_t aux[4],
                                     const std::unordered_map<const Node *, Variant> *scalars = nullptr,
                                     bool out_maps = false);

// Every node `targets` depend on (themselves included), in id (= topological) order.
std::vector<Node *> collect_nodes(const std::vector<Node *> &targets);

struct EvalStats {
  int launches = 0;
  int groups = 0;
  int compiled = 0;
  int bands = 0;     // row bands of a streamed evaluation (0: whole rasters)
  int predicted = 0; // groups filled with their one known value instead of launched
  double host_ms = 0;
};

class Executor {
 public:
  static Executor &get();
  // Evaluates `targets` (and the sinks' nodes). Blocks until done unless `async`
  // is set and nothing needs the host (no sinks with host memory, no writes,
  // no scalar read-backs).
  void evaluate(const std::vector<Node *> &targets, const std::vector<Sink> &sinks, bool async = false);
  // Evaluates rows [y0, y1) of a program of Local / Focal groups over one raster
  // shape: every sink goes to device memory holding those rows (its `dev` is the
  // address of row y0), inputs are device rasters, whole or row bands holding at
  // least the rows the range reads (the program's halo beyond it). Border
  // decisions are made in whole-raster coordinates, so the rows equal those of a
  // whole-raster evaluation. Blocks until done.
  void evaluate_rows(const std::vector<Node *> &targets, const std::vector<Sink> &sinks, int y0, int y1);
  // Rows beyond [y0, y1) (above and below, clipped to the raster) that
  // evaluate_rows reads from the inputs of `targets`.
  int row_margin(const std::vector<Node *> &targets);
  // Evaluates `nodes` in one evaluation and returns, for each, a node that
  // holds its value: a D2 result in a device buffer the library owns (freed
  // with the returned node), a D0 result as a constant. Device inputs holding a
  // whole raster and constants are returned as they are. Loop-carried values
  // of a while-loop stay resident this way between iterations.
  std::vector<Node *> materialize(const std::vector<Node *> &nodes);
  // Fusion + code generation + compilation only (no device needed).
  std::vector<std::string> compile_only(const std::vector<Node *> &targets, bool compile);
  std::string describe_groups(const std::vector<Node *> &targets);
  std::vector<PlainJob> schedule_for(const std::vector<Node *> &targets);
  EvalStats last;
  void sync();

 private:
  struct Prepared {
    FusionResult fr;
    std::vector<KernelPlan> plans;
    std::vector<Node *> order;
  };
  Prepared prepare(const std::vector<Node *> &targets, const std::set<Node *> &tset, bool compile);
  // Programs evaluated again (same target nodes, same launch mode, same known
  // scalar values, no node destroyed since) reuse their fusion and kernel plans.
  struct CacheEntry {
    std::shared_ptr<Prepared> P;
    std::vector<char> d0sig;   // has_value of every D0 node of P.order
    uint64_t epoch = 0;
    uint64_t used = 0;
  };
  std::map<std::string, CacheEntry> cache_;
  uint64_t cache_tick_ = 0;
  std::shared_ptr<Prepared> prepare_cached(const std::vector<Node *> &targets, const std::set<Node *> &tset);
  // Row-band streaming of host-to-host Local / Focal programs; false (and no
  // work done) when the program does not qualify.
  bool evaluate_streamed(const Prepared &P, const std::vector<Node *> &targets, const std::vector<Sink> &sinks);
};

}  // namespace mapb

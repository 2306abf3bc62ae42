// Batched persistent execution: many independent programs (instances), e.g. the
// same script over hundreds of rasters of uneven size, run as ONE persistent
// kernel per dependency level, driven by a device work-list of
// (kind, instance, tile) items and replayed from a CUDA graph.
//
//  * each instance is fused on its own; its Local / Focal groups are bucketed by
//    kernel body ("kind"): instances with the same program share one compiled
//    tile function, with per-instance arguments in a device array;
//  * the batch module holds every kind's tile function in its own namespace and
//    a persistent kernel that pulls items with an atomic counter and dispatches
//    on the kind (the TMA staging mbarrier is initialised once per CTA and
//    tracked by phase parity across items);
//  * tile shapes are chosen per kind by an autotuner that times candidate shapes
//    on the batch's largest raster of that kind and caches the winner per
//    (skeleton, halo, dtype, shape bucket) in memory and on disk;
//  * intermediate rasters live in buffers owned by the batch.
#pragma once

#include "codegen.hpp"
#include "executor.hpp"

#include <memory>
#include <string>
#include <vector>

namespace mapb {

struct BatchInstance {
  std::vector<Node *> outs;
  std::vector<void *> dst;
  std::vector<long long> pitch;
};

class Batch {
 public:
  Batch();
  ~Batch();
  void add(const std::vector<Node *> &outs, const std::vector<void *> &dst, const std::vector<long long> &pitch);
  void prepare(bool autotune);
  void run(bool sync);
  std::string info() const;
  int instances() const { return (int)inst_.size(); }

 private:
  struct Kind;
  struct Impl;
  std::vector<BatchInstance> inst_;
  std::unique_ptr<Impl> impl_;
};

// Persistent dispatcher over several kinds of tile function (Local / Focal
// plans with 256 threads): one kernel `kname` taking
//   struct { u64 items; s64 n; u64 counter; u64 err; u64 args[kinds]; }
// that pulls (kind, instance, tile) items with an atomic counter.
struct PersistentModule {
  std::string source, kname;
  size_t smem = 0;
};
PersistentModule build_persistent_module(const std::vector<const KernelPlan *> &kinds);

// Autotuned tile shape for a kind (groups of identical code, inputs / outputs bound
// through `get` / `bufs`): times one persistent launch over all members' tiles per
// candidate shape on the library stream.
TileCfg autotune_kind(const std::vector<const Group *> &members, const std::function<DevRaster &(Node *)> &get,
                      std::unordered_map<Node *, DevRaster> &bufs);
std::string tune_key(const Group &g, const KernelPlan &p);

}  // namespace mapb

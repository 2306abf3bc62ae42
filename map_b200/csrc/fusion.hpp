// Fusion compiler: partitions the nodes of one evaluation into groups, each of
// which becomes one kernel (or one host step for scalar-only work).
//
// The legality tables are the reference's (runtime/Pattern.cpp:53-184,
// canPipeFuse / canFlatFuse); the grouping procedure is this project's own:
//   1. every device node starts in its own group;
//   2. pipe fusion merges a consumer into its producer's group when the edge
//      (producer pattern -> consumer pattern) may be pipe-fused, the group
//      patterns may be flat-fused, a scalar (D0) result is not consumed by a
//      raster op, and no third group lies on a path between the two;
//   3. flat fusion merges sibling groups that read a common raster;
//   4. steps 2-3 repeat until nothing changes.
// FREE raster nodes (constants, index) are recomputed inside every group that
// reads them, as the reference forwards them (runtime/visitor/Fusioner.cpp:343).
#pragma once

#include "graph.hpp"

#include <memory>
#include <set>
#include <vector>

namespace mapb {

enum SkeletonKind : int { SK_HOST = 0, SK_LOCAL, SK_FOCAL, SK_ZONAL, SK_RADIAL, SK_SPREAD };
const char *skeleton_name(int sk);

bool can_pipe_fuse(int top, int bot);
bool can_flat_fuse(int left, int right);

struct Group {
  int id = 0;
  int pattern = P_NONE;
  int skeleton = SK_LOCAL;
  std::vector<Node *> nodes;    // nodes computed by the group, in id order (includes inlined FREE nodes)
  std::vector<Node *> inputs;   // rasters and scalars read from outside, in id order
  std::vector<Node *> outputs;  // nodes whose values leave the group, in id order
  std::vector<Group *> prev, next;
  // geometry shared by every raster node of the group
  int W = 0, H = 0, BS0 = 0, BS1 = 0;
};

struct FusionResult {
  std::vector<std::unique_ptr<Group>> groups;   // topological order
};

// `order`: every node to evaluate, in id (= topological) order.
// `targets`: nodes whose values the caller needs after evaluation.
FusionResult fuse(const std::vector<Node *> &order, const std::set<Node *> &targets, bool enable_fusion = true);

}  // namespace mapb

// Kernel generation and execution for the Radiating (viewshed-style radial
// scans) and Spreading (flow accumulation) skeletons.
#include "codegen.hpp"
#include "executor.hpp"

#include <functional>
#include <unordered_map>

namespace mapb {

std::string codegen_scan(const Group &g, KernelPlan &plan) {
  (void)plan;
  throw MapError(std::string(skeleton_name(g.skeleton)) + " groups are not supported by this build yet");
}

void run_scan_group(const Group &g, const KernelPlan &P, std::unordered_map<Node *, DevRaster> &bufs,
                    const std::function<DevRaster &(Node *)> &get, const std::function<DevRaster(Node *)> &alloc_out) {
  (void)P; (void)bufs; (void)get; (void)alloc_out;
  throw MapError(std::string(skeleton_name(g.skeleton)) + " groups are not supported by this build yet");
}

}  // namespace mapb

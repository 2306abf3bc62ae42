// Serving: a request loop over a device-resident DEM with continuous batching.
//
// Requests name a program (hillshade, slope, viewshed, D8 flow + accumulation)
// and a window of the resident DEM. A dispatcher thread admits waiting
// requests while their memory fits the HBM budget (window copy, outputs,
// scratch), builds each request's program on the IR (compiled code is shared:
// every program kind compiles once), and enqueues the whole admitted set as one
// batch on one of two streams:
//   * Local / Focal groups of all requests: one persistent launch over a
//     (kind, request, tile) work-list (the batch dispatcher);
//   * radial scans: one launch, 8 CTAs per request;
//   * flow accumulations: one launch, one CTA per request, after the D8 groups.
// Requests that arrive while a batch runs are admitted into the next batch as
// soon as memory frees up, and the next batch's work overlaps the running one
// on the other stream (continuous batching). A completion thread retires
// batches in order, stamps each request's completion time and frees memory.
// A window is an independent raster (border rule applied at the window edge),
// so a request's result does not depend on what it was batched with.
#pragma once

#include "graph.hpp"

#include <cstddef>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace mapb {

enum RequestType : int { REQ_HILLSHADE = 0, REQ_SLOPE = 1, REQ_VIEWSHED = 2, REQ_FLOW = 3 };

struct ServerStats;

class Server {
 public:
  Server(void *dem, long long pitch, int W, int H, size_t budget_bytes, int max_batch);
  ~Server();
  // Returns the request id; the request runs asynchronously.
  long long submit(int type, int x0, int y0, int w, int h, int obs_x, int obs_y, float obs_h, double radius,
                   bool auto_release);
  // Waits for completion (timeout in seconds, <0 forever); 0 done, 1 timeout.
  int wait(long long id, double timeout_s);
  // Copies the result (F32 for hillshade/slope/viewshed, S32 for flow) to host memory and releases it.
  void result(long long id, void *dst, size_t bytes);
  void release(long long id);
  double latency_ms(long long id);
  std::string stats_json();
  // Open-loop load: Poisson arrivals at `rate` requests/s for `seconds`, program
  // mix weights mix[4], windows 256^2 / 512^2 / 1024^2 uniformly, offsets and
  // observers uniform; returns latency percentiles and throughput as JSON.
  std::string run_load(double rate, double seconds, const double *mix, unsigned seed, double obs_h, double radius);
  // Closed-loop load: `outstanding` requests are kept in flight for `seconds`
  // (each completion is replaced at once by a new request of the same mix).
  std::string run_closed(int outstanding, double seconds, const double *mix, unsigned seed, double obs_h, double radius);

 private:
  std::string load_report(const std::vector<long long> &ids, const std::vector<int> &types, const std::vector<int> &wsz,
                          double t0, double t_end, long long cells, long long batches0, long long batched0,
                          const std::string &head);
  struct Impl;
  std::unique_ptr<Impl> impl_;
};

}  // namespace mapb

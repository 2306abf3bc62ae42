// Per-zone statistics of a float32 value raster over an int32 zone raster
// (count / min / max / sum / mean per zone); see zonestats.cu for the rules.
#pragma once

#include "types.hpp"

#include <cstddef>

struct CUstream_st;

namespace mapb {

struct ZoneStatsArgs {
  const void *value = nullptr;   // device, float32, row-major with value_pitch bytes per row
  long long value_pitch = 0;
  const void *zone = nullptr;    // device, int32, row-major with zone_pitch bytes per row
  long long zone_pitch = 0;
  int W = 0, H = 0;
  int nzones = 0;
  // device output arrays of nzones elements; any may be null
  unsigned long long *count = nullptr;
  float *vmin = nullptr, *vmax = nullptr, *sum = nullptr, *mean = nullptr;
};

// Stream-ordered; allocates its working bins (nzones x 24 bytes) from the
// stream's memory pool and frees them after use.
void zone_stats(const ZoneStatsArgs &a, CUstream_st *stream);

// Same computation without allocating device memory: the working bins are a
// fixed per-device array of 16384 zones, shared by every call on the device
// (overlapping calls race). Runs on the calling thread's current device; the
// first call there does the set-up. See zonestats.cu for who needs it.
void zone_stats_no_alloc(const ZoneStatsArgs &a, CUstream_st *stream);

}  // namespace mapb

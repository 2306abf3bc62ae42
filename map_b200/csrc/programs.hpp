// The reference's example programs built directly on the IR (C++), operator by
// operator in the order the reference scripts create them, so the node graph,
// dtypes and floating-point evaluation order equal those of the Python scripts:
//   hillshade / slope -- python/hill.py:15-50 (dist = 1, zfactor = 1)
//   viewshed          -- python/view.py:18-31 and front/Raster.cpp:558-569
//   flow              -- D8 directions (front/Raster.cpp:485-557) + flow
//                        accumulation of ones (front/Raster.cpp:571-579)
#pragma once

#include "graph.hpp"

namespace mapb {

Node *prog_slope(Runtime &rt, Node *dem);
Node *prog_aspect(Runtime &rt, Node *dem);
Node *prog_hillshade(Runtime &rt, Node *dem, double zenith = 45.0, double azimuth = 315.0);
// The observer's coordinates and height are kernel arguments (ox_out, oy_out,
// oh_out receive their nodes), so every observer shares one kernel.
Node *prog_viewshed(Runtime &rt, Node *dem, int obs_x, int obs_y, float obs_h, double radius, Node **ox_out = nullptr,
                    Node **oy_out = nullptr, Node **oh_out = nullptr);
Node *prog_flow(Runtime &rt, Node *dem, Node **dirs_out = nullptr);

}  // namespace mapb

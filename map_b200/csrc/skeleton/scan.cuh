// Device building blocks of the Radiating and Spreading skeletons.
#pragma once
#include "map_common.cuh"

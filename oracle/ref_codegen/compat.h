// Forced-include compatibility header for compiling the reference's runtime
// sources with a current GCC / libstdc++ (TEST INFRASTRUCTURE ONLY): the
// headers the sources use without including them, on top of the util/ shim.
#pragma once
#include "../ref_util/compat.h"
#include <cmath>
#include <functional>
#include <algorithm>
#include <string>

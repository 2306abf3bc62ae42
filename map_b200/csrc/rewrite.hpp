// Algebraic rewrite of the hillshade composition at code generation.
//
// python/hill.py:15-50 evaluates, per cell,
//   hs = cz * cos(s) + sz * sin(s) * cos(ar - aspect)
//   s = atan(k * sqrt(x*x + y*y)),  aspect = atan2(y, -x) wrapped to [0, 2 PI')
// with x == 0 handled by its own branch (PI' = the script's 3.141593). The
// identities cos(atan t) = 1 / sqrt(1 + t^2), sin(atan t) = t / sqrt(1 + t^2),
// cos(a - atan2(y, -x)) = (y sin a - x cos a) / sqrt(x^2 + y^2) and
// cos(a - b - 2 PI') = cos((a - (2 PI' - 2 PI)) - b) turn it into
//   hs = (cz + sz k (y S - x C)) / sqrt(1 + k^2 (x^2 + y^2))
// where (S, C) = (sin a', cos a') with a' = ar, or ar - (2 PI' - 2 PI) where the
// script's atan2 is negative and wraps; for x == 0 the script's constant angles
// PI'/2 and 3 PI'/2 give S = cos(ar - PI'/2) (y > 0) or -cos(ar - 3 PI'/2)
// (y < 0). The script's inexact PI therefore enters exactly as the constants
// the reference chain uses, not as an approximation of pi.
//
// The matcher below recognises that composition in a fusion group's IR (any
// operand order of the commutative operators, any constants cz, sz, ar, k > 0
// and wrap constants within 1e-5 of 2 pi, pi / 2 and 3 pi / 2) and reports the
// constants of the rewritten form. Cells whose x^2 + y^2 is not finite run the
// literal chain instead (the generated code keeps it in a separate function).
#pragma once

#include "graph.hpp"

#include <functional>
#include <set>
#include <vector>

namespace mapb {

struct ShadeMatch {
  Node *hs = nullptr;          // the node whose value the rewrite computes
  Node *x = nullptr, *y = nullptr;
  std::vector<Node *> pattern; // every node of the composition except x, y and constants, id order
  // constants of the rewritten form (float32 values)
  float cz = 0, szk = 0, kk = 1;
  float S0 = 0, C0 = 0;        // x != 0, atan2 >= 0: sin(ar), cos(ar)
  float S1 = 0, C1 = 0;        // x != 0, atan2 < 0:  sin(ar - d), cos(ar - d), d = 2 PI' - 2 pi
  float SH = 0, S3 = 0;        // x == 0: cos(ar - PI'/2) (y > 0), -cos(ar - 3 PI'/2) (y < 0)
  bool k_one = true;           // k == 1: 1 + q without the multiply
};

// `lit(n, v)`: whether n is a constant whose value (as generated code sees it) is v.
// `member(n)`: whether n is computed by the group.
bool match_shade(Node *hs, const std::function<bool(Node *, double &)> &lit,
                 const std::function<bool(Node *)> &member, ShadeMatch &m);

}  // namespace mapb

// A C++ client of the front end (include/map_b200.hpp) that writes the reference
// scripts' programs the way a C++ user of front/Raster.hpp would:
//   frontend_programs source W H            prints the generated kernels of hillshade
//   frontend_programs eval in.f32 W H out   hillshade, viewshed, D8 + flow accumulation
// The tests compare both against the Python module on the same inputs.
#include "map_b200.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace map;

static const double PI = 3.141593;   // the constant the reference scripts use

// python/hill.py:15-50, operator by operator. Each node is made in its own
// statement, in the script's left-to-right order: C++ leaves the order in which
// an expression's operands are evaluated unspecified, and the order nodes are
// created in is the order statements appear in the generated kernels.
static Raster hori(const Raster &dem) {
  Raster c = convolve(dem, Mask({3, 3}, {-1, 0, 1, -2, 0, 2, -1, 0, 1}));
  return c / 8;
}
static Raster vert(const Raster &dem) {
  Raster c = convolve(dem, Mask({3, 3}, {-1, -2, -1, 0, 0, 0, 1, 2, 1}));
  return c / 8;
}
static Raster slope(const Raster &dem) {
  Raster x = hori(dem);
  Raster y = vert(dem);
  Raster xx = x * x;
  Raster yy = y * y;
  Raster r = sqrt(xx + yy);
  return atan(1 * r);
}
static Raster aspect(const Raster &dem) {
  Raster x = hori(dem);
  Raster y = vert(dem);
  Raster nz = x != 0;
  Raster nx = -x;
  Raster at = atan2(y, nx);
  Raster z1 = nz * at;
  Raster neg = z1 < 0;
  Raster wrap = neg * Variant((float)(PI * 2));
  z1 = z1 + wrap;
  Raster zx = x == 0;
  Raster up = y > 0;
  Raster a = up * Variant((float)(PI / 2));
  Raster down = y < 0;
  Raster b = down * Variant((float)(PI * 2 - PI / 2));
  Raster z0 = zx * (a + b);
  return z1 + z0;
}
static Raster hillshade(const Raster &dem) {
  const double zr = (90 - 45.0) / 180 * PI;
  double ar = 360 - 315.0 + 90;
  ar = ar > 360 ? ar - 360 : ar;
  ar = ar / 180 * PI;
  Raster c1 = cos(slope(dem));
  Raster t1 = Variant((float)std::cos(zr)) * c1;
  Raster s2 = sin(slope(dem));
  Raster t2 = Variant((float)std::sin(zr)) * s2;
  Raster d = Variant((float)ar) - aspect(dem);
  Raster t3 = t2 * cos(d);
  return t1 + t3;
}

int main(int argc, char **argv) {
  try {
    if (argc >= 4 && std::string(argv[1]) == "source") {
      const int W = std::atoi(argv[2]), H = std::atoi(argv[3]);
      std::vector<float> dem((size_t)W * H, 0.0f);
      Raster d = fromHost(dem.data(), {W, H}, F32, {W, H});
      Raster hs = hillshade(d);
      ma_Node *n = hs.node;
      std::vector<char> buf(ma_generatedSource(&n, 1, nullptr, 0) + 1);
      ma_generatedSource(&n, 1, buf.data(), buf.size());
      std::fputs(buf.data(), stdout);
      return 0;
    }
    if (argc >= 2 && std::string(argv[1]) == "loop") {
      // a scalar loop with its carried rasters materialised every iteration
      Raster x = zeros(DataSize(), S32);
      int k = 0;
      while (truth(x < Variant((int32_t)10))) {
        x = x + Variant((int32_t)3);
        materialize({&x});
        k++;
      }
      std::printf("%d %d %d\n", (int)value(x).get(), k, ma_nodeCount());
      return 0;
    }
    if (argc >= 6 && std::string(argv[1]) == "eval") {
      const int W = std::atoi(argv[3]), H = std::atoi(argv[4]);
      const size_t n = (size_t)W * H;
      std::vector<float> dem(n);
      FILE *f = std::fopen(argv[2], "rb");
      if (!f || std::fread(dem.data(), 4, n, f) != n) return 2;
      std::fclose(f);
      Raster d = fromHost(dem.data(), {W, H}, F32, {W, H});
      std::vector<float> hs(n), vs(n);
      std::vector<int32_t> acc(n);
      toHost(hillshade(d), hs.data(), n * 4);
      toHost(viewshed(d, {W / 3, H / 2}, 10.0f), vs.data(), n * 4);
      Raster dirs = flowDirection(d);
      toHost(flowAccumulation(ones_like(d, S32), dirs), acc.data(), n * 4);
      FILE *o = std::fopen(argv[5], "wb");
      if (!o) return 2;
      std::fwrite(hs.data(), 4, n, o);
      std::fwrite(vs.data(), 4, n, o);
      std::fwrite(acc.data(), 4, n, o);
      std::fclose(o);
      return 0;
    }
  } catch (const Error &e) {
    std::fprintf(stderr, "map error: %s\n", e.what());
    return 3;
  }
  std::fprintf(stderr, "usage: frontend_programs source W H | eval in.f32 W H out | loop\n");
  return 1;
}

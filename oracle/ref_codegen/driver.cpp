// Driver of the reference's runtime for the kernel dump (TEST INFRASTRUCTURE
// ONLY). Builds the programs of the reference's example scripts through the
// reference's own C ABI (front/bindings.hpp), creating scalar constants the way
// its Python bindings do (python/map.py: a Python float becomes an F32 Variant,
// an int an S32 one), and evaluates them with ma_write, which makes the
// reference fuse, generate and print its OpenCL kernels (the stand-in OpenCL of
// stubs.cpp runs nothing).
//
// usage: ref_codegen hill|life|wsum|stats|view|percent <work dir>
//        ref_codegen binwrite <path> <W> <H> <BS> <dtype>
//        ref_codegen binread <path> <out>
#include "front/bindings.hpp"
#include "util/util.hpp"
#include "file/File.hpp"
#include "file/binary.hpp"
#include "runtime/Block.hpp"
#include "runtime/Entry.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

using namespace map::detail;

namespace {

Node *fconst(double v) {   // Variant(float) (python/map.py:113-115)
  VariantType var((float)v);
  return ma_constant(var, DataSize(), F32, ROW + BLK, BlockSize());
}
Node *iconst(int v) {      // Variant(int) (python/map.py:119-121)
  VariantType var((int32_t)v);
  return ma_constant(var, DataSize(), S32, ROW + BLK, BlockSize());
}
Node *bin(Node *l, Node *r, BinaryEnum op) { return ma_binary(l, r, op); }
Node *un(Node *a, UnaryEnum op) { return ma_unary(a, op); }

Node *convolve(Node *a, const std::vector<int> &m, int side) {
  std::vector<VariantType> v;
  for (int x : m) v.push_back(VariantType((int32_t)x));   // convolve(raster, list of ints)
  return ma_convolution(a, v.data(), (int)v.size(), DataSize{side, side});
}

void write_bin(const std::string &path, int w, int h, int bs, DataTypeEnum dt) {
  // a zero raster of the given shape in the reference's .bin layout is written
  // by the reference itself: zeros -> write
  VariantType zero = VariantType(0).convert(DataType(dt));
  Node *z = ma_constant(zero, DataSize{w, h}, dt, ROW + BLK, BlockSize{bs, bs});
  ma_increaseRef(z);
  ma_write(z, path.c_str());
  ma_decreaseRef(z);
}

// python/hill.py:15-54
Node *hill(Node *dem) {
  const double PI = 3.141593;
  auto hori = [&](Node *d) {
    return bin(convolve(d, {-1, 0, 1, -2, 0, 2, -1, 0, 1}, 3), iconst(8 * 1), DIV);
  };
  auto vert = [&](Node *d) {
    return bin(convolve(d, {-1, -2, -1, 0, 0, 0, 1, 2, 1}, 3), iconst(8 * 1), DIV);
  };
  auto slope = [&](Node *d) {
    Node *x = hori(d), *y = vert(d);
    return un(bin(iconst(1), un(bin(bin(x, x, MUL), bin(y, y, MUL), ADD), SQRT), MUL), ATAN);
  };
  auto aspect = [&](Node *d) {
    Node *x = hori(d), *y = vert(d);
    Node *z1 = bin(bin(x, iconst(0), NE), ma_binary(y, un(x, NEG), ATAN2), MUL);
    z1 = bin(z1, bin(bin(z1, iconst(0), LT), fconst(PI * 2), MUL), ADD);
    Node *z0 = bin(bin(x, iconst(0), EQ),
                   bin(bin(bin(y, iconst(0), GT), fconst(PI / 2), MUL), bin(bin(y, iconst(0), LT), fconst(PI * 2 - PI / 2), MUL), ADD),
                   MUL);
    return bin(z1, z0, ADD);
  };
  const double zr = (90 - 45.0) / 180 * PI;
  double ar = 360 - 315.0 + 90;
  ar = ar > 360 ? ar - 360 : ar;
  ar = ar / 180 * PI;
  Node *a = bin(fconst(std::cos(zr)), un(slope(dem), COS), MUL);
  Node *b = bin(bin(fconst(std::sin(zr)), un(slope(dem), SIN), MUL), un(bin(fconst(ar), aspect(dem), SUB), COS), MUL);
  return bin(a, b, ADD);
}

// .bin files through the reference's own File<binary> (file/binary.cpp):
// bin_write creates a W x H raster of dtype dt (F32, U8 or S32) in BS x BS
// blocks whose cell (x, y) holds pattern(x, y), block by block with writeBlock
// (cells of edge blocks beyond the raster hold pattern of their padded
// coordinate); bin_read reads a file block by block with readBlock and writes
// its cells as dense row-major bytes to `out`.
double pattern(int x, int y) { return (double)((x * 7 + y * 13) % 251) + 0.25 * (x % 4); }

int bin_write(const std::string &path, int W, int H, int BS, int dt) {
  MetaData meta(DataSize{W, H}, DataType((DataTypeEnum)dt), MemOrder(ROW + BLK), BlockSize{BS, BS});
  File<binary> f(meta);
  f.open(path, OUT);
  const int es = DataType((DataTypeEnum)dt).sizeOf();
  std::vector<char> buf((size_t)BS * BS * es);
  Entry entry(nullptr);
  entry.host_mem = buf.data();
  for (int by = 0; by * BS < H; by++)
    for (int bx = 0; bx * BS < W; bx++) {
      for (int j = 0; j < BS; j++)
        for (int i = 0; i < BS; i++) {
          const double v = pattern(bx * BS + i, by * BS + j);
          char *c = buf.data() + ((size_t)j * BS + i) * es;
          if (dt == F32) { float t = (float)v; std::memcpy(c, &t, 4); }
          else if (dt == S32) { int32_t t = (int32_t)v; std::memcpy(c, &t, 4); }
          else { uint8_t t = (uint8_t)v; std::memcpy(c, &t, 1); }
        }
      Block blk(Key(nullptr, Coord{bx, by}));
      blk.entry = &entry;
      f.writeBlock(blk);
      blk.entry = nullptr;
    }
  f.close();
  return 0;
}

int bin_read(const std::string &path, const std::string &out) {
  File<binary> f;
  f.open(path, IN);
  const DataSize ds = f.getDataSize();
  const BlockSize bs = f.getBlockSize();
  const int es = f.getDataType().sizeOf();
  const int W = ds[0], H = ds[1];
  std::vector<char> buf((size_t)bs[0] * bs[1] * es), dense((size_t)W * H * es);
  Entry entry(nullptr);
  entry.host_mem = buf.data();
  for (int by = 0; by * bs[1] < H; by++)
    for (int bx = 0; bx * bs[0] < W; bx++) {
      Block blk(Key(nullptr, Coord{bx, by}));
      blk.entry = &entry;
      f.readBlock(blk);
      blk.entry = nullptr;
      for (int j = 0; j < bs[1] && by * bs[1] + j < H; j++)
        for (int i = 0; i < bs[0] && bx * bs[0] + i < W; i++)
          std::memcpy(dense.data() + ((size_t)(by * bs[1] + j) * W + bx * bs[0] + i) * es,
                      buf.data() + ((size_t)j * bs[0] + i) * es, es);
    }
  f.close();
  FILE *o = std::fopen(out.c_str(), "wb");
  if (!o) return 1;
  std::fprintf(o, "%d %d %d %d %d %d\n", (int)f.getDataType().get(), W, H, (int)f.getMemOrder().get(), bs[0], bs[1]);
  std::fwrite(dense.data(), 1, dense.size(), o);
  std::fclose(o);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc >= 7 && std::string(argv[1]) == "binwrite")
    return bin_write(argv[2], std::atoi(argv[3]), std::atoi(argv[4]), std::atoi(argv[5]), std::atoi(argv[6]));
  if (argc >= 4 && std::string(argv[1]) == "binread") return bin_read(argv[2], argv[3]);
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s hill|life|wsum|stats|view|percent <work dir>\n", argv[0]);
    return 2;
  }
  const std::string what = argv[1], dir = argv[2];
  ma_setupDevices("", DEV_GPU, "");
  Node *out = nullptr;
  if (what == "hill") {
    write_bin(dir + "/dem.bin", 512, 512, 256, F32);
    Node *dem = ma_read((dir + "/dem.bin").c_str());
    out = hill(dem);
  } else if (what == "life") {
    // python/life.py:24-34, two generations of a rand(N, ds, U8, ROW+BLK, bs) > 128 state
    VariantType seed = VariantType((int32_t)16).convert(DataType(U8));
    Node *s = ma_constant(seed, DataSize{512, 512}, U8, ROW + BLK, BlockSize{256, 256});
    Node *state = bin(ma_rand(s, U8, ROW + BLK), iconst(128), GT);
    for (int g = 0; g < 2; g++) {
      Node *nbh = convolve(state, {1, 1, 1, 1, 0, 1, 1, 1, 1}, 3);
      state = bin(bin(nbh, iconst(3), EQ), bin(bin(nbh, iconst(2), EQ), state, MUL), ADD);
    }
    out = state;
  } else if (what == "wsum") {
    // python/wsum.py:11
    Node *r[4];
    for (int i = 0; i < 4; i++) write_bin(dir + "/r" + std::to_string(i) + ".bin", 512, 512, 256, F32);
    for (int i = 0; i < 4; i++) r[i] = ma_read((dir + "/r" + std::to_string(i) + ".bin").c_str());
    Node *o = bin(iconst(0), bin(fconst(0.1), r[0], MUL), ADD);
    o = bin(o, bin(r[1], fconst(0.2), MUL), ADD);
    o = bin(o, bin(fconst(0.3), r[2], MUL), ADD);
    o = bin(o, bin(r[3], fconst(0.4), MUL), ADD);
    out = bin(o, iconst(0), ADD);
  } else if (what == "stats") {
    // python/stats.py:12-35 (N = prod(datasize) is a Python int, 1.0/N a float)
    write_bin(dir + "/dem.bin", 512, 512, 256, F32);
    Node *dem = ma_read((dir + "/dem.bin").c_str());
    const int N = 512 * 512;
    Node *maxv = ma_zonalReduc(dem, MAX), *minv = ma_zonalReduc(dem, MIN);
    Node *rang = bin(maxv, minv, SUB);
    Node *mean = bin(ma_zonalReduc(dem, SUM), iconst(N), DIV);
    Node *geom = bin(ma_zonalReduc(dem, PROD), fconst(1.0 / N), POW);
    Node *harm = bin(iconst(N), ma_zonalReduc(bin(fconst(1.0), dem, DIV), SUM), DIV);
    Node *quam = un(bin(ma_zonalReduc(bin(dem, iconst(2), POW), SUM), iconst(N), DIV), SQRT);
    Node *cubm = un(bin(ma_zonalReduc(bin(dem, iconst(3), POW), SUM), iconst(N), DIV), CBRT);
    Node *dev = bin(bin(dem, mean, SUB), iconst(2), POW);
    Node *std_ = un(bin(ma_zonalReduc(dev, SUM), iconst(N), DIV), SQRT);
    Node *norm = bin(bin(dev, minv, SUB), rang, DIV);
    Node *nstd = un(bin(ma_zonalReduc(norm, SUM), iconst(N), DIV), SQRT);
    Node *all[] = {maxv, minv, rang, mean, geom, harm, quam, cubm, std_, nstd};
    for (Node *n : all) ma_increaseRef(n);
    std::fflush(stdout);
    ma_eval(all, 10);
    std::fflush(stdout);
    for (Node *n : all) ma_decreaseRef(n);
    return 0;
  } else if (what == "percent") {
    // FocalPercent (front/Raster.cpp:438-447): percentage (AGE) and percentile
    // (ILE) of an F32 raster over a 3 x 3 window, summed into one output
    write_bin(dir + "/dem.bin", 512, 512, 256, F32);
    Node *dem = ma_read((dir + "/dem.bin").c_str());
    std::vector<VariantType> m(9, VariantType(1.0f));
    Node *age = ma_focalPercent(dem, m.data(), 9, DataSize{3, 3}, AGE);
    Node *ile = ma_focalPercent(dem, m.data(), 9, DataSize{3, 3}, ILE);
    out = bin(age, ile, ADD);
  } else if (what == "view") {
    // python/view.py:17-43 with observer (100, 150) and h = 10.0
    write_bin(dir + "/dem.bin", 512, 512, 256, F32);
    Node *dem = ma_read((dir + "/dem.bin").c_str());
    Node *norm = bin(bin(dem, ma_zonalReduc(dem, MIN), SUB),
                     bin(ma_zonalReduc(dem, MAX), ma_zonalReduc(dem, MIN), SUB), DIV);
    const int ox = 100, oy = 150;
    const double h = 10.0;
    Node *shift = bin(norm, fconst(h), SUB);
    Node *x = bin(iconst(ox), ma_index(norm, D1), SUB);
    Node *y = bin(iconst(oy), ma_index(norm, D2), SUB);
    Node *dist = un(bin(bin(bin(x, x, MUL), bin(y, y, MUL), ADD), fconst(0.0), ADD), SQRT);
    Node *slope = bin(shift, dist, DIV);
    Node *maxr = ma_radialScan(slope, MAX, Coord{ox, oy});
    Node *view = bin(bin(bin(maxr, dist, MUL), fconst(h), ADD), norm, SUB);
    std::vector<VariantType> f;
    for (double v : {1.0 / 16, 1.0 / 8, 1.0 / 16, 1.0 / 8, 1.0 / 4, 1.0 / 8, 1.0 / 16, 1.0 / 8, 1.0 / 16})
      f.push_back(VariantType((float)v));
    Node *soft = ma_convolution(view, f.data(), 9, DataSize{3, 3});
    VariantType zero = VariantType(0.0f);
    Node *zeros = ma_constant(zero, DataSize{512, 512}, F32, ROW + BLK, BlockSize{256, 256});
    out = ma_conditional(bin(soft, fconst(0.1), LT), dem, zeros);
  } else {
    std::fprintf(stderr, "unknown program %s\n", what.c_str());
    return 2;
  }
  ma_increaseRef(out);
  std::fflush(stdout);
  const int rc = ma_write(out, (dir + "/out.bin").c_str());
  ma_decreaseRef(out);
  return rc;
}

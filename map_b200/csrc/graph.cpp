// Node factories, hash-consing and garbage collection.
#include "graph.hpp"
#include "binfile.hpp"

#include <algorithm>
#include <cstdlib>
#include <functional>
#include <unordered_set>

namespace mapb {

const char *kind_name(int k) {
  static const char *n[] = {"Constant", "Read", "HostInput", "DeviceInput", "Index", "Rand", "Cast", "Unary", "Binary",
                            "Conditional", "Neighbor", "Convolution", "FocalFunc", "FocalFlow", "ZonalReduc",
                            "RadialScan", "SpreadScan", "Write", "Barrier", "FocalPercent"};
  return (k >= 0 && k <= K_FOCALPERCENT) ? n[k] : "?";
}

std::string arr_str(const Arr2 &a) {
  return "[" + std::to_string(a.arr[0]) + "," + std::to_string(a.arr[1]) + "/" + std::to_string(a.n) + "]";
}

int Node::halo_x() const {
  switch (kind) {
    case K_CONVOLUTION: case K_FOCALFUNC: case K_FOCALPERCENT: return mask_ds.arr[0] / 2;   // Convolution.cpp:85 (size/2)
    case K_NEIGHBOR: return std::abs(coord.arr[0]);                     // Neighbor.cpp:86
    case K_FOCALFLOW: return 1;                                         // FocalFlow.cpp:75
    default: return 0;
  }
}
int Node::halo_y() const {
  switch (kind) {
    case K_CONVOLUTION: case K_FOCALFUNC: case K_FOCALPERCENT: return mask_ds.arr[1] / 2;
    case K_NEIGHBOR: return std::abs(coord.arr[1]);
    case K_FOCALFLOW: return 1;
    default: return 0;
  }
}

Runtime &Runtime::get() {
  static Runtime rt;
  return rt;
}

static Arr2 d0_size() { return Arr2{{-1, -1}, 0}; }

static bool same_arr(const Arr2 &a, const Arr2 &b) {
  if (a.n != b.n) return false;
  for (int i = 0; i < a.n; i++) if (a.arr[i] != b.arr[i]) return false;
  return true;
}

static std::string meta_key(const Meta &m) {
  return std::to_string(m.dtype) + ":" + std::to_string(m.numdim) + ":" + std::to_string(m.memorder) + ":" +
         arr_str(m.ds) + ":" + arr_str(m.bs);
}

static std::string var_key(const Variant &v) {
  uint64_t bits = 0;
  std::memcpy(&bits, &v.u, dt_size(v.dtype));
  return std::to_string(v.dtype) + "#" + std::to_string(bits);
}

static std::string pid(const Node *n) { return "#" + std::to_string(n->id); }

Node *Runtime::add(std::unique_ptr<Node> n, const std::string &key) {
  std::lock_guard<std::recursive_mutex> lk(mtx);
  if (!key.empty()) {
    auto it = cse.find(key);
    if (it != cse.end()) return it->second;   // hash-consing: equal node already exists
  }
  n->id = next_id++;
  for (Node *p : n->prev) p->next.push_back(n.get());
  Node *raw = n.get();
  live_set.insert(raw);
  nodes.push_back(std::move(n));
  if (!key.empty()) cse[key] = raw;
  return raw;
}

bool Runtime::owns(const Node *n) const { return live_set.count(n) > 0; }

static void check_node(Node *n, const char *what) {
  if (n == nullptr) throw MapError(std::string(what) + ": null node argument");
}

// Result metadata of an element-wise op over two operands (Binary.cpp:34-60):
// a D0 operand takes the other's shape, otherwise both shapes must agree.
static Meta merge_meta(const Meta &l, const Meta &r) {
  if (l.numdim == D0) return r;
  if (r.numdim == D0) return l;
  if (l.numdim != r.numdim || !same_arr(l.ds, r.ds) || !same_arr(l.bs, r.bs) || l.memorder != r.memorder)
    throw MapError("operands differ in shape: " + arr_str(l.ds) + " vs " + arr_str(r.ds) + ", blocks " + arr_str(l.bs) +
                   " vs " + arr_str(r.bs));
  return l;
}

Node *Runtime::constant(Variant v, Arr2 ds, int dt, int mo, Arr2 bs) {
  if (dt <= NONE_DATATYPE || dt >= N_DATATYPE) throw MapError("constant: invalid data type");
  auto n = std::make_unique<Node>();
  n->kind = K_CONSTANT;
  n->pattern = P_FREE;
  n->meta.dtype = dt;
  n->meta.memorder = mo;
  n->meta.ds = ds.n == 0 ? d0_size() : ds;
  n->meta.numdim = numdim_fromsize(n->meta.ds);
  if (n->meta.numdim == D2) {
    if (ds.arr[0] <= 0 || ds.arr[1] <= 0) throw MapError("constant: invalid data size " + arr_str(ds));
    n->meta.bs = (bs.n == 0) ? default_bs : bs;
  } else if (n->meta.numdim != D0) {
    throw MapError("constant: only D0 and D2 rasters are supported");
  }
  n->cnst = var_convert(v, dt);
  n->has_value = (n->meta.numdim == D0);
  n->value = n->cnst;
  std::string key = "C|" + meta_key(n->meta) + "|" + var_key(n->cnst);
  return add(std::move(n), key);
}

Node *Runtime::scalar_param(Variant v) {
  dt_size(v.dtype);
  auto n = std::make_unique<Node>();
  n->kind = K_CONSTANT;
  n->pattern = P_FREE;
  n->meta.dtype = v.dtype;
  n->meta.numdim = D0;
  n->cnst = v;
  n->as_param = true;
  n->has_value = true;
  n->value = v;
  return add(std::move(n), "P|" + var_key(v));
}

Node *Runtime::read(const std::string &path) {
  if (path.empty()) throw MapError("read: empty path");
  auto n = std::make_unique<Node>();
  n->kind = K_READ;
  n->pattern = P_FREE;
  n->path = path;
  BinHeader h = bin_read_header(path);
  n->meta.dtype = h.dtype;
  n->meta.numdim = D2;
  n->meta.memorder = h.memorder;
  n->meta.ds = Arr2{{h.ds0, h.ds1}, 2};
  n->meta.bs = Arr2{{h.bs0, h.bs1}, 2};
  return add(std::move(n), "R|" + path);   // Read.cpp:16-22 keys reads by path
}

Node *Runtime::host_input(const void *ptr, Arr2 ds, int dt, Arr2 bs, bool copy) {
  if (ptr == nullptr) throw MapError("host input: null pointer");
  if (ds.n != 2 || ds.arr[0] <= 0 || ds.arr[1] <= 0) throw MapError("host input: data size must be 2-D and positive");
  auto n = std::make_unique<Node>();
  n->kind = K_HOSTIN;
  n->pattern = P_FREE;
  n->meta.dtype = dt;
  n->meta.numdim = D2;
  n->meta.ds = ds;
  n->meta.bs = (bs.n == 0) ? default_bs : bs;
  dt_size(dt);
  n->host = std::make_shared<HostData>();
  if (copy) {
    size_t bytes = (size_t)ds.arr[0] * ds.arr[1] * dt_size(dt);
    n->host->own.assign((const unsigned char *)ptr, (const unsigned char *)ptr + bytes);
    n->host->ptr = n->host->own.data();
  } else {
    n->host->ptr = ptr;
  }
  return add(std::move(n), "");
}

Node *Runtime::dev_input(void *ptr, long long pitch, Arr2 ds, int dt, Arr2 bs) {
  if (ptr == nullptr) throw MapError("device input: null pointer");
  if (ds.n != 2 || ds.arr[0] <= 0 || ds.arr[1] <= 0) throw MapError("device input: data size must be 2-D and positive");
  if (pitch < (long long)ds.arr[0] * (long long)dt_size(dt)) throw MapError("device input: pitch smaller than a row");
  auto n = std::make_unique<Node>();
  n->kind = K_DEVIN;
  n->pattern = P_FREE;
  n->meta.dtype = dt;
  n->meta.numdim = D2;
  n->meta.ds = ds;
  n->meta.bs = (bs.n == 0) ? default_bs : bs;
  n->dev = std::make_shared<DevData>();
  n->dev->ptr = ptr;
  n->dev->pitch = pitch;
  return add(std::move(n), "");
}

Node *Runtime::dev_input_rows(void *ptr, long long pitch, Arr2 ds, int dt, Arr2 bs, int row0, int rows) {
  if (ds.n != 2 || ds.arr[0] <= 0 || ds.arr[1] <= 0) throw MapError("device input: data size must be 2-D and positive");
  if (row0 < 0 || rows <= 0 || (long long)row0 + rows > (long long)ds.arr[1])
    throw MapError("device row band: rows [" + std::to_string(row0) + ", " + std::to_string((long long)row0 + rows) +
                   ") are not inside the raster's " + std::to_string(ds.arr[1]) + " rows");
  Node *n = dev_input(ptr, pitch, ds, dt, bs);
  n->dev->row0 = row0;
  n->dev->rows = rows;
  return n;
}

Node *Runtime::index(Node *arg, int dim) {
  check_node(arg, "index");
  if (dim != D1 && dim != D2) throw MapError("index: dimension must be D1 or D2");
  if (arg->meta.numdim != D2) throw MapError("index: argument must be a 2-D raster");
  auto n = std::make_unique<Node>();
  n->kind = K_INDEX;
  n->pattern = P_FREE;
  n->op = dim;
  n->meta = arg->meta;
  n->meta.dtype = S64;   // Index.cpp:30
  return add(std::move(n), "I|" + std::to_string(dim) + "|" + meta_key(n->meta));
}

Node *Runtime::rand(Node *seed, int dt, int mo) {
  check_node(seed, "rand");
  if (seed->meta.numdim != D2) throw MapError("rand: seed must be a 2-D raster");
  auto n = std::make_unique<Node>();
  n->kind = K_RAND;
  n->pattern = P_LOCAL;
  n->meta = seed->meta;
  n->meta.dtype = (dt != NONE_DATATYPE) ? dt : seed->meta.dtype;
  n->meta.memorder = (mo != NONE_MEMORDER) ? mo : seed->meta.memorder;
  if (dt_size(n->meta.dtype) > 4) throw MapError("rand: 64-bit output types are not supported");
  n->prev = {seed};
  return add(std::move(n), "RND|" + pid(seed) + "|" + meta_key(n->meta));
}

Node *Runtime::cast(Node *arg, int dt) {
  check_node(arg, "cast");
  if (dt <= NONE_DATATYPE || dt >= N_DATATYPE) throw MapError("cast: invalid data type");
  auto n = std::make_unique<Node>();
  n->kind = K_CAST;
  n->pattern = P_LOCAL;
  n->op = dt;
  n->meta = arg->meta;
  n->meta.dtype = dt;
  n->prev = {arg};
  return add(std::move(n), "CAST|" + std::to_string(dt) + "|" + pid(arg));
}

Node *Runtime::unary(Node *arg, int op) {
  check_node(arg, "unary");
  unary_name(op);
  if (op == bNOT && !dt_is_unsigned(arg->meta.dtype)) throw MapError("bitwise not requires an unsigned type");
  auto n = std::make_unique<Node>();
  n->kind = K_UNARY;
  n->pattern = P_LOCAL;
  n->op = op;
  n->meta = arg->meta;
  if (op == NOT) n->meta.dtype = U8;   // Unary.cpp:41-42
  n->prev = {arg};
  return add(std::move(n), "U|" + std::to_string(op) + "|" + pid(arg));
}

Node *Runtime::binary(Node *l, Node *r, int op) {
  check_node(l, "binary");
  check_node(r, "binary");
  binary_name(op);
  if (binary_is_bitwise(op) && !(dt_is_unsigned(l->meta.dtype) && dt_is_unsigned(r->meta.dtype)))
    throw MapError(std::string("bitwise ") + binary_name(op) + " requires unsigned operands");
  auto n = std::make_unique<Node>();
  n->kind = K_BINARY;
  n->pattern = P_LOCAL;
  n->op = op;
  n->meta = merge_meta(l->meta, r->meta);
  n->meta.dtype = binary_is_relational(op) ? U8 : dt_promote(l->meta.dtype, r->meta.dtype);   // Binary.cpp:54-58
  n->prev = {l, r};
  return add(std::move(n), "B|" + std::to_string(op) + "|" + pid(l) + "|" + pid(r));
}

Node *Runtime::conditional(Node *c, Node *l, Node *r) {
  check_node(c, "conditional");
  check_node(l, "conditional");
  check_node(r, "conditional");
  if (l->meta.dtype != r->meta.dtype)
    throw MapError(std::string("conditional: branches differ in type (") + dt_name(l->meta.dtype) + " vs " +
                   dt_name(r->meta.dtype) + ")");
  auto n = std::make_unique<Node>();
  n->kind = K_CONDITIONAL;
  n->pattern = P_LOCAL;
  n->meta = merge_meta(merge_meta(c->meta, l->meta), r->meta);   // Conditional.cpp Factory
  n->meta.dtype = l->meta.dtype;
  n->prev = {c, l, r};
  return add(std::move(n), "CON|" + pid(c) + "|" + pid(l) + "|" + pid(r));
}

static void check_focal_arg(Node *arg, const char *what) {
  check_node(arg, what);
  if (arg->meta.numdim != D2) throw MapError(std::string(what) + ": argument must be a 2-D raster");
}

Node *Runtime::neighbor(Node *arg, Arr2 coord) {
  check_focal_arg(arg, "neighbor");
  if (coord.n != 2) throw MapError("neighbor: coordinate must have 2 components");
  auto n = std::make_unique<Node>();
  n->kind = K_NEIGHBOR;
  n->pattern = P_FOCAL;
  n->coord = coord;
  n->meta = arg->meta;
  n->prev = {arg};
  if (n->halo_x() > 16 || n->halo_y() > 16) throw MapError("neighbor: offset larger than 16 cells");
  return add(std::move(n), "NB|" + arr_str(coord) + "|" + pid(arg));
}

static std::string mask_key(const std::vector<Variant> &m, const Arr2 &ds) {
  std::string k = arr_str(ds);
  for (auto &v : m) k += "," + var_key(v);
  return k;
}

static void check_mask(const Variant *mask, int n, Arr2 mds, const char *what) {
  if (mask == nullptr || n <= 0) throw MapError(std::string(what) + ": empty mask");
  if (mds.n != 2 || mds.arr[0] <= 0 || mds.arr[1] <= 0 || mds.arr[0] * mds.arr[1] != n)
    throw MapError(std::string(what) + ": mask size does not match its shape");
  if (mds.arr[0] % 2 == 0 || mds.arr[1] % 2 == 0) throw MapError(std::string(what) + ": mask sides must be odd");
  if (mds.arr[0] > 33 || mds.arr[1] > 33) throw MapError(std::string(what) + ": mask larger than 33x33");
  for (int i = 1; i < n; i++)
    if (mask[i].dtype != mask[0].dtype) throw MapError(std::string(what) + ": mask values must share one type");
  dt_size(mask[0].dtype);
}

Node *Runtime::convolution(Node *arg, const Variant *mask, int cnt, Arr2 mds) {
  check_focal_arg(arg, "convolution");
  check_mask(mask, cnt, mds, "convolution");
  auto n = std::make_unique<Node>();
  n->kind = K_CONVOLUTION;
  n->pattern = P_FOCAL;
  n->mask.assign(mask, mask + cnt);
  n->mask_ds = mds;
  n->meta = arg->meta;
  n->meta.dtype = dt_promote(arg->meta.dtype, mask[0].dtype);   // Convolution.cpp:37
  n->prev = {arg};
  return add(std::move(n), "CONV|" + mask_key(n->mask, mds) + "|" + pid(arg));
}

Node *Runtime::focal_func(Node *arg, const Variant *mask, int cnt, Arr2 mds, int red) {
  check_focal_arg(arg, "focalFunc");
  check_mask(mask, cnt, mds, "focalFunc");
  reduction_name(red);
  auto n = std::make_unique<Node>();
  n->kind = K_FOCALFUNC;
  n->pattern = P_FOCAL;
  n->op = red;
  n->mask.assign(mask, mask + cnt);
  n->mask_ds = mds;
  n->meta = arg->meta;   // FocalFunc.cpp: keeps the argument's type
  n->prev = {arg};
  return add(std::move(n), "FF|" + std::to_string(red) + "|" + mask_key(n->mask, mds) + "|" + pid(arg));
}

// FocalPercent (runtime/dag/FocalPercent.cpp Factory, runtime/skeleton/FocalSkeleton.cpp:375-403,
// util/PercentType.cpp): the result keeps the argument's type; the mask gives
// the window's extent only (its values are not read, as in the reference).
Node *Runtime::focal_percent(Node *arg, const Variant *mask, int cnt, Arr2 mds, int type) {
  check_focal_arg(arg, "focalPercent");
  check_mask(mask, cnt, mds, "focalPercent");
  if (type != 1 && type != 2) throw MapError("focalPercent: type must be AGE (1) or ILE (2)");
  auto n = std::make_unique<Node>();
  n->kind = K_FOCALPERCENT;
  n->pattern = P_FOCAL;
  n->op = type;
  n->mask.assign(mask, mask + cnt);
  n->mask_ds = mds;
  n->meta = arg->meta;
  n->prev = {arg};
  return add(std::move(n), "FP|" + std::to_string(type) + "|" + mask_key(n->mask, mds) + "|" + pid(arg));
}

Node *Runtime::focal_flow(Node *arg) {
  check_focal_arg(arg, "focalFlow");
  auto n = std::make_unique<Node>();
  n->kind = K_FOCALFLOW;
  n->pattern = P_FOCAL;
  n->meta = arg->meta;
  n->meta.dtype = U8;   // FocalFlow.cpp Factory
  n->prev = {arg};
  return add(std::move(n), "FLOW|" + pid(arg));
}

Node *Runtime::zonal_reduc(Node *arg, int red) {
  check_node(arg, "zonalReduc");
  if (arg->meta.numdim == D0) throw MapError("zonalReduc: argument must be a raster");
  reduction_name(red);
  if ((red == rAND || red == rOR) && dt_is_float(arg->meta.dtype))
    throw MapError("zonalReduc: bitwise reductions need an integer raster");
  auto n = std::make_unique<Node>();
  n->kind = K_ZONALREDUC;
  n->pattern = P_ZONAL;
  n->op = red;
  n->meta.dtype = arg->meta.dtype;   // ZonalReduc.cpp:34-40: D0 result of the argument's type
  n->meta.memorder = arg->meta.memorder;
  n->meta.numdim = D0;
  n->prev = {arg};
  return add(std::move(n), "Z|" + std::to_string(red) + "|" + pid(arg));
}

Node *Runtime::radial_scan(Node *arg, int red, Arr2 start, double radius) {
  check_focal_arg(arg, "radialScan");
  reduction_name(red);
  if (start.n != 2) throw MapError("radialScan: start must have 2 components");
  if (start.arr[0] < 0 || start.arr[1] < 0 || start.arr[0] >= arg->meta.W() || start.arr[1] >= arg->meta.H())
    throw MapError("radialScan: start " + arr_str(start) + " outside the raster");
  if (!dt_is_float(arg->meta.dtype)) throw MapError("radialScan: the scanned raster must be floating point");
  auto n = std::make_unique<Node>();
  n->kind = K_RADIALSCAN;
  n->pattern = P_RADIAL;
  n->op = red;
  if (radius < 0) throw MapError("radialScan: negative radius");
  n->coord = start;
  n->radius = radius;
  n->meta = arg->meta;
  n->prev = {arg};
  return add(std::move(n), "RAD|" + std::to_string(red) + "|" + arr_str(start) + "|" + std::to_string(radius) + "|" + pid(arg));
}

Node *Runtime::spread_scan(Node *arg, Node *dir, int red) {
  check_node(arg, "spreadScan");
  check_focal_arg(dir, "spreadScan");
  if (dir->meta.dtype != U8) throw MapError("spreadScan: directions must be U8");   // SpreadScan.cpp Factory
  if (arg->meta.numdim != D0 && !same_arr(arg->meta.ds, dir->meta.ds))
    throw MapError("spreadScan: value and direction rasters differ in size");
  if (red != SUM) throw MapError("spreadScan: only SUM is supported");
  auto n = std::make_unique<Node>();
  n->kind = K_SPREADSCAN;
  n->pattern = P_SPREAD;
  n->op = red;
  n->meta = (arg->meta.numdim == D0) ? dir->meta : arg->meta;
  n->meta.dtype = arg->meta.dtype;
  n->prev = {arg, dir};
  return add(std::move(n), "SPR|" + std::to_string(red) + "|" + pid(arg) + "|" + pid(dir));
}

Node *Runtime::barrier(Node *arg) {
  check_node(arg, "barrier");
  auto n = std::make_unique<Node>();
  n->kind = K_BARRIER;
  n->pattern = P_BARRIER;
  n->meta = arg->meta;
  n->prev = {arg};
  return add(std::move(n), "BAR|" + pid(arg));
}

Node *Runtime::write(Node *arg, const std::string &path) {
  check_node(arg, "write");
  if (arg->meta.numdim != D2) throw MapError("write: only 2-D rasters can be written");
  if (path.empty()) throw MapError("write: empty path");
  auto n = std::make_unique<Node>();
  n->kind = K_WRITE;
  n->pattern = P_FREE;
  n->path = path;
  n->meta = arg->meta;
  n->prev = {arg};
  return add(std::move(n), "");
}

// Unlinks every node that no referenced node depends on (the reference drops
// unreferenced nodes at the next evaluation, runtime/Runtime.cpp:380-395).
void Runtime::collect_garbage() {
  std::lock_guard<std::recursive_mutex> lk(mtx);
  std::unordered_set<Node *> live;
  std::vector<Node *> stack;
  for (auto &u : nodes)
    if (u->ref > 0) stack.push_back(u.get());
  while (!stack.empty()) {
    Node *n = stack.back();
    stack.pop_back();
    if (!live.insert(n).second) continue;
    for (Node *p : n->prev) stack.push_back(p);
  }
  if (live.size() == nodes.size()) return;
  for (auto it = cse.begin(); it != cse.end();) {
    if (!live.count(it->second)) it = cse.erase(it);
    else ++it;
  }
  for (auto &u : nodes) {
    if (!live.count(u.get())) continue;
    auto &nx = u->next;
    nx.erase(std::remove_if(nx.begin(), nx.end(), [&](Node *m) { return !live.count(m); }), nx.end());
  }
  for (auto &u : nodes)
    if (!live.count(u.get())) live_set.erase(u.get());
  nodes.erase(std::remove_if(nodes.begin(), nodes.end(), [&](const std::unique_ptr<Node> &u) { return !live.count(u.get()); }),
              nodes.end());
  epoch++;
}

void Runtime::reset() {
  std::lock_guard<std::recursive_mutex> lk(mtx);
  epoch++;
  cse.clear();
  live_set.clear();
  nodes.clear();
}

}  // namespace mapb

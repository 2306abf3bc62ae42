// Map-algebra IR: nodes, their factories (metadata and type rules), hash-consing
// of structurally equal nodes, reference counting and garbage collection.
//
// Factories restate the metadata rules of the reference's node classes
// (runtime/dag/*.cpp, Factory functions); hash-consing restates the online
// simplifier (runtime/visitor/SimplifierOnline.tpl:13-37): creating a node equal
// to an existing one returns the existing node.
#pragma once

#include "types.hpp"

#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace mapb {

enum NodeKind : int {
  K_CONSTANT, K_READ, K_HOSTIN, K_DEVIN, K_INDEX, K_RAND, K_CAST, K_UNARY, K_BINARY, K_CONDITIONAL,
  K_NEIGHBOR, K_CONVOLUTION, K_FOCALFUNC, K_FOCALFLOW, K_ZONALREDUC, K_RADIALSCAN, K_SPREADSCAN,
  K_WRITE, K_BARRIER, K_FOCALPERCENT
};

const char *kind_name(int k);

struct Meta {
  int dtype = NONE_DATATYPE;
  int numdim = D0;
  int memorder = ROW + BLK;
  Arr2 ds{{-1, -1}, 0};   // data size (cells); ds.arr[0] = width (x), ds.arr[1] = height (y)
  Arr2 bs{{-1, -1}, 0};   // block size
  int W() const { return ds.arr[0]; }
  int H() const { return ds.arr[1]; }
  int BS0() const { return bs.arr[0]; }
  int BS1() const { return bs.arr[1]; }
  bool is_d0() const { return numdim == D0; }
};

// Host-provided raster data attached to an input node.
struct HostData {
  const void *ptr = nullptr;      // caller-owned host memory, row-major, dense
  std::vector<unsigned char> own; // owned copy (file reads)
};

struct DevData {
  void *ptr = nullptr;    // device memory (address of raster row `row0`), caller-owned unless `owned`
  long long pitch = 0;    // bytes between rows
  // Row band: the memory holds raster rows row0 .. row0 + rows - 1 only
  // (rows == 0: the whole raster). Such an input is evaluated by row ranges
  // (Executor::evaluate_rows) that read no row outside the band.
  int row0 = 0, rows = 0;
  // The library allocated the memory (Executor::materialize) and frees it,
  // stream-ordered, with the last node that holds it.
  bool owned = false;
  DevData() = default;
  DevData(const DevData &) = delete;
  DevData &operator=(const DevData &) = delete;
  ~DevData();
};

struct Node {
  int id = 0;
  int kind = K_CONSTANT;
  int pattern = P_FREE;
  Meta meta;
  std::vector<Node *> prev;
  std::vector<Node *> next;
  int ref = 0;

  // parameters
  int op = 0;                  // unary/binary/reduction op; index dim; cast target
  Variant cnst{};              // constant value
  std::vector<Variant> mask;   // focal mask, row-major (mask_ds.arr[0] columns)
  Arr2 mask_ds{{-1, -1}, 0};
  Arr2 coord{{0, 0}, 2};       // neighbour offset / radial start
  double radius = 0;           // radial scan: fronts farther than this are not swept (0 = all)
  bool as_param = false;       // scalar constant passed to kernels as an argument, not written into their source
  std::string path;            // read / write path
  std::shared_ptr<HostData> host;
  std::shared_ptr<DevData> dev;

  // evaluation state
  bool has_value = false;  // D0 value known on the host
  Variant value{};

  int halo_x() const;
  int halo_y() const;
  bool is_input() const { return kind == K_READ || kind == K_HOSTIN || kind == K_DEVIN; }
};

struct Runtime {
  static Runtime &get();

  std::recursive_mutex mtx;
  std::vector<std::unique_ptr<Node>> nodes;
  std::unordered_map<std::string, Node *> cse;
  std::unordered_set<const Node *> live_set;   // fast ownership test of node handles
  int next_id = 0;

  // configuration
  int border = BORDER_BLOCK_MIRROR;
  int exec_mode = EXEC_FUSED;
  // Row bands of streamed evaluations (host rasters in, host rasters out):
  // 0 automatic, < 0 never stream, > 0 stream whenever a raster has more rows.
  int stream_rows = 0;
  // Focal groups of float math compute two cells per thread step on packed
  // f32x2 instructions (bit-identical to one cell at a time); 0 turns it off.
  int paired_cells = 1;
  long long flow_jump_cells = -1;   // < 0: the default limit of pointer-jumping flow accumulation
  int dependent_launch = 1;           // Local / Focal kernels as programmatic dependent launches
  // Hillshade compositions (python/hill.py:41-49) are generated through the
  // shading identity of rewrite.hpp; 0 keeps the literal operator chain; 2 uses
  // the identity without its fast form (derivatives computed as written).
  int algebraic_rewrite = 1;
  // Local / Focal groups whose every output is one known value are filled, not
  // launched (the reference's Predictor, runtime/visitor/Predictor.cpp); 0 turns it off.
  int prediction = 1;
  // incremented whenever nodes are destroyed (caches keyed by node ids check it)
  uint64_t epoch = 0;
  Arr2 default_bs{{256, 256}, 2};

  // factories (each returns a node owned by the runtime, possibly pre-existing)
  Node *constant(Variant v, Arr2 ds, int dt, int mo, Arr2 bs);
  Node *read(const std::string &path);
  // A scalar whose value is a kernel argument rather than part of the kernel's
  // source, so programs differing only in this value share compiled code.
  Node *scalar_param(Variant v);
  Node *host_input(const void *ptr, Arr2 ds, int dt, Arr2 bs, bool copy);
  Node *dev_input(void *ptr, long long pitch, Arr2 ds, int dt, Arr2 bs);
  // Device input holding rows [row0, row0 + rows) of a ds raster; ptr is the address of row row0.
  Node *dev_input_rows(void *ptr, long long pitch, Arr2 ds, int dt, Arr2 bs, int row0, int rows);
  Node *index(Node *arg, int dim);
  Node *rand(Node *seed, int dt, int mo);
  Node *cast(Node *arg, int dt);
  Node *unary(Node *arg, int op);
  Node *binary(Node *l, Node *r, int op);
  Node *conditional(Node *c, Node *l, Node *r);
  Node *neighbor(Node *arg, Arr2 coord);
  Node *convolution(Node *arg, const Variant *mask, int n, Arr2 mask_ds);
  Node *focal_func(Node *arg, const Variant *mask, int n, Arr2 mask_ds, int red);
  // type 1 (AGE): fraction of the window's cells equal to the centre cell;
  // type 2 (ILE): fraction of the window's cells the centre cell exceeds
  Node *focal_percent(Node *arg, const Variant *mask, int n, Arr2 mask_ds, int type);
  Node *focal_flow(Node *arg);
  Node *zonal_reduc(Node *arg, int red);
  Node *radial_scan(Node *arg, int red, Arr2 start, double radius = 0);
  Node *spread_scan(Node *arg, Node *dir, int red);
  Node *barrier(Node *arg);
  Node *write(Node *arg, const std::string &path);

  // drops nodes unreachable from any referenced node
  void collect_garbage();
  bool owns(const Node *n) const;
  void reset();

 private:
  Node *add(std::unique_ptr<Node> n, const std::string &key);
};

std::string arr_str(const Arr2 &a);

}  // namespace mapb

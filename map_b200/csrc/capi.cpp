// C ABI (include/map_b200.h): the reference's ma_* entry points
// (front/bindings.cpp:14-273) plus the extensions documented in the header.
// Every entry point converts C++ exceptions into a recorded error.
#include "../../include/map_b200.h"
#include "batch.hpp"
#include "server.hpp"
#include "zonestats.hpp"
#include "codegen.hpp"
#include "cuda_env.hpp"
#include "binfile.hpp"
#include "executor.hpp"
#include "graph.hpp"

#include <cuda_runtime.h>

#include <cstring>
#include <sstream>
#include <string>

using namespace mapb;

static_assert(sizeof(ma_Variant) == sizeof(Variant), "ma_Variant layout");
static_assert(sizeof(ma_Array) == sizeof(Arr2), "ma_Array layout");

namespace {

thread_local std::string t_err;
thread_local int t_code = 0;

void ok() { t_code = 0; }
void fail(const std::string &m) {
  t_err = m;
  t_code = 1;
}

Variant V(ma_Variant v) {
  Variant r;
  std::memcpy(&r, &v, sizeof r);
  return r;
}
ma_Variant MV(const Variant &v) {
  ma_Variant r;
  std::memcpy(&r, &v, sizeof r);
  return r;
}
Arr2 A(ma_Array a) {
  Arr2 r;
  std::memcpy(&r, &a, sizeof r);
  return r;
}
ma_Array MA(const Arr2 &a) {
  ma_Array r;
  std::memcpy(&r, &a, sizeof r);
  return r;
}
Node *N(ma_Node *n) { return reinterpret_cast<Node *>(n); }
ma_Node *MN(Node *n) { return reinterpret_cast<ma_Node *>(n); }

Node *checked(ma_Node *n) {
  if (n == nullptr) throw MapError("null node");
  Node *p = N(n);
  if (!Runtime::get().owns(p)) throw MapError("node handle does not belong to the runtime");
  return p;
}

template <class F> ma_Node *node_call(F f) {
  try {
    Node *n = f();
    ok();
    return MN(n);
  } catch (const std::exception &e) {
    fail(e.what());
    return nullptr;
  }
}

template <class F> int int_call(F f) {
  try {
    int r = f();
    ok();
    return r;
  } catch (const std::exception &e) {
    fail(e.what());
    return -1;
  }
}

template <class F> void void_call(F f) {
  try {
    f();
    ok();
  } catch (const std::exception &e) {
    fail(e.what());
  }
}

size_t copy_out(const std::string &s, char *buf, size_t len) {
  if (buf && len) {
    size_t n = std::min(len - 1, s.size());
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
  }
  return s.size() + 1;
}

std::vector<Node *> node_vec(ma_Node **vec, int num) {
  if (num <= 0 || vec == nullptr) throw MapError("empty node list");
  std::vector<Node *> v;
  for (int i = 0; i < num; i++) v.push_back(checked(vec[i]));
  return v;
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

void ma_setupDevices(const char *plat_name, int dev_type, const char *dev_name) {
  // The platform / device strings select an OpenCL platform in the reference
  // (runtime/Runtime.cpp:100-154); here the device is the CUDA device set by
  // ma_setDevice (default 0), initialised lazily on first use.
  (void)plat_name;
  (void)dev_type;
  (void)dev_name;
  ok();
}

void ma_increaseRef(ma_Node *node) {
  void_call([&] {
    if (node) checked(node)->ref++;
  });
}

void ma_decreaseRef(ma_Node *node) {
  void_call([&] {
    if (node && Runtime::get().owns(N(node)) && N(node)->ref > 0) N(node)->ref--;
  });
}

void ma_eval(ma_Node **vec, int num) {
  void_call([&] { Executor::get().evaluate(node_vec(vec, num), {}); });
}

ma_Variant ma_value(ma_Node *node) {
  try {
    Node *n = checked(node);
    if (n->meta.numdim != D0) throw MapError("value: node is not a scalar (D0)");
    if (!n->has_value) throw MapError("value: node has not been evaluated");
    ok();
    return MV(n->value);
  } catch (const std::exception &e) {
    fail(e.what());
    ma_Variant v;
    std::memset(&v, 0, sizeof v);
    return v;
  }
}

int ma_nodeid(ma_Node *node) {
  return int_call([&] { return checked(node)->id; });
}
int ma_datatype(ma_Node *node) {
  return int_call([&] { return checked(node)->meta.dtype; });
}
int ma_numdim(ma_Node *node) {
  return int_call([&] { return checked(node)->meta.numdim; });
}
int ma_memorder(ma_Node *node) {
  return int_call([&] { return checked(node)->meta.memorder; });
}
int ma_streamdir(ma_Node *node) {
  return int_call([&] {
    checked(node);
    return 0;
  });
}
ma_Array ma_datasize(ma_Node *node) {
  try {
    ma_Array r = MA(checked(node)->meta.ds);
    ok();
    return r;
  } catch (const std::exception &e) {
    fail(e.what());
    return ma_Array{{-1, -1}, 0};
  }
}
ma_Array ma_blocksize(ma_Node *node) {
  try {
    ma_Array r = MA(checked(node)->meta.bs);
    ok();
    return r;
  } catch (const std::exception &e) {
    fail(e.what());
    return ma_Array{{-1, -1}, 0};
  }
}
ma_Array ma_numblock(ma_Node *node) {
  try {
    const Meta &m = checked(node)->meta;
    ma_Array r{{-1, -1}, 0};
    if (m.numdim == D2) r = ma_Array{{(m.W() + m.BS0() - 1) / m.BS0(), (m.H() + m.BS1() - 1) / m.BS1()}, 2};
    ok();
    return r;
  } catch (const std::exception &e) {
    fail(e.what());
    return ma_Array{{-1, -1}, 0};
  }
}

ma_Node *ma_read(const char *file_path) {
  return node_call([&] {
    if (!file_path) throw MapError("read: null path");
    return Runtime::get().read(file_path);
  });
}

// Evaluates eagerly, as the reference does (front/bindings.cpp:99-106).
int ma_write(ma_Node *node, const char *file_path) {
  try {
    if (!file_path) throw MapError("write: null path");
    Node *w = Runtime::get().write(checked(node), file_path);
    w->ref++;
    try {
      Executor::get().evaluate({w}, {});
    } catch (...) {
      w->ref--;
      throw;
    }
    w->ref--;
    ok();
    return 0;
  } catch (const std::exception &e) {
    fail(e.what());
    return 1;
  }
}

ma_Node *ma_constant(ma_Variant var, ma_Array ds, int dt, int mo, ma_Array bs) {
  return node_call([&] { return Runtime::get().constant(V(var), A(ds), dt, mo, A(bs)); });
}
ma_Node *ma_rand(ma_Node *seed, int dt, int mo) {
  return node_call([&] { return Runtime::get().rand(checked(seed), dt, mo); });
}
ma_Node *ma_cast(ma_Node *node, int type) {
  return node_call([&] { return Runtime::get().cast(checked(node), type); });
}
ma_Node *ma_index(ma_Node *node, int dim) {
  return node_call([&] { return Runtime::get().index(checked(node), dim); });
}
ma_Node *ma_conditional(ma_Node *c, ma_Node *l, ma_Node *r) {
  return node_call([&] { return Runtime::get().conditional(checked(c), checked(l), checked(r)); });
}
ma_Node *ma_unary(ma_Node *node, int type) {
  return node_call([&] { return Runtime::get().unary(checked(node), type); });
}
ma_Node *ma_binary(ma_Node *l, ma_Node *r, int type) {
  return node_call([&] { return Runtime::get().binary(checked(l), checked(r), type); });
}
ma_Node *ma_diversity(ma_Node **, int, int) {
  return node_call([&]() -> Node * { throw MapError("diversity is not supported by this engine"); });
}
ma_Node *ma_access(ma_Node *, ma_Array) {
  return node_call([&]() -> Node * { throw MapError("access is not supported by this engine"); });
}
ma_Node *ma_lhsAccess(ma_Node *, ma_Node *, ma_Array) {
  return node_call([&]() -> Node * { throw MapError("lhsAccess is not supported by this engine"); });
}
ma_Node *ma_neighbor(ma_Node *node, ma_Array coord) {
  return node_call([&] { return Runtime::get().neighbor(checked(node), A(coord)); });
}
ma_Node *ma_boundedNbh(ma_Node *, ma_Node *, ma_Node *) {
  return node_call([&]() -> Node * { throw MapError("boundedNbh is not supported by this engine"); });
}
ma_Node *ma_spreadNeighbor(ma_Node *, ma_Node *, int) {
  return node_call([&]() -> Node * { throw MapError("spreadNeighbor is not supported by this engine"); });
}
ma_Node *ma_convolution(ma_Node *node, ma_Variant *mask_v, int mask_s, ma_Array mask_ds) {
  return node_call([&] {
    return Runtime::get().convolution(checked(node), reinterpret_cast<Variant *>(mask_v), mask_s, A(mask_ds));
  });
}
ma_Node *ma_focalFunc(ma_Node *node, ma_Variant *mask_v, int mask_s, ma_Array mask_ds, int type) {
  return node_call([&] {
    return Runtime::get().focal_func(checked(node), reinterpret_cast<Variant *>(mask_v), mask_s, A(mask_ds), type);
  });
}
ma_Node *ma_focalPercent(ma_Node *node, ma_Variant *mask_v, int mask_s, ma_Array mask_ds, int type) {
  return node_call([&] {
    return Runtime::get().focal_percent(checked(node), reinterpret_cast<Variant *>(mask_v), mask_s, A(mask_ds), type);
  });
}
ma_Node *ma_zonalReduc(ma_Node *node, int type) {
  return node_call([&] { return Runtime::get().zonal_reduc(checked(node), type); });
}
ma_Node *ma_radialScan(ma_Node *node, int type, ma_Array coord) {
  return node_call([&] { return Runtime::get().radial_scan(checked(node), type, A(coord)); });
}
ma_Node *ma_radialScanRadius(ma_Node *node, int type, ma_Array coord, double radius) {
  return node_call([&] { return Runtime::get().radial_scan(checked(node), type, A(coord), radius); });
}
ma_Node *ma_spreadScan(ma_Node *node, ma_Node *dir, int type) {
  return node_call([&] { return Runtime::get().spread_scan(checked(node), checked(dir), type); });
}
ma_Node *ma_focalFlow(ma_Node *node) {
  return node_call([&] { return Runtime::get().focal_flow(checked(node)); });
}
ma_Node *ma_stats(ma_Node *) {
  return node_call([&]() -> Node * { throw MapError("stats is not supported by this engine"); });
}
ma_Node *ma_barrier(ma_Node *node) {
  return node_call([&] { return Runtime::get().barrier(checked(node)); });
}

static void loops_unsupported() {
  fail("symbolic loop capture entries are not supported: the Python module runs while-loops itself (ma_materialize)");
}
void ma_loopStart(void) { loops_unsupported(); }
void ma_loopCond(ma_Node *) { loops_unsupported(); }
void ma_loopBody(void) { loops_unsupported(); }
void ma_loopAgain(void) { loops_unsupported(); }
ma_Node *ma_loopAssemble(void) {
  loops_unsupported();
  return nullptr;
}
void ma_loopEnd(void) { loops_unsupported(); }
void ma_loopAgainTail(ma_Node *, ma_Node ***agains, ma_Node ***tails, int *num) {
  if (agains) *agains = nullptr;
  if (tails) *tails = nullptr;
  if (num) *num = 0;
  loops_unsupported();
}

// ---- extensions

const char *ma_lastError(void) { return t_err.c_str(); }
int ma_errorCode(void) { return t_code; }
void ma_clearError(void) {
  t_err.clear();
  t_code = 0;
}

void ma_setBorder(int mode) {
  void_call([&] {
    if (mode < BORDER_BLOCK_MIRROR || mode > BORDER_DEAD) throw MapError("setBorder: invalid mode");
    Runtime::get().border = mode;
  });
}
int ma_getBorder(void) { return Runtime::get().border; }
void ma_setExecMode(int mode) {
  void_call([&] {
    if (mode != EXEC_FUSED && mode != EXEC_PLAIN) throw MapError("setExecMode: invalid mode");
    Runtime::get().exec_mode = mode;
  });
}
int ma_getExecMode(void) { return Runtime::get().exec_mode; }
void ma_setStreamRows(int rows) {
  void_call([&] { Runtime::get().stream_rows = rows; });
}
int ma_getStreamRows(void) { return Runtime::get().stream_rows; }
void ma_setPairedCells(int on) {
  void_call([&] { Runtime::get().paired_cells = on ? 1 : 0; });
}
int ma_getPairedCells(void) { return Runtime::get().paired_cells; }
void ma_setFlowJumpCells(long long cells) {
  void_call([&] { Runtime::get().flow_jump_cells = cells < 0 ? -1 : cells; });
}
long long ma_getFlowJumpCells(void) { return (long long)spread_pj_cells(); }

void ma_setPrediction(int on) {
  void_call([&] { Runtime::get().prediction = on ? 1 : 0; });
}
int ma_getPrediction(void) { return Runtime::get().prediction; }
int ma_lastPredictedCount(void) { return Executor::get().last.predicted; }

void ma_setAlgebraicRewrite(int on) {
  void_call([&] { Runtime::get().algebraic_rewrite = on < 0 ? 0 : on > 2 ? 2 : on; });
}
int ma_getAlgebraicRewrite(void) { return Runtime::get().algebraic_rewrite; }
void ma_setDefaultBlockSize(ma_Array bs) {
  void_call([&] {
    if (bs.n != 2 || bs.arr[0] <= 0 || bs.arr[1] <= 0) throw MapError("setDefaultBlockSize: invalid size");
    Runtime::get().default_bs = A(bs);
  });
}
void ma_setDevice(int device) {
  void_call([&] { CudaEnv::get().set_device(device); });
}

ma_Node *ma_fromHost(const void *data, ma_Array ds, int dt, ma_Array bs, int copy) {
  return node_call([&] { return Runtime::get().host_input(data, A(ds), dt, A(bs), copy != 0); });
}
ma_Node *ma_fromDevice(void *dptr, long long pitch, ma_Array ds, int dt, ma_Array bs) {
  return node_call([&] { return Runtime::get().dev_input(dptr, pitch, A(ds), dt, A(bs)); });
}

ma_Node *ma_fromDeviceRows(void *dptr, long long pitch, ma_Array ds, int dt, ma_Array bs, int row0, int rows) {
  return node_call([&] { return Runtime::get().dev_input_rows(dptr, pitch, A(ds), dt, A(bs), row0, rows); });
}

int ma_evalRows(ma_Node **nodes, int n, void **dst, const long long *pitch, int y0, int y1) {
  return int_call([&] {
    std::vector<Node *> v = node_vec(nodes, n);
    if (!dst || !pitch) throw MapError("evalRows: null destination arrays");
    std::vector<Sink> sinks;
    for (int i = 0; i < n; i++) {
      if (!dst[i]) throw MapError("evalRows: null destination");
      Sink s;
      s.node = v[i];
      s.dev = dst[i];
      s.dev_pitch = pitch[i];
      sinks.push_back(s);
    }
    Executor::get().evaluate_rows({}, sinks, y0, y1);
    return 0;
  });
}

int ma_rowMargin(ma_Node **nodes, int n) {
  return int_call([&] { return Executor::get().row_margin(node_vec(nodes, n)); });
}

int ma_binInfo(const char *path, int *info7) {
  return int_call([&] {
    if (!path || !info7) throw MapError("binInfo: null argument");
    BinHeader h = bin_read_header(path);
    const int v[7] = {h.dtype, h.numdim, h.ds0, h.ds1, h.memorder, h.bs0, h.bs1};
    std::memcpy(info7, v, sizeof v);
    return 0;
  });
}

int ma_binReadHost(const char *path, void *dst, size_t bytes) {
  return int_call([&] {
    if (!path || !dst) throw MapError("binRead: null argument");
    BinHeader h = bin_read_header(path);
    const size_t need = (size_t)h.ds0 * h.ds1 * dt_size(h.dtype);
    if (bytes < need) throw MapError("binRead: destination holds " + std::to_string(bytes) + " bytes, " +
                                     std::to_string(need) + " needed");
    bin_read_dense(path, h, dst);
    return 0;
  });
}

int ma_binWriteHost(const char *path, const void *src, ma_Array ds, int dt, int mo, ma_Array bs) {
  return int_call([&] {
    if (!path || !src) throw MapError("binWrite: null argument");
    BinHeader h;
    h.dtype = dt;
    h.numdim = D2;
    h.ds0 = ds.arr[0];
    h.ds1 = ds.arr[1];
    h.memorder = mo;
    h.bs0 = mo == ROW ? h.ds0 : bs.arr[0];
    h.bs1 = mo == ROW ? h.ds1 : bs.arr[1];
    if (h.ds0 <= 0 || h.ds1 <= 0 || h.bs0 <= 0 || h.bs1 <= 0) throw MapError("binWrite: invalid sizes");
    dt_size(dt);
    bin_write_dense(path, h, src);
    return 0;
  });
}

int ma_toHost(ma_Node *node, void *dst, size_t bytes) {
  return int_call([&] {
    Node *n = checked(node);
    if (!dst) throw MapError("toHost: null destination");
    if (n->meta.numdim != D2) throw MapError("toHost: node is not a 2-D raster");
    size_t need = (size_t)n->meta.W() * n->meta.H() * dt_size(n->meta.dtype);
    if (bytes < need) throw MapError("toHost: destination holds " + std::to_string(bytes) + " bytes, " + std::to_string(need) + " needed");
    Sink s;
    s.node = n;
    s.host = dst;
    Executor::get().evaluate({}, {s});
    return 0;
  });
}

int ma_toDevice(ma_Node *node, void *dptr, long long pitch, int async) {
  return int_call([&] {
    Node *n = checked(node);
    if (!dptr) throw MapError("toDevice: null destination");
    if (n->meta.numdim != D2) throw MapError("toDevice: node is not a 2-D raster");
    if (pitch < (long long)n->meta.W() * (long long)dt_size(n->meta.dtype)) throw MapError("toDevice: pitch smaller than a row");
    Sink s;
    s.node = n;
    s.dev = dptr;
    s.dev_pitch = pitch;
    Executor::get().evaluate({}, {s}, async != 0);
    return 0;
  });
}

int ma_materialize(ma_Node **vec, int num, ma_Node **out) {
  return int_call([&] {
    std::vector<Node *> v = node_vec(vec, num);
    if (!out) throw MapError("materialize: null output array");
    std::vector<Node *> r = Executor::get().materialize(v);
    for (int i = 0; i < num; i++) out[i] = MN(r[i]);
    return 0;
  });
}

int ma_evalAsync(ma_Node **vec, int num) {
  return int_call([&] {
    Executor::get().evaluate(node_vec(vec, num), {}, true);
    return 0;
  });
}

int ma_sync(void) {
  return int_call([&] {
    Executor::get().sync();
    return 0;
  });
}

void *ma_stream(void) {
  try {
    CudaEnv::get().ensure_device();
    ok();
    return (void *)CudaEnv::get().stream();
  } catch (const std::exception &e) {
    fail(e.what());
    return nullptr;
  }
}

void *ma_hostAlloc(size_t bytes) {
  try {
    CudaEnv::get().ensure_device();
    void *p = nullptr;
    cuda_check(cudaMallocHost(&p, bytes), "cudaMallocHost");
    ok();
    return p;
  } catch (const std::exception &e) {
    fail(e.what());
    return nullptr;
  }
}
void ma_hostFree(void *p) {
  if (p) cudaFreeHost(p);
}
void *ma_devAlloc(size_t bytes) {
  try {
    CudaEnv::get().ensure_device();
    void *p = nullptr;
    cuda_check(cudaMalloc(&p, bytes), "cudaMalloc");
    ok();
    return p;
  } catch (const std::exception &e) {
    fail(e.what());
    return nullptr;
  }
}
void ma_devFree(void *p) {
  if (p) cudaFree(p);
}
int ma_memcpy(void *dst, const void *src, size_t bytes, int kind) {
  return int_call([&] {
    CudaEnv::get().ensure_device();
    cuda_check(cudaMemcpy(dst, src, bytes, (cudaMemcpyKind)kind), "cudaMemcpy");
    return 0;
  });
}

int ma_lastLaunchCount(void) { return Executor::get().last.launches; }
int ma_lastGroupCount(void) { return Executor::get().last.groups; }
int ma_lastBandCount(void) { return Executor::get().last.bands; }
int ma_totalLaunchCount(void) { return CudaEnv::get().launches(); }

int ma_compileOnly(ma_Node **vec, int num, int compile) {
  return int_call([&] { return (int)Executor::get().compile_only(node_vec(vec, num), compile != 0).size(); });
}

size_t ma_describeGroups(ma_Node **vec, int num, char *buf, size_t len) {
  try {
    std::string s = Executor::get().describe_groups(node_vec(vec, num));
    ok();
    return copy_out(s, buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

size_t ma_generatedSource(ma_Node **vec, int num, char *buf, size_t len) {
  try {
    auto srcs = Executor::get().compile_only(node_vec(vec, num), false);
    std::string s;
    for (auto &x : srcs) s += x + "\n//----\n";
    ok();
    return copy_out(s, buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

size_t ma_plainSchedule(ma_Node **vec, int num, char *buf, size_t len) {
  try {
    auto jobs = Executor::get().schedule_for(node_vec(vec, num));
    std::ostringstream s;
    for (auto &j : jobs) s << j.group << " " << j.bx << " " << j.by << " " << j.kind << "\n";
    ok();
    return copy_out(s.str(), buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

// ---- batches

struct ma_Batch {
  Batch b;
  std::vector<Node *> held;   // output nodes kept alive while the batch exists
};

ma_Batch *ma_batchCreate(void) {
  try {
    ok();
    return new ma_Batch();
  } catch (const std::exception &e) {
    fail(e.what());
    return nullptr;
  }
}

int ma_batchAdd(ma_Batch *b, ma_Node **outs, int n, void **dst, const long long *pitch) {
  return int_call([&] {
    if (!b) throw MapError("batch: null handle");
    std::vector<Node *> o = node_vec(outs, n);
    std::vector<void *> d(dst, dst + n);
    std::vector<long long> p(pitch, pitch + n);
    b->b.add(o, d, p);
    for (Node *x : o) {
      x->ref++;
      b->held.push_back(x);
    }
    return b->b.instances() - 1;
  });
}

int ma_batchPrepare(ma_Batch *b, int autotune) {
  return int_call([&] {
    if (!b) throw MapError("batch: null handle");
    b->b.prepare(autotune != 0);
    return 0;
  });
}

int ma_batchRun(ma_Batch *b, int sync) {
  return int_call([&] {
    if (!b) throw MapError("batch: null handle");
    b->b.run(sync != 0);
    return 0;
  });
}

size_t ma_batchInfo(ma_Batch *b, char *buf, size_t len) {
  try {
    if (!b) throw MapError("batch: null handle");
    ok();
    return copy_out(b->b.info(), buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

void ma_batchDestroy(ma_Batch *b) {
  if (!b) return;
  for (Node *x : b->held)
    if (Runtime::get().owns(x) && x->ref > 0) x->ref--;
  delete b;
}

// ---- serving

struct ma_Server {
  std::unique_ptr<Server> s;
};

ma_Server *ma_serverCreate(void *dem, long long pitch, int W, int H, size_t budget_bytes, int max_batch) {
  try {
    auto *h = new ma_Server();
    h->s = std::make_unique<Server>(dem, pitch, W, H, budget_bytes, max_batch);
    ok();
    return h;
  } catch (const std::exception &e) {
    fail(e.what());
    return nullptr;
  }
}

long long ma_serverSubmit(ma_Server *h, int type, int x0, int y0, int w, int hh, int obs_x, int obs_y, float obs_h,
                          double radius) {
  try {
    if (!h) throw MapError("server: null handle");
    long long id = h->s->submit(type, x0, y0, w, hh, obs_x, obs_y, obs_h, radius, false);
    ok();
    return id;
  } catch (const std::exception &e) {
    fail(e.what());
    return -1;
  }
}

int ma_serverWait(ma_Server *h, long long id, double timeout_s) {
  return int_call([&] {
    if (!h) throw MapError("server: null handle");
    return h->s->wait(id, timeout_s);
  });
}

int ma_serverResult(ma_Server *h, long long id, void *dst, size_t bytes) {
  return int_call([&] {
    if (!h) throw MapError("server: null handle");
    h->s->result(id, dst, bytes);
    return 0;
  });
}

int ma_serverRelease(ma_Server *h, long long id) {
  return int_call([&] {
    if (!h) throw MapError("server: null handle");
    h->s->release(id);
    return 0;
  });
}

double ma_serverLatency(ma_Server *h, long long id) {
  try {
    if (!h) throw MapError("server: null handle");
    double v = h->s->latency_ms(id);
    ok();
    return v;
  } catch (const std::exception &e) {
    fail(e.what());
    return -1;
  }
}

size_t ma_serverStats(ma_Server *h, char *buf, size_t len) {
  try {
    if (!h) throw MapError("server: null handle");
    ok();
    return copy_out(h->s->stats_json(), buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

size_t ma_serverLoad(ma_Server *h, double rate, double seconds, const double *mix, unsigned seed, double obs_h,
                     double radius, char *buf, size_t len) {
  try {
    if (!h || !mix) throw MapError("server: null argument");
    std::string j = h->s->run_load(rate, seconds, mix, seed, obs_h, radius);
    ok();
    return copy_out(j, buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

size_t ma_serverLoadClosed(ma_Server *h, int outstanding, double seconds, const double *mix, unsigned seed, double obs_h,
                           double radius, char *buf, size_t len) {
  try {
    if (!h || !mix) throw MapError("server: null argument");
    std::string j = h->s->run_closed(outstanding, seconds, mix, seed, obs_h, radius);
    ok();
    return copy_out(j, buf, len);
  } catch (const std::exception &e) {
    fail(e.what());
    return 0;
  }
}

void ma_serverDestroy(ma_Server *h) {
  try {
    delete h;
    ok();
  } catch (const std::exception &e) {
    fail(e.what());
  }
}

int ma_zoneStats(const void *value, long long value_pitch, const void *zone, long long zone_pitch, int W, int H,
                 int nzones, unsigned long long *count, float *vmin, float *vmax, float *sum, float *mean,
                 void *stream) {
  return int_call([&] {
    CudaEnv::get().ensure_device();
    ZoneStatsArgs a;
    a.value = value;
    a.value_pitch = value_pitch;
    a.zone = zone;
    a.zone_pitch = zone_pitch;
    a.W = W;
    a.H = H;
    a.nzones = nzones;
    a.count = count;
    a.vmin = vmin;
    a.vmax = vmax;
    a.sum = sum;
    a.mean = mean;
    zone_stats(a, (CUstream_st *)stream);
    return 0;
  });
}

int ma_zoneStatsNoAlloc(const void *value, long long value_pitch, const void *zone, long long zone_pitch, int W,
                        int H, int nzones, unsigned long long *count, float *vmin, float *vmax, float *sum,
                        float *mean, void *stream) {
  return int_call([&] {
    CudaEnv::get().ensure_device();
    ZoneStatsArgs a;
    a.value = value;
    a.value_pitch = value_pitch;
    a.zone = zone;
    a.zone_pitch = zone_pitch;
    a.W = W;
    a.H = H;
    a.nzones = nzones;
    a.count = count;
    a.vmin = vmin;
    a.vmax = vmax;
    a.sum = sum;
    a.mean = mean;
    zone_stats_no_alloc(a, (CUstream_st *)stream);
    return 0;
  });
}

int ma_nodeCount(void) { return (int)Runtime::get().nodes.size(); }
void ma_collectGarbage(void) {
  void_call([&] { Runtime::get().collect_garbage(); });
}

}  // extern "C"
#pragma GCC visibility pop

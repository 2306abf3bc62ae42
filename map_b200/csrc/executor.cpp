// Evaluation engine (see executor.hpp).
#include "executor.hpp"
#include "binfile.hpp"
#include "cuda_env.hpp"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <chrono>
#include <functional>
#include <cstring>
#include <future>
#include <queue>
#include <sstream>
#include <unordered_map>
#include <unordered_set>

namespace mapb {

void run_scan_group(const Group &g, const KernelPlan &P, std::unordered_map<Node *, DevRaster> &bufs,
                    const std::function<DevRaster &(Node *)> &get, const std::function<DevRaster(Node *)> &alloc_out);

namespace {

long long pitch_for(int W, int dt) {
  long long b = (long long)W * (long long)dt_size(dt);
  return (b + 127) / 128 * 128;
}

uint64_t spread_bits(uint32_t v) {
  uint64_t x = v & 0x1fffff;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}
// Morton interleave of (x, y, group): x bits highest in each triple, as the
// reference's Order interleaves (h, t, y, x) with x highest (runtime/Job.cpp:22-45).
uint64_t morton3(uint32_t x, uint32_t y, uint32_t t) { return spread_bits(x) << 2 | spread_bits(y) << 1 | spread_bits(t); }

}  // namespace

std::vector<Node *> collect_nodes(const std::vector<Node *> &targets) {
  std::unordered_set<Node *> seen;
  std::vector<Node *> st(targets.begin(), targets.end()), out;
  while (!st.empty()) {
    Node *n = st.back();
    st.pop_back();
    if (!seen.insert(n).second) continue;
    out.push_back(n);
    for (Node *p : n->prev) st.push_back(p);
  }
  std::sort(out.begin(), out.end(), [](Node *a, Node *b) { return a->id < b->id; });
  return out;
}

namespace {

std::vector<Node *> collect(const std::vector<Node *> &targets) { return collect_nodes(targets); }

bool per_block(int sk) { return sk == SK_LOCAL || sk == SK_FOCAL || sk == SK_ZONAL; }

bool reads_focal(const Group &g, Node *in) {
  for (Node *n : g.nodes)
    if ((n->kind == K_NEIGHBOR || n->kind == K_CONVOLUTION || n->kind == K_FOCALFUNC || n->kind == K_FOCALFLOW ||
         n->kind == K_FOCALPERCENT) &&
        n->prev[0] == in)
      return true;
  return false;
}

Variant host_eval(Node *n) {
  for (Node *p : n->prev)
    if (!p->has_value) throw MapError(std::string("scalar input of ") + kind_name(n->kind) + " has no value");
  switch (n->kind) {
    case K_UNARY: return var_convert(host_unary(n->op, n->prev[0]->value), n->meta.dtype);
    case K_BINARY: return var_convert(host_binary(n->op, n->prev[0]->value, n->prev[1]->value), n->meta.dtype);
    case K_CAST: return var_convert(n->prev[0]->value, n->meta.dtype);
    case K_BARRIER: return n->prev[0]->value;
    case K_CONDITIONAL: {
      bool c = var_as_f64(n->prev[0]->value) != 0.0;
      return var_convert(c ? n->prev[1]->value : n->prev[2]->value, n->meta.dtype);
    }
    default: throw MapError(std::string("cannot evaluate ") + kind_name(n->kind) + " on the host");
  }
}

double now_ms() {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Whole-raster form of the reference's Predictor (runtime/visitor/Predictor.cpp:22-200,
// called before every block's computation, runtime/Worker.cpp:83-91): a node is
// fixed when every cell holds the same value, known on the host. Constants are
// fixed; element-wise nodes of fixed operands are evaluated with the host
// operator tables; a focal node over a fixed raster is fixed under the mirror
// border rules (every tap reads the same value) and is folded in the kernel's
// order; an integer product with a fixed zero operand is zero. Cell-dependent
// nodes (index, rand, flow directions, percentages) and raster inputs are not
// fixed. Returns whether every raster output of the group is fixed (and how
// many bytes each holds: 1, 2 or 4, the sizes a fill writes without a kernel).
bool predict_group(const Group &g, const KernelPlan &K, std::unordered_map<Node *, Variant> &fixed, int border) {
  if (g.skeleton != SK_LOCAL && g.skeleton != SK_FOCAL) return false;
  auto known = [&](Node *p, Variant &v) {
    auto it = fixed.find(p);
    if (it != fixed.end()) { v = it->second; return true; }
    if (p->meta.numdim == D0 && p->kind == K_CONSTANT) { v = p->cnst; return true; }
    if (p->meta.numdim == D0 && p->has_value) { v = p->value; return true; }
    return false;
  };
  const bool mirror = border == BORDER_BLOCK_MIRROR || border == BORDER_RASTER_MIRROR;
  for (Node *n : g.nodes) {
    Variant a, b, c;
    const int dt = n->meta.dtype;
    switch (n->kind) {
      case K_CONSTANT: fixed[n] = var_convert(n->cnst, dt); break;
      case K_CAST: case K_BARRIER:
        if (known(n->prev[0], a)) fixed[n] = var_convert(a, dt);
        break;
      case K_UNARY:
        if (known(n->prev[0], a)) fixed[n] = var_convert(host_unary(n->op, a), dt);
        break;
      case K_BINARY: {
        const bool la = known(n->prev[0], a), lb = known(n->prev[1], b);
        if (la && lb) fixed[n] = var_convert(host_binary(n->op, a, b), dt);
        else if (n->op == MUL && !dt_is_float(dt) && ((la && var_is_zero(a)) || (lb && var_is_zero(b))))
          fixed[n] = var_make_f64(0.0, dt);
        break;
      }
      case K_CONDITIONAL:
        if (known(n->prev[0], c)) {
          Node *pick = var_as_f64(c) != 0.0 ? n->prev[1] : n->prev[2];
          if (known(pick, a)) fixed[n] = var_convert(a, dt);
        }
        break;
      case K_NEIGHBOR:
        if (mirror && known(n->prev[0], a)) fixed[n] = var_convert(a, dt);
        break;
      case K_CONVOLUTION:
        if (mirror && known(n->prev[0], a)) {   // acc = acc + tap * w, rows outer, columns inner
          Variant acc = var_make_f64(0.0, dt);
          for (const Variant &w : n->mask) acc = var_convert(host_binary(ADD, acc, host_binary(MUL, a, w)), dt);
          fixed[n] = acc;
        }
        break;
      case K_FOCALFUNC:
        if (mirror && known(n->prev[0], a)) {
          Variant acc = reduction_neutral(n->op, dt);
          for (size_t i = 0; i < n->mask.size(); i++) acc = host_reduce(n->op, acc, var_convert(a, dt));
          fixed[n] = acc;
        }
        break;
      default:
        break;
    }
  }
  if (K.out_rasters.empty()) return false;
  for (Node *o : K.out_rasters) {
    if (!fixed.count(o)) return false;
    const size_t s = dt_size(o->meta.dtype);
    if (s != 1 && s != 2 && s != 4) return false;
  }
  return true;
}

}  // namespace

std::vector<PlainJob> plain_schedule(const std::vector<std::unique_ptr<Group>> &groups, const std::vector<KernelPlan> &plans) {
  (void)plans;
  struct J { PlainJob j; std::vector<int> succ; int indeg = 0; uint64_t key = 0; };
  std::vector<J> jobs;
  std::unordered_map<Node *, const Group *> owner;
  for (auto &g : groups)
    for (Node *o : g->outputs) owner[o] = g.get();
  for (auto &g : groups)
    for (Node *n : g->nodes) if (!owner.count(n)) owner[n] = g.get();
  // job index tables
  std::vector<std::vector<int>> block_job(groups.size());
  std::vector<int> single_job(groups.size(), -1);
  std::vector<int> nbx(groups.size(), 1), nby(groups.size(), 1);
  for (auto &gp : groups) {
    const Group &g = *gp;
    if (per_block(g.skeleton)) {
      nbx[g.id] = (g.W + g.BS0 - 1) / g.BS0;
      nby[g.id] = (g.H + g.BS1 - 1) / g.BS1;
      for (int by = 0; by < nby[g.id]; by++)
        for (int bx = 0; bx < nbx[g.id]; bx++) {
          J j;
          j.j = PlainJob{g.id, bx, by, 0};
          j.key = morton3(bx, by, g.id);
          block_job[g.id].push_back((int)jobs.size());
          jobs.push_back(j);
        }
      if (g.skeleton == SK_ZONAL) {
        J j;
        j.j = PlainJob{g.id, -1, -1, 2};
        j.key = morton3(nbx[g.id], nby[g.id], g.id);
        single_job[g.id] = (int)jobs.size();
        jobs.push_back(j);
        for (int b : block_job[g.id]) { jobs[b].succ.push_back(single_job[g.id]); jobs[single_job[g.id]].indeg++; }
      }
    } else {
      J j;
      j.j = PlainJob{g.id, -1, -1, g.skeleton == SK_HOST ? 3 : 1};
      j.key = morton3(0, 0, g.id);
      single_job[g.id] = (int)jobs.size();
      jobs.push_back(j);
    }
  }
  auto dep = [&](int from, int to) {
    jobs[from].succ.push_back(to);
    jobs[to].indeg++;
  };
  for (auto &gp : groups) {
    const Group &g = *gp;
    for (Node *in : g.inputs) {
      auto it = owner.find(in);
      if (it == owner.end()) continue;
      const Group &src = *it->second;
      const bool scalar = in->meta.numdim == D0;
      const bool src_blocks = per_block(src.skeleton) && !scalar;
      auto whole_of = [&](const Group &s) -> std::vector<int> {
        if (single_job[s.id] >= 0 && (s.skeleton != SK_ZONAL || scalar)) return {single_job[s.id]};
        return block_job[s.id];
      };
      if (per_block(g.skeleton)) {
        for (int b : block_job[g.id]) {
          const PlainJob &pj = jobs[b].j;
          if (src_blocks && src.W == g.W && src.H == g.H && src.BS0 == g.BS0 && src.BS1 == g.BS1) {
            const int r = reads_focal(g, in) ? 1 : 0;
            for (int dy = -r; dy <= r; dy++)
              for (int dx = -r; dx <= r; dx++) {
                int bx = pj.bx + dx, by = pj.by + dy;
                if (bx < 0 || by < 0 || bx >= nbx[src.id] || by >= nby[src.id]) continue;
                dep(block_job[src.id][by * nbx[src.id] + bx], b);
              }
          } else {
            for (int s : whole_of(src)) dep(s, b);
          }
        }
      } else {
        for (int s : whole_of(src)) dep(s, single_job[g.id]);
      }
    }
  }
  // ready queue: smallest key first, ties by creation order
  typedef std::pair<uint64_t, int> KI;
  std::priority_queue<KI, std::vector<KI>, std::greater<KI>> ready;
  for (int i = 0; i < (int)jobs.size(); i++)
    if (jobs[i].indeg == 0) ready.push({jobs[i].key, i});
  std::vector<PlainJob> out;
  while (!ready.empty()) {
    int i = ready.top().second;
    ready.pop();
    out.push_back(jobs[i].j);
    for (int s : jobs[i].succ)
      if (--jobs[s].indeg == 0) ready.push({jobs[s].key, s});
  }
  if (out.size() != jobs.size()) throw MapError("plain schedule: dependency cycle");
  return out;
}

std::vector<unsigned char> pack_args(const Group &g, const KernelPlan &K, const std::function<DevRaster &(Node *)> &get,
                                     std::unordered_map<Node *, DevRaster> &bufs, int rx0, int ry0, int rx1, int ry1,
                                     const uint64_t aux[4], const std::unordered_map<const Node *, Variant> *scalars,
                                     bool out_maps) {
  CudaEnv &env = CudaEnv::get();
  std::vector<unsigned char> a(K.args_size, 0);
  int32_t oy = 0;
  for (size_t k = 0; k < K.tma.size(); k++) {
    const TmaSpec &t = K.tma[k];
    DevRaster &r = get(K.in_rasters[t.in_index]);
    alignas(64) unsigned char desc[128];
    // a row band is mapped from its buffer's first row; the kernel subtracts Geom::oy from row coordinates
    void *base = r.rows ? (void *)((uintptr_t)r.ptr + (uintptr_t)(r.org * r.pitch)) : r.ptr;
    const uint64_t rows = r.rows ? (uint64_t)r.rows : (uint64_t)r.H;
    if (k == 0) oy = (int32_t)(r.rows ? r.org : 0);
    else if (oy != (int32_t)(r.rows ? r.org : 0)) throw MapError("staged inputs of one group must share their row origin");
    env.encode_tma_2d(desc, r.dtype, base, (uint64_t)r.W, rows, (uint64_t)r.pitch, (uint32_t)t.box_w, (uint32_t)t.box_h);
    std::memcpy(a.data() + K.off_tm + 128 * k, desc, 128);
  }
  for (size_t k = 0; k < K.in_rasters.size(); k++) {
    DevRaster &r = get(K.in_rasters[k]);
    uint64_t p = (uint64_t)(uintptr_t)r.ptr;
    int64_t pitch = r.pitch;
    std::memcpy(a.data() + K.off_in + 16 * k, &p, 8);
    std::memcpy(a.data() + K.off_in + 16 * k + 8, &pitch, 8);
  }
  for (size_t k = 0; k < K.out_rasters.size(); k++) {
    DevRaster &r = bufs.at(K.out_rasters[k]);
    uint64_t p = (uint64_t)(uintptr_t)r.ptr;
    int64_t pitch = r.pitch;
    std::memcpy(a.data() + K.off_out + 16 * k, &p, 8);
    std::memcpy(a.data() + K.off_out + 16 * k + 8, &pitch, 8);
  }
  for (size_t k = 0; k < K.scalars.size(); k++) {
    Node *s = K.scalars[k];
    const Variant *sv = &s->value;
    if (scalars) {
      auto it = scalars->find(s);
      if (it != scalars->end()) sv = &it->second;
      else if (!s->has_value) throw MapError(std::string("scalar input ") + kind_name(s->kind) + " has no value");
    } else if (!s->has_value) {
      throw MapError(std::string("scalar input ") + kind_name(s->kind) + " has no value");
    }
    Variant v = var_convert(*sv, s->meta.dtype);
    std::memcpy(a.data() + K.off_s + 8 * k, &v.u, dt_size(v.dtype));
  }
  int32_t geom[12] = {g.W, g.H, g.BS0, g.BS1, rx0, ry0, rx1, ry1, 0, 0, Runtime::get().border, oy};
  const int tx = (rx1 - rx0 + K.tile_w - 1) / K.tile_w, ty = (ry1 - ry0 + K.tile_h - 1) / K.tile_h;
  geom[8] = tx;
  geom[9] = tx * ty;
  std::memcpy(a.data() + K.off_geom, geom, sizeof geom);
  uint64_t errp = (uint64_t)(uintptr_t)env.err_word();
  std::memcpy(a.data() + K.off_err, &errp, 8);
  uint64_t ax[4] = {aux[0], aux[1], aux[2], aux[3]};
  // output tile stores: maps over the whole output rasters, after the inputs' maps
  bool omaps = out_maps && !K.tma_out.empty();
  for (size_t j = 0; omaps && j < K.tma_out.size(); j++) {
    const TmaSpec &t = K.tma_out[j];
    const DevRaster &r = bufs.at(K.out_rasters[t.in_index]);
    if (((uintptr_t)r.ptr & 15) != 0 || (r.pitch & 15) != 0 || r.rows != 0) {
      omaps = false;
      break;
    }
    alignas(64) unsigned char desc[128];
    env.encode_tma_2d(desc, r.dtype, r.ptr, (uint64_t)r.W, (uint64_t)r.H, (uint64_t)r.pitch, (uint32_t)t.box_w,
                      (uint32_t)t.box_h);
    std::memcpy(a.data() + K.off_tm + 128 * (K.tma.size() + j), desc, 128);
  }
  if (!K.tma_out.empty()) ax[2] = omaps ? 1 : 0;
  std::memcpy(a.data() + K.off_aux, ax, 4 * sizeof(uint64_t));
  return a;
}

// Largest grid height of a launch (CUDA's limit on gridDim.y): taller regions of
// Local / Focal tiles are launched in pieces of this many tile rows.
constexpr int kMaxGridY = 65535;

Executor &Executor::get() {
  static Executor e;
  return e;
}

Executor::Prepared Executor::prepare(const std::vector<Node *> &targets, const std::set<Node *> &tset, bool compile) {
  Prepared P;
  P.order = collect(targets);
  P.fr = fuse(P.order, tset);
  P.plans.resize(P.fr.groups.size());
  std::vector<std::future<void>> jobs;
  std::set<std::string> seen;
  for (auto &g : P.fr.groups) {
    if (g->skeleton == SK_HOST) { P.plans[g->id].skeleton = SK_HOST; continue; }
    // standalone focal kernels: 128 threads on a 64 x 32 tile (16 rows per thread),
    // measured 1.5% faster than 256 threads on the hillshade and 2% on life
    TileCfg cfg;
    if (g->skeleton == SK_FOCAL && focal_quad_form(*g)) {
      // packed byte form: 128 x 16 tiles of 128 threads, a warp on the 32 words of
      // one tile row, 4 rows per thread (Life at 4096^2 with dependent launches:
      // 1021 Gcell-updates/s, against 996 for 64 x 32 and 981 for 128 x 32 of 256)
      const FocalTune &ft = focal_tune();
      cfg.tw = ft.qtw ? ft.qtw : 128;
      cfg.th = ft.qth ? ft.qth : 16;
      cfg.nt = ft.qnt ? ft.qnt : 128;
    } else if (g->skeleton == SK_FOCAL) {
      cfg.nt = 128;
      if (focal_fast_shade(*g)) {
        // fast hillshade form: 64 x 64 tiles of 256 threads, 16 rows per thread
        // (532 Gcells/s at 16384^2, against 530 for 32 x 128 of 256 threads and
        // 513 for 32 x 128 of 128, the same box, with per-thread store addresses),
        // registers capped for 6 resident CTAs per SM (533 against 521 with the
        // 5 that 48 registers allow, the same box)
        cfg.tw = 64;
        cfg.th = 64;
        cfg.nt = 256;
        cfg.minb = 6;
      }
      const FocalTune &ft = focal_tune();
      if (ft.nt) cfg.nt = ft.nt;
      if (ft.tw) cfg.tw = ft.tw;
      if (ft.th) cfg.th = ft.th;
    } else if (g->skeleton == SK_LOCAL) {
      const FocalTune &ft = focal_tune();
      if (ft.lnt) cfg.nt = ft.lnt;
      if (ft.ltw) cfg.tw = ft.ltw;
      if (ft.lth) cfg.th = ft.lth;
    }
    cfg.tile_store = g->skeleton == SK_FOCAL;   // whole-raster launches: the output tile store where it applies
    P.plans[g->id] = generate_kernel(*g, cfg);
    if (compile && seen.insert(P.plans[g->id].source).second) {
      const std::string *src = &P.plans[g->id].source;
      jobs.push_back(std::async(std::launch::async, [src]() { CudaEnv::get().compile(*src); }));
    }
  }
  for (auto &f : jobs) f.get();
  return P;
}

std::shared_ptr<Executor::Prepared> Executor::prepare_cached(const std::vector<Node *> &targets,
                                                             const std::set<Node *> &tset) {
  Runtime &rt = Runtime::get();
  std::string key = std::to_string(rt.exec_mode) + "," + std::to_string(rt.paired_cells) + "," +
                    std::to_string(rt.algebraic_rewrite) + ";";   // prediction runs per evaluation (not cached)
  for (Node *t : targets) key += std::to_string(t->id) + ",";
  key += ";";
  for (Node *t : tset) key += std::to_string(t->id) + ",";
  auto sig = [](const Prepared &P) {
    std::vector<char> v;
    for (Node *n : P.order)
      if (n->meta.numdim == D0) v.push_back(n->has_value ? 1 : 0);
    return v;
  };
  auto it = cache_.find(key);
  if (it != cache_.end() && it->second.epoch == rt.epoch && it->second.d0sig == sig(*it->second.P)) {
    it->second.used = ++cache_tick_;
    return it->second.P;
  }
  auto P = std::make_shared<Prepared>(prepare(targets, tset, true));
  if (cache_.size() >= 64) {   // evict the least recently used entry
    auto lru = cache_.begin();
    for (auto c = cache_.begin(); c != cache_.end(); ++c)
      if (c->second.used < lru->second.used) lru = c;
    cache_.erase(lru);
  }
  CacheEntry &e = cache_[key];
  e.P = P;
  e.d0sig = sig(*P);
  e.epoch = rt.epoch;
  e.used = ++cache_tick_;
  return P;
}

namespace {
// Set by an exit handler registered at the first materialisation (so it runs
// before the runtime's and the device environment's destructors): buffers of
// nodes destroyed during process teardown are left to the driver.
std::atomic<bool> g_exiting{false};
std::once_flag g_exit_hook;
}  // namespace

DevData::~DevData() {
  if (!owned || ptr == nullptr || g_exiting.load()) return;
  try {
    CudaEnv &env = CudaEnv::get();
    if (env.device_ready()) cudaFreeAsync(ptr, (cudaStream_t)env.stream());
  } catch (...) {
  }
}

std::vector<Node *> Executor::materialize(const std::vector<Node *> &nodes) {
  Runtime &rt = Runtime::get();
  std::lock_guard<std::recursive_mutex> lk(rt.mtx);
  std::call_once(g_exit_hook, [] { std::atexit([] { g_exiting.store(true); }); });
  std::vector<Node *> out(nodes.size(), nullptr);
  std::vector<Node *> d0;
  std::vector<Sink> sinks;
  struct Held { Node *node; void *ptr; long long pitch; };
  std::vector<Held> held;
  std::unordered_map<Node *, size_t> slot;   // a node given twice is evaluated once
  for (size_t i = 0; i < nodes.size(); i++) {
    Node *n = nodes[i];
    if (!rt.owns(n)) throw MapError("materialize: unknown node");
    if (n->meta.numdim == D0) {
      d0.push_back(n);
      continue;
    }
    if (n->meta.numdim != D2) throw MapError("materialize: only D0 and D2 rasters are supported");
    if (n->kind == K_CONSTANT || (n->kind == K_DEVIN && n->dev->rows == 0)) {
      out[i] = n;
      continue;
    }
    if (slot.count(n)) continue;
    CudaEnv &env = CudaEnv::get();
    env.ensure_device();
    Held h{n, nullptr, pitch_for(n->meta.W(), n->meta.dtype)};
    const cudaError_t e = cudaMallocAsync(&h.ptr, (size_t)h.pitch * n->meta.H(), (cudaStream_t)env.stream());
    if (e != cudaSuccess) {
      for (const Held &o : held) cudaFreeAsync(o.ptr, (cudaStream_t)env.stream());
      cuda_check(e, "cudaMallocAsync(materialize)");
    }
    slot[n] = held.size();
    held.push_back(h);
    Sink s;
    s.node = n;
    s.dev = h.ptr;
    s.dev_pitch = h.pitch;
    sinks.push_back(s);
  }
  if (!d0.empty() || !sinks.empty()) {
    try {
      evaluate(d0, sinks);
    } catch (...) {
      for (const Held &o : held) cudaFreeAsync(o.ptr, (cudaStream_t)CudaEnv::get().stream());
      throw;
    }
  }
  std::vector<Node *> made(held.size(), nullptr);
  for (size_t k = 0; k < held.size(); k++) {
    const Held &h = held[k];
    Node *m = rt.dev_input(h.ptr, h.pitch, h.node->meta.ds, h.node->meta.dtype, h.node->meta.bs);
    m->dev->owned = true;
    m->meta.memorder = h.node->meta.memorder;
    made[k] = m;
  }
  for (size_t i = 0; i < nodes.size(); i++) {
    Node *n = nodes[i];
    if (out[i]) continue;
    if (n->meta.numdim == D0) {
      if (!n->has_value) throw MapError("materialize: a scalar was not computed");
      out[i] = rt.constant(n->value, Arr2(), n->meta.dtype, n->meta.memorder, Arr2());
    } else {
      out[i] = made[slot.at(n)];
    }
  }
  return out;
}

std::vector<std::string> Executor::compile_only(const std::vector<Node *> &targets, bool compile) {
  std::lock_guard<std::recursive_mutex> lk(Runtime::get().mtx);
  std::set<Node *> tset(targets.begin(), targets.end());
  Prepared P = prepare(targets, tset, compile);
  std::vector<std::string> srcs;
  for (auto &p : P.plans)
    if (!p.source.empty()) srcs.push_back(p.source);
  return srcs;
}

std::string Executor::describe_groups(const std::vector<Node *> &targets) {
  std::lock_guard<std::recursive_mutex> lk(Runtime::get().mtx);
  std::set<Node *> tset(targets.begin(), targets.end());
  FusionResult fr = fuse(collect(targets), tset);
  std::ostringstream s;
  for (auto &g : fr.groups) {
    s << skeleton_name(g->skeleton) << " in=[";
    for (Node *n : g->inputs) s << kind_name(n->kind) << ":" << n->id << " ";
    s << "] nodes=[";
    for (Node *n : g->nodes) s << kind_name(n->kind) << ":" << n->id << " ";
    s << "] out=[";
    for (Node *n : g->outputs) s << kind_name(n->kind) << ":" << n->id << " ";
    s << "]\n";
  }
  return s.str();
}

std::vector<PlainJob> Executor::schedule_for(const std::vector<Node *> &targets) {
  std::lock_guard<std::recursive_mutex> lk(Runtime::get().mtx);
  std::set<Node *> tset(targets.begin(), targets.end());
  Prepared P = prepare(targets, tset, false);
  return plain_schedule(P.fr.groups, P.plans);
}

void Executor::sync() {
  CudaEnv &env = CudaEnv::get();
  if (!env.device_ready()) return;
  cuda_check(cudaStreamSynchronize((cudaStream_t)env.stream()), "stream synchronize");
  uint32_t err = 0;
  cuda_check(cudaMemcpy(&err, env.err_word(), sizeof err, cudaMemcpyDeviceToHost), "error word read");
  if (err) {
    cuda_check(cudaMemset(env.err_word(), 0, sizeof err), "error word reset");
    std::string m = "device kernel reported an error:";
    if (err & 1) m += " shared-memory staging timed out;";
    if (err & 2) m += " invalid launch shape;";
    if (err & 4) m += " iteration limit reached before convergence;";
    if (err & 8) m += " spin-wait limit reached;";
    throw MapError(m);
  }
}

void Executor::evaluate(const std::vector<Node *> &targets_in, const std::vector<Sink> &sinks, bool async) {
  const double t0 = now_ms();
  Runtime &rt = Runtime::get();
  std::lock_guard<std::recursive_mutex> lk(rt.mtx);
  CudaEnv &env = CudaEnv::get();
  std::vector<Node *> targets = targets_in;
  for (auto &s : sinks) targets.push_back(s.node);
  for (Node *t : targets)
    if (!rt.owns(t)) throw MapError("evaluate: unknown node");
  std::set<Node *> tset(targets.begin(), targets.end());
  std::shared_ptr<Prepared> PP = prepare_cached(targets, tset);
  const Prepared &P = *PP;
  last = EvalStats();
  last.groups = (int)P.fr.groups.size();
  const int launches0 = env.launches();

  bool need_device = false;
  for (auto &g : P.fr.groups) if (g->skeleton != SK_HOST) need_device = true;
  for (Node *t : targets) if (t->meta.numdim != D0) need_device = true;
  if (!need_device) {
    for (auto &g : P.fr.groups) {
      Node *n = g->nodes[0];
      n->value = host_eval(n);
      n->has_value = true;
    }
    last.host_ms = now_ms() - t0;
    return;
  }
  env.ensure_device();
  cudaStream_t st = (cudaStream_t)env.stream();
  if (evaluate_streamed(P, targets, sinks)) {
    last.launches = env.launches() - launches0;
    last.host_ms = now_ms() - t0;
    return;
  }
  static bool pool_cfg = false;
  if (!pool_cfg) {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, env.device()) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    pool_cfg = true;
  }

  std::unordered_map<Node *, DevRaster> bufs;
  std::vector<void *> pinned;
  bool must_sync = !async;
  std::unordered_map<Node *, const Sink *> dev_sink;
  for (auto &s : sinks)
    if (s.dev) dev_sink[s.node] = &s;

  auto alloc_raster = [&](int dtype, int W, int H) {
    DevRaster r;
    r.dtype = dtype;
    r.W = W;
    r.H = H;
    r.pitch = pitch_for(W, dtype);
    cuda_check(cudaMallocAsync(&r.ptr, (size_t)r.pitch * H, st), "cudaMallocAsync");
    r.owned = true;
    return r;
  };
  std::function<DevRaster &(Node *)> get = [&](Node *n) -> DevRaster & {
    auto it = bufs.find(n);
    if (it != bufs.end()) return it->second;
    const int W = n->meta.W(), H = n->meta.H(), dt = n->meta.dtype;
    const size_t row = (size_t)W * dt_size(dt);
    if (n->kind == K_DEVIN) {
      if (n->dev->rows) throw MapError("a device input holding a row band is evaluated by row ranges only (ma_evalRows)");
      DevRaster r;
      r.ptr = n->dev->ptr;
      r.pitch = n->dev->pitch;
      r.dtype = dt;
      r.W = W;
      r.H = H;
      if (((uintptr_t)r.ptr & 127) != 0 || (r.pitch & 15) != 0) {   // realign for TMA and coalescing
        DevRaster c = alloc_raster(dt, W, H);
        cuda_check(cudaMemcpy2DAsync(c.ptr, c.pitch, r.ptr, r.pitch, row, H, cudaMemcpyDeviceToDevice, st), "realign copy");
        return bufs[n] = c;
      }
      return bufs[n] = r;
    }
    if (n->kind == K_HOSTIN) {
      DevRaster r = alloc_raster(dt, W, H);
      cuda_check(cudaMemcpy2DAsync(r.ptr, r.pitch, n->host->ptr, row, row, H, cudaMemcpyHostToDevice, st), "upload");
      return bufs[n] = r;
    }
    if (n->kind == K_READ) {
      BinHeader h = bin_read_header(n->path);
      void *pin = nullptr;
      cuda_check(cudaMallocHost(&pin, row * H), "cudaMallocHost");
      pinned.push_back(pin);
      bin_read_dense(n->path, h, pin);
      DevRaster r = alloc_raster(dt, W, H);
      cuda_check(cudaMemcpy2DAsync(r.ptr, r.pitch, pin, row, row, H, cudaMemcpyHostToDevice, st), "upload");
      must_sync = true;
      return bufs[n] = r;
    }
    throw MapError(std::string("raster of ") + kind_name(n->kind) + " #" + std::to_string(n->id) + " was not computed");
  };
  std::function<DevRaster(Node *)> alloc_out = [&](Node *o) -> DevRaster {
    auto ds = dev_sink.find(o);
    if (ds != dev_sink.end()) {
      const Sink *s = ds->second;
      if (((uintptr_t)s->dev & 127) == 0 && (s->dev_pitch & 15) == 0 &&
          s->dev_pitch >= (long long)o->meta.W() * (long long)dt_size(o->meta.dtype)) {
        DevRaster r;
        r.ptr = s->dev;
        r.pitch = s->dev_pitch;
        r.dtype = o->meta.dtype;
        r.W = o->meta.W();
        r.H = o->meta.H();
        return r;
      }
    }
    return alloc_raster(o->meta.dtype, o->meta.W(), o->meta.H());
  };

  // partial-result storage of zonal groups
  struct ZonalState { void *part = nullptr; long long slots = 0; long long cap = 0; void *res = nullptr; };
  std::unordered_map<int, ZonalState> zst;

  auto build_args = [&](const Group &g, const KernelPlan &K, int rx0, int ry0, int rx1, int ry1, uint64_t aux0,
                        uint64_t aux1) {
    uint64_t aux[4] = {aux0, aux1, 0, 0};
    return pack_args(g, K, get, bufs, rx0, ry0, rx1, ry1, aux, nullptr, true);
  };

  auto ensure_outputs = [&](const Group &g, const KernelPlan &K) {
    for (Node *o : K.out_rasters)
      if (!bufs.count(o)) bufs[o] = alloc_out(o);
    (void)g;
  };

  auto launch_region = [&](const Group &g, const KernelPlan &K, int rx0, int ry0, int rx1, int ry1) {
    const int tx = (rx1 - rx0 + K.tile_w - 1) / K.tile_w, ty = (ry1 - ry0 + K.tile_h - 1) / K.tile_h;
    const int tiles = tx * ty;
    KernelHandle kh = env.kernel(K.source, K.kname, K.smem_bytes);
    if (g.skeleton == SK_ZONAL) {
      ZonalState &z = zst[g.id];
      const int nz = (int)K.zonal.size();
      const int grid = std::min(tiles, env.sm_count() * 8);
      if (z.slots + grid > z.cap) throw MapError("zonal partial storage overflow");
      auto a = build_args(g, K, rx0, ry0, rx1, ry1, (uint64_t)(uintptr_t)z.part, (uint64_t)z.slots);
      env.launch(kh, grid, K.threads, K.smem_bytes, (CUstream_st *)st, a.data(), a.size());
      z.slots += grid;
      (void)nz;
    } else {
      // Local / Focal kernels run one CTA per tile on a tx x ty grid (regions of
      // more than kMaxGridY tile rows in vertical pieces) and wait for their
      // predecessor in the kernel (griddep_wait), so they are dependent launches
      for (int y = ry0; y < ry1; y += kMaxGridY * K.tile_h) {
        const int ye = std::min(ry1, y + kMaxGridY * K.tile_h);
        const int pty = (ye - y + K.tile_h - 1) / K.tile_h;
        auto a = build_args(g, K, rx0, y, rx1, ye, 0, 0);
        if (rt.dependent_launch && focal_tune().pdl)
          env.launch_pdl(kh, tx, pty, K.threads, K.smem_bytes, (CUstream_st *)st, a.data());
        else
          env.launch_2d(kh, tx, pty, K.threads, K.smem_bytes, (CUstream_st *)st, a.data());
      }
      (void)ty;
    }
  };

  auto zonal_begin = [&](const Group &g, const KernelPlan &K) {
    ZonalState &z = zst[g.id];
    if (z.part) return;
    const int nz = (int)K.zonal.size();
    long long cap;
    if (rt.exec_mode == EXEC_PLAIN) {
      const int nbx = (g.W + g.BS0 - 1) / g.BS0, nby = (g.H + g.BS1 - 1) / g.BS1;
      const int tpb = ((g.BS0 + K.tile_w - 1) / K.tile_w) * ((g.BS1 + K.tile_h - 1) / K.tile_h);
      cap = (long long)nbx * nby * std::min(tpb, env.sm_count() * 8);
    } else {
      cap = env.sm_count() * 8;
    }
    cuda_check(cudaMallocAsync(&z.part, (size_t)cap * nz * 8, st), "cudaMallocAsync(partials)");
    cuda_check(cudaMallocAsync(&z.res, (size_t)nz * 8, st), "cudaMallocAsync(results)");
    z.cap = cap;
    z.slots = 0;
  };

  auto zonal_finish = [&](const Group &g, const KernelPlan &K) {
    ZonalState &z = zst[g.id];
    const int nz = (int)K.zonal.size();
    KernelHandle kf = env.kernel(K.source, K.kname_final, 0);
    struct { uint64_t part; int64_t nslots; uint64_t res; uint64_t pad; } fa{(uint64_t)(uintptr_t)z.part, z.slots,
                                                                              (uint64_t)(uintptr_t)z.res, 0};
    env.launch(kf, 1, K.threads, 0, (CUstream_st *)st, &fa, sizeof fa);
    std::vector<uint64_t> res(nz);
    cuda_check(cudaMemcpyAsync(res.data(), z.res, (size_t)nz * 8, cudaMemcpyDeviceToHost, st), "result read-back");
    cuda_check(cudaStreamSynchronize(st), "stream synchronize");
    for (int i = 0; i < nz; i++) {
      Node *n = K.zonal[i];
      Variant v;
      std::memset(&v, 0, sizeof v);
      v.dtype = n->meta.dtype;
      std::memcpy(&v.u, &res[i], dt_size(v.dtype));
      n->value = v;
      n->has_value = true;
    }
    cudaFreeAsync(z.part, st);
    cudaFreeAsync(z.res, st);
    z.part = z.res = nullptr;
  };

  auto run_host = [&](const Group &g) {
    Node *n = g.nodes[0];
    n->value = host_eval(n);
    n->has_value = true;
  };

  // groups whose every output is one known value (Predictor): filled, not launched
  std::unordered_map<Node *, Variant> fixed;
  std::vector<char> predicted(P.fr.groups.size(), 0), filled(P.fr.groups.size(), 0);
  if (rt.prediction)
    for (auto &gp : P.fr.groups)
      predicted[gp->id] = predict_group(*gp, P.plans[gp->id], fixed, rt.border) ? 1 : 0;
  auto fill_predicted = [&](const Group &g, const KernelPlan &K) {
    ensure_outputs(g, K);
    for (Node *o : K.out_rasters) {
      DevRaster &r = bufs.at(o);
      const Variant v = fixed.at(o);
      const int es = (int)dt_size(o->meta.dtype);
      if (!env.fill_2d(r.ptr, (size_t)r.pitch, &v.u, es, (size_t)o->meta.W(), (size_t)o->meta.H(), (CUstream_st *)st))
        throw MapError("prediction: no fill for this element size");
    }
    last.predicted++;
  };

  try {
    if (rt.exec_mode == EXEC_FUSED) {
      for (auto &gp : P.fr.groups) {
        const Group &g = *gp;
        const KernelPlan &K = P.plans[g.id];
        if (g.skeleton == SK_HOST) { run_host(g); continue; }
        if (predicted[g.id]) { fill_predicted(g, K); continue; }
        if (g.skeleton == SK_RADIAL || g.skeleton == SK_SPREAD) {
          run_scan_group(g, K, bufs, get, alloc_out);
          continue;
        }
        ensure_outputs(g, K);
        if (g.skeleton == SK_ZONAL) zonal_begin(g, K);
        launch_region(g, K, 0, 0, g.W, g.H);
        if (g.skeleton == SK_ZONAL) zonal_finish(g, K);
      }
    } else {
      std::vector<PlainJob> jobs = plain_schedule(P.fr.groups, P.plans);
      for (const PlainJob &j : jobs) {
        const Group &g = *P.fr.groups[j.group];
        const KernelPlan &K = P.plans[g.id];
        switch (j.kind) {
          case 3: run_host(g); break;
          case 1: run_scan_group(g, K, bufs, get, alloc_out); break;
          case 2: zonal_finish(g, K); break;
          default: {
            if (predicted[g.id]) {
              if (!filled[g.id]) fill_predicted(g, K);   // one fill, at the group's first block, for all its blocks
              filled[g.id] = 1;
              break;
            }
            ensure_outputs(g, K);
            if (g.skeleton == SK_ZONAL) zonal_begin(g, K);
            const int rx0 = j.bx * g.BS0, ry0 = j.by * g.BS1;
            launch_region(g, K, rx0, ry0, std::min(rx0 + g.BS0, g.W), std::min(ry0 + g.BS1, g.H));
          }
        }
      }
    }
    // sinks
    for (const Sink &s : sinks) {
      Node *n = s.node;
      if (n->meta.numdim == D0) continue;
      DevRaster &r = get(n);
      const size_t row = (size_t)n->meta.W() * dt_size(n->meta.dtype);
      if (s.host) {
        cuda_check(cudaMemcpy2DAsync(s.host, row, r.ptr, r.pitch, row, n->meta.H(), cudaMemcpyDeviceToHost, st), "download");
        must_sync = true;
      }
      if (s.dev && r.ptr != s.dev)
        cuda_check(cudaMemcpy2DAsync(s.dev, s.dev_pitch, r.ptr, r.pitch, row, n->meta.H(), cudaMemcpyDeviceToDevice, st),
                   "device copy");
    }
    // writes
    for (Node *t : P.order) {
      if (t->kind != K_WRITE) continue;
      Node *src = t->prev[0];
      DevRaster &r = get(src);
      const size_t row = (size_t)src->meta.W() * dt_size(src->meta.dtype);
      void *pin = nullptr;
      cuda_check(cudaMallocHost(&pin, row * src->meta.H()), "cudaMallocHost");
      pinned.push_back(pin);
      cuda_check(cudaMemcpy2DAsync(pin, row, r.ptr, r.pitch, row, src->meta.H(), cudaMemcpyDeviceToHost, st), "download");
      cuda_check(cudaStreamSynchronize(st), "stream synchronize");
      BinHeader h;
      h.dtype = src->meta.dtype;
      h.numdim = D2;
      h.ds0 = src->meta.W();
      h.ds1 = src->meta.H();
      h.memorder = (src->meta.memorder == ROW) ? ROW : ROW + BLK;
      h.bs0 = src->meta.BS0();
      h.bs1 = src->meta.BS1();
      bin_write_dense(t->path, h, pin);
    }
  } catch (...) {
    cudaStreamSynchronize(st);
    for (auto &kv : bufs) if (kv.second.owned) cudaFree(kv.second.ptr);
    for (void *p : pinned) cudaFreeHost(p);
    throw;
  }
  for (auto &kv : bufs)
    if (kv.second.owned) cudaFreeAsync(kv.second.ptr, st);
  if (must_sync || !pinned.empty()) {
    sync();
    for (void *p : pinned) cudaFreeHost(p);
  }
  last.launches = env.launches() - launches0;
  last.host_ms = now_ms() - t0;
}

// ------------------------------------------------------------ streamed bands
//
// A program from host rasters to host rasters made of Local / Focal groups runs
// band by band: band b covers raster rows [y0, y1); group g computes rows
// [y0 - need(g), y1 + need(g)) where need(g) is the halo its consumers still
// require, so the output rows of the band only ever see values computed from
// true neighbours, and border decisions use the whole raster's geometry
// (kernels address rasters in raster rows through a virtual base), making the
// result identical to whole-raster evaluation. Each of kSlots buffer sets holds
// every raster's rows [y0 - M, y1 + M) plus a tile of padding (M = the largest
// margin); uploads run on one stream, kernels on the engine's stream and
// downloads on a third, chained by events, so band b+1 uploads while band b
// computes and band b-1 downloads.

namespace {

constexpr int kSlots = 3;

struct BandStreams {
  cudaStream_t up = nullptr, down = nullptr;
  cudaEvent_t ev_up[kSlots] = {}, ev_comp[kSlots] = {}, ev_down[kSlots] = {}, ev_alloc = nullptr;
  bool ready = false;
  void init() {
    if (ready) return;
    cuda_check(cudaStreamCreateWithFlags(&up, cudaStreamNonBlocking), "cudaStreamCreate");
    cuda_check(cudaStreamCreateWithFlags(&down, cudaStreamNonBlocking), "cudaStreamCreate");
    for (int i = 0; i < kSlots; i++) {
      cuda_check(cudaEventCreateWithFlags(&ev_up[i], cudaEventDisableTiming), "cudaEventCreate");
      cuda_check(cudaEventCreateWithFlags(&ev_comp[i], cudaEventDisableTiming), "cudaEventCreate");
      cuda_check(cudaEventCreateWithFlags(&ev_down[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    cuda_check(cudaEventCreateWithFlags(&ev_alloc, cudaEventDisableTiming), "cudaEventCreate");
    ready = true;
  }
};

BandStreams &band_streams() {
  static BandStreams b;
  return b;
}

}  // namespace

// Row structure of a program made only of Local / Focal groups over one raster
// shape: need[g] = rows beyond a requested row range that group g must still
// produce for the groups that read it; M = rows beyond the range that the
// program reads from its inputs. False (with the reason) for other programs.
struct RowPlan {
  int W = -1, H = -1, th_max = 1, hy_max = 0, M = 0;
  std::map<const Group *, int> need;
  std::set<Node *> produced;
  std::map<Node *, const Group *> producer;
  std::set<Node *> inputs;
};
static bool row_plan(const FusionResult &fr, const std::vector<KernelPlan> &plans, RowPlan &R, std::string &why) {
  for (auto &gp : fr.groups) {
    const Group &g = *gp;
    if (g.skeleton != SK_LOCAL && g.skeleton != SK_FOCAL) {
      why = std::string("group of skeleton ") + skeleton_name(g.skeleton) + " (only Local and Focal groups run by rows)";
      return false;
    }
    if (R.W < 0) {
      R.W = g.W;
      R.H = g.H;
    } else if (g.W != R.W || g.H != R.H) {
      why = "groups of different raster shapes";
      return false;
    }
    const KernelPlan &K = plans[g.id];
    R.th_max = std::max(R.th_max, K.tile_h);
    R.hy_max = std::max(R.hy_max, K.halo_y);
    for (Node *o : K.out_rasters) {
      R.produced.insert(o);
      R.producer[o] = &g;
    }
  }
  if (R.W <= 0 || R.H <= 0) {
    why = "no raster group";
    return false;
  }
  for (auto &gp : fr.groups)
    for (Node *n : plans[gp->id].in_rasters)
      if (!R.produced.count(n)) R.inputs.insert(n);
  for (auto it = fr.groups.rbegin(); it != fr.groups.rend(); ++it) {
    const Group *c = it->get();
    const KernelPlan &K = plans[c->id];
    const int nc = R.need[c];
    for (Node *n : K.in_rasters) {
      auto p = R.producer.find(n);
      if (p != R.producer.end()) R.need[p->second] = std::max(R.need[p->second], nc + K.halo_y);
    }
  }
  for (auto &gp : fr.groups) R.M = std::max(R.M, R.need[gp.get()] + plans[gp->id].halo_y);
  return true;
}

void Executor::evaluate_rows(const std::vector<Node *> &targets_in, const std::vector<Sink> &sinks, int y0, int y1) {
  const double t0 = now_ms();
  Runtime &rt = Runtime::get();
  std::lock_guard<std::recursive_mutex> lk(rt.mtx);
  CudaEnv &env = CudaEnv::get();
  if (rt.exec_mode != EXEC_FUSED) throw MapError("evalRows: row ranges run fused launches only");
  std::vector<Node *> targets = targets_in;
  for (auto &s : sinks) {
    if (!s.dev || s.host) throw MapError("evalRows: every output goes to device memory");
    targets.push_back(s.node);
  }
  for (Node *t : targets) {
    if (!rt.owns(t)) throw MapError("evalRows: unknown node");
    if (t->meta.numdim != D2) throw MapError("evalRows: every output is a 2-D raster");
  }
  std::set<Node *> tset(targets.begin(), targets.end());
  std::shared_ptr<Prepared> PP = prepare_cached(targets, tset);
  const Prepared &P = *PP;
  for (Node *n : P.order)
    if (n->kind == K_WRITE) throw MapError("evalRows: a program with file writes runs whole");
  RowPlan R;
  std::string why;
  if (!row_plan(P.fr, P.plans, R, why)) throw MapError("evalRows: " + why);
  const int W = R.W, H = R.H;
  if (y0 < 0 || y1 > H || y0 >= y1)
    throw MapError("evalRows: rows [" + std::to_string(y0) + ", " + std::to_string(y1) + ") are not a range of the " +
                   std::to_string(H) + " rows");
  for (const Sink &s : sinks) {
    if (!R.produced.count(s.node)) throw MapError("evalRows: an output is not computed by a raster group");
    if (s.dev_pitch < (long long)W * (long long)dt_size(s.node->meta.dtype)) throw MapError("evalRows: pitch smaller than a row");
  }
  const int ya = std::max(0, y0 - R.M), yb = std::min(H, y1 + R.M);
  last = EvalStats();
  last.groups = (int)P.fr.groups.size();
  const int launches0 = env.launches();
  env.ensure_device();
  cudaStream_t st = (cudaStream_t)env.stream();
  std::unordered_map<Node *, DevRaster> bufs;
  for (Node *n : R.inputs) {
    if (n->kind != K_DEVIN) throw MapError("evalRows: every input is a device raster (ma_fromDevice / ma_fromDeviceRows)");
    if (n->meta.W() != W || n->meta.H() != H) throw MapError("evalRows: inputs of different raster shapes");
    const DevData &d = *n->dev;
    if (((uintptr_t)d.ptr & 15) != 0 || (d.pitch & 15) != 0)
      throw MapError("evalRows: device inputs must start on 16 bytes with a pitch multiple of 16 bytes");
    DevRaster r;
    r.dtype = n->meta.dtype;
    r.W = W;
    r.H = H;
    r.pitch = d.pitch;
    if (d.rows) {
      if (d.row0 > ya || d.row0 + d.rows < yb)
        throw MapError("evalRows: an input holds rows [" + std::to_string(d.row0) + ", " + std::to_string(d.row0 + d.rows) +
                       ") but rows [" + std::to_string(ya) + ", " + std::to_string(yb) + ") are read");
      r.org = d.row0;
      r.rows = d.rows;
      r.ptr = (void *)((uintptr_t)d.ptr - (uintptr_t)((long long)d.row0 * d.pitch));
    } else {
      r.org = ya;
      r.rows = H - ya;
      r.ptr = d.ptr;
    }
    bufs[n] = r;
  }
  std::map<Node *, const Sink *> sink_of;
  for (const Sink &s : sinks) sink_of[s.node] = &s;
  std::vector<void *> allocs;
  std::vector<std::pair<const Sink *, Node *>> copies;
  try {
    const int rows_alloc = (yb - ya) + R.th_max + R.hy_max + 1;
    for (Node *n : R.produced) {
      DevRaster r;
      r.dtype = n->meta.dtype;
      r.W = W;
      r.H = H;
      auto sk = sink_of.find(n);
      if (sk != sink_of.end() && R.need[R.producer[n]] == 0 && ((uintptr_t)sk->second->dev & 15) == 0 &&
          (sk->second->dev_pitch & 15) == 0) {
        // written straight into the caller's rows [y0, y1)
        r.pitch = sk->second->dev_pitch;
        r.org = y0;
        r.rows = y1 - y0;
        r.ptr = (void *)((uintptr_t)sk->second->dev - (uintptr_t)((long long)y0 * r.pitch));
      } else {
        r.pitch = pitch_for(W, r.dtype);
        void *p = nullptr;
        cuda_check(cudaMallocAsync(&p, (size_t)r.pitch * rows_alloc, st), "cudaMallocAsync(rows)");
        allocs.push_back(p);
        r.org = ya;
        r.rows = rows_alloc;
        r.ptr = (void *)((uintptr_t)p - (uintptr_t)((long long)ya * r.pitch));
        if (sk != sink_of.end()) copies.push_back({sk->second, n});
      }
      bufs[n] = r;
    }
    std::function<DevRaster &(Node *)> get = [&](Node *n) -> DevRaster & {
      auto it = bufs.find(n);
      if (it == bufs.end()) throw MapError("evalRows: raster not bound");
      return it->second;
    };
    for (auto &gp : P.fr.groups) {
      const Group &g = *gp;
      const KernelPlan &K = P.plans[g.id];
      const int ry0 = std::max(0, y0 - R.need[&g]), ry1 = std::min(H, y1 + R.need[&g]);
      const int tx = (W + K.tile_w - 1) / K.tile_w;
      KernelHandle kh = env.kernel(K.source, K.kname, K.smem_bytes);
      uint64_t aux[4] = {0, 0, 0, 0};
      for (int y = ry0; y < ry1; y += kMaxGridY * K.tile_h) {
        const int ye = std::min(ry1, y + kMaxGridY * K.tile_h);
        auto a = pack_args(g, K, get, bufs, 0, y, W, ye, aux);
        env.launch_2d(kh, tx, (ye - y + K.tile_h - 1) / K.tile_h, K.threads, K.smem_bytes, (CUstream_st *)st, a.data());
      }
    }
    for (auto &c : copies) {
      const DevRaster &r = bufs.at(c.second);
      const size_t row = (size_t)W * dt_size(c.second->meta.dtype);
      cuda_check(cudaMemcpy2DAsync(c.first->dev, c.first->dev_pitch, (const char *)r.ptr + (long long)y0 * r.pitch, r.pitch,
                                   row, y1 - y0, cudaMemcpyDeviceToDevice, st),
                 "row copy");
    }
    for (void *p : allocs) cudaFreeAsync(p, st);
    allocs.clear();
    sync();
  } catch (...) {
    cudaStreamSynchronize(st);
    for (void *p : allocs) cudaFreeAsync(p, st);
    throw;
  }
  last.launches = env.launches() - launches0;
  last.host_ms = now_ms() - t0;
}

int Executor::row_margin(const std::vector<Node *> &targets) {
  Runtime &rt = Runtime::get();
  std::lock_guard<std::recursive_mutex> lk(rt.mtx);
  for (Node *t : targets)
    if (!rt.owns(t)) throw MapError("rowMargin: unknown node");
  std::set<Node *> tset(targets.begin(), targets.end());
  Prepared P = prepare(targets, tset, false);
  RowPlan R;
  std::string why;
  if (!row_plan(P.fr, P.plans, R, why)) throw MapError("rowMargin: " + why);
  return R.M;
}

bool Executor::evaluate_streamed(const Prepared &P, const std::vector<Node *> &targets, const std::vector<Sink> &sinks) {
  Runtime &rt = Runtime::get();
  if (rt.exec_mode != EXEC_FUSED || rt.stream_rows < 0 || sinks.empty()) return false;
  std::set<Node *> sink_nodes;
  for (const Sink &s : sinks) {
    if (!s.host || s.dev || s.node->meta.numdim != D2) return false;
    sink_nodes.insert(s.node);
  }
  for (Node *t : targets)
    if (!sink_nodes.count(t)) return false;
  for (Node *n : P.order)
    if (n->kind == K_WRITE) return false;
  RowPlan R;
  std::string why;
  if (!row_plan(P.fr, P.plans, R, why)) return false;
  const int W = R.W, H = R.H, th_max = R.th_max, hy_max = R.hy_max, M = R.M;
  const std::set<Node *> &produced = R.produced;
  std::map<const Group *, int> &need = R.need;
  for (Node *s : sink_nodes)
    if (!produced.count(s)) return false;
  std::vector<Node *> host_in, dev_in;
  for (Node *n : R.inputs) {
    if (n->meta.W() != W || n->meta.H() != H) return false;
    if (n->kind == K_HOSTIN) {
      host_in.push_back(n);
    } else if (n->kind == K_DEVIN) {
      if (n->dev->rows || ((uintptr_t)n->dev->ptr & 127) != 0 || (n->dev->pitch & 15) != 0) return false;
      dev_in.push_back(n);
    } else {
      return false;
    }
  }
  size_t row_bytes = 0;
  for (Node *n : host_in) row_bytes += (size_t)W * dt_size(n->meta.dtype);
  for (Node *n : sink_nodes) row_bytes += (size_t)W * dt_size(n->meta.dtype);
  int B;
  if (rt.stream_rows > 0) {
    B = rt.stream_rows;
    if (B >= H) return false;
  } else {
    B = (int)std::min<size_t>((size_t)H, std::max<size_t>(64, ((size_t)32 << 20) / std::max<size_t>(row_bytes, 1)));
    B = std::max(32, B / 32 * 32);
    if ((long long)H < 4LL * B) return false;
  }

  CudaEnv &env = CudaEnv::get();
  cudaStream_t st = (cudaStream_t)env.stream();
  BandStreams &bs = band_streams();
  bs.init();
  const int nb = (H + B - 1) / B;
  const int slots = std::min(kSlots, nb);
  const int rows_alloc = std::min(H, B + 2 * M) + th_max + hy_max + 1;
  std::vector<Node *> banded(host_in.begin(), host_in.end());
  banded.insert(banded.end(), produced.begin(), produced.end());
  std::vector<std::unordered_map<Node *, DevRaster>> slot_buf(slots);
  std::vector<void *> allocs;
  auto release = [&]() {
    for (void *p : allocs) cudaFreeAsync(p, st);
    allocs.clear();
  };
  try {
    for (int sidx = 0; sidx < slots; sidx++)
      for (Node *n : banded) {
        DevRaster r;
        r.dtype = n->meta.dtype;
        r.W = W;
        r.H = H;
        r.pitch = pitch_for(W, r.dtype);
        void *p = nullptr;
        cuda_check(cudaMallocAsync(&p, (size_t)r.pitch * rows_alloc, st), "cudaMallocAsync(band)");
        allocs.push_back(p);
        r.ptr = p;   // real address until a band is bound
        r.rows = rows_alloc;
        slot_buf[sidx][n] = r;
      }
    cuda_check(cudaEventRecord(bs.ev_alloc, st), "cudaEventRecord");
    cuda_check(cudaStreamWaitEvent(bs.up, bs.ev_alloc, 0), "cudaStreamWaitEvent");
    std::vector<void *> real(allocs);
    std::unordered_map<Node *, DevRaster> bufs;
    std::function<DevRaster &(Node *)> get = [&](Node *n) -> DevRaster & {
      auto it = bufs.find(n);
      if (it == bufs.end()) throw MapError("streamed evaluation: raster not bound");
      return it->second;
    };
    for (int b = 0; b < nb; b++) {
      const int sidx = b % slots;
      const int y0 = b * B, y1 = std::min(H, y0 + B);
      const int ya = std::max(0, y0 - M), yb = std::min(H, y1 + M);
      if (b >= slots) cuda_check(cudaStreamWaitEvent(bs.up, bs.ev_down[sidx], 0), "cudaStreamWaitEvent");
      bufs.clear();
      size_t ai = (size_t)sidx * banded.size();
      for (Node *n : banded) {
        DevRaster r = slot_buf[sidx][n];
        void *base = real[ai++];
        r.org = ya;
        r.ptr = (void *)((uintptr_t)base - (uintptr_t)((long long)ya * r.pitch));
        bufs[n] = r;
      }
      for (Node *n : dev_in) {
        DevRaster r;
        r.ptr = n->dev->ptr;
        r.pitch = n->dev->pitch;
        r.dtype = n->meta.dtype;
        r.W = W;
        r.H = H;
        r.org = ya;
        r.rows = H - ya;
        bufs[n] = r;
      }
      for (Node *n : host_in) {
        const DevRaster &r = bufs[n];
        const size_t row = (size_t)W * dt_size(n->meta.dtype);
        cuda_check(cudaMemcpy2DAsync((char *)r.ptr + (long long)ya * r.pitch, r.pitch,
                                     (const char *)n->host->ptr + (size_t)ya * row, row, row, yb - ya,
                                     cudaMemcpyHostToDevice, bs.up),
                   "band upload");
      }
      cuda_check(cudaEventRecord(bs.ev_up[sidx], bs.up), "cudaEventRecord");
      cuda_check(cudaStreamWaitEvent(st, bs.ev_up[sidx], 0), "cudaStreamWaitEvent");
      for (auto &gp : P.fr.groups) {
        const Group &g = *gp;
        const KernelPlan &K = P.plans[g.id];
        const int ry0 = std::max(0, y0 - need[&g]), ry1 = std::min(H, y1 + need[&g]);
        const int tx = (W + K.tile_w - 1) / K.tile_w;
        KernelHandle kh = env.kernel(K.source, K.kname, K.smem_bytes);
        uint64_t aux[4] = {0, 0, 0, 0};
        for (int y = ry0; y < ry1; y += kMaxGridY * K.tile_h) {
          const int ye = std::min(ry1, y + kMaxGridY * K.tile_h);
          auto a = pack_args(g, K, get, bufs, 0, y, W, ye, aux);
          env.launch_2d(kh, tx, (ye - y + K.tile_h - 1) / K.tile_h, K.threads, K.smem_bytes, (CUstream_st *)st,
                        a.data());
        }
      }
      cuda_check(cudaEventRecord(bs.ev_comp[sidx], st), "cudaEventRecord");
      cuda_check(cudaStreamWaitEvent(bs.down, bs.ev_comp[sidx], 0), "cudaStreamWaitEvent");
      for (const Sink &s : sinks) {
        const DevRaster &r = bufs.at(s.node);
        const size_t row = (size_t)W * dt_size(s.node->meta.dtype);
        cuda_check(cudaMemcpy2DAsync((char *)s.host + (size_t)y0 * row, row, (const char *)r.ptr + (long long)y0 * r.pitch,
                                     r.pitch, row, y1 - y0, cudaMemcpyDeviceToHost, bs.down),
                   "band download");
      }
      cuda_check(cudaEventRecord(bs.ev_down[sidx], bs.down), "cudaEventRecord");
    }
    cuda_check(cudaStreamSynchronize(bs.down), "stream synchronize");
    cuda_check(cudaStreamSynchronize(bs.up), "stream synchronize");
    release();
    sync();
  } catch (...) {
    cudaStreamSynchronize(bs.up);
    cudaStreamSynchronize(bs.down);
    cudaStreamSynchronize(st);
    release();
    throw;
  }
  last.bands = nb;
  return true;
}

}  // namespace mapb

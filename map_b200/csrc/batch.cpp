// Batched persistent execution and tile-shape autotuning (see batch.hpp).
#include "batch.hpp"
#include "binfile.hpp"
#include "cuda_env.hpp"
#include "fusion.hpp"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <unordered_map>

namespace mapb {

namespace {

std::string hex16(const std::string &s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) { h ^= c; h *= 1099511628211ull; }
  char b[17];
  std::snprintf(b, sizeof b, "%016llx", (unsigned long long)h);
  return b;
}

long long pitch_for(int W, int dt) {
  long long b = (long long)W * (long long)dt_size(dt);
  return (b + 127) / 128 * 128;
}

// ------------------------------------------------------------------ tuning cache

std::mutex g_tune_mtx;
std::map<std::string, TileCfg> g_tune;
bool g_tune_loaded = false;

std::string tune_file() { return CudaEnv::cache_dir() + "/tune.txt"; }

void tune_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  std::ifstream f(tune_file());
  std::string key;
  TileCfg c;
  while (f >> key >> c.tw >> c.th >> c.nt)
    if (tile_cfg_valid(c)) g_tune[key] = c;
}

void tune_store(const std::string &key, const TileCfg &c) {
  g_tune[key] = c;
  std::ofstream f(tune_file(), std::ios::app);
  if (f) f << key << " " << c.tw << " " << c.th << " " << c.nt << "\n";
}

}  // namespace

// (skeleton, halo, staged and output dtypes, shape bucket = log2 of the short side)
std::string tune_key(const Group &g, const KernelPlan &p) {
  std::ostringstream k;
  k << skeleton_name(g.skeleton) << "/h" << p.halo_x << "x" << p.halo_y << "/in";
  for (Node *n : p.in_rasters) k << dt_name(n->meta.dtype);
  k << "/out";
  for (Node *n : p.out_rasters) k << dt_name(n->meta.dtype);
  int side = std::max(1, std::min(g.W, g.H));
  k << "/b" << (int)std::floor(std::log2((double)side));
  k << "/n" << hex16(p.body).substr(0, 8);
  return k.str();
}

// Tile shape of a kind chosen in the form it runs: for each candidate shape, one
// persistent launch over the tiles of all the kind's members, timed with events;
// the winner is cached per (skeleton, halo, dtypes, largest member's shape bucket,
// body). Candidates that do not fit the persistent module's 256 threads are skipped.
TileCfg autotune_kind(const std::vector<const Group *> &members, const std::function<DevRaster &(Node *)> &get,
                      std::unordered_map<Node *, DevRaster> &bufs) {
  const Group *big = members[0];
  for (const Group *g : members)
    if ((long long)g->W * g->H > (long long)big->W * big->H) big = g;
  if (big->skeleton != SK_LOCAL && big->skeleton != SK_FOCAL) return TileCfg();
  KernelPlan base = generate_kernel(*big);
  const std::string key = tune_key(*big, base) + "/m" + std::to_string(members.size());
  {
    std::lock_guard<std::mutex> lk(g_tune_mtx);
    tune_load();
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  CudaEnv &env = CudaEnv::get();
  cudaStream_t st = (cudaStream_t)env.stream();
  static const int cand[][2] = {{64, 32}, {128, 16}, {32, 32}, {64, 16}, {128, 32}, {32, 64}, {64, 64}, {32, 128}};
  TileCfg best;
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  cuda_check(cudaEventCreate(&e0), "cudaEventCreate");
  cuda_check(cudaEventCreate(&e1), "cudaEventCreate");
  for (auto &c : cand) {
    TileCfg cfg;
    cfg.tw = c[0];
    cfg.th = c[1];
    cfg.nt = 256;
    if (!tile_cfg_valid(cfg)) continue;
    KernelPlan P0 = generate_kernel(*big, cfg);
    std::vector<unsigned char> args;
    std::vector<uint32_t> items;   // (kind 0, member, tile, pad)
    uint32_t mi = 0;
    for (const Group *g : members) {
      KernelPlan P = generate_kernel(*g, cfg);
      uint64_t aux[4] = {0, 0, 0, 0};
      auto a = pack_args(*g, P, get, bufs, 0, 0, g->W, g->H, aux);
      args.insert(args.end(), a.begin(), a.end());
      const int tiles = ((g->W + cfg.tw - 1) / cfg.tw) * ((g->H + cfg.th - 1) / cfg.th);
      for (int t = 0; t < tiles; t++) {
        items.push_back(0u);
        items.push_back(mi);
        items.push_back((uint32_t)t);
        items.push_back(0u);
      }
      mi++;
    }
    PersistentModule pm = build_persistent_module({&P0});
    KernelHandle kh = env.kernel(pm.source, pm.kname, pm.smem);
    const int grid = env.sm_count() * std::max(1, env.occupancy(kh, 256, pm.smem));
    void *d = nullptr;
    const size_t nitem = items.size() / 4;
    const size_t bytes = 256 + args.size() + items.size() * 4;
    cuda_check(cudaMallocAsync(&d, bytes, st), "cudaMallocAsync(tuning)");
    char *dargs = (char *)d + 256, *ditems = dargs + args.size();
    cuda_check(cudaMemcpyAsync(dargs, args.data(), args.size(), cudaMemcpyHostToDevice, st), "upload");
    cuda_check(cudaMemcpyAsync(ditems, items.data(), items.size() * 4, cudaMemcpyHostToDevice, st), "upload");
    struct {
      uint64_t items;
      int64_t n;
      uint64_t counter;
      uint64_t err;
      uint64_t args[1];
    } ba{(uint64_t)(uintptr_t)ditems, (int64_t)nitem, (uint64_t)(uintptr_t)d, (uint64_t)(uintptr_t)env.err_word(),
         {(uint64_t)(uintptr_t)dargs}};
    auto run = [&]() {
      cuda_check(cudaMemsetAsync(d, 0, 4, st), "cudaMemsetAsync");
      env.launch(kh, std::min<int>(grid, (int)nitem), 256, pm.smem, (CUstream_st *)st, &ba, sizeof ba);
    };
    run();
    cuda_check(cudaEventRecord(e0, st), "cudaEventRecord");
    for (int r = 0; r < 3; r++) run();
    cuda_check(cudaEventRecord(e1, st), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0;
    cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    cuda_check(cudaFreeAsync(d, st), "cudaFreeAsync");
    if (ms < best_ms) {
      best_ms = ms;
      best = cfg;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lk(g_tune_mtx);
  tune_store(key, best);
  return best;
}

// ------------------------------------------------------------------ persistent module

PersistentModule build_persistent_module(const std::vector<const KernelPlan *> &kinds) {
  size_t bar_off = 16;
  for (const KernelPlan *p : kinds) {
    if (p->threads != 256) throw MapError("persistent module: tile configurations must use 256 threads");
    if (!p->tma.empty()) bar_off = std::max(bar_off, (p->bar_off + 15) / 16 * 16);
  }
  PersistentModule pm;
  pm.smem = bar_off + 16;
  std::ostringstream src;
  src << "#include \"map_common.cuh\"\n";
  for (size_t k = 0; k < kinds.size(); k++) src << "namespace k" << k << " {\n" << kinds[k]->body << "}\n";
  src << "struct BItem { u32 kind, inst, tile, pad; };\n"
      << "struct BatchArgs { u64 items; s64 n; u64 counter; u64 err; u64 args[" << kinds.size() << "]; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(256) KNAME(const __grid_constant__ BatchArgs b) {\n"
      << "  extern __shared__ __align__(128) unsigned char smem[];\n"
      << "  __shared__ int item_s[2];\n"
      << "  u64 *bar = (u64 *)(smem + " << bar_off << ");\n"
      << "  if (threadIdx.x == 0) { mbar_init(bar, 1); fence_mbar_init(); item_s[0] = atomicAdd((int *)b.counter, 1); }\n"
      << "  __syncthreads();\n"
      << "  u32 phase = 0;\n"
      << "  const BItem *items = (const BItem *)b.items;\n"
      // the next item's index is claimed while the current tile runs (its atomic's latency is hidden)
      << "  for (int slot = 0;; slot ^= 1) {\n"
      << "    const int i = item_s[slot];\n"
      << "    if (i >= b.n) break;\n"
      << "    if (threadIdx.x == 0) item_s[slot ^ 1] = atomicAdd((int *)b.counter, 1);\n"
      << "    const BItem w = items[i];\n"
      << "    bool ok = true;\n"
      << "    switch (w.kind) {\n";
  for (size_t k = 0; k < kinds.size(); k++)
    src << "      case " << k << ": ok = k" << k << "::run_tile(((const k" << k << "::Args *)b.args[" << k
        << "])[w.inst], (int)w.tile, smem, bar, phase, true); break;\n";
  src << "      default: skel_fail((u32 *)b.err, ERR_BAD_LAUNCH); ok = false;\n"
      << "    }\n"
      // a barrier that also makes the stop decision uniform: the claimed index is
      // visible afterwards, and this slot may be rewritten
      << "    if (__syncthreads_or(!ok)) break;\n"
      << "  }\n"
      << "}\n";
  pm.source = src.str();
  pm.kname = "map_batch_" + hex16(pm.source).substr(0, 12);
  size_t pos;
  while ((pos = pm.source.find("KNAME")) != std::string::npos) pm.source.replace(pos, 5, pm.kname);
  return pm;
}

// ------------------------------------------------------------------ batch

struct Batch::Kind {
  std::string key;            // default-shape body (kind identity)
  const Group *proto = nullptr;
  TileCfg cfg;
  KernelPlan plan;            // plan at the tuned shape (layout shared by every member)
  std::vector<unsigned char> args;   // one Args struct per member, back to back
  int members = 0;
  void *d_args = nullptr;
  // the kind's own persistent module: its register and shared-memory needs alone
  // set its occupancy
  PersistentModule pm;
  KernelHandle kh;
  int grid = 0;
};

struct Batch::Impl {
  std::vector<FusionResult> fused;
  std::vector<Kind> kinds;
  std::unordered_map<Node *, DevRaster> bufs;
  std::vector<void *> owned;
  struct Item { uint32_t kind, inst, tile, pad; };
  std::vector<std::vector<Item>> phases;
  void *d_items = nullptr;
  void *d_counter = nullptr;
  // per dependency level, the contiguous item ranges of one kind (one launch each)
  struct Segment { int kind; size_t off, n; };
  std::vector<std::vector<Segment>> segments;
  std::vector<cudaStream_t> branch;   // streams the kinds of one level fork onto while capturing
  std::vector<cudaEvent_t> fork_ev;
  int launches = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long cells = 0;
  size_t tiles = 0;
  bool tuned = false;
};

Batch::Batch() = default;

Batch::~Batch() {
  if (!impl_) return;
  if (impl_->exec) cudaGraphExecDestroy(impl_->exec);
  if (impl_->graph) cudaGraphDestroy(impl_->graph);
  for (auto &k : impl_->kinds)
    if (k.d_args) cudaFree(k.d_args);
  if (impl_->d_items) cudaFree(impl_->d_items);
  for (cudaStream_t b : impl_->branch) cudaStreamDestroy(b);
  for (cudaEvent_t e : impl_->fork_ev) cudaEventDestroy(e);
  if (impl_->d_counter) cudaFree(impl_->d_counter);
  for (void *p : impl_->owned) cudaFree(p);
}

void Batch::add(const std::vector<Node *> &outs, const std::vector<void *> &dst, const std::vector<long long> &pitch) {
  if (impl_) throw MapError("batch: cannot add after prepare");
  if (outs.empty() || outs.size() != dst.size() || outs.size() != pitch.size()) throw MapError("batch: bad instance");
  for (size_t i = 0; i < outs.size(); i++) {
    if (!outs[i] || outs[i]->meta.numdim != D2) throw MapError("batch: outputs must be 2-D rasters");
    if (!dst[i]) throw MapError("batch: null output buffer");
    if (((uintptr_t)dst[i] & 15) || (pitch[i] & 15) || pitch[i] < (long long)outs[i]->meta.W() * (long long)dt_size(outs[i]->meta.dtype))
      throw MapError("batch: output buffers need a 16-byte aligned base and pitch of at least one row");
  }
  inst_.push_back(BatchInstance{outs, dst, pitch});
}

void Batch::prepare(bool autotune) {
  if (impl_) return;
  if (inst_.empty()) throw MapError("batch: no instances");
  std::lock_guard<std::recursive_mutex> lk(Runtime::get().mtx);
  CudaEnv &env = CudaEnv::get();
  env.ensure_device();
  cudaStream_t st = (cudaStream_t)env.stream();
  impl_ = std::make_unique<Impl>();
  Impl &I = *impl_;
  auto &bufs = I.bufs;

  std::function<DevRaster &(Node *)> get = [&](Node *n) -> DevRaster & {
    auto it = bufs.find(n);
    if (it != bufs.end()) return it->second;
    const int W = n->meta.W(), H = n->meta.H(), dt = n->meta.dtype;
    const size_t row = (size_t)W * dt_size(dt);
    DevRaster r;
    r.dtype = dt;
    r.W = W;
    r.H = H;
    if (n->kind == K_DEVIN && n->dev->rows)
      throw MapError("batch: a device input holding a row band is evaluated by row ranges only (ma_evalRows)");
    if (n->kind == K_DEVIN && ((uintptr_t)n->dev->ptr & 15) == 0 && (n->dev->pitch & 15) == 0) {
      r.ptr = n->dev->ptr;
      r.pitch = n->dev->pitch;
      return bufs[n] = r;
    }
    r.pitch = pitch_for(W, dt);
    cuda_check(cudaMalloc(&r.ptr, (size_t)r.pitch * H), "cudaMalloc(batch input)");
    I.owned.push_back(r.ptr);
    if (n->kind == K_DEVIN) {
      cuda_check(cudaMemcpy2DAsync(r.ptr, r.pitch, n->dev->ptr, n->dev->pitch, row, H, cudaMemcpyDeviceToDevice, st), "copy");
    } else if (n->kind == K_HOSTIN) {
      cuda_check(cudaMemcpy2DAsync(r.ptr, r.pitch, n->host->ptr, row, row, H, cudaMemcpyHostToDevice, st), "upload");
    } else if (n->kind == K_READ) {
      std::vector<unsigned char> tmp(row * H);
      bin_read_dense(n->path, bin_read_header(n->path), tmp.data());
      cuda_check(cudaMemcpy2D(r.ptr, r.pitch, tmp.data(), row, row, H, cudaMemcpyHostToDevice), "upload");
    } else {
      throw MapError(std::string("batch: raster of ") + kind_name(n->kind) + " is not available");
    }
    return bufs[n] = r;
  };

  // fuse every instance; bind outputs; bucket groups into kinds
  std::map<std::string, int> kind_of_body;
  struct Member { int kind; const Group *g; int level; };
  std::vector<Member> members;
  for (auto &in : inst_) {
    std::set<Node *> tset(in.outs.begin(), in.outs.end());
    I.fused.push_back(fuse(collect_nodes(in.outs), tset));
    FusionResult &fr = I.fused.back();
    std::map<const Group *, int> level;
    for (size_t i = 0; i < in.outs.size(); i++) {
      DevRaster r;
      r.ptr = in.dst[i];
      r.pitch = in.pitch[i];
      r.dtype = in.outs[i]->meta.dtype;
      r.W = in.outs[i]->meta.W();
      r.H = in.outs[i]->meta.H();
      bufs[in.outs[i]] = r;
    }
    for (auto &gp : fr.groups) {
      const Group &g = *gp;
      if (g.skeleton != SK_LOCAL && g.skeleton != SK_FOCAL)
        throw MapError(std::string("batch: ") + skeleton_name(g.skeleton) + " groups cannot be batched");
      int lv = 0;
      for (Group *p : g.prev) lv = std::max(lv, level[p] + 1);
      level[&g] = lv;
      KernelPlan proto = generate_kernel(g);
      for (Node *o : proto.out_rasters) {
        if (bufs.count(o)) continue;
        DevRaster r;
        r.dtype = o->meta.dtype;
        r.W = o->meta.W();
        r.H = o->meta.H();
        r.pitch = pitch_for(r.W, r.dtype);
        cuda_check(cudaMalloc(&r.ptr, (size_t)r.pitch * r.H), "cudaMalloc(batch intermediate)");
        I.owned.push_back(r.ptr);
        bufs[o] = r;
      }
      auto it = kind_of_body.find(proto.body);
      int k;
      if (it == kind_of_body.end()) {
        k = (int)I.kinds.size();
        kind_of_body[proto.body] = k;
        Kind kd;
        kd.key = proto.body;
        kd.proto = &g;
        I.kinds.push_back(std::move(kd));
      } else {
        k = it->second;
        // the largest member represents the kind when tuning
        const Group *p = I.kinds[k].proto;
        if ((long long)g.W * g.H > (long long)p->W * p->H) I.kinds[k].proto = &g;
      }
      members.push_back(Member{k, &g, lv});
    }
  }
  cuda_check(cudaStreamSynchronize(st), "stream synchronize");

  // tile shapes: tuned per kind over all its members, in the persistent form
  std::vector<std::vector<const Group *>> kind_members(I.kinds.size());
  for (auto &m : members) kind_members[m.kind].push_back(m.g);
  for (size_t k = 0; k < I.kinds.size(); k++) {
    Kind &kd = I.kinds[k];
    kd.cfg = autotune ? autotune_kind(kind_members[k], get, bufs) : TileCfg();
    kd.plan = generate_kernel(*kd.proto, kd.cfg);
    if (kd.cfg.nt != 256) throw MapError("batch: tile configurations must use 256 threads");
  }
  I.tuned = autotune;

  // per-member arguments and work items
  int nphase = 0;
  for (auto &m : members) nphase = std::max(nphase, m.level + 1);
  I.phases.assign(nphase, {});
  for (auto &m : members) {
    Kind &kd = I.kinds[m.kind];
    KernelPlan P = generate_kernel(*m.g, kd.cfg);
    if (P.body != kd.plan.body) throw MapError("batch: members of one kind generated different code");
    uint64_t aux[4] = {0, 0, 0, 0};
    auto a = pack_args(*m.g, P, get, bufs, 0, 0, m.g->W, m.g->H, aux);
    const uint32_t idx = (uint32_t)kd.members++;
    kd.args.insert(kd.args.end(), a.begin(), a.end());
    const int tiles = ((m.g->W + kd.cfg.tw - 1) / kd.cfg.tw) * ((m.g->H + kd.cfg.th - 1) / kd.cfg.th);
    for (int t = 0; t < tiles; t++) I.phases[m.level].push_back(Impl::Item{(uint32_t)m.kind, idx, (uint32_t)t, 0});
    I.cells += (long long)m.g->W * m.g->H;
    I.tiles += tiles;
  }

  // items of one level are independent: run them kind by kind, so the CTAs of an
  // SM mostly execute one tile function at a time (instruction-cache locality)
  for (auto &p : I.phases)
    std::stable_sort(p.begin(), p.end(), [](const Impl::Item &x, const Impl::Item &y) { return x.kind < y.kind; });

  // one persistent module per kind; a level's items are contiguous per kind
  for (auto &kd : I.kinds) {
    kd.pm = build_persistent_module({&kd.plan});
    kd.kh = env.kernel(kd.pm.source, kd.pm.kname, kd.pm.smem);
    kd.grid = env.sm_count() * std::max(1, env.occupancy(kd.kh, 256, kd.pm.smem));
  }
  std::vector<Impl::Item> all;
  I.segments.assign(nphase, {});
  size_t nseg = 0;
  for (int ph = 0; ph < nphase; ph++) {
    const auto &p = I.phases[ph];
    for (size_t a = 0; a < p.size();) {
      size_t b = a;
      while (b < p.size() && p[b].kind == p[a].kind) b++;
      I.segments[ph].push_back(Impl::Segment{(int)p[a].kind, all.size(), b - a});
      for (size_t q = a; q < b; q++) all.push_back(Impl::Item{0u, p[q].inst, p[q].tile, 0u});   // kind 0 of its module
      nseg++;
      a = b;
    }
  }
  I.launches = (int)nseg;

  // device arrays
  for (auto &kd : I.kinds) {
    cuda_check(cudaMalloc(&kd.d_args, kd.args.size()), "cudaMalloc(batch args)");
    cuda_check(cudaMemcpy(kd.d_args, kd.args.data(), kd.args.size(), cudaMemcpyHostToDevice), "upload args");
  }
  cuda_check(cudaMalloc(&I.d_items, std::max<size_t>(1, all.size()) * sizeof(Impl::Item)), "cudaMalloc(items)");
  cuda_check(cudaMalloc(&I.d_counter, std::max<size_t>(1, nseg) * 256), "cudaMalloc(counter)");
  if (!all.empty())
    cuda_check(cudaMemcpy(I.d_items, all.data(), all.size() * sizeof(Impl::Item), cudaMemcpyHostToDevice), "upload items");
  size_t maxk = 1;
  for (auto &segs : I.segments) maxk = std::max(maxk, segs.size());
  for (size_t b = 1; b < maxk; b++) {
    cudaStream_t bs;
    cuda_check(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking), "cudaStreamCreate");
    I.branch.push_back(bs);
  }
  for (size_t e = 0; e < 2 * maxk; e++) {
    cudaEvent_t ev;
    cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    I.fork_ev.push_back(ev);
  }

  // capture: per dependency level, the level's kinds run side by side (one branch
  // each: reset the segment's counter, then its persistent launch), joined before
  // the next level
  cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  try {
    size_t si = 0;
    for (int ph = 0; ph < nphase; ph++) {
      const auto &segs = I.segments[ph];
      cuda_check(cudaEventRecord(I.fork_ev[0], st), "cudaEventRecord");
      for (size_t b = 1; b < segs.size(); b++) cuda_check(cudaStreamWaitEvent(I.branch[b - 1], I.fork_ev[0], 0), "fork");
      for (size_t b = 0; b < segs.size(); b++) {
        const Impl::Segment &sg = segs[b];
        const Kind &kd = I.kinds[sg.kind];
        cudaStream_t bst = b == 0 ? st : I.branch[b - 1];
        void *ctr = (char *)I.d_counter + 256 * (si++);
        cuda_check(cudaMemsetAsync(ctr, 0, 4, bst), "cudaMemsetAsync");
        struct {
          uint64_t items;
          int64_t n;
          uint64_t counter;
          uint64_t err;
          uint64_t args[1];
        } ba;
        ba.items = (uint64_t)(uintptr_t)((Impl::Item *)I.d_items + sg.off);
        ba.n = (int64_t)sg.n;
        ba.counter = (uint64_t)(uintptr_t)ctr;
        ba.err = (uint64_t)(uintptr_t)env.err_word();
        ba.args[0] = (uint64_t)(uintptr_t)kd.d_args;
        env.launch(kd.kh, std::min<int>(kd.grid, (int)sg.n), 256, kd.pm.smem, (CUstream_st *)bst, &ba, sizeof ba);
      }
      for (size_t b = 1; b < segs.size(); b++) {
        cuda_check(cudaEventRecord(I.fork_ev[b], I.branch[b - 1]), "cudaEventRecord");
        cuda_check(cudaStreamWaitEvent(st, I.fork_ev[b], 0), "join");
      }
    }
  } catch (...) {
    cudaGraph_t g;
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  cuda_check(cudaStreamEndCapture(st, &I.graph), "cudaStreamEndCapture");
  cuda_check(cudaGraphInstantiate(&I.exec, I.graph, 0), "cudaGraphInstantiate");
}

void Batch::run(bool sync) {
  if (!impl_) prepare(true);
  CudaEnv &env = CudaEnv::get();
  cuda_check(cudaGraphLaunch(impl_->exec, (cudaStream_t)env.stream()), "cudaGraphLaunch");
  env.count_launch();
  if (!sync) return;
  try {
    Executor::get().sync();
  } catch (const MapError &e) {
    // A CTA that gave up on its staging wait left its tile's copy in flight; the
    // copy can land in shared memory that another CTA reuses, so no output of
    // this run can be trusted, not only the tile that failed.
    throw MapError(std::string(e.what()) + " every output of this batch run is void");
  }
}

std::string Batch::info() const {
  std::ostringstream s;
  s << "{\"instances\": " << inst_.size();
  if (impl_) {
    s << ", \"cells\": " << impl_->cells << ", \"tiles\": " << impl_->tiles << ", \"phases\": " << impl_->phases.size()
      << ", \"launches\": " << impl_->launches << ", \"kinds\": [";
    for (size_t k = 0; k < impl_->kinds.size(); k++) {
      auto &kd = impl_->kinds[k];
      s << (k ? ", " : "") << "{\"skeleton\": \"" << skeleton_name(kd.proto->skeleton) << "\", \"members\": " << kd.members
        << ", \"tile\": [" << kd.cfg.tw << ", " << kd.cfg.th << "], \"threads\": " << kd.cfg.nt
        << ", \"tma\": " << (kd.plan.tma.empty() ? "false" : "true") << ", \"kernel\": \"" << kd.pm.kname
        << "\", \"grid\": " << kd.grid << "}";
    }
    s << "], \"autotuned\": " << (impl_->tuned ? "true" : "false");
  }
  s << "}";
  return s.str();
}

}  // namespace mapb

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

TileCfg autotune_group(const Group &g, const std::function<DevRaster &(Node *)> &get,
                       std::unordered_map<Node *, DevRaster> &bufs) {
  KernelPlan base = generate_kernel(g);
  if (g.skeleton != SK_LOCAL && g.skeleton != SK_FOCAL) return TileCfg();
  const std::string key = tune_key(g, base);
  {
    std::lock_guard<std::mutex> lk(g_tune_mtx);
    tune_load();
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  CudaEnv &env = CudaEnv::get();
  cudaStream_t st = (cudaStream_t)env.stream();
  static const int cand[][2] = {{64, 32}, {128, 16}, {32, 32}, {64, 16}, {128, 32}, {32, 64}, {64, 64}};
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
    KernelPlan P = generate_kernel(g, cfg);
    KernelHandle kh = env.kernel(P.source, P.kname, P.smem_bytes);
    uint64_t aux[4] = {0, 0, 0, 0};
    auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux);
    const int tiles = ((g.W + cfg.tw - 1) / cfg.tw) * ((g.H + cfg.th - 1) / cfg.th);
    env.launch(kh, tiles, cfg.nt, P.smem_bytes, (CUstream_st *)st, a.data(), a.size());
    cuda_check(cudaEventRecord(e0, st), "cudaEventRecord");
    for (int r = 0; r < 3; r++) env.launch(kh, tiles, cfg.nt, P.smem_bytes, (CUstream_st *)st, a.data(), a.size());
    cuda_check(cudaEventRecord(e1, st), "cudaEventRecord");
    cuda_check(cudaEventSynchronize(e1), "cudaEventSynchronize");
    float ms = 0;
    cuda_check(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
    if (ms < best_ms) { best_ms = ms; best = cfg; }
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
      << "  __shared__ int item_s;\n"
      << "  u64 *bar = (u64 *)(smem + " << bar_off << ");\n"
      << "  if (threadIdx.x == 0) { mbar_init(bar, 1); fence_mbar_init(); }\n"
      << "  __syncthreads();\n"
      << "  u32 phase = 0;\n"
      << "  const BItem *items = (const BItem *)b.items;\n"
      << "  for (;;) {\n"
      << "    if (threadIdx.x == 0) item_s = atomicAdd((int *)b.counter, 1);\n"
      << "    __syncthreads();\n"
      << "    const int i = item_s;\n"
      << "    __syncthreads();\n"
      << "    if (i >= b.n) break;\n"
      << "    const BItem w = items[i];\n"
      << "    bool ok = true;\n"
      << "    switch (w.kind) {\n";
  for (size_t k = 0; k < kinds.size(); k++)
    src << "      case " << k << ": ok = k" << k << "::run_tile(((const k" << k << "::Args *)b.args[" << k
        << "])[w.inst], (int)w.tile, smem, bar, phase, true); break;\n";
  src << "      default: skel_fail((u32 *)b.err, ERR_BAD_LAUNCH); ok = false;\n"
      << "    }\n"
      << "    if (!ok) break;\n"
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
  std::string source, kname;
  KernelHandle kh;
  size_t smem = 0;
  int grid = 0;
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

  // tile shapes: tuned on each kind's largest member
  for (auto &kd : I.kinds) {
    kd.cfg = autotune ? autotune_group(*kd.proto, get, bufs) : TileCfg();
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

  // batch module: every kind's tile function in its own namespace + a persistent dispatcher
  std::vector<const KernelPlan *> kp;
  for (auto &kd : I.kinds) kp.push_back(&kd.plan);
  PersistentModule pm = build_persistent_module(kp);
  I.source = pm.source;
  I.kname = pm.kname;
  I.smem = pm.smem;
  I.kh = env.kernel(I.source, I.kname, I.smem);
  int occ = std::max(1, env.occupancy(I.kh, 256, I.smem));
  I.grid = env.sm_count() * occ;

  // device arrays
  for (auto &kd : I.kinds) {
    cuda_check(cudaMalloc(&kd.d_args, kd.args.size()), "cudaMalloc(batch args)");
    cuda_check(cudaMemcpy(kd.d_args, kd.args.data(), kd.args.size(), cudaMemcpyHostToDevice), "upload args");
  }
  size_t nitems = 0;
  for (auto &p : I.phases) nitems += p.size();
  cuda_check(cudaMalloc(&I.d_items, std::max<size_t>(1, nitems) * sizeof(Impl::Item)), "cudaMalloc(items)");
  cuda_check(cudaMalloc(&I.d_counter, (size_t)std::max(1, nphase) * 256), "cudaMalloc(counter)");
  size_t off = 0;
  for (auto &p : I.phases) {
    cuda_check(cudaMemcpy((char *)I.d_items + off * sizeof(Impl::Item), p.data(), p.size() * sizeof(Impl::Item),
                          cudaMemcpyHostToDevice),
               "upload items");
    off += p.size();
  }

  // capture: per dependency level, reset its counter then one persistent launch
  cuda_check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  try {
    off = 0;
    for (int ph = 0; ph < nphase; ph++) {
      void *ctr = (char *)I.d_counter + 256 * ph;
      cuda_check(cudaMemsetAsync(ctr, 0, 4, st), "cudaMemsetAsync");
      struct {
        uint64_t items;
        int64_t n;
        uint64_t counter;
        uint64_t err;
        uint64_t args[64];
      } ba;
      if (I.kinds.size() > 64) throw MapError("batch: too many kernel kinds");
      ba.items = (uint64_t)(uintptr_t)((Impl::Item *)I.d_items + off);
      ba.n = (int64_t)I.phases[ph].size();
      ba.counter = (uint64_t)(uintptr_t)ctr;
      ba.err = (uint64_t)(uintptr_t)env.err_word();
      for (size_t k = 0; k < I.kinds.size(); k++) ba.args[k] = (uint64_t)(uintptr_t)I.kinds[k].d_args;
      env.launch(I.kh, I.grid, 256, I.smem, (CUstream_st *)st, &ba, 32 + 8 * I.kinds.size());
      off += I.phases[ph].size();
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
  if (sync) Executor::get().sync();
}

std::string Batch::info() const {
  std::ostringstream s;
  s << "{\"instances\": " << inst_.size();
  if (impl_) {
    s << ", \"cells\": " << impl_->cells << ", \"tiles\": " << impl_->tiles << ", \"grid\": " << impl_->grid
      << ", \"phases\": " << impl_->phases.size() << ", \"kernel\": \"" << impl_->kname << "\", \"kinds\": [";
    for (size_t k = 0; k < impl_->kinds.size(); k++) {
      auto &kd = impl_->kinds[k];
      s << (k ? ", " : "") << "{\"skeleton\": \"" << skeleton_name(kd.proto->skeleton) << "\", \"members\": " << kd.members
        << ", \"tile\": [" << kd.cfg.tw << ", " << kd.cfg.th << "], \"threads\": " << kd.cfg.nt
        << ", \"tma\": " << (kd.plan.tma.empty() ? "false" : "true") << "}";
    }
    s << "], \"autotuned\": " << (impl_->tuned ? "true" : "false");
  }
  s << "}";
  return s.str();
}

}  // namespace mapb

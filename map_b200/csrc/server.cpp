// Serving with continuous batching (see server.hpp).
#include "server.hpp"
#include "batch.hpp"
#include "codegen.hpp"
#include "cuda_env.hpp"
#include "executor.hpp"
#include "fusion.hpp"
#include "programs.hpp"

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <random>
#include <set>
#include <sstream>
#include <thread>
#include <unordered_map>

namespace mapb {

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

long long pitch_for(int W, int dt) {
  long long b = (long long)W * (long long)dt_size(dt);
  return (b + 127) / 128 * 128;
}

// Launch phases of a batch, in stream order. A request is complete once the
// last phase its program uses has finished.
enum Phase { PH_LEVEL0 = 0, PH_RADIAL = 1, PH_LEVEL1 = 2, PH_SPREAD = 3, N_PHASES = 4 };

struct Req {
  long long id = 0;
  int type = 0, x0 = 0, y0 = 0, w = 0, h = 0, ox = 0, oy = 0;
  float oh = 0;
  double radius = 0;
  bool auto_release = false;
  double t_submit = 0, t_done = 0;
  int state = 0;   // 0 queued, 1 running, 2 done, 3 failed
  std::string err;
  size_t bytes = 0;
  int stream = 0;
  void *win = nullptr;
  long long win_pitch = 0;
  void *out = nullptr;
  long long out_pitch = 0;
  int out_dt = F32;
  std::vector<void *> scratch;
};

// Flow windows above 64 K cells with integer accumulations use pointer jumping
// (MAP_B200_SERVE_PJ=0: the one-CTA frontier sweep instead).
bool serve_pj() {
  static const bool v = [] {
    const char *e = std::getenv("MAP_B200_SERVE_PJ");
    return !(e && e[0] == '0');
  }();
  return v;
}

size_t request_bytes(int type, int w, int h) {
  size_t b = (size_t)pitch_for(w, F32) * h * 2;   // window copy + output
  if (type == REQ_FLOW) b += (size_t)pitch_for(w, U8) * h + (size_t)w * h * 32;   // directions + sweep scratch
  return b;
}

// A program kind over a window size, fused and code-generated once. Its nodes
// stand for any request of that shape: a request binds its own buffers to the
// template's rasters and its own observer to the template's scalar arguments.
struct Template {
  FusionResult fr;
  std::vector<KernelPlan> plans;   // per group, in group order
  std::vector<int> level;          // dependency level per group
  std::vector<int> kind;           // persistent-module kind per Local / Focal group (-1 otherwise)
  Node *win = nullptr, *out = nullptr;
  Node *ox = nullptr, *oy = nullptr, *oh = nullptr;   // viewshed observer arguments
  int last_phase = PH_LEVEL0;
};

// Flow accumulations run one CTA per request; batches take turns over several
// streams so that consecutive batches' accumulations run side by side.
constexpr int kSpreadStreams = 8;
constexpr int kQueues = 2 + kSpreadStreams;   // two batch streams, then the spreading streams

// One phase of one batch: the requests that complete with it.
struct PhaseDone {
  cudaEvent_t ev = nullptr;
  std::vector<Req *> reqs;
  void *batch_mem = nullptr;   // freed with the batch's last phase
};

}  // namespace

struct Server::Impl {
  void *dem = nullptr;
  long long pitch = 0;
  int W = 0, H = 0;
  size_t budget = 0;
  int max_batch = 0;

  std::mutex m;
  std::condition_variable cv_pending, cv_done, cv_inflight;
  std::deque<Req *> pending;
  std::map<long long, std::unique_ptr<Req>> reqs;
  std::deque<PhaseDone> inflight[kQueues];   // per stream, in stream order
  size_t used = 0;
  long long next_id = 1;
  bool stop = false;
  std::thread dispatcher, completer;
  cudaStream_t streams[kQueues] = {};   // two batch streams, then the spreading streams
  cudaEvent_t staged[2] = {nullptr, nullptr};               // upload of the stream's last batch done
  int next_stream = 0, next_spread = 0;
  // pinned staging for argument / work-list uploads, one per batch stream
  void *stage[2] = {nullptr, nullptr};
  size_t stage_cap[2] = {0, 0};

  // Local / Focal kinds seen so far, in registration order; the persistent
  // module holds all of them, so it is rebuilt (compiled) only when a new kind appears
  std::vector<KernelPlan> reg_plans;
  std::map<std::string, int> reg_index;
  int module_kinds = -1;
  PersistentModule pm;
  KernelHandle pk;
  int pk_grid = 0;
  std::map<std::string, std::unique_ptr<Template>> templates;
  static constexpr size_t kMaxTemplates = 512;
  std::vector<std::unique_ptr<Template>> transient;   // templates built past the cache limit (one batch)
  void drop(Template &T) {
    Runtime &rt = Runtime::get();
    std::lock_guard<std::recursive_mutex> lk(rt.mtx);
    if (T.out && rt.owns(T.out) && T.out->ref > 0) T.out->ref--;
  }

  // statistics
  long long batches = 0, completed = 0, failed = 0, max_batch_seen = 0, batched_requests = 0;
  size_t peak_used = 0;

  int register_kind(const KernelPlan &P) {
    auto it = reg_index.find(P.body);
    if (it != reg_index.end()) return it->second;
    int k = (int)reg_plans.size();
    reg_index[P.body] = k;
    reg_plans.push_back(P);
    return k;
  }
  void ensure_module() {
    if (module_kinds == (int)reg_plans.size() || reg_plans.empty()) return;
    CudaEnv &env = CudaEnv::get();
    std::vector<const KernelPlan *> kp;
    for (auto &p : reg_plans) kp.push_back(&p);
    pm = build_persistent_module(kp);
    pk = env.kernel(pm.source, pm.kname, pm.smem);
    pk_grid = env.sm_count() * std::max(1, env.occupancy(pk, 256, pm.smem));
    module_kinds = (int)reg_plans.size();
  }
  // compile = false defers the persistent module's (re)compilation to the caller
  Template &template_for(int type, int w, int h, bool compile = true);
  void warm_up();
  void dispatch_loop();
  void complete_loop();
  bool idle() const {
    for (int i = 0; i < kQueues; i++)
      if (!inflight[i].empty()) return false;
    return true;
  }
  void run_batch(std::vector<Req *> &batch);
  void free_request(Req *r, cudaStream_t st);
};

void Server::Impl::free_request(Req *r, cudaStream_t st) {
  if (r->win) cudaFreeAsync(r->win, st);
  if (r->out) cudaFreeAsync(r->out, st);
  for (void *p : r->scratch) cudaFreeAsync(p, st);
  r->win = r->out = nullptr;
  r->scratch.clear();
}

Template &Server::Impl::template_for(int type, int w, int h, bool compile) {
  const std::string key = std::to_string(type) + "|" + std::to_string(w) + "x" + std::to_string(h);
  auto it = templates.find(key);
  if (it != templates.end()) return *it->second;
  Runtime &rt = Runtime::get();
  std::lock_guard<std::recursive_mutex> lk(rt.mtx);
  CudaEnv &env = CudaEnv::get();
  auto T = std::make_unique<Template>();
  // the pointer only identifies the input: requests bind their own window buffers
  T->win = rt.dev_input(dem, pitch_for(w, F32), Arr2{{w, h}, 2}, F32, Arr2{{w, h}, 2});
  switch (type) {
    case REQ_HILLSHADE: T->out = prog_hillshade(rt, T->win); break;
    case REQ_SLOPE: T->out = prog_slope(rt, T->win); break;
    // distinct placeholder coordinates keep the two argument nodes distinct
    case REQ_VIEWSHED: T->out = prog_viewshed(rt, T->win, 1, 2, 3.0f, 0.0, &T->ox, &T->oy, &T->oh); break;
    case REQ_FLOW: T->out = prog_flow(rt, T->win); break;
    default: throw MapError("unknown request type");
  }
  T->out->ref++;
  T->fr = fuse(collect_nodes({T->out}), {T->out});
  std::map<const Group *, int> level;
  for (auto &gp : T->fr.groups) {
    const Group &g = *gp;
    int lv = 0;
    for (Group *p : g.prev) lv = std::max(lv, level[p] + 1);
    level[&g] = lv;
    if (g.skeleton == SK_HOST) throw MapError(std::string("serving: unexpected host step ") + kind_name(g.nodes[0]->kind));
    KernelPlan P = generate_kernel(g);
    int k = -1;
    if (g.skeleton == SK_LOCAL || g.skeleton == SK_FOCAL) {
      if (lv > 1) throw MapError("serving: program too deep");
      k = register_kind(P);
      T->last_phase = std::max(T->last_phase, lv == 0 ? (int)PH_LEVEL0 : (int)PH_LEVEL1);
    } else if (g.skeleton == SK_RADIAL) {
      env.kernel(P.source, P.kname + "_many", 0);
      T->last_phase = std::max(T->last_phase, (int)PH_RADIAL);
    } else if (g.skeleton == SK_SPREAD) {
      env.kernel(P.source, P.kname + "_prep_many", 0);
      env.kernel(P.source, P.kname + "_kahnp_many", 0);
      if (spread_pj_type(P.core->meta.dtype))
        for (const char *k : {"_pj_init_many", "_pj_step_many", "_pj_final_many"}) env.kernel(P.source, P.kname + k, 0);
      T->last_phase = std::max(T->last_phase, (int)PH_SPREAD);
    } else {
      throw MapError("serving: zonal groups are not served");
    }
    T->plans.push_back(std::move(P));
    T->level.push_back(lv);
    T->kind.push_back(k);
  }
  if (compile) ensure_module();
  Template &ref = *T;
  if (templates.size() < kMaxTemplates) templates[key] = std::move(T);
  else transient.push_back(std::move(T));   // a window size beyond the cache: used for this batch only
  return ref;
}

void Server::Impl::run_batch(std::vector<Req *> &batch) {
  // templates built past the cache limit serve this batch only (every exit path)
  struct TransientRelease {
    Impl &I;
    ~TransientRelease() {
      for (auto &T : I.transient) I.drop(*T);
      I.transient.clear();
    }
  } release_transient{*this};
  CudaEnv &env = CudaEnv::get();
  const int si = next_stream;
  next_stream ^= 1;
  cudaStream_t st = streams[si];
  const int spi = 2 + next_spread;
  next_spread = (next_spread + 1) % kSpreadStreams;
  cudaStream_t sp = streams[spi];
  // the pinned staging buffer of this stream is free once its last upload is done
  if (staged[si]) cuda_check(cudaEventSynchronize(staged[si]), "cudaEventSynchronize");

  std::vector<std::vector<unsigned char>> kind_args;   // per registered kind, this batch's members
  std::vector<int> kind_members;
  struct Item { uint32_t kind, inst, tile, pad; };
  std::vector<std::vector<Item>> levels(2);
  struct Many {
    const KernelPlan *plan = nullptr;
    std::vector<unsigned char> args;
    int n = 0;
    int max_dim = 0;   // largest window side (radial front buffers)
    size_t max_cells = 0;
    bool pj = false;   // flow accumulation by pointer jumping (integer type, windows above 64 K cells)
  };
  std::map<std::string, Many> radial, spread;
  std::vector<Req *> ok;
  std::vector<int> phase_of;

  for (Req *r : batch) {
    try {
      Template &T = template_for(r->type, r->w, r->h, false);
      r->stream = si;
      r->win_pitch = pitch_for(r->w, F32);
      cuda_check(cudaMallocAsync(&r->win, (size_t)r->win_pitch * r->h, st), "cudaMallocAsync(window)");
      cuda_check(cudaMemcpy2DAsync(r->win, r->win_pitch, (char *)dem + (size_t)r->y0 * pitch + (size_t)r->x0 * 4, pitch,
                                   (size_t)r->w * 4, r->h, cudaMemcpyDeviceToDevice, st),
                 "window copy");
      r->out_dt = T.out->meta.dtype;
      r->out_pitch = pitch_for(r->w, r->out_dt);
      cuda_check(cudaMallocAsync(&r->out, (size_t)r->out_pitch * r->h, st), "cudaMallocAsync(output)");
      std::unordered_map<Node *, DevRaster> bufs;
      DevRaster wr;
      wr.ptr = r->win;
      wr.pitch = r->win_pitch;
      wr.dtype = F32;
      wr.W = r->w;
      wr.H = r->h;
      bufs[T.win] = wr;
      DevRaster orr;
      orr.ptr = r->out;
      orr.pitch = r->out_pitch;
      orr.dtype = r->out_dt;
      orr.W = r->w;
      orr.H = r->h;
      bufs[T.out] = orr;
      std::function<DevRaster &(Node *)> get = [&](Node *n) -> DevRaster & {
        auto it = bufs.find(n);
        if (it == bufs.end()) throw MapError("serving: raster not bound");
        return it->second;
      };
      std::unordered_map<const Node *, Variant> scal;
      if (T.ox) {
        Variant vx{}, vy{}, vh{};
        vx.dtype = vy.dtype = S32;
        vx.u.s32 = r->ox;
        vy.u.s32 = r->oy;
        vh.dtype = F32;
        vh.u.f32 = r->oh;
        scal[T.ox] = vx;
        scal[T.oy] = vy;
        scal[T.oh] = vh;
      }
      for (size_t gi = 0; gi < T.fr.groups.size(); gi++) {
        const Group &g = *T.fr.groups[gi];
        const KernelPlan &P = T.plans[gi];
        for (Node *o : P.out_rasters) {
          if (bufs.count(o)) continue;
          DevRaster t;
          t.dtype = o->meta.dtype;
          t.W = o->meta.W();
          t.H = o->meta.H();
          t.pitch = pitch_for(t.W, t.dtype);
          cuda_check(cudaMallocAsync(&t.ptr, (size_t)t.pitch * t.H, st), "cudaMallocAsync(intermediate)");
          r->scratch.push_back(t.ptr);
          bufs[o] = t;
        }
        if (g.skeleton == SK_LOCAL || g.skeleton == SK_FOCAL) {
          const int k = T.kind[gi];
          if ((int)kind_args.size() <= k) {
            kind_args.resize(k + 1);
            kind_members.resize(k + 1, 0);
          }
          uint64_t aux[4] = {0, 0, 0, 0};
          auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux, &scal);
          kind_args[k].insert(kind_args[k].end(), a.begin(), a.end());
          const uint32_t idx = (uint32_t)kind_members[k]++;
          const int tiles = ((g.W + P.tile_w - 1) / P.tile_w) * ((g.H + P.tile_h - 1) / P.tile_h);
          for (int t = 0; t < tiles; t++) levels[T.level[gi]].push_back(Item{(uint32_t)k, idx, (uint32_t)t, 0});
        } else if (g.skeleton == SK_RADIAL) {
          Many &mn = radial[P.source];
          mn.plan = &P;
          const long long lim = r->radius > 0 ? (long long)r->radius : -1;
          int ri = 0;
          for (size_t k = 0; k < P.out_rasters.size(); k++)
            if (P.out_rasters[k] == P.core) ri = (int)k;
          if (lim >= 0)
            for (Node *o : P.out_rasters) {
              DevRaster &d = bufs.at(o);
              cuda_check(cudaMemset2DAsync(d.ptr, d.pitch, 0xFF, (size_t)d.W * dt_size(d.dtype), d.H, st), "memset");
            }
          uint64_t aux[4] = {(uint64_t)r->ox, (uint64_t)r->oy, (uint64_t)lim, (uint64_t)ri};
          auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux, &scal);
          mn.args.insert(mn.args.end(), a.begin(), a.end());
          mn.n++;
          mn.max_dim = std::max(mn.max_dim, std::max(g.W, g.H));
        } else {   // SK_SPREAD
          const size_t N = (size_t)g.W * g.H;
          const bool pj = serve_pj() && N > ((size_t)1 << 16) && spread_pj_type(P.core->meta.dtype);
          // windows of one template share one launch per phase, so each form keys its own
          Many &mn = spread[P.source + (pj ? "#pj" : "")];
          mn.plan = &P;
          mn.pj = pj;
          mn.max_cells = std::max(mn.max_cells, N);
          void *work = nullptr;
          const size_t wbytes = pj ? spread_pj_scratch(N, P.core->meta.dtype) : 6 * N * sizeof(int32_t);
          cuda_check(cudaMallocAsync(&work, wbytes, st), "cudaMallocAsync(spread work)");
          r->scratch.push_back(work);
          uint64_t aux[4] = {(uint64_t)(uintptr_t)work, (uint64_t)(uintptr_t)((int32_t *)work + 2 * N),
                             (uint64_t)(uintptr_t)((int32_t *)work + 4 * N), (uint64_t)(N + 1)};
          auto a = pack_args(g, P, get, bufs, 0, 0, g.W, g.H, aux, &scal);
          mn.args.insert(mn.args.end(), a.begin(), a.end());
          mn.n++;
        }
      }
      ok.push_back(r);
      phase_of.push_back(T.last_phase);
    } catch (const std::exception &e) {
      std::lock_guard<std::mutex> lk(m);
      r->state = 3;
      r->err = e.what();
      failed++;
      cv_done.notify_all();
    }
  }
  batch = ok;
  if (batch.empty()) return;
  ensure_module();
  // items of one level are independent: run them kind by kind (instruction-cache locality)
  for (auto &lv : levels)
    std::stable_sort(lv.begin(), lv.end(), [](const Item &x, const Item &y) { return x.kind < y.kind; });

  // stage every upload into this stream's pinned buffer
  kind_args.resize(reg_plans.size());
  kind_members.resize(reg_plans.size(), 0);
  std::vector<std::pair<const void *, size_t>> blobs;
  for (auto &a : kind_args) blobs.push_back({a.data(), a.size()});   // empty for kinds absent from this batch
  for (auto &lv : levels) blobs.push_back({lv.data(), lv.size() * sizeof(Item)});
  for (auto &kv : radial) blobs.push_back({kv.second.args.data(), kv.second.args.size()});
  for (auto &kv : spread) blobs.push_back({kv.second.args.data(), kv.second.args.size()});
  size_t total = 512;
  for (auto &b : blobs) total += (b.second + 255) / 256 * 256;
  if (total > stage_cap[si]) {
    if (stage[si]) cudaFreeHost(stage[si]);
    stage[si] = nullptr;
    stage_cap[si] = std::max(total, (size_t)1 << 20);
    cuda_check(cudaMallocHost(&stage[si], stage_cap[si]), "cudaMallocHost(staging)");
  }
  void *dbuf = nullptr;
  cuda_check(cudaMallocAsync(&dbuf, total, st), "cudaMallocAsync(batch arrays)");
  std::vector<void *> dptr;
  size_t off = 256;   // first 256 bytes: work-list counters
  std::memset(stage[si], 0, 256);
  for (auto &b : blobs) {
    if (b.second) std::memcpy((char *)stage[si] + off, b.first, b.second);
    dptr.push_back((char *)dbuf + off);
    off += (b.second + 255) / 256 * 256;
  }
  cuda_check(cudaMemcpyAsync(dbuf, stage[si], off, cudaMemcpyHostToDevice, st), "upload batch arrays");
  if (!staged[si]) cuda_check(cudaEventCreateWithFlags(&staged[si], cudaEventDisableTiming), "cudaEventCreate");
  cuda_check(cudaEventRecord(staged[si], st), "cudaEventRecord");
  size_t bi = 0;
  std::vector<void *> d_kind_args;
  for (size_t k = 0; k < kind_args.size(); k++) d_kind_args.push_back(dptr[bi++]);
  std::vector<void *> d_levels;
  for (size_t l = 0; l < levels.size(); l++) d_levels.push_back(dptr[bi++]);

  // phases: persistent launch over level-0 Local / Focal groups; radial scans;
  // level-1 groups; flow accumulations on the spreading stream (so their long
  // sweeps hold up neither stream's next batch nor this batch's other requests)
  cudaEvent_t ev[N_PHASES];
  for (int p = 0; p < N_PHASES; p++) cuda_check(cudaEventCreateWithFlags(&ev[p], cudaEventDisableTiming), "cudaEventCreate");
  const size_t smem = pm.smem;
  const int grid = pk_grid;
  auto launch_level = [&](int l) {
    if (levels[l].empty()) return;
    struct {
      uint64_t items;
      int64_t n;
      uint64_t counter;
      uint64_t err;
      uint64_t args[64];
    } ba;
    if (reg_plans.size() > 64) throw MapError("serving: too many kinds");
    ba.items = (uint64_t)(uintptr_t)d_levels[l];
    ba.n = (int64_t)levels[l].size();
    ba.counter = (uint64_t)(uintptr_t)((char *)dbuf + 16 * l);
    ba.err = (uint64_t)(uintptr_t)env.err_word();
    for (size_t k = 0; k < reg_plans.size(); k++) ba.args[k] = (uint64_t)(uintptr_t)d_kind_args[k];
    env.launch(pk, std::min<int>(grid, (int)levels[l].size()), 256, smem, (CUstream_st *)st, &ba,
               32 + 8 * reg_plans.size());
  };
  launch_level(0);
  cuda_check(cudaEventRecord(ev[PH_LEVEL0], st), "cudaEventRecord");
  for (auto &kv : radial) {
    Many &mn = kv.second;
    const size_t smem = radial_front_smem(mn.max_dim, mn.max_dim, mn.plan->core->meta.dtype);
    KernelHandle kh = env.kernel(mn.plan->source, mn.plan->kname + "_many", smem);
    struct { uint64_t args; int64_t n; } ma{(uint64_t)(uintptr_t)dptr[bi++], mn.n};
    env.launch(kh, 8 * mn.n, 512, smem, (CUstream_st *)st, &ma, sizeof ma);
  }
  cuda_check(cudaEventRecord(ev[PH_RADIAL], st), "cudaEventRecord");
  launch_level(1);
  cuda_check(cudaEventRecord(ev[PH_LEVEL1], st), "cudaEventRecord");
  if (!spread.empty()) {
    cuda_check(cudaStreamWaitEvent(sp, ev[PH_LEVEL1], 0), "cudaStreamWaitEvent");
    for (auto &kv : spread) {
      Many &mn = kv.second;
      if (mn.pj) {
        // pointer jumping: a fixed number of rounds, `slices` CTAs per window
        const int rounds = spread_pj_rounds(mn.max_cells);
        const int64_t slices = std::max<int64_t>(32, std::min<int64_t>(256, (int64_t)(2 * mn.max_cells / 8192)));
        struct { uint64_t args; int64_t n, slices, round; } pa{(uint64_t)(uintptr_t)dptr[bi++], mn.n, slices, 0};
        const int grid = (int)(mn.n * slices);
        env.launch(env.kernel(mn.plan->source, mn.plan->kname + "_pj_init_many", 0), grid, 256, 0, (CUstream_st *)sp,
                   &pa, sizeof pa);
        KernelHandle ks = env.kernel(mn.plan->source, mn.plan->kname + "_pj_step_many", 0);
        for (int k = 0; k < rounds; k++) {
          pa.round = k;
          env.launch(ks, grid, 256, 0, (CUstream_st *)sp, &pa, sizeof pa);
        }
        pa.round = rounds;
        env.launch(env.kernel(mn.plan->source, mn.plan->kname + "_pj_final_many", 0), grid, 256, 0, (CUstream_st *)sp,
                   &pa, sizeof pa);
        continue;
      }
      // in-degrees by 32 CTAs per window, then one CTA per window sweeps the
      // frontiers (the lowest latency at window sizes)
      KernelHandle kp = env.kernel(mn.plan->source, mn.plan->kname + "_prep_many", 0);
      KernelHandle kh = env.kernel(mn.plan->source, mn.plan->kname + "_kahnp_many", 0);
      struct { uint64_t args; int64_t n; } ma{(uint64_t)(uintptr_t)dptr[bi++], mn.n};
      env.launch(kp, (int)(mn.n * 32), 256, 0, (CUstream_st *)sp, &ma, sizeof ma);
      env.launch(kh, mn.n, 1024, 0, (CUstream_st *)sp, &ma, sizeof ma);
    }
    cuda_check(cudaEventRecord(ev[PH_SPREAD], sp), "cudaEventRecord");
  }
  {
    std::lock_guard<std::mutex> lk2(m);
    batches++;
    batched_requests += (long long)batch.size();
    max_batch_seen = std::max<long long>(max_batch_seen, (long long)batch.size());
    // completion records, one per phase; the batch arrays go with the batch's last one
    const int last = spread.empty() ? (int)PH_LEVEL1 : (int)PH_SPREAD;
    for (int p = 0; p < N_PHASES; p++) {
      if (p == PH_SPREAD && spread.empty()) {
        cudaEventDestroy(ev[p]);
        continue;
      }
      PhaseDone d;
      d.ev = ev[p];
      for (size_t i = 0; i < batch.size(); i++)
        if (phase_of[i] == p) d.reqs.push_back(batch[i]);
      if (p == last) d.batch_mem = dbuf;
      inflight[p == PH_SPREAD ? spi : si].push_back(std::move(d));
    }
  }
  cv_inflight.notify_all();
}

void Server::Impl::dispatch_loop() {
  CudaEnv &env = CudaEnv::get();
  cudaSetDevice(env.device());
  while (true) {
    std::vector<Req *> batch;
    {
      std::unique_lock<std::mutex> lk(m);
      cv_pending.wait(lk, [&] { return stop || !pending.empty(); });
      if (stop) return;
      while (!pending.empty() && (int)batch.size() < max_batch) {
        Req *r = pending.front();
        if (used + r->bytes > budget && !(batch.empty() && idle() && used == 0)) break;
        used += r->bytes;
        peak_used = std::max(peak_used, used);
        r->state = 1;
        pending.pop_front();
        batch.push_back(r);
      }
      if (batch.empty()) {
        // memory is held by running batches: wait for a completion
        cv_done.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
    }
    try {
      run_batch(batch);
    } catch (const std::exception &e) {
      std::lock_guard<std::mutex> lk(m);
      for (Req *r : batch) {
        if (r->state >= 2) continue;
        r->state = 3;
        r->err = e.what();
        failed++;
      }
      cv_done.notify_all();
    }
  }
}

// Retires phases as their events fire. Each stream's queue completes in order,
// but independently of the others, so the completion thread polls the head of
// every queue.
void Server::Impl::complete_loop() {
  CudaEnv &env = CudaEnv::get();
  cudaSetDevice(env.device());
  while (true) {
    PhaseDone d;
    int q = -1;
    cudaError_t e = cudaSuccess;
    {
      std::unique_lock<std::mutex> lk(m);
      cv_inflight.wait(lk, [&] { return stop || !idle(); });
      if (stop && idle()) return;
      for (int i = 0; i < kQueues && q < 0; i++) {
        if (inflight[i].empty()) continue;
        e = cudaEventQuery(inflight[i].front().ev);
        if (e != cudaErrorNotReady) q = i;
      }
      if (q >= 0) {
        d = std::move(inflight[q].front());
        inflight[q].pop_front();
      }
    }
    if (q < 0) {
      std::this_thread::sleep_for(std::chrono::microseconds(20));
      continue;
    }
    const double t = now_s();
    cudaEventDestroy(d.ev);
    cudaStream_t st = streams[q];
    if (d.batch_mem) cudaFreeAsync(d.batch_mem, st);
    {
      std::lock_guard<std::mutex> lk(m);
      for (Req *r : d.reqs) {
        r->t_done = t;
        if (e != cudaSuccess) {
          r->state = 3;
          r->err = cudaGetErrorString(e);
          failed++;
        } else {
          r->state = 2;
          completed++;
        }
        if (r->auto_release) {
          free_request(r, st);
          used -= r->bytes;
          r->bytes = 0;
        }
      }
    }
    cv_done.notify_all();
    cv_pending.notify_all();
  }
}

// Builds the templates of every program kind at the load generator's window
// sizes, which registers and compiles every kernel up front, so no request
// waits for a compilation.
void Server::Impl::warm_up() {
  for (int s : {256, 512, 1024})
    if (s <= W && s <= H)
      for (int type = REQ_HILLSHADE; type <= REQ_FLOW; type++) template_for(type, s, s, false);
  const int w = std::min(64, W), h = std::min(64, H);
  for (int type = REQ_HILLSHADE; type <= REQ_FLOW; type++) template_for(type, w, h, false);
  ensure_module();
  // Grow the stream-ordered pool to the memory budget (at most 4 GiB) now: the
  // pool keeps freed memory, so requests later allocate from it instead of
  // stalling every stream while the pool maps new memory (measured: ~60 ms).
  CudaEnv &env = CudaEnv::get();
  cudaStream_t st = (cudaStream_t)env.stream();
  const size_t chunk = (size_t)256 << 20;
  const size_t want = std::min(budget, (size_t)4 << 30);
  std::vector<void *> held;
  for (size_t got = 0; got + chunk <= want; got += chunk) {
    void *p = nullptr;
    if (cudaMallocAsync(&p, chunk, st) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    held.push_back(p);
  }
  for (void *p : held) cudaFreeAsync(p, st);
  cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize(pool reserve)");
}

Server::Server(void *dem, long long pitch, int W, int H, size_t budget_bytes, int max_batch) : impl_(new Impl) {
  if (!dem || W <= 0 || H <= 0 || pitch < (long long)W * 4) throw MapError("server: invalid DEM");
  CudaEnv &env = CudaEnv::get();
  env.ensure_device();
  Impl &I = *impl_;
  I.dem = dem;
  I.pitch = pitch;
  I.W = W;
  I.H = H;
  I.budget = budget_bytes;
  I.max_batch = std::max(1, max_batch);
  // keep freed pool memory mapped: requests allocate and free continuously
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, env.device()) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  for (int i = 0; i < kQueues; i++)
    cuda_check(cudaStreamCreateWithFlags(&I.streams[i], cudaStreamNonBlocking), "cudaStreamCreate");
  I.warm_up();
  I.dispatcher = std::thread([&I] { I.dispatch_loop(); });
  I.completer = std::thread([&I] { I.complete_loop(); });
}

Server::~Server() {
  Impl &I = *impl_;
  {
    std::lock_guard<std::mutex> lk(I.m);
    I.stop = true;
  }
  I.cv_pending.notify_all();
  I.cv_inflight.notify_all();
  I.dispatcher.join();
  // drain what is still running
  {
    std::unique_lock<std::mutex> lk(I.m);
    I.stop = false;
  }
  I.cv_inflight.notify_all();
  for (;;) {
    std::unique_lock<std::mutex> lk(I.m);
    if (I.idle()) break;
    I.cv_done.wait_for(lk, std::chrono::milliseconds(5));
  }
  {
    std::lock_guard<std::mutex> lk(I.m);
    I.stop = true;
  }
  I.cv_inflight.notify_all();
  I.completer.join();
  for (int i = 0; i < kQueues; i++) cudaStreamSynchronize(I.streams[i]);
  for (auto &kv : I.reqs) I.free_request(kv.second.get(), I.streams[0]);
  cudaStreamSynchronize(I.streams[0]);
  for (int i = 0; i < 2; i++) {
    if (I.staged[i]) cudaEventDestroy(I.staged[i]);
    if (I.stage[i]) cudaFreeHost(I.stage[i]);
  }
  for (int i = 0; i < kQueues; i++) cudaStreamDestroy(I.streams[i]);
  for (auto &kv : I.templates) I.drop(*kv.second);
}

long long Server::submit(int type, int x0, int y0, int w, int h, int obs_x, int obs_y, float obs_h, double radius,
                         bool auto_release) {
  Impl &I = *impl_;
  if (type < REQ_HILLSHADE || type > REQ_FLOW) throw MapError("server: unknown request type");
  if (w <= 0 || h <= 0 || x0 < 0 || y0 < 0 || x0 + w > I.W || y0 + h > I.H) throw MapError("server: window outside the DEM");
  if (type == REQ_VIEWSHED && (obs_x < 0 || obs_y < 0 || obs_x >= w || obs_y >= h))
    throw MapError("server: observer outside the window");
  auto r = std::make_unique<Req>();
  r->type = type;
  r->x0 = x0;
  r->y0 = y0;
  r->w = w;
  r->h = h;
  r->ox = obs_x;
  r->oy = obs_y;
  r->oh = obs_h;
  r->radius = radius;
  r->auto_release = auto_release;
  r->bytes = request_bytes(type, w, h);
  if (r->bytes > I.budget) throw MapError("server: request larger than the memory budget");
  r->t_submit = now_s();
  long long id;
  {
    std::lock_guard<std::mutex> lk(I.m);
    id = I.next_id++;
    r->id = id;
    I.pending.push_back(r.get());
    I.reqs[id] = std::move(r);
  }
  I.cv_pending.notify_one();
  return id;
}

int Server::wait(long long id, double timeout_s) {
  Impl &I = *impl_;
  std::unique_lock<std::mutex> lk(I.m);
  auto it = I.reqs.find(id);
  if (it == I.reqs.end()) throw MapError("server: unknown request");
  Req *r = it->second.get();
  auto done = [&] { return r->state >= 2; };
  if (timeout_s < 0) I.cv_done.wait(lk, done);
  else if (!I.cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) return 1;
  if (r->state == 3) throw MapError("server: request failed: " + r->err);
  return 0;
}

void Server::result(long long id, void *dst, size_t bytes) {
  wait(id, -1);
  Impl &I = *impl_;
  Req *r;
  {
    std::lock_guard<std::mutex> lk(I.m);
    r = I.reqs.at(id).get();
    if (!r->out) throw MapError("server: result already released");
  }
  const size_t row = (size_t)r->w * dt_size(r->out_dt);
  if (bytes < row * r->h) throw MapError("server: destination too small");
  cuda_check(cudaMemcpy2D(dst, row, r->out, r->out_pitch, row, r->h, cudaMemcpyDeviceToHost), "result download");
  release(id);
}

void Server::release(long long id) {
  Impl &I = *impl_;
  std::lock_guard<std::mutex> lk(I.m);
  auto it = I.reqs.find(id);
  if (it == I.reqs.end()) return;
  Req *r = it->second.get();
  if (r->state < 2) throw MapError("server: request still running");
  I.free_request(r, I.streams[r->stream]);
  I.used -= r->bytes;
  r->bytes = 0;
  I.cv_pending.notify_all();
}

double Server::latency_ms(long long id) {
  Impl &I = *impl_;
  std::lock_guard<std::mutex> lk(I.m);
  Req *r = I.reqs.at(id).get();
  return r->state == 2 ? (r->t_done - r->t_submit) * 1e3 : -1.0;
}

std::string Server::stats_json() {
  Impl &I = *impl_;
  std::lock_guard<std::mutex> lk(I.m);
  std::ostringstream s;
  s << "{\"batches\": " << I.batches << ", \"completed\": " << I.completed << ", \"failed\": " << I.failed
    << ", \"mean_batch\": " << (I.batches ? (double)I.batched_requests / I.batches : 0.0)
    << ", \"max_batch\": " << I.max_batch_seen << ", \"peak_bytes\": " << I.peak_used << ", \"budget_bytes\": " << I.budget
    << ", \"templates\": " << I.templates.size() << ", \"kinds\": " << I.reg_plans.size() << "}";
  return s.str();
}

namespace {
double pct(std::vector<double> v, double p) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  double idx = p / 100.0 * (v.size() - 1);
  size_t lo = (size_t)std::floor(idx), hi = (size_t)std::ceil(idx);
  return v[lo] + (v[hi] - v[lo]) * (idx - lo);
}
}  // namespace

namespace {
// one generated request of the synthetic load (program, window, observer)
struct GenReq {
  int type, w, h, x0, y0, ox, oy;
};
struct LoadGen {
  std::mt19937_64 rng;
  std::discrete_distribution<int> pick;
  std::uniform_int_distribution<int> pick_size{0, 2};
  int W, H;
  LoadGen(unsigned seed, const double *mix, int W, int H) : rng(seed), pick(mix, mix + 4), W(W), H(H) {}
  GenReq next() {
    static const int sizes[3] = {256, 512, 1024};
    GenReq r;
    r.type = pick(rng);
    r.w = r.h = sizes[pick_size(rng)];
    std::uniform_int_distribution<int> px(0, W - r.w), py(0, H - r.h), po(0, r.w - 1);
    r.x0 = px(rng);
    r.y0 = py(rng);
    r.ox = po(rng);
    r.oy = po(rng);
    return r;
  }
};
}  // namespace

std::string Server::load_report(const std::vector<long long> &ids, const std::vector<int> &types,
                                const std::vector<int> &wsz, double t0, double t_end, long long cells,
                                long long batches0, long long batched0, const std::string &head) {
  Impl &I = *impl_;
  const int sizes[3] = {256, 512, 1024};
  std::vector<double> all, by_size[3], by_type[4];
  for (size_t i = 0; i < ids.size(); i++) {
    double l = latency_ms(ids[i]);
    if (l < 0) continue;
    all.push_back(l);
    by_size[wsz[i] == 256 ? 0 : wsz[i] == 512 ? 1 : 2].push_back(l);
    by_type[types[i]].push_back(l);
  }
  long long nb, nr;
  {
    std::lock_guard<std::mutex> lk(I.m);
    nb = I.batches - batches0;
    nr = I.batched_requests - batched0;
  }
  std::ostringstream s;
  s.setf(std::ios::fixed);
  s.precision(3);
  const double wall = t_end - t0;
  s << "{" << head << ", \"requests\": " << ids.size() << ", \"completed\": " << all.size() << ", \"wall_s\": " << wall
    << ", \"throughput_req_s\": " << ids.size() / wall << ", \"gcells_s\": " << cells / wall / 1e9
    << ", \"p50_ms\": " << pct(all, 50) << ", \"p99_ms\": " << pct(all, 99) << ", \"batches\": " << nb
    << ", \"mean_batch\": " << (nb ? (double)nr / nb : 0.0) << ", \"by_window\": {";
  for (int k = 0; k < 3; k++)
    s << (k ? ", " : "") << "\"" << sizes[k] << "\": {\"n\": " << by_size[k].size() << ", \"p50_ms\": " << pct(by_size[k], 50)
      << ", \"p99_ms\": " << pct(by_size[k], 99) << "}";
  const char *tn[4] = {"hillshade", "slope", "viewshed", "flow"};
  s << "}, \"by_program\": {";
  for (int k = 0; k < 4; k++)
    s << (k ? ", " : "") << "\"" << tn[k] << "\": {\"n\": " << by_type[k].size() << ", \"p50_ms\": " << pct(by_type[k], 50)
      << ", \"p99_ms\": " << pct(by_type[k], 99) << "}";
  s << "}, \"server\": " << stats_json() << "}";
  return s.str();
}

std::string Server::run_load(double rate, double seconds, const double *mix, unsigned seed, double obs_h, double radius) {
  Impl &I = *impl_;
  LoadGen gen(seed, mix, I.W, I.H);
  std::exponential_distribution<double> gap(rate);
  std::vector<long long> ids;
  std::vector<int> types, wsz;
  long long batches0, batched0;
  {
    std::lock_guard<std::mutex> lk(I.m);
    batches0 = I.batches;
    batched0 = I.batched_requests;
  }
  const double t0 = now_s();
  double t = 0;
  long long cells = 0;
  while (true) {
    t += gap(gen.rng);
    if (t > seconds) break;
    const GenReq r = gen.next();
    const double target = t0 + t;
    double dt = target - now_s();
    if (dt > 0) std::this_thread::sleep_for(std::chrono::duration<double>(dt));
    ids.push_back(submit(r.type, r.x0, r.y0, r.w, r.h, r.ox, r.oy, (float)obs_h, radius, true));
    types.push_back(r.type);
    wsz.push_back(r.w);
    cells += (long long)r.w * r.h;
  }
  for (long long id : ids) wait(id, 120.0);
  std::ostringstream head;
  head.setf(std::ios::fixed);
  head.precision(3);
  head << "\"mode\": \"open\", \"rate_req_s\": " << rate << ", \"seconds\": " << seconds;
  return load_report(ids, types, wsz, t0, now_s(), cells, batches0, batched0, head.str());
}

std::string Server::run_closed(int outstanding, double seconds, const double *mix, unsigned seed, double obs_h,
                               double radius) {
  Impl &I = *impl_;
  if (outstanding < 1) throw MapError("server: a closed-loop load needs at least one outstanding request");
  LoadGen gen(seed, mix, I.W, I.H);
  std::vector<long long> ids;
  std::vector<int> types, wsz;
  std::vector<size_t> inflight;   // indices into ids
  long long batches0, batched0;
  {
    std::lock_guard<std::mutex> lk(I.m);
    batches0 = I.batches;
    batched0 = I.batched_requests;
  }
  const double t0 = now_s();
  long long cells = 0;
  while (now_s() - t0 < seconds) {
    while ((int)inflight.size() < outstanding) {
      const GenReq r = gen.next();
      inflight.push_back(ids.size());
      ids.push_back(submit(r.type, r.x0, r.y0, r.w, r.h, r.ox, r.oy, (float)obs_h, radius, true));
      types.push_back(r.type);
      wsz.push_back(r.w);
      cells += (long long)r.w * r.h;
    }
    bool any = false;
    for (size_t k = 0; k < inflight.size();) {
      if (wait(ids[inflight[k]], 0.0) == 0) {
        inflight[k] = inflight.back();
        inflight.pop_back();
        any = true;
      } else {
        k++;
      }
    }
    if (!any) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
  for (size_t k : inflight) wait(ids[k], 120.0);
  std::ostringstream head;
  head.setf(std::ios::fixed);
  head.precision(3);
  head << "\"mode\": \"closed\", \"outstanding\": " << outstanding << ", \"seconds\": " << seconds;
  return load_report(ids, types, wsz, t0, now_s(), cells, batches0, batched0, head.str());
}

}  // namespace mapb

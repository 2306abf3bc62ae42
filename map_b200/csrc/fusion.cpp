// Fusion compiler (see fusion.hpp for the procedure).
#include "fusion.hpp"

#include <algorithm>
#include <functional>
#include <map>
#include <queue>
#include <unordered_map>
#include <unordered_set>

namespace mapb {

const char *skeleton_name(int sk) {
  switch (sk) {
    case SK_HOST: return "Host"; case SK_LOCAL: return "Local"; case SK_FOCAL: return "Focal";
    case SK_ZONAL: return "Zonal"; case SK_RADIAL: return "Radiating"; case SK_SPREAD: return "Spreading";
    default: return "?";
  }
}

namespace {

struct Rule { int a, b; bool r; };

bool match(int x, int bits) { return (x & bits) == bits; }

}  // namespace

// runtime/Pattern.cpp:53-135: first matching (top,bot) rule wins.
bool can_pipe_fuse(int top, int bot) {
  static const Rule rules[] = {
      {P_SPREAD, P_SPREAD, false}, {P_SPREAD, P_RADIAL, false}, {P_SPREAD, P_ZONAL, false}, {P_SPREAD, P_FOCAL, false},
      {P_SPREAD, P_LOCAL, false}, {P_SPREAD, P_FREE, true}, {P_SPREAD, P_SPECIAL, false}, {P_SPREAD, P_BARRIER, false},
      {P_RADIAL, P_SPREAD, false}, {P_RADIAL, P_RADIAL, false}, {P_RADIAL, P_ZONAL, false}, {P_RADIAL, P_FOCAL, false},
      {P_RADIAL, P_LOCAL, true}, {P_RADIAL, P_FREE, true}, {P_RADIAL, P_SPECIAL, false}, {P_RADIAL, P_BARRIER, false},
      {P_ZONAL, P_SPREAD, false}, {P_ZONAL, P_RADIAL, false}, {P_ZONAL, P_ZONAL, false}, {P_ZONAL, P_FOCAL, false},
      {P_ZONAL, P_LOCAL, false}, {P_ZONAL, P_FREE, true}, {P_ZONAL, P_SPECIAL, true}, {P_ZONAL, P_BARRIER, false},
      {P_FOCAL, P_SPREAD, false}, {P_FOCAL, P_RADIAL, false}, {P_FOCAL, P_ZONAL, false}, {P_FOCAL, P_FOCAL, false},
      {P_FOCAL, P_LOCAL, true}, {P_FOCAL, P_FREE, true}, {P_FOCAL, P_SPECIAL, false}, {P_FOCAL, P_BARRIER, false},
      {P_LOCAL, P_SPREAD, false}, {P_LOCAL, P_RADIAL, true}, {P_LOCAL, P_ZONAL, true}, {P_LOCAL, P_FOCAL, false},
      {P_LOCAL, P_LOCAL, true}, {P_LOCAL, P_FREE, true}, {P_LOCAL, P_SPECIAL, false}, {P_LOCAL, P_BARRIER, true},
      {P_SPECIAL, P_SPREAD, false}, {P_SPECIAL, P_RADIAL, false}, {P_SPECIAL, P_ZONAL, false}, {P_SPECIAL, P_FOCAL, false},
      {P_SPECIAL, P_LOCAL, false}, {P_SPECIAL, P_FREE, true}, {P_SPECIAL, P_SPECIAL, false}, {P_SPECIAL, P_BARRIER, false},
      {P_BARRIER, P_SPREAD, false}, {P_BARRIER, P_RADIAL, false}, {P_BARRIER, P_ZONAL, false}, {P_BARRIER, P_FOCAL, false},
      {P_BARRIER, P_LOCAL, false}, {P_BARRIER, P_FREE, true}, {P_BARRIER, P_SPECIAL, false}, {P_BARRIER, P_BARRIER, false},
  };
  for (const Rule &r : rules)
    if (match(top, r.a) && match(bot, r.b)) return r.r;
  if (match(top, P_FREE) || match(bot, P_FREE)) return true;
  throw MapError("pipe-fusion rule missing for patterns " + std::to_string(top) + " / " + std::to_string(bot));
}

// runtime/Pattern.cpp:137-184.
bool can_flat_fuse(int left, int right) {
  static const Rule rules[] = {
      {P_SPREAD, P_SPREAD, false}, {P_SPREAD, P_RADIAL, false}, {P_SPREAD, P_ZONAL, false}, {P_SPREAD, P_FOCAL, false},
      {P_SPREAD, P_LOCAL, false}, {P_SPREAD, P_FREE, true},
      {P_RADIAL, P_SPREAD, false}, {P_RADIAL, P_RADIAL, false}, {P_RADIAL, P_ZONAL, false}, {P_RADIAL, P_FOCAL, false},
      {P_RADIAL, P_LOCAL, true}, {P_RADIAL, P_FREE, true},
      {P_ZONAL, P_SPREAD, false}, {P_ZONAL, P_RADIAL, false}, {P_ZONAL, P_ZONAL, true}, {P_ZONAL, P_FOCAL, false},
      {P_ZONAL, P_LOCAL, true}, {P_ZONAL, P_FREE, true},
      {P_FOCAL, P_SPREAD, false}, {P_FOCAL, P_RADIAL, false}, {P_FOCAL, P_ZONAL, false}, {P_FOCAL, P_FOCAL, true},
      {P_FOCAL, P_LOCAL, true}, {P_FOCAL, P_FREE, true},
  };
  for (const Rule &r : rules)
    if (match(left, r.a) && match(right, r.b)) return r.r;
  return true;   // LOCAL / SPECIAL / BARRIER / FREE on either side
}

namespace {

bool is_free_raster(const Node *n) {
  return (n->kind == K_CONSTANT || n->kind == K_INDEX) && n->meta.numdim != D0;
}
bool is_leaf(const Node *n) { return n->is_input() || (n->kind == K_CONSTANT && n->meta.numdim == D0); }
bool is_host_scalar(const Node *n) {
  return n->meta.numdim == D0 && !is_leaf(n) && n->kind != K_ZONALREDUC;
}
// Consumers that read their argument over a neighbourhood (or a whole-raster
// dependency) need that argument materialised in memory.
bool needs_materialised_arg(const Node *n) {
  return n->pattern == P_FOCAL || n->pattern == P_SPREAD;
}

struct UF {
  std::vector<int> p;
  int find(int x) { while (p[x] != x) x = p[x] = p[p[x]]; return x; }
};

}  // namespace

FusionResult fuse(const std::vector<Node *> &order, const std::set<Node *> &targets, bool enable_fusion) {
  // ---- which nodes get a group
  std::unordered_set<Node *> in_order(order.begin(), order.end());
  std::unordered_set<Node *> materialise;
  for (Node *n : order) {
    if (!needs_materialised_arg(n)) continue;
    for (size_t j = 0; j < n->prev.size(); j++) {
      Node *p = n->prev[j];
      // a spread scan reads its water at the cell itself; only the directions
      // are read over the neighbourhood
      if (n->pattern == P_SPREAD && j == 0) continue;
      if (is_free_raster(p)) materialise.insert(p);
    }
  }
  for (Node *t : targets)
    if (is_free_raster(t)) materialise.insert(t);
  for (Node *n : order)
    if (n->kind == K_WRITE && is_free_raster(n->prev[0])) materialise.insert(n->prev[0]);

  std::unordered_map<Node *, int> gid;
  std::vector<Node *> grouped;
  for (Node *n : order) {
    if (n->kind == K_WRITE || is_leaf(n)) continue;
    if (is_free_raster(n) && !materialise.count(n)) continue;
    gid[n] = (int)grouped.size();
    grouped.push_back(n);
  }
  const int G = (int)grouped.size();
  UF uf;
  uf.p.resize(G);
  for (int i = 0; i < G; i++) uf.p[i] = i;
  std::vector<int> pat(G);
  for (int i = 0; i < G; i++) {
    Node *n = grouped[i];
    pat[i] = materialise.count(n) ? P_LOCAL : n->pattern;
  }
  auto host = [&](int i) { return is_host_scalar(grouped[i]); };
  // geometry key of a group: its rasters' (or a zonal node's argument's) size and blocks
  auto geo = [&](Node *n) -> std::string {
    const Meta &m = (n->meta.numdim == D0 && !n->prev.empty()) ? n->prev[0]->meta : n->meta;
    return arr_str(m.ds) + arr_str(m.bs);
  };
  std::vector<std::string> geom(G);
  for (int i = 0; i < G; i++) geom[i] = geo(grouped[i]);

  // group-level successor sets, rebuilt after each merge round
  auto build_edges = [&]() {
    std::vector<std::set<int>> succ(G);
    for (int i = 0; i < G; i++) {
      Node *n = grouped[i];
      int c = uf.find(i);
      for (Node *p : n->prev) {
        auto it = gid.find(p);
        if (it == gid.end()) continue;
        int g = uf.find(it->second);
        if (g != c) succ[g].insert(c);
      }
    }
    return succ;
  };
  auto reach = [&](const std::vector<std::set<int>> &succ, int from, int to, bool skip_direct) {
    std::vector<char> seen(G, 0);
    std::vector<int> st;
    for (int s : succ[from])
      if (!(skip_direct && s == to)) st.push_back(s);
    while (!st.empty()) {
      int x = st.back();
      st.pop_back();
      if (x == to) return true;
      if (seen[x]) continue;
      seen[x] = 1;
      for (int s : succ[x]) st.push_back(s);
    }
    return false;
  };
  auto merge = [&](int a, int b) {
    a = uf.find(a);
    b = uf.find(b);
    int lo = std::min(a, b), hi = std::max(a, b);
    uf.p[hi] = lo;
    pat[lo] |= pat[hi];
  };

  bool changed = enable_fusion;
  while (changed) {
    changed = false;
    // pipe fusion: legal only when every edge from the producer group into the
    // consumer group may be pipe-fused (a consumer group that already holds a
    // focal reader of the producer's raster must stay separate)
    auto node_pat = [&](Node *x) { return materialise.count(x) ? (int)P_LOCAL : x->pattern; };
    auto pipe_ok = [&](int gp, int gc) {
      for (int j = 0; j < G; j++) {
        if (uf.find(j) != gc) continue;
        Node *m = grouped[j];
        for (Node *q : m->prev) {
          auto it = gid.find(q);
          if (it == gid.end() || uf.find(it->second) != gp) continue;
          if (!can_pipe_fuse(node_pat(q), node_pat(m))) return false;
          if (q->meta.numdim == D0 && m->meta.numdim != D0) return false;   // scalar result feeds a raster op
        }
      }
      return true;
    };
    for (int i = 0; i < G; i++) {
      if (host(i)) continue;
      Node *n = grouped[i];
      for (Node *p : n->prev) {
        auto it = gid.find(p);
        if (it == gid.end() || host(it->second)) continue;
        int gp = uf.find(it->second), gc = uf.find(i);
        if (gp == gc) continue;
        if (!can_flat_fuse(pat[gp], pat[gc]) || !can_flat_fuse(pat[gc], pat[gp])) continue;
        if (geom[gp] != geom[gc]) continue;
        if (!pipe_ok(gp, gc)) continue;
        auto succ = build_edges();
        if (reach(succ, gp, gc, true)) continue;
        merge(gp, gc);
        changed = true;
      }
    }
    // flat fusion of groups reading a common raster
    std::map<Node *, std::vector<int>> readers;
    for (int i = 0; i < G; i++) {
      if (host(i)) continue;
      for (Node *p : grouped[i]->prev)
        if (p->meta.numdim != D0 && !is_free_raster(p)) readers[p].push_back(i);
    }
    for (auto &kv : readers) {
      auto &v = kv.second;
      for (size_t a = 0; a < v.size(); a++) {
        for (size_t b = a + 1; b < v.size(); b++) {
          int ga = uf.find(v[a]), gb = uf.find(v[b]);
          if (ga == gb) continue;
          if (!can_flat_fuse(pat[ga], pat[gb]) || !can_flat_fuse(pat[gb], pat[ga])) continue;
          if (geom[ga] != geom[gb]) continue;
          auto succ = build_edges();
          if (reach(succ, ga, gb, false) || reach(succ, gb, ga, false)) continue;
          merge(ga, gb);
          changed = true;
        }
      }
    }
  }

  // ---- materialise Group structs
  std::map<int, Group *> by_root;
  std::vector<std::unique_ptr<Group>> groups;
  for (int i = 0; i < G; i++) {
    int r = uf.find(i);
    if (!by_root.count(r)) {
      groups.push_back(std::make_unique<Group>());
      by_root[r] = groups.back().get();
      by_root[r]->pattern = pat[r];
    }
    by_root[r]->nodes.push_back(grouped[i]);
  }
  std::unordered_map<Node *, Group *> owner;
  for (auto &g : groups)
    for (Node *n : g->nodes) owner[n] = g.get();

  for (auto &gp : groups) {
    Group &g = *gp;
    // inline the FREE rasters read by the group (transitively)
    std::unordered_set<Node *> members(g.nodes.begin(), g.nodes.end());
    std::vector<Node *> stack(g.nodes.begin(), g.nodes.end());
    while (!stack.empty()) {
      Node *n = stack.back();
      stack.pop_back();
      for (Node *p : n->prev) {
        if (is_free_raster(p) && !materialise.count(p) && !members.count(p)) {
          members.insert(p);
          g.nodes.push_back(p);
          stack.push_back(p);
        }
      }
    }
    std::sort(g.nodes.begin(), g.nodes.end(), [](Node *a, Node *b) { return a->id < b->id; });
    std::set<Node *, bool (*)(Node *, Node *)> ins([](Node *a, Node *b) { return a->id < b->id; });
    for (Node *n : g.nodes)
      for (Node *p : n->prev)
        if (!members.count(p)) ins.insert(p);
    g.inputs.assign(ins.begin(), ins.end());
    // skeleton
    if (g.nodes.size() == 1 && is_host_scalar(g.nodes[0])) g.skeleton = SK_HOST;
    else if (g.pattern & P_SPREAD) g.skeleton = SK_SPREAD;
    else if (g.pattern & P_RADIAL) g.skeleton = SK_RADIAL;
    else if (g.pattern & P_ZONAL) g.skeleton = SK_ZONAL;
    else if (g.pattern & P_FOCAL) g.skeleton = SK_FOCAL;
    else g.skeleton = SK_LOCAL;
    // geometry
    for (Node *n : g.nodes) {
      const Meta &m = (n->meta.numdim == D0 && !n->prev.empty()) ? n->prev[0]->meta : n->meta;
      if (m.numdim == D2) { g.W = m.W(); g.H = m.H(); g.BS0 = m.BS0(); g.BS1 = m.BS1(); break; }
    }
  }
  // outputs: consumed outside the group, requested, written, or scanned in place
  for (auto &gp : groups) {
    Group &g = *gp;
    std::unordered_set<Node *> members(g.nodes.begin(), g.nodes.end());
    for (Node *n : g.nodes) {
      if (is_free_raster(n) && !materialise.count(n)) continue;
      bool out = targets.count(n) > 0 || n->kind == K_RADIALSCAN || n->kind == K_SPREADSCAN ||
                 (n->meta.numdim == D0 && n->kind == K_ZONALREDUC);
      for (Node *c : n->next) {
        if (!in_order.count(c)) continue;
        if (c->kind == K_WRITE) out = true;
        else if (!members.count(c)) out = true;
      }
      if (out) g.outputs.push_back(n);
    }
  }
  // group edges + topological order (ties broken by the last node id)
  for (auto &gp : groups) {
    for (Node *in : gp->inputs) {
      auto it = owner.find(in);
      if (it == owner.end()) continue;
      Group *src = it->second;
      if (std::find(gp->prev.begin(), gp->prev.end(), src) == gp->prev.end()) {
        gp->prev.push_back(src);
        src->next.push_back(gp.get());
      }
    }
  }
  std::vector<std::unique_ptr<Group>> sorted;
  std::unordered_map<Group *, int> indeg;
  for (auto &gp : groups) indeg[gp.get()] = (int)gp->prev.size();
  auto cmp = [](Group *a, Group *b) { return a->nodes.back()->id > b->nodes.back()->id; };
  std::priority_queue<Group *, std::vector<Group *>, decltype(cmp)> ready(cmp);
  for (auto &gp : groups)
    if (indeg[gp.get()] == 0) ready.push(gp.get());
  std::unordered_map<Group *, std::unique_ptr<Group>> hold;
  for (auto &gp : groups) hold[gp.get()] = std::move(gp);
  while (!ready.empty()) {
    Group *g = ready.top();
    ready.pop();
    g->id = (int)sorted.size();
    sorted.push_back(std::move(hold[g]));
    for (Group *nx : g->next)
      if (--indeg[nx] == 0) ready.push(nx);
  }
  if (sorted.size() != hold.size()) throw MapError("fusion produced a cyclic group graph");
  FusionResult res;
  res.groups = std::move(sorted);
  return res;
}

}  // namespace mapb

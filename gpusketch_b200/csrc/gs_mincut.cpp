// gs_mincut.cpp - exact global minimum cut of a small multigraph (the k-forest certificate).
//
// The reference hands the certificate to VieCut (src/mc_sketch_alg.cpp:966-1002), which is fetched
// at configure time and not part of the reference tree.  This is the Nagamochi-Ono-Ibaraki
// contraction algorithm built on CAPFOREST (a maximum-adjacency ordering):
//   * lambda starts at the minimum weighted degree;
//   * one MA ordering from an arbitrary vertex visits x_1..x_n; the cut value of every prefix
//     {x_1..x_i} (i < n) is a candidate for lambda;
//   * when the adjacency r(y) of an unvisited vertex y crosses lambda through edge (x,y), the edge
//     is marked: contracting it keeps every cut of value < lambda;
//   * the marked edges are contracted and the ordering repeats until one vertex is left.
// The last vertex of each ordering has r(x_n) = deg(x_n) >= lambda, so each ordering marks at
// least one edge; a Stoer-Wagner style contraction of the last two vertices is the fallback.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <queue>
#include <vector>

#include "gs_internal.h"

namespace {

struct WGraph {
  uint32_t n = 0;
  std::vector<uint64_t> off;   // CSR
  std::vector<uint32_t> adj;
  std::vector<uint64_t> w;
};

// build a CSR multigraph from (a, b, weight) triples over n vertices, merging parallel edges
WGraph build(uint32_t n, std::vector<uint64_t>& keys, std::vector<uint64_t>& wts) {
  // keys: (min << 32) | max ; sort with weights
  std::vector<uint64_t> idx(keys.size());
  std::iota(idx.begin(), idx.end(), 0);
  std::sort(idx.begin(), idx.end(), [&](uint64_t a, uint64_t b) { return keys[a] < keys[b]; });
  std::vector<uint64_t> uk;
  std::vector<uint64_t> uw;
  for (size_t t = 0; t < idx.size();) {
    size_t s = t;
    uint64_t sum = 0;
    while (s < idx.size() && keys[idx[s]] == keys[idx[t]]) sum += wts[idx[s++]];
    uk.push_back(keys[idx[t]]);
    uw.push_back(sum);
    t = s;
  }
  WGraph g;
  g.n = n;
  g.off.assign(n + 1, 0);
  for (uint64_t k : uk) { g.off[(k >> 32) + 1]++; g.off[(uint32_t)k + 1]++; }
  for (uint32_t i = 0; i < n; i++) g.off[i + 1] += g.off[i];
  g.adj.resize(g.off[n]);
  g.w.resize(g.off[n]);
  std::vector<uint64_t> cur(g.off.begin(), g.off.end() - 1);
  for (size_t t = 0; t < uk.size(); t++) {
    uint32_t a = (uint32_t)(uk[t] >> 32), b = (uint32_t)uk[t];
    g.adj[cur[a]] = b; g.w[cur[a]++] = uw[t];
    g.adj[cur[b]] = a; g.w[cur[b]++] = uw[t];
  }
  return g;
}

uint32_t find(std::vector<uint32_t>& p, uint32_t x) {
  while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
  return x;
}

}  // namespace

uint64_t gs_exact_min_cut_host(uint32_t V, const uint32_t* pairs, uint64_t m, uint8_t* side) {
  if (V < 2) return UINT64_MAX;
  std::vector<uint64_t> keys, wts;
  keys.reserve(m);
  wts.reserve(m);
  for (uint64_t i = 0; i < m; i++) {
    uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
    if (a == b || a >= V || b >= V) continue;
    keys.push_back(((uint64_t)std::min(a, b) << 32) | std::max(a, b));
    wts.push_back(1);
  }
  WGraph g = build(V, keys, wts);
  std::vector<uint32_t> comp(V);  // original vertex -> current super vertex
  std::iota(comp.begin(), comp.end(), 0);

  // initial bound: minimum weighted degree
  uint64_t best = UINT64_MAX;
  std::vector<uint8_t> best_side(V, 0);
  for (uint32_t v = 0; v < g.n; v++) {
    uint64_t d = 0;
    for (uint64_t e = g.off[v]; e < g.off[v + 1]; e++) d += g.w[e];
    if (d < best) {
      best = d;
      std::fill(best_side.begin(), best_side.end(), 0);
      best_side[v] = 1;
    }
  }

  std::vector<uint64_t> r, deg;
  std::vector<uint32_t> order_idx, dsu;
  std::vector<uint8_t> visited;
  while (g.n > 1 && best > 0) {
    const uint32_t n = g.n;
    r.assign(n, 0);
    deg.assign(n, 0);
    for (uint32_t v = 0; v < n; v++)
      for (uint64_t e = g.off[v]; e < g.off[v + 1]; e++) deg[v] += g.w[e];
    visited.assign(n, 0);
    order_idx.assign(n, 0);
    dsu.resize(n);
    std::iota(dsu.begin(), dsu.end(), 0);
    std::priority_queue<std::pair<uint64_t, uint32_t>> pq;
    uint64_t alpha = 0;
    int64_t best_prefix = -1;
    uint32_t nvis = 0, last = 0, prev = 0;
    uint32_t unions = 0;
    uint32_t next_unvisited = 0;
    while (nvis < n) {
      uint32_t x = UINT32_MAX;
      while (!pq.empty()) {
        auto t = pq.top();
        pq.pop();
        if (!visited[t.second] && t.first == r[t.second]) { x = t.second; break; }
      }
      if (x == UINT32_MAX) {  // disconnected remainder: start from any unvisited vertex (r = 0)
        while (visited[next_unvisited]) next_unvisited++;
        x = next_unvisited;
      }
      visited[x] = 1;
      order_idx[x] = nvis;
      prev = last;
      last = x;
      alpha = alpha + deg[x] - 2 * r[x];
      if (nvis + 1 < n && alpha < best) { best = alpha; best_prefix = nvis; }
      for (uint64_t e = g.off[x]; e < g.off[x + 1]; e++) {
        const uint32_t y = g.adj[e];
        if (visited[y]) continue;
        const uint64_t w = g.w[e];
        if (r[y] < best && r[y] + w >= best) {
          uint32_t a = find(dsu, x), b = find(dsu, y);
          if (a != b) { dsu[b] = a; unions++; }
        }
        r[y] += w;
        pq.push({r[y], y});
      }
      nvis++;
    }
    if (best_prefix >= 0) {
      for (uint32_t v = 0; v < V; v++) best_side[v] = order_idx[comp[v]] <= (uint32_t)best_prefix ? 1 : 0;
    }
    if (best == 0) break;
    if (unions == 0) {  // fallback: merge the last two vertices of the ordering
      uint32_t a = find(dsu, prev), b = find(dsu, last);
      if (a != b) dsu[b] = a;
    }
    // contract
    std::vector<uint32_t> newid(n, UINT32_MAX);
    uint32_t nn = 0;
    for (uint32_t v = 0; v < n; v++) {
      uint32_t rt = find(dsu, v);
      if (newid[rt] == UINT32_MAX) newid[rt] = nn++;
    }
    for (uint32_t v = 0; v < V; v++) comp[v] = newid[find(dsu, comp[v])];
    keys.clear();
    wts.clear();
    for (uint32_t v = 0; v < n; v++) {
      const uint32_t a = newid[find(dsu, v)];
      for (uint64_t e = g.off[v]; e < g.off[v + 1]; e++) {
        const uint32_t y = g.adj[e];
        if (y <= v) continue;  // each undirected edge once
        const uint32_t b = newid[find(dsu, y)];
        if (a == b) continue;
        keys.push_back(((uint64_t)std::min(a, b) << 32) | std::max(a, b));
        wts.push_back(g.w[e]);
      }
    }
    g = build(nn, keys, wts);
  }
  if (side) std::memcpy(side, best_side.data(), V);
  return best;
}

extern "C" gs_status gs_exact_min_cut(uint32_t num_vertices, const uint32_t* pairs, uint64_t num_edges,
                                      uint64_t* value, uint8_t* side) {
  if (!value || (num_edges && !pairs) || num_vertices < 2) {
    gs_set_error("gs_exact_min_cut: bad arguments");
    return GS_ERR_BAD_ARG;
  }
  *value = gs_exact_min_cut_host(num_vertices, pairs, num_edges, side);
  return GS_OK;
}

// Seeded synthetic grids, bridge detection and N-1 outage selection.
//
// The reference reads MATPOWER cases (src/files/loadMatpowerFormat.h:14-209);
// its benchmark matrix uses grids of 14..9241 buses (README.md:3).  This file
// generates grids of those sizes deterministically from a seed: points in the
// unit square, a random spanning tree over the k-nearest-neighbour graph and
// extra branches among nearby buses (geometrically local, like a real grid),
// so the LU fill of the Newton system matches a real grid's.  A uniform-random
// variant (topology = 1) exists only as a stress input.
//
// Determinism: own PRNG (splitmix64 seeding xoshiro256**), no std::
// distributions, all ties broken by index.
#include "mpf.h"
#include "internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace mpf {

uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

Rng::Rng(uint64_t seed) {
  uint64_t z = seed;
  for (int i = 0; i < 4; ++i) s[i] = splitmix64(z);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

uint64_t Rng::next() {
  const uint64_t result = rotl(s[1] * 5, 7) * 9;
  const uint64_t t = s[1] << 17;
  s[2] ^= s[0];
  s[3] ^= s[1];
  s[1] ^= s[2];
  s[0] ^= s[3];
  s[2] ^= t;
  s[3] = rotl(s[3], 45);
  return result;
}

double Rng::uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }

uint64_t Rng::below(uint64_t n) {
  // rejection sampling for an unbiased integer in [0, n)
  if (n <= 1) return 0;
  const uint64_t lim = UINT64_MAX - (UINT64_MAX % n);
  uint64_t v;
  do { v = next(); } while (v >= lim);
  return v % n;
}

double Rng::normal() {
  // Box-Muller; u1 in (0, 1]
  const double u1 = 1.0 - uniform();
  const double u2 = uniform();
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586476925 * u2);
}

template <class T>
static void shuffle(std::vector<T>& v, Rng& rng) {
  for (size_t i = v.size(); i > 1; --i) {
    size_t j = (size_t)rng.below(i);
    std::swap(v[i - 1], v[j]);
  }
}

struct Dsu {
  std::vector<int> p, r;
  explicit Dsu(int n) : p(n), r(n, 0) { std::iota(p.begin(), p.end(), 0); }
  int find(int x) {
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
  }
  bool unite(int a, int b) {
    a = find(a); b = find(b);
    if (a == b) return false;
    if (r[a] < r[b]) std::swap(a, b);
    p[b] = a;
    if (r[a] == r[b]) ++r[a];
    return true;
  }
};

// k nearest neighbours of every point (brute force, ties by index).
static std::vector<std::pair<int, int>> knn_edges(const std::vector<double>& px,
                                                  const std::vector<double>& py, int k) {
  const int n = (int)px.size();
  std::vector<std::pair<int, int>> edges;
  std::vector<std::pair<double, int>> d(n);
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < n; ++j) {
      const double dx = px[i] - px[j], dy = py[i] - py[j];
      d[j] = {j == i ? INFINITY : dx * dx + dy * dy, j};
    }
    const int kk = std::min(k, n - 1);
    std::nth_element(d.begin(), d.begin() + kk, d.end());
    for (int t = 0; t < kk; ++t) {
      int j = d[t].second;
      edges.push_back({std::min(i, j), std::max(i, j)});
    }
  }
  std::sort(edges.begin(), edges.end());
  edges.erase(std::unique(edges.begin(), edges.end()), edges.end());
  return edges;
}

static int synth_topology(const mpf_synth_params& p, Rng& rng,
                          std::vector<std::pair<int, int>>& out) {
  const int n = p.n_bus;
  const int n_extra = p.n_branch - (n - 1);
  std::vector<double> px(n), py(n);
  for (int i = 0; i < n; ++i) { px[i] = rng.uniform(); py[i] = rng.uniform(); }

  auto dist = [&](int a, int b) {
    const double dx = px[a] - px[b], dy = py[a] - py[b];
    return std::sqrt(dx * dx + dy * dy);
  };

  int k = 8;
  for (;;) {
    std::vector<std::pair<int, int>> cand = knn_edges(px, py, k);
    // random spanning tree over the kNN graph: Kruskal on dist * U(1, 2)
    std::vector<std::pair<double, int>> order(cand.size());
    for (size_t e = 0; e < cand.size(); ++e)
      order[e] = {dist(cand[e].first, cand[e].second) * (1.0 + rng.uniform()), (int)e};
    std::sort(order.begin(), order.end());
    Dsu dsu(n);
    std::vector<char> in_tree(cand.size(), 0);
    std::vector<std::pair<int, int>> tree;
    for (auto& o : order) {
      const auto& e = cand[o.second];
      if (dsu.unite(e.first, e.second)) { in_tree[o.second] = 1; tree.push_back(e); }
    }
    // join leftover components through their closest pair of points
    for (;;) {
      int root0 = dsu.find(0);
      int other = -1;
      for (int i = 0; i < n; ++i)
        if (dsu.find(i) != root0) { other = dsu.find(i); break; }
      if (other < 0) break;
      double best = INFINITY; int ba = -1, bb = -1;
      for (int a = 0; a < n; ++a) {
        if (dsu.find(a) != other) continue;
        for (int b = 0; b < n; ++b) {
          if (dsu.find(b) == other) continue;
          const double d = dist(a, b);
          if (d < best) { best = d; ba = a; bb = b; }
        }
      }
      dsu.unite(ba, bb);
      tree.push_back({std::min(ba, bb), std::max(ba, bb)});
    }
    std::vector<std::pair<int, int>> extras;
    if (p.topology == 0) {
      for (size_t e = 0; e < cand.size(); ++e)
        if (!in_tree[e]) extras.push_back(cand[e]);
      if ((int)extras.size() < n_extra) { k *= 2; if (k > n) return -1; continue; }
      shuffle(extras, rng);
      extras.resize(n_extra);
    } else {
      std::vector<std::pair<int, int>> used(tree);
      std::sort(used.begin(), used.end());
      int guard = 0;
      while ((int)extras.size() < n_extra) {
        if (++guard > 100 * (n_extra + 10)) return -1;
        int a = (int)rng.below(n), b = (int)rng.below(n);
        if (a == b) continue;
        std::pair<int, int> e{std::min(a, b), std::max(a, b)};
        auto it = std::lower_bound(used.begin(), used.end(), e);
        if (it != used.end() && *it == e) continue;
        used.insert(it, e);
        extras.push_back(e);
      }
    }
    out = tree;
    out.insert(out.end(), extras.begin(), extras.end());
    shuffle(out, rng);
    return 0;
  }
}

}  // namespace mpf

using namespace mpf;

extern "C" void mpf_synth_default(mpf_synth_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->n_bus = 30;
  p->n_branch = 41;
  p->n_pv = 5;
  p->topology = 0;
  p->tap_fraction = 0.0;
  p->tap_lo = 0.95; p->tap_hi = 1.05;
  p->r_lo = 0.01; p->r_hi = 0.10;
  p->xr_lo = 2.0; p->xr_hi = 6.0;
  p->b_hi = 0.05;
  p->vset_lo = 1.00; p->vset_hi = 1.06;
  p->pload_hi = 0.5;
  p->qp_lo = 0.2; p->qp_hi = 0.5;
  p->gen_factor = 1.02;
  p->loading = 0.2;
  p->seed = 1;
}

extern "C" int32_t mpf_synth_grid(const mpf_synth_params* p, mpf_bus* buses, mpf_branch* branches) {
  if (!p || !buses || !branches) return MPF_ERR_BAD_INPUT;
  if (p->n_bus < 2 || p->n_branch < p->n_bus - 1 || p->n_pv < 0 || p->n_pv > p->n_bus - 1)
    return MPF_ERR_BAD_INPUT;
  const int n = p->n_bus;
  Rng rng(p->seed);
  std::vector<std::pair<int, int>> edges;
  if (synth_topology(*p, rng, edges) != 0) return MPF_ERR_BAD_INPUT;

  // bus roles: one slack (random), n_pv PV buses spread over the grid by
  // farthest-first traversal in hops from the buses already chosen (random
  // tie-break), the rest PQ.  Spreading the voltage-controlled buses avoids long
  // radial chains of PQ buses that collapse under load.
  std::vector<int> head(n + 1, 0), adj;
  for (auto& e : edges) { head[e.first + 1]++; head[e.second + 1]++; }
  for (int i = 0; i < n; ++i) head[i + 1] += head[i];
  adj.resize(head[n]);
  {
    std::vector<int> f(head.begin(), head.end() - 1);
    for (auto& e : edges) { adj[f[e.first]++] = e.second; adj[f[e.second]++] = e.first; }
  }
  std::vector<int> type(n, MPF_BUS_PQ);
  std::vector<int> sources;  // slack first, then PV buses in the order chosen
  {
    std::vector<int> dist(n, INT32_MAX), queue;
    auto relax_from = [&](int s0) {
      dist[s0] = 0;
      queue.assign(1, s0);
      for (size_t h = 0; h < queue.size(); ++h) {
        const int v = queue[h];
        for (int k = head[v]; k < head[v + 1]; ++k) {
          const int u = adj[k];
          if (dist[u] > dist[v] + 1) { dist[u] = dist[v] + 1; queue.push_back(u); }
        }
      }
    };
    const int slack = (int)rng.below(n);
    type[slack] = MPF_BUS_SLACK;
    sources.push_back(slack);
    relax_from(slack);
    std::vector<int> far;
    for (int k = 0; k < p->n_pv; ++k) {
      int dmax = -1;
      far.clear();
      for (int i = 0; i < n; ++i) {
        if (type[i] != MPF_BUS_PQ) continue;
        if (dist[i] > dmax) { dmax = dist[i]; far.clear(); }
        if (dist[i] == dmax) far.push_back(i);
      }
      const int pick = far[(size_t)rng.below(far.size())];
      type[pick] = MPF_BUS_PV;
      sources.push_back(pick);
      relax_from(pick);
    }
  }
  double total_load = 0.0;
  for (int i = 0; i < n; ++i) {
    mpf_bus& b = buses[i];
    std::memset(&b, 0, sizeof(b));
    b.type = type[i];
    b.vm = 1.0;
    b.va = 0.0;
    if (type[i] == MPF_BUS_PQ) {
      const double pl = p->pload_hi * rng.uniform();
      const double ql = pl * (p->qp_lo + (p->qp_hi - p->qp_lo) * rng.uniform());
      b.p = -pl * p->loading;
      b.q = -ql * p->loading;
      total_load += pl * p->loading;
    } else {
      b.vm = p->vset_lo + (p->vset_hi - p->vset_lo) * rng.uniform();
    }
  }
  // PV generation: gen_factor * total load, each PV bus dispatched in proportion
  // to the load of its graph-Voronoi cell (buses whose nearest PV/slack bus, in
  // hops over the branch graph, it is; ties to the lower bus index) times U(0.75, 1.25).
  // Generation placed near the load keeps the synthetic grid solvable at the
  // stated load level; a split with purely random weights makes most grids
  // infeasible (long transfers over r ~ U(0.01, 0.1) lines).
  if (p->n_pv > 0) {
    std::vector<int> owner(n, -1), queue;
    for (int i = 0; i < n; ++i)
      if (type[i] != MPF_BUS_PQ) { owner[i] = i; queue.push_back(i); }
    for (size_t h = 0; h < queue.size(); ++h) {
      const int v = queue[h];
      for (int k = head[v]; k < head[v + 1]; ++k) {
        const int u = adj[k];
        if (owner[u] < 0) { owner[u] = owner[v]; queue.push_back(u); }
      }
    }
    std::vector<double> cell(n, 0.0);
    for (int i = 0; i < n; ++i)
      if (type[i] == MPF_BUS_PQ && owner[i] >= 0) cell[owner[i]] += -buses[i].p;
    std::vector<double> w(p->n_pv);
    double ws = 0.0;
    for (int k = 0; k < p->n_pv; ++k) {
      const int b = sources[1 + k];
      w[k] = (cell[b] + 1e-3) * (0.75 + 0.5 * rng.uniform());
      ws += w[k];
    }
    for (int k = 0; k < p->n_pv; ++k)
      buses[sources[1 + k]].p = p->gen_factor * total_load * w[k] / ws;
  }
  for (int e = 0; e < p->n_branch; ++e) {
    mpf_branch& br = branches[e];
    std::memset(&br, 0, sizeof(br));
    int a = edges[e].first, c = edges[e].second;
    if (rng.uniform() < 0.5) std::swap(a, c);
    br.from = a;
    br.to = c;
    br.status = 1;
    br.r = p->r_lo + (p->r_hi - p->r_lo) * rng.uniform();
    br.x = br.r * (p->xr_lo + (p->xr_hi - p->xr_lo) * rng.uniform());
    br.b = p->b_hi * rng.uniform();
    const double u = rng.uniform();
    br.tap = (u < p->tap_fraction) ? p->tap_lo + (p->tap_hi - p->tap_lo) * rng.uniform() : 0.0;
    br.shift = 0.0;
  }
  return MPF_OK;
}

namespace mpf {

// Bridges of the in-service multigraph (iterative Tarjan low-link; a parallel
// branch is not a bridge because the DFS skips only the tree edge's own id).
int find_bridges(const mpf_branch* br, int nbr, int nb, std::vector<uint8_t>& is_bridge) {
  is_bridge.assign(nbr, 0);
  std::vector<int> head(nb + 1, 0), adj_to, adj_e;
  for (int e = 0; e < nbr; ++e) {
    if (!br[e].status) continue;
    if (br[e].from < 0 || br[e].from >= nb || br[e].to < 0 || br[e].to >= nb) return -1;
    head[br[e].from + 1]++;
    head[br[e].to + 1]++;
  }
  for (int i = 0; i < nb; ++i) head[i + 1] += head[i];
  adj_to.resize(head[nb]);
  adj_e.resize(head[nb]);
  std::vector<int> fill(head.begin(), head.end() - 1);
  for (int e = 0; e < nbr; ++e) {
    if (!br[e].status) continue;
    adj_to[fill[br[e].from]] = br[e].to; adj_e[fill[br[e].from]++] = e;
    adj_to[fill[br[e].to]] = br[e].from; adj_e[fill[br[e].to]++] = e;
  }
  std::vector<int> tin(nb, -1), low(nb, 0), it(nb, 0), parent_e(nb, -1), stack;
  int timer = 0;
  for (int s = 0; s < nb; ++s) {
    if (tin[s] >= 0) continue;
    stack.push_back(s);
    tin[s] = low[s] = timer++;
    it[s] = head[s];
    while (!stack.empty()) {
      int v = stack.back();
      if (it[v] < head[v + 1]) {
        int k = it[v]++;
        int u = adj_to[k], e = adj_e[k];
        if (e == parent_e[v]) continue;
        if (tin[u] >= 0) {
          low[v] = std::min(low[v], tin[u]);
        } else {
          parent_e[u] = e;
          tin[u] = low[u] = timer++;
          it[u] = head[u];
          stack.push_back(u);
        }
      } else {
        stack.pop_back();
        if (!stack.empty()) {
          int w = stack.back();
          low[w] = std::min(low[w], low[v]);
          if (low[v] > tin[w]) is_bridge[parent_e[v]] = 1;
        }
      }
    }
  }
  return 0;
}

}  // namespace mpf

extern "C" int32_t mpf_find_bridges(const mpf_branch* branches, int32_t n_branch, int32_t n_bus,
                                    uint8_t* is_bridge) {
  if (!branches || !is_bridge || n_branch < 0 || n_bus < 1) return MPF_ERR_BAD_INPUT;
  std::vector<uint8_t> b;
  if (find_bridges(branches, n_branch, n_bus, b) != 0) return MPF_ERR_BAD_INPUT;
  std::memcpy(is_bridge, b.data(), (size_t)n_branch);
  return MPF_OK;
}

extern "C" int32_t mpf_select_outages(const mpf_branch* branches, int32_t n_branch, int32_t n_bus,
                                      int32_t n_out, uint64_t seed, int32_t* out) {
  if (!branches || !out || n_out < 0) return MPF_ERR_BAD_INPUT;
  std::vector<uint8_t> bridge;
  if (find_bridges(branches, n_branch, n_bus, bridge) != 0) return MPF_ERR_BAD_INPUT;
  std::vector<int> cand;
  for (int e = 0; e < n_branch; ++e)
    if (branches[e].status && !bridge[e]) cand.push_back(e);
  if ((int)cand.size() < n_out) return MPF_ERR_BAD_INPUT;
  Rng rng(seed);
  shuffle(cand, rng);
  std::memcpy(out, cand.data(), sizeof(int32_t) * (size_t)n_out);
  return MPF_OK;
}

extern "C" int32_t mpf_synth_load_scenarios(const mpf_bus* buses, int32_t n_bus, int32_t n_cases,
                                            double sigma, uint64_t seed, double* sbus) {
  if (!buses || !sbus || n_bus < 1 || n_cases < 0 || !(sigma >= 0.0)) return MPF_ERR_BAD_INPUT;
  Rng rng(seed);
  for (int c = 0; c < n_cases; ++c) {
    for (int i = 0; i < n_bus; ++i) {
      double pp = buses[i].p, qq = buses[i].q;
      if (pp < 0.0) {
        const double s = 1.0 + sigma * rng.normal();
        pp *= s;
        qq *= s;
      }
      sbus[((size_t)c * n_bus + i) * 2 + 0] = pp;
      sbus[((size_t)c * n_bus + i) * 2 + 1] = qq;
    }
  }
  return MPF_OK;
}

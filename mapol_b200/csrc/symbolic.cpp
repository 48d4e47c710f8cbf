// Host symbolic layer: done once per grid, shared by every case of a batch.
//
//  * superset Ybus pattern (every branch, in or out of service) and base values,
//    the reference's Ybus = Cf*Yf + Ct*Yt + Ysh (makeYbus.h:113-274 CPU,
//    :372-510 GPU) whose pattern already keeps out-of-service branches;
//  * per-branch admittances and their Ybus positions, so a case's Ybus is the
//    base minus its outaged branches (no SpGEMM per case);
//  * the Newton system: the reference's J (newtonpf.h:215-310) with rows
//    [P_pv, P_pq, Q_pq] x cols [Va_pv, Va_pq, Vm_pq], renumbered bus by bus in a
//    minimum-degree order so each PQ bus is a 2x2 block, and its symbolic LU;
//  * B' and B'' of the fast-decoupled methods (makeB.h:311-501) with their
//    symbolic LU and base values.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <set>
#include <string>
#include <tuple>
#include <vector>

#include "internal.h"

namespace mpf {

BranchY branch_admittance(double r, double x, double b, double tap, double shift_deg, int stat) {
  BranchY y;
  std::memset(&y, 0, sizeof(y));
  if (!stat) return y;
  // Ys = 1 / (r + jx)
  const double den = r * r + x * x;
  const double ysr = r / den, ysi = -x / den;
  // t = tap e^{j shift}, tap 0 -> 1
  const double a = (tap != 0.0) ? tap : 1.0;
  const double ang = M_PI / 180.0 * shift_deg;
  const double tr = a * std::cos(ang), ti = a * std::sin(ang);
  const double t2 = tr * tr + ti * ti;
  // Ytt = Ys + j b/2
  const double ytr = ysr, yti = ysi + 0.5 * b;
  y.tt[0] = ytr;
  y.tt[1] = yti;
  y.ff[0] = ytr / t2;
  y.ff[1] = yti / t2;
  // Yft = -Ys / conj(t) = -Ys * t / |t|^2
  y.ft[0] = -(ysr * tr - ysi * ti) / t2;
  y.ft[1] = -(ysr * ti + ysi * tr) / t2;
  // Ytf = -Ys / t = -Ys * conj(t) / |t|^2
  y.tf[0] = -(ysr * tr + ysi * ti) / t2;
  y.tf[1] = -(ysi * tr - ysr * ti) / t2;
  return y;
}

std::vector<int> minimum_degree(int n, const std::vector<std::vector<int>>& adj0) {
  std::vector<std::vector<int>> adj(adj0);
  for (auto& a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  std::set<std::pair<int, int>> pq;
  for (int v = 0; v < n; ++v) pq.insert({(int)adj[v].size(), v});
  std::vector<int> perm;
  perm.reserve(n);
  std::vector<int> tmp;
  while (!pq.empty()) {
    const int v = pq.begin()->second;
    pq.erase(pq.begin());
    perm.push_back(v);
    const std::vector<int> nv = adj[v];
    for (int a : nv) {
      pq.erase({(int)adj[a].size(), a});
      // adj[a] <- (adj[a] u nv) \ {a, v}
      tmp.clear();
      std::set_union(adj[a].begin(), adj[a].end(), nv.begin(), nv.end(), std::back_inserter(tmp));
      adj[a].clear();
      for (int u : tmp)
        if (u != a && u != v) adj[a].push_back(u);
      pq.insert({(int)adj[a].size(), a});
    }
    adj[v].clear();
    adj[v].shrink_to_fit();
  }
  return perm;
}

std::vector<int> minimum_fill(int n, const std::vector<std::vector<int>>& adj0, const std::vector<int>* weight,
                              long long max_work) {
  std::vector<std::vector<int>> adj(n);
  for (int v = 0; v < n; ++v)
    for (int a : adj0[v])
      if (a != v) {
        adj[v].push_back(a);
        adj[a].push_back(v);
      }
  for (auto& a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  auto W = [&](int v) -> long long { return weight ? (*weight)[v] : 1; };
  std::vector<int> mark(n, -1);
  int stamp = 0;
  long long work = 0;  // inner steps of the fill counts (their cost grows with the fill)
  // weighted count of the edges that eliminating v would add (pairs of its
  // neighbours not yet adjacent)
  auto fill_of = [&](int v) {
    long long f = 0;
    const std::vector<int>& nb = adj[v];
    for (size_t i = 0; i + 1 < nb.size(); ++i) {
      ++stamp;
      for (int x : adj[nb[i]]) mark[x] = stamp;
      work += (long long)adj[nb[i]].size() + (long long)(nb.size() - i);
      for (size_t j = i + 1; j < nb.size(); ++j)
        if (mark[nb[j]] != stamp) f += W(nb[i]) * W(nb[j]);
    }
    return f;
  };
  auto degree_of = [&](int v) {
    long long d = 0;
    for (int a : adj[v]) d += W(a);
    return d;
  };
  std::vector<long long> fill(n), deg(n);
  std::set<std::tuple<long long, long long, int>> pq;
  for (int v = 0; v < n; ++v) {
    fill[v] = fill_of(v);
    deg[v] = degree_of(v);
    pq.insert({fill[v], deg[v], v});
  }
  std::vector<int> perm;
  perm.reserve(n);
  std::vector<char> done(n, 0);
  std::vector<int> tmp, touched;
  std::vector<int> seen(n, -1);
  while (!pq.empty()) {
    const int v = std::get<2>(*pq.begin());
    pq.erase(pq.begin());
    perm.push_back(v);
    done[v] = 1;
    const std::vector<int> nv = adj[v];
    for (int a : nv) {
      // adj[a] <- (adj[a] u nv) \ {a, v}: the neighbours of v become a clique
      tmp.clear();
      std::set_union(adj[a].begin(), adj[a].end(), nv.begin(), nv.end(), std::back_inserter(tmp));
      adj[a].clear();
      for (int u : tmp)
        if (u != a && u != v) adj[a].push_back(u);
    }
    adj[v].clear();
    // the fill of every vertex within two steps of v may have changed
    touched.clear();
    for (int a : nv) {
      if (seen[a] != v) {
        seen[a] = v;
        touched.push_back(a);
      }
      for (int b : adj[a])
        if (!done[b] && seen[b] != v) {
          seen[b] = v;
          touched.push_back(b);
        }
    }
    for (int u : touched) {
      pq.erase({fill[u], deg[u], u});
      fill[u] = fill_of(u);
      deg[u] = degree_of(u);
      pq.insert({fill[u], deg[u], u});
    }
    if (max_work > 0 && work > max_work) return {};  // too dense for this method
  }
  if (const char* e = std::getenv("MPF_ORDER_WORK_LOG")) std::fprintf(stderr, "minimum_fill work %lld\n", work);
  return perm;
}

int LUSymbolic::local(int s, int var) const {
  const int* b = sn_rows.data() + sn_rptr[s];
  const int* e = sn_rows.data() + sn_rptr[s + 1];
  const int* p = std::lower_bound(b, e, var);
  if (p == e || *p != var) return -1;
  return (int)(p - b);
}

int64_t LUSymbolic::entry_pos(int row, int col) const {
  const int s = sn_of[std::min(row, col)];
  const int lr = local(s, row), lc = local(s, col);
  if (lr < 0 || lc < 0) return -1;
  const int w = sn_w[s], f = sn_f[s];
  if (lr < w) return pan_off[s] + (int64_t)lr * f + lc;
  if (lc < w) return pan_off[s] + (int64_t)w * f + (int64_t)(lr - w) * w + lc;
  return -1;
}

void lu_symbolic(int n, const std::vector<std::vector<int>>& adj, LUSymbolic& s, const Relax& relax) {
  s = LUSymbolic();
  s.n = n;
  // elimination tree (Liu), using the entries left of the diagonal of each row
  std::vector<int> parent(n, -1), ancestor(n, -1);
  for (int j = 0; j < n; ++j) {
    for (int i : adj[j]) {
      if (i >= j) continue;
      int r = i;
      while (ancestor[r] != -1 && ancestor[r] != j) {
        const int t = ancestor[r];
        ancestor[r] = j;
        r = t;
      }
      if (ancestor[r] == -1) {
        ancestor[r] = j;
        parent[r] = j;
      }
    }
  }
  s.etree_parent = parent;
  // L column structures: below-diagonal entries of A(:,j) plus children's structures
  std::vector<std::vector<int>> children(n);
  for (int j = 0; j < n; ++j)
    if (parent[j] >= 0) children[parent[j]].push_back(j);
  std::vector<std::vector<int>> Ls(n);
  std::vector<int> mark(n, -1);
  for (int j = 0; j < n; ++j) {
    auto& out = Ls[j];
    mark[j] = j;
    for (int i : adj[j])
      if (i > j && mark[i] != j) { mark[i] = j; out.push_back(i); }
    for (int c : children[j])
      for (int i : Ls[c])
        if (i > j && mark[i] != j) { mark[i] = j; out.push_back(i); }
    std::sort(out.begin(), out.end());
  }
  // fundamental supernodes: j joins j-1 when j is j-1's parent, its only child,
  // and L(:,j) = L(:,j-1) minus row j
  std::vector<int> fs_c0;
  for (int j = 0; j < n; ++j) {
    const bool join = j > 0 && parent[j - 1] == j && children[j].size() == 1 &&
                      Ls[j].size() + 1 == Ls[j - 1].size();
    if (!join) fs_c0.push_back(j);
  }
  const int nfs = (int)fs_c0.size();
  fs_c0.push_back(n);
  std::vector<int> fs_of(n);
  for (int q = 0; q < nfs; ++q)
    for (int j = fs_c0[q]; j < fs_c0[q + 1]; ++j) fs_of[j] = q;
  std::vector<int> fs_parent(nfs, -1);
  std::vector<std::vector<int>> fs_children(nfs);
  for (int q = 0; q < nfs; ++q) {
    const int last = fs_c0[q + 1] - 1;
    if (parent[last] >= 0) {
      fs_parent[q] = fs_of[parent[last]];
      fs_children[fs_parent[q]].push_back(q);
    }
  }
  // Relaxed amalgamation: merge a child supernode into its parent when the merged
  // front stays small and gains few explicit zeros.  The child's pivots join the
  // parent's front (all its contribution-block rows are already there), so its
  // contribution block never leaves the front.  Merged pivot sets need not be
  // consecutive; siblings' pivots are independent.  Children have lower indices
  // than parents, so one increasing pass sees every child before its parent.
  std::vector<int> grp(nfs);                  // group representative (a parent-most supernode)
  std::vector<int> gw(nfs), gf(nfs);          // pivots and front size of the group rooted here
  std::vector<long long> gnnz(nfs);           // true panel entries of the group
  for (int q = 0; q < nfs; ++q) {
    grp[q] = q;
    gw[q] = fs_c0[q + 1] - fs_c0[q];
    gf[q] = 1 + (int)Ls[fs_c0[q]].size();
    gnnz[q] = 2LL * gw[q] * gf[q] - (long long)gw[q] * gw[q];
  }
  if (relax.max_pivots > 1) {
    for (int q = 0; q < nfs; ++q) {
      std::vector<int> ch = fs_children[q];
      std::sort(ch.begin(), ch.end(), [&](int a, int b) { return gw[a] < gw[b] || (gw[a] == gw[b] && a < b); });
      for (int c : ch) {
        const int wm = gw[q] + gw[c], fm = gf[q] + gw[c];
        if (wm > relax.max_pivots || fm > relax.max_front) continue;
        const long long size = 2LL * wm * fm - (long long)wm * wm;
        const long long zeros = size - (gnnz[q] + gnnz[c]);
        if (zeros > relax.max_zeros && (double)zeros > relax.max_zero_frac * (double)size) continue;
        grp[c] = q;
        gw[q] = wm;
        gf[q] = fm;
        gnnz[q] += gnnz[c];
      }
    }
  }
  // resolve groups to their final representative (a merged child's own children
  // that merged into it are already pointing at it)
  std::vector<int> rep(nfs);
  for (int q = nfs - 1; q >= 0; --q) rep[q] = (grp[q] == q) ? q : rep[grp[q]];
  std::vector<int> final_id(nfs, -1);
  int ns = 0;
  for (int q = 0; q < nfs; ++q)
    if (rep[q] == q) final_id[q] = ns++;
  s.nsn = ns;
  s.sn_w.assign(ns, 0);
  s.sn_f.assign(ns, 0);
  s.sn_of.assign(n, -1);
  std::vector<std::vector<int>> piv(ns);
  for (int q = 0; q < nfs; ++q) {
    const int t = final_id[rep[q]];
    for (int j = fs_c0[q]; j < fs_c0[q + 1]; ++j) {
      piv[t].push_back(j);
      s.sn_of[j] = t;
    }
  }
  s.sn_rptr.assign(ns + 1, 0);
  s.sn_parent.assign(ns, -1);
  for (int q = 0; q < nfs; ++q) {
    if (rep[q] != q) continue;
    const int t = final_id[q];
    std::vector<int>& pv = piv[t];
    std::sort(pv.begin(), pv.end());
    const int last = fs_c0[q + 1] - 1;  // the representative's last pivot: its L rows form the CB
    std::vector<int> rows(pv);
    for (int i : Ls[last]) rows.push_back(i);
    s.sn_w[t] = (int)pv.size();
    s.sn_f[t] = (int)rows.size();
    s.sn_rptr[t + 1] = s.sn_rptr[t] + s.sn_f[t];
    s.sn_rows.insert(s.sn_rows.end(), rows.begin(), rows.end());
    s.max_front = std::max(s.max_front, s.sn_f[t]);
    if (parent[last] >= 0) s.sn_parent[t] = s.sn_of[parent[last]];
  }
  // children lists, levels
  s.child_ptr.assign(ns + 1, 0);
  for (int q = 0; q < ns; ++q)
    if (s.sn_parent[q] >= 0) s.child_ptr[s.sn_parent[q] + 1]++;
  for (int q = 0; q < ns; ++q) s.child_ptr[q + 1] += s.child_ptr[q];
  s.child_list.resize(s.child_ptr[ns]);
  {
    std::vector<int> f(s.child_ptr.begin(), s.child_ptr.end() - 1);
    for (int q = 0; q < ns; ++q)
      if (s.sn_parent[q] >= 0) s.child_list[f[s.sn_parent[q]]++] = q;
  }
  s.sn_level.assign(ns, 0);
  s.nlevels = ns > 0 ? 1 : 0;
  for (int q = 0; q < ns; ++q) {  // children have smaller indices than parents
    if (s.sn_parent[q] >= 0) {
      int& lp = s.sn_level[s.sn_parent[q]];
      lp = std::max(lp, s.sn_level[q] + 1);
      s.nlevels = std::max(s.nlevels, lp + 1);
    }
  }
  s.lev_ptr.assign(s.nlevels + 1, 0);
  for (int q = 0; q < ns; ++q) s.lev_ptr[s.sn_level[q] + 1]++;
  for (int l = 0; l < s.nlevels; ++l) s.lev_ptr[l + 1] += s.lev_ptr[l];
  s.lev_sn.resize(ns);
  {
    std::vector<int> f(s.lev_ptr.begin(), s.lev_ptr.end() - 1);
    for (int q = 0; q < ns; ++q) s.lev_sn[f[s.sn_level[q]]++] = q;
    for (int l = 0; l < s.nlevels; ++l)
      std::stable_sort(s.lev_sn.begin() + s.lev_ptr[l], s.lev_sn.begin() + s.lev_ptr[l + 1],
                       [&](int a, int b) { return s.sn_f[a] < s.sn_f[b]; });
  }
  // storage offsets, relative maps, flops (of the dense fronts, explicit zeros included)
  s.pan_off.assign(ns + 1, 0);
  s.cb_off.assign(ns + 1, 0);
  s.cbr_off.assign(ns + 1, 0);
  s.rel_ptr.assign(ns + 1, 0);
  for (int q = 0; q < ns; ++q) {
    const int w = s.sn_w[q], f = s.sn_f[q];
    s.pan_off[q + 1] = s.pan_off[q] + (int64_t)w * f + (int64_t)(f - w) * w;
    s.cb_off[q + 1] = s.cb_off[q] + (int64_t)(f - w) * (f - w);
    s.cbr_off[q + 1] = s.cbr_off[q] + (f - w);
    s.rel_ptr[q + 1] = s.rel_ptr[q] + (s.sn_parent[q] >= 0 ? f - w : 0);
    for (int p = 0; p < w; ++p) {
      const int64_t m = f - p - 1;
      s.flops += m + 2 * m * m;  // column scaling + rank-1 update
      s.nnz_l += m;
    }
    s.sum_cb += (int64_t)(f - w) * (f - w);
  }
  // contribution blocks are stored parent by parent, the children of a supernode
  // adjacent in child_list order, so that everything a front assembles from its
  // children is one contiguous range (cb_off[nsn] / cbr_off[nsn] stay the totals)
  {
    int64_t off = 0, roff = 0;
    auto place = [&](int q) {
      const int64_t m = s.sn_f[q] - s.sn_w[q];
      s.cb_off[q] = off;
      s.cbr_off[q] = roff;
      off += m * m;
      roff += m;
    };
    for (int q = 0; q < ns; ++q)
      for (int c = s.child_ptr[q]; c < s.child_ptr[q + 1]; ++c) place(s.child_list[c]);
    for (int q = 0; q < ns; ++q)
      if (s.sn_parent[q] < 0) place(q);
    s.cb_off[ns] = off;
    s.cbr_off[ns] = roff;
  }
  s.nnz = s.pan_off[ns];
  s.relmap.resize(s.rel_ptr[ns]);
  for (int q = 0; q < ns; ++q) {
    const int par = s.sn_parent[q];
    if (par < 0) continue;
    const int w = s.sn_w[q], f = s.sn_f[q];
    for (int t = 0; t < f - w; ++t) {
      const int var = s.sn_rows[s.sn_rptr[q] + w + t];
      s.relmap[s.rel_ptr[q] + t] = s.local(par, var);  // always >= 0 (CB rows are in the parent's front)
    }
  }
}

void arrowhead_layout(const LUSymbolic& s, const std::vector<int>& rows,
                      const std::vector<int>& cols, std::vector<int>& a_index,
                      std::vector<int>& ah_ptr, std::vector<int>& ah_loc) {
  const size_t m = rows.size();
  std::vector<int> owner(m);
  ah_ptr.assign(s.nsn + 1, 0);
  for (size_t e = 0; e < m; ++e) {
    owner[e] = s.sn_of[std::min(rows[e], cols[e])];
    ah_ptr[owner[e] + 1]++;
  }
  for (int q = 0; q < s.nsn; ++q) ah_ptr[q + 1] += ah_ptr[q];
  std::vector<int> fill(ah_ptr.begin(), ah_ptr.end() - 1);
  a_index.resize(m);
  ah_loc.resize(m);
  for (size_t e = 0; e < m; ++e) {
    const int q = owner[e];
    const int k = fill[q]++;
    a_index[e] = k;
    const int f = s.sn_f[q];
    ah_loc[k] = s.local(q, rows[e]) * ((f + 1) | 1) + s.local(q, cols[e]);
  }
}

// B' / B'' of one fast-decoupled variant: -Im of the modified Ybus restricted to
// the system's buses (makeB.h:326-381 take -Im(Ybus(k)) over pvpq x pvpq / pq x pq).
static void build_fd(GridSymbolic& g, const mpf_bus* buses, const mpf_branch* br,
                     bool is_bp, int variant, const std::vector<int>& var_of_bus, int nvar,
                     const std::vector<std::vector<int>>& adj_var, GridSymbolic::FDSystem& fd) {
  fd.var = var_of_bus;
  lu_symbolic(nvar, adj_var, fd.lu);
  // matrix entries = Ybus positions whose row and column buses are in the system
  const int nnzY = g.y_rowptr[g.nb];
  std::vector<int> rows, cols, ypos_of_entry;
  std::vector<int> y_to_entry(nnzY, -1);
  for (int i = 0; i < g.nb; ++i) {
    if (var_of_bus[i] < 0) continue;
    for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
      const int j = g.y_col[p];
      if (var_of_bus[j] < 0) continue;
      y_to_entry[p] = (int)rows.size();
      rows.push_back(var_of_bus[i]);
      cols.push_back(var_of_bus[j]);
    }
  }
  std::vector<int> a_index;
  arrowhead_layout(fd.lu, rows, cols, a_index, fd.ah_ptr, fd.ah_loc);
  fd.base.assign(rows.size(), 0.0);
  fd.br_pos.assign(4 * (size_t)g.nbr, -1);
  fd.br_val.assign(4 * (size_t)g.nbr, 0.0);
  for (int e = 0; e < g.nbr; ++e) {
    const mpf_branch& b = br[e];
    double r = b.r, chg = b.b, tap = b.tap, shift = b.shift;
    if (is_bp) {
      // B': zero line charging and taps; XB also zeroes R (makeB.h:311-324)
      chg = 0.0;
      tap = 0.0;
      if (variant == 0) r = 0.0;
    } else {
      // B'': zero phase shifters; BX also zeroes R (makeB.h:383-390)
      shift = 0.0;
      if (variant == 1) r = 0.0;
    }
    const BranchY y = branch_admittance(r, b.x, chg, tap, shift, b.status);
    const double vals[4] = {-y.ff[1], -y.ft[1], -y.tf[1], -y.tt[1]};
    for (int q = 0; q < 4; ++q) {
      fd.br_val[4 * e + q] = vals[q];
      const int ent = y_to_entry[g.br_pos[4 * e + q]];
      if (ent >= 0) fd.br_pos[4 * e + q] = a_index[ent];
    }
  }
  // base = sum of branch contributions (CfYf then CtYt order) + shunts
  for (int e = 0; e < g.nbr; ++e)
    for (int q : {0, 1})
      if (fd.br_pos[4 * e + q] >= 0) fd.base[fd.br_pos[4 * e + q]] += fd.br_val[4 * e + q];
  for (int e = 0; e < g.nbr; ++e)
    for (int q : {2, 3})
      if (fd.br_pos[4 * e + q] >= 0) fd.base[fd.br_pos[4 * e + q]] += fd.br_val[4 * e + q];
  fd.diag_pos.assign(g.nb, -1);
  for (int i = 0; i < g.nb; ++i) {
    if (var_of_bus[i] < 0) continue;
    // B' has Bsh zeroed (makeB.h:320-323); B'' keeps the bus shunt: -Im(j Bsh)
    const double sh = is_bp ? 0.0 : -buses[i].bsh;
    fd.diag_pos[i] = a_index[y_to_entry[g.y_diag[i]]];
    fd.base[fd.diag_pos[i]] += sh;
  }
}

std::string build_symbolic(const mpf_bus* buses, int nb, const mpf_branch* br, int nbr,
                           GridSymbolic& g, const std::vector<char>* vm_free, int ordering) {
  g = GridSymbolic();
  if (nb < 2) return "grid needs at least 2 buses";
  if (nbr < 1) return "grid needs at least 1 branch";
  g.nb = nb;
  g.nbr = nbr;
  g.bus_type.resize(nb);
  for (int i = 0; i < nb; ++i) {
    const int t = buses[i].type;
    if (t < MPF_BUS_NONE || t > MPF_BUS_ISOLATED) return "bus " + std::to_string(i) + " has an invalid type";
    if (!std::isfinite(buses[i].vm) || !std::isfinite(buses[i].va) || !std::isfinite(buses[i].p) ||
        !std::isfinite(buses[i].q) || !std::isfinite(buses[i].gsh) || !std::isfinite(buses[i].bsh))
      return "bus " + std::to_string(i) + " has a non-finite field";
    g.bus_type[i] = t;
    if (t == MPF_BUS_SLACK) {
      if (g.slack < 0) g.slack = i;
      ++g.n_slack;
    } else if (t == MPF_BUS_PV) {
      g.pv.push_back(i);
    } else if (t == MPF_BUS_PQ) {
      g.pq.push_back(i);
    }
  }
  if (g.slack < 0) return "no slack bus";
  g.npv = (int)g.pv.size();
  g.npq = (int)g.pq.size();
  for (int e = 0; e < nbr; ++e) {
    const mpf_branch& b = br[e];
    if (b.from < 0 || b.from >= nb || b.to < 0 || b.to >= nb)
      return "branch " + std::to_string(e) + " has a bus index out of range";
    if (b.from == b.to) return "branch " + std::to_string(e) + " connects a bus to itself";
    if (!std::isfinite(b.r) || !std::isfinite(b.x) || !std::isfinite(b.b) || !std::isfinite(b.tap) ||
        !std::isfinite(b.shift))
      return "branch " + std::to_string(e) + " has a non-finite field";
    if (b.x == 0.0) return "branch " + std::to_string(e) + " has zero reactance";
    if (b.status != 0 && b.status != 1) return "branch " + std::to_string(e) + " status must be 0 or 1";
  }
  // Islands: connected components over every branch (in or out of service).  Each
  // component with PV/PQ buses needs exactly one slack; several islands make a
  // multi-grid handle whose Jacobian is block-diagonal (one block per island).
  {
    std::vector<int> comp(nb);
    for (int i = 0; i < nb; ++i) comp[i] = i;
    std::function<int(int)> root = [&](int i) {
      while (comp[i] != i) {
        comp[i] = comp[comp[i]];
        i = comp[i];
      }
      return i;
    };
    for (int e = 0; e < nbr; ++e) {
      const int a = root(br[e].from), b = root(br[e].to);
      if (a != b) comp[std::max(a, b)] = std::min(a, b);
    }
    std::vector<int> slack_of(nb, -1), free_of(nb, 0);
    for (int i = 0; i < nb; ++i) {
      const int r = root(i);
      if (g.bus_type[i] == MPF_BUS_SLACK) {
        if (slack_of[r] >= 0)
          return "more than one slack bus in one connected island (buses " + std::to_string(slack_of[r]) + " and " +
                 std::to_string(i) + ")";
        slack_of[r] = i;
      } else if (g.bus_type[i] == MPF_BUS_PV || g.bus_type[i] == MPF_BUS_PQ) {
        ++free_of[r];
      }
    }
    std::vector<int> island_of_root(nb, -1);
    for (int i = 0; i < nb; ++i)  // islands numbered in the order of their slack buses
      if (g.bus_type[i] == MPF_BUS_SLACK) island_of_root[root(i)] = g.n_islands++;
    g.bus_island.assign(nb, -1);
    for (int i = 0; i < nb; ++i) {
      const int r = root(i);
      if (free_of[r] > 0 && slack_of[r] < 0)
        return "bus " + std::to_string(i) + " is in a connected island without a slack bus";
      g.bus_island[i] = island_of_root[r];
    }
    g.br_island.resize(nbr);
    for (int e = 0; e < nbr; ++e) g.br_island[e] = g.bus_island[br[e].from];
  }
  // Ybus superset pattern
  std::vector<std::vector<int>> rows(nb);
  for (int i = 0; i < nb; ++i) rows[i].push_back(i);
  for (int e = 0; e < nbr; ++e) {
    rows[br[e].from].push_back(br[e].to);
    rows[br[e].to].push_back(br[e].from);
  }
  g.y_rowptr.assign(nb + 1, 0);
  for (int i = 0; i < nb; ++i) {
    auto& r = rows[i];
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    g.y_rowptr[i + 1] = g.y_rowptr[i] + (int)r.size();
  }
  const int nnzY = g.y_rowptr[nb];
  g.y_col.resize(nnzY);
  g.y_diag.resize(nb);
  for (int i = 0; i < nb; ++i) {
    std::copy(rows[i].begin(), rows[i].end(), g.y_col.begin() + g.y_rowptr[i]);
  }
  auto ypos = [&](int i, int j) {
    const int* b = g.y_col.data() + g.y_rowptr[i];
    const int* e = g.y_col.data() + g.y_rowptr[i + 1];
    const int* p = std::lower_bound(b, e, j);
    return (int)(p - g.y_col.data());
  };
  for (int i = 0; i < nb; ++i) g.y_diag[i] = ypos(i, i);
  g.br_pos.resize(4 * (size_t)nbr);
  g.br_y.resize(8 * (size_t)nbr);
  g.br_from.resize(nbr);
  g.br_to.resize(nbr);
  g.br_status.resize(nbr);
  g.y_val.assign(2 * (size_t)nnzY, 0.0);
  for (int e = 0; e < nbr; ++e) {
    const mpf_branch& b = br[e];
    const int f = b.from, t = b.to;
    g.br_from[e] = f;
    g.br_to[e] = t;
    g.br_status[e] = b.status;
    g.br_pos[4 * e + 0] = g.y_diag[f];
    g.br_pos[4 * e + 1] = ypos(f, t);
    g.br_pos[4 * e + 2] = ypos(t, f);
    g.br_pos[4 * e + 3] = g.y_diag[t];
    const BranchY y = branch_admittance(b.r, b.x, b.b, b.tap, b.shift, b.status);
    const double* parts[4] = {y.ff, y.ft, y.tf, y.tt};
    for (int q = 0; q < 4; ++q) {
      g.br_y[8 * e + 2 * q + 0] = parts[q][0];
      g.br_y[8 * e + 2 * q + 1] = parts[q][1];
    }
  }
  // base values: Cf*Yf, then Ct*Yt, then Ysh (makeYbus.h:194-273)
  for (int e = 0; e < nbr; ++e)
    for (int q : {0, 1}) {
      const int p = g.br_pos[4 * e + q];
      g.y_val[2 * p] += g.br_y[8 * e + 2 * q];
      g.y_val[2 * p + 1] += g.br_y[8 * e + 2 * q + 1];
    }
  for (int e = 0; e < nbr; ++e)
    for (int q : {2, 3}) {
      const int p = g.br_pos[4 * e + q];
      g.y_val[2 * p] += g.br_y[8 * e + 2 * q];
      g.y_val[2 * p + 1] += g.br_y[8 * e + 2 * q + 1];
    }
  for (int i = 0; i < nb; ++i) {
    g.y_val[2 * g.y_diag[i]] += buses[i].gsh;
    g.y_val[2 * g.y_diag[i] + 1] += buses[i].bsh;
  }
  // injections and start point (runpf.h:211-226)
  g.sbus.resize(2 * (size_t)nb);
  g.v0.resize(2 * (size_t)nb);
  for (int i = 0; i < nb; ++i) {
    g.sbus[2 * i] = buses[i].p;
    g.sbus[2 * i + 1] = buses[i].q;
    double vr = buses[i].vm * std::cos(buses[i].va);
    double vi = buses[i].vm * std::sin(buses[i].va);
    if (buses[i].type == MPF_BUS_PV || buses[i].type == MPF_BUS_SLACK) {
      const double a = std::hypot(vr, vi);
      if (a > 0.0) {
        vr *= buses[i].vm / a;
        vi *= buses[i].vm / a;
      }
    }
    g.v0[2 * i] = vr;
    g.v0[2 * i + 1] = vi;
  }
  // Newton system ordering at bus level (PV and PQ buses)
  std::vector<int> free_idx(nb, -1), free_bus;
  for (int i = 0; i < nb; ++i)
    if (g.bus_type[i] == MPF_BUS_PV || g.bus_type[i] == MPF_BUS_PQ) {
      free_idx[i] = (int)free_bus.size();
      free_bus.push_back(i);
    }
  const int nfree = (int)free_bus.size();
  if (nfree == 0) return "grid has no PV or PQ bus";
  std::vector<std::vector<int>> badj(nfree);
  for (int a = 0; a < nfree; ++a) {
    const int i = free_bus[a];
    for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
      const int j = g.y_col[p];
      if (j != i && free_idx[j] >= 0) badj[a].push_back(free_idx[j]);
    }
  }
  // Vm is a variable of every PQ bus, and of PV buses that may switch to PQ (their Q
  // limits are enforced): a superset pattern shared by all cases
  auto has_vm = [&](int i) {
    return g.bus_type[i] == MPF_BUS_PQ || (vm_free && (*vm_free)[i] && g.bus_type[i] == MPF_BUS_PV);
  };
  // the Newton system's numbering and symbolic LU for one bus elimination order
  auto newton_symbolic = [&](const std::vector<int>& border) {
    g.bus_order.resize(nfree);
    g.var_va.assign(nb, -1);
    g.var_vm.assign(nb, -1);
    int nv = 0;
    for (int k = 0; k < nfree; ++k) {
      const int i = free_bus[border[k]];
      g.bus_order[k] = i;
      g.var_va[i] = nv++;
      if (has_vm(i)) g.var_vm[i] = nv++;
    }
    std::vector<std::vector<int>> vadj(nv);
    for (int i : g.bus_order) {
      const int vi[2] = {g.var_va[i], g.var_vm[i]};
      if (vi[1] >= 0) {
        vadj[vi[0]].push_back(vi[1]);
        vadj[vi[1]].push_back(vi[0]);
      }
      for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
        const int j = g.y_col[p];
        if (j == i || free_idx[j] < 0) continue;
        const int vj[2] = {g.var_va[j], g.var_vm[j]};
        for (int a : vi)
          for (int b : vj)
            if (a >= 0 && b >= 0) vadj[a].push_back(b);
      }
    }
    for (auto& a : vadj) {
      std::sort(a.begin(), a.end());
      a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    lu_symbolic(nv, vadj, g.jac);
  };
  // Bus elimination order.  Candidates: minimum degree; minimum fill (deficiency); and
  // minimum fill with each bus weighted by its variables (2 for a bus with Va and Vm, 1
  // for Va alone), which counts the fill of the Newton system itself.  Automatic choice:
  // the candidate with the least estimated factorisation time per case,
  //   flops + kLevelFlops x levels,
  // a level (one launch of the level-synchronous factorisation and backward solve)
  // costing about as much as 53k flops per case: fitted on measured B200 times of the
  // 9241-bus synthetic workload and case9241pegase, 1000 N-1 cases each, four orderings
  // (factorisation + backward solve = 3.24 ms per MFLOP per case + 0.172 ms per level).
  std::vector<int> wvar(nfree);
  for (int a = 0; a < nfree; ++a) wvar[a] = has_vm(free_bus[a]) ? 2 : 1;
  // budget of the automatic choice's minimum-fill runs: their cost grows with the fill,
  // so on densely meshed grids (where fronts are large anyway) they give way to
  // minimum degree; a method asked for explicitly always runs
  const long long work_cap = 400LL * 1000 * 1000;
  auto order_of = [&](int method, long long cap) {
    if (method == MPF_ORDER_MIN_FILL) return minimum_fill(nfree, badj, nullptr, cap);
    if (method == MPF_ORDER_MIN_FILL_WEIGHTED) return minimum_fill(nfree, badj, &wvar, cap);
    return minimum_degree(nfree, badj);
  };
  int method = ordering;
  if (method == MPF_ORDER_AUTO) {
    constexpr double kLevelFlops = 53000.0;
    double best = 0.0;
    for (int m : {MPF_ORDER_MIN_DEGREE, MPF_ORDER_MIN_FILL, MPF_ORDER_MIN_FILL_WEIGHTED}) {
      const std::vector<int> ord = order_of(m, work_cap);
      if (ord.empty()) continue;
      newton_symbolic(ord);
      const double cost = (double)g.jac.flops + kLevelFlops * g.jac.nlevels;
      if (method == MPF_ORDER_AUTO || cost < best) {
        best = cost;
        method = m;
      }
    }
  }
  newton_symbolic(order_of(method, 0));
  g.ordering = method;
  // J entries: the (Va,Va), (Va,Vm), (Vm,Va), (Vm,Vm) quadrants of every Ybus entry
  // between PV/PQ buses (newtonpf.h:215-295 enumerate the same set)
  std::vector<int> jr, jc, jsrc;
  for (int i = 0; i < nb; ++i) {
    if (free_idx[i] < 0) continue;
    for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
      const int j = g.y_col[p];
      if (free_idx[j] < 0) continue;
      const int r[4] = {g.var_va[i], g.var_va[i], g.var_vm[i], g.var_vm[i]};
      const int c[4] = {g.var_va[j], g.var_vm[j], g.var_va[j], g.var_vm[j]};
      for (int q = 0; q < 4; ++q) {
        if (r[q] < 0 || c[q] < 0) continue;
        jr.push_back(r[q]);
        jc.push_back(c[q]);
        jsrc.push_back(4 * p + q);
      }
    }
  }
  std::vector<int> a_index;
  arrowhead_layout(g.jac, jr, jc, a_index, g.ah_ptr, g.ah_loc);
  g.jpos.assign(4 * (size_t)nnzY, -1);
  for (size_t e = 0; e < jsrc.size(); ++e) g.jpos[jsrc[e]] = a_index[e];
  g.nnz_jac = (int)jsrc.size();
  g.mis_rows = g.bus_order;

  // fast-decoupled systems
  {
    std::vector<int> var_bp(nb, -1);
    for (int k = 0; k < nfree; ++k) var_bp[g.bus_order[k]] = k;
    std::vector<std::vector<int>> adj_bp(nfree);
    for (int k = 0; k < nfree; ++k) {
      const int i = g.bus_order[k];
      for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
        const int j = g.y_col[p];
        if (j != i && var_bp[j] >= 0) adj_bp[k].push_back(var_bp[j]);
      }
      std::sort(adj_bp[k].begin(), adj_bp[k].end());
    }
    // B'': PQ buses ordered by minimum degree on the PQ-induced subgraph
    std::vector<int> pq_idx(nb, -1);
    for (int k = 0; k < g.npq; ++k) pq_idx[g.pq[k]] = k;
    std::vector<std::vector<int>> adj_pq(g.npq);
    for (int k = 0; k < g.npq; ++k) {
      const int i = g.pq[k];
      for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
        const int j = g.y_col[p];
        if (j != i && pq_idx[j] >= 0) adj_pq[k].push_back(pq_idx[j]);
      }
    }
    const std::vector<int> pord = minimum_degree(g.npq, adj_pq);
    g.bpp_order.resize(g.npq);
    std::vector<int> var_bpp(nb, -1);
    for (int k = 0; k < g.npq; ++k) {
      g.bpp_order[k] = g.pq[pord[k]];
      var_bpp[g.bpp_order[k]] = k;
    }
    std::vector<std::vector<int>> adj_bpp(g.npq);
    for (int k = 0; k < g.npq; ++k) {
      const int i = g.bpp_order[k];
      for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
        const int j = g.y_col[p];
        if (j != i && var_bpp[j] >= 0) adj_bpp[k].push_back(var_bpp[j]);
      }
      std::sort(adj_bpp[k].begin(), adj_bpp[k].end());
    }
    for (int variant = 0; variant < 2; ++variant) {
      build_fd(g, buses, br, true, variant, var_bp, nfree, adj_bp, g.bp[variant]);
      build_fd(g, buses, br, false, variant, var_bpp, g.npq, adj_bpp, g.bpp[variant]);
    }
  }
  return std::string();
}

}  // namespace mpf

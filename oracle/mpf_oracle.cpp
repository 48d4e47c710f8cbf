// mpf_oracle.cpp — CPU FP64 oracle for the batched power flow.  TEST INFRASTRUCTURE:
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
// load it, always as the checker or the timed CPU baseline, never as the product.
//
// It restates the reference's CPU path (the mkl_* functions of
// src/powerflow/{runpf,makeYbus,newtonpf,makeB,fdpf}.h) case by case:
//   Ybus          makeYbus.h:40-107 (pi model) and :113-274 (Cf*Yf + Ct*Yt + Ysh)
//   start point   runpf.h:211-226
//   mismatch      newtonpf.h:18-71      (F = [Re mis_pv; Re mis_pq; Im mis_pq], max |F|)
//   Ibus          newtonpf.h:73-95
//   Jacobian      newtonpf.h:97-186 with the pattern/order of :215-310
//   update        newtonpf.h:188-213    (polar, dx subtracted)
//   NR loop       newtonpf.h:365-523    (tol strict '<', at most max_it iterations)
//   B', B''       makeB.h:311-501       (XB: R=0 in B'; BX: R=0 in B'')
//   FDPF loop     fdpf.h:369-596        (P half, check, Q half, check)
//   branch loss   runpf.h:228-257
// A case = the base grid with its outaged branches' status set to 0, which is how
// the reference itself removes a branch (makeYbus.h:69-73: Ys and Bc scaled by
// status, the pattern kept).
//
// Linear solvers: ORACLE_SOLVER_GP, a sparse LU with partial pivoting (left-looking
// Gilbert-Peierls) after a minimum-degree column ordering, written here; and, when
// compiled with -DORACLE_WITH_EIGEN against the reference's vendored Eigen 3.2.8
// (src/Eigen), ORACLE_SOLVER_EIGEN = SparseLU<SparseMatrix<double>, COLAMDOrdering<int>>
// with compute() on every solve, exactly the reference's Eigen_SparseLU option
// (newtonpf.h:341-363).
//
// Parity pin: the reference's own CPU power flow, compiled unmodified from its sources
// into oracle/_ref/librefpf.so (oracle/ref_pf.cu, with in-project MKL stand-ins),
// produces the same converged flags and iteration counts and voltages within ~1e-13 on
// its bundled MATPOWER cases with N-1 outages, for NR, FDXB and FDBX
// (tests/test_oracle_reference_pin.py).  Also cross-checked against an independent
// numpy/scipy polar-form Newton-Raphson and hand-solvable 2-bus cases.
//
// Quirk policy (reference behaviours the oracle chooses explicitly):
//   * convergence uses max |F| (CPU path, newtonpf.h:59-67), not the GPU path's
//     max F without abs (newtonpf.h:1451);
//   * the angle of V uses atan2 unless angle_mode = 1, which reproduces
//     cuCangle = atan(y/x) (util/complexUtils.h:21-23);
//   * iteration counts are per case (the reference's GPU path counts globally).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <set>
#include <vector>

#include "mpf.h"

#ifdef ORACLE_WITH_EIGEN
#include <Eigen/SparseLU>
#endif

#define ORACLE_SOLVER_GP 0
#define ORACLE_SOLVER_EIGEN 1
#define ORACLE_SOLVER_EIGEN_REUSE 2  // Eigen SparseLU, analyzePattern once per case, factorize per solve

namespace {

struct Cx {
  double re, im;
};
inline Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
inline Cx csub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
inline Cx cconj(Cx a) { return {a.re, -a.im}; }
inline Cx cdiv(Cx a, Cx b) {
  const double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
inline double cabs_(Cx a) { return std::hypot(a.re, a.im); }
inline Cx cexpj(double th) { return {std::cos(th), std::sin(th)}; }

struct Grid {
  int nb = 0, nbr = 0;
  std::vector<mpf_bus> bus;
  std::vector<mpf_branch> br;
  std::vector<int> pv, pq;
  std::vector<int> idx;  // indicePVPQ (Topology.h:60-80): PV 0..npv-1, PQ npv..npv+npq-1
};

void classify(Grid& g) {
  g.pv.clear();
  g.pq.clear();
  for (int i = 0; i < g.nb; ++i) {
    if (g.bus[i].type == MPF_BUS_PV) g.pv.push_back(i);
    else if (g.bus[i].type == MPF_BUS_PQ) g.pq.push_back(i);
  }
  g.idx.assign(g.nb, -1);
  for (size_t k = 0; k < g.pv.size(); ++k) g.idx[g.pv[k]] = (int)k;
  for (size_t k = 0; k < g.pq.size(); ++k) g.idx[g.pq[k]] = (int)(g.pv.size() + k);
}

struct CsrC {  // complex CSR
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<Cx> val;
};

// makeYbus.h:40-107 (pi model per branch) and :113-274 (sum).  The pattern holds
// the diagonal of every bus and both off-diagonals of every branch.
CsrC make_ybus(const Grid& g, const std::vector<mpf_branch>& br, const std::vector<double>& bsh) {
  CsrC y;
  y.n = g.nb;
  std::vector<std::vector<int>> rows(g.nb);
  for (int i = 0; i < g.nb; ++i) rows[i].push_back(i);
  for (const auto& b : br) {
    rows[b.from].push_back(b.to);
    rows[b.to].push_back(b.from);
  }
  y.ptr.assign(g.nb + 1, 0);
  for (int i = 0; i < g.nb; ++i) {
    std::sort(rows[i].begin(), rows[i].end());
    rows[i].erase(std::unique(rows[i].begin(), rows[i].end()), rows[i].end());
    y.ptr[i + 1] = y.ptr[i] + (int)rows[i].size();
  }
  y.col.resize(y.ptr[g.nb]);
  for (int i = 0; i < g.nb; ++i) std::copy(rows[i].begin(), rows[i].end(), y.col.begin() + y.ptr[i]);
  y.val.assign(y.col.size(), Cx{0, 0});
  auto at = [&](int i, int j) -> Cx& {
    const int p = (int)(std::lower_bound(y.col.begin() + y.ptr[i], y.col.begin() + y.ptr[i + 1], j) - y.col.begin());
    return y.val[p];
  };
  std::vector<Cx> yff(br.size()), yft(br.size()), ytf(br.size()), ytt(br.size());
  for (size_t k = 0; k < br.size(); ++k) {
    const mpf_branch& b = br[k];
    const double stat = b.status ? 1.0 : 0.0;
    const Cx ys = cdiv(Cx{stat, 0}, Cx{b.r, b.x});
    const Cx bc = Cx{0, stat * b.b};
    Cx tap = Cx{b.tap != 0.0 ? b.tap : 1.0, 0.0};
    tap = cmul(tap, cexpj(M_PI / 180.0 * b.shift));
    ytt[k] = cadd(ys, Cx{bc.re / 2, bc.im / 2});
    yff[k] = cdiv(ytt[k], cmul(tap, cconj(tap)));
    yft[k] = cdiv(Cx{-ys.re, -ys.im}, cconj(tap));
    ytf[k] = cdiv(Cx{-ys.re, -ys.im}, tap);
  }
  // Cf*Yf, then Ct*Yt, then Ysh (makeYbus.h:194-273)
  for (size_t k = 0; k < br.size(); ++k) {
    at(br[k].from, br[k].from) = cadd(at(br[k].from, br[k].from), yff[k]);
    at(br[k].from, br[k].to) = cadd(at(br[k].from, br[k].to), yft[k]);
  }
  for (size_t k = 0; k < br.size(); ++k) {
    at(br[k].to, br[k].from) = cadd(at(br[k].to, br[k].from), ytf[k]);
    at(br[k].to, br[k].to) = cadd(at(br[k].to, br[k].to), ytt[k]);
  }
  for (int i = 0; i < g.nb; ++i) at(i, i) = cadd(at(i, i), Cx{g.bus[i].gsh, bsh[i]});
  return y;
}

double angle_of(Cx v, int angle_mode) {
  return angle_mode == 1 ? std::atan(v.im / v.re) : std::atan2(v.im, v.re);
}

// newtonpf.h:18-71: F = [Re mis_pv; Re mis_pq; Im mis_pq], returns max |F|
double nr_mismatch(const Grid& g, const CsrC& y, const std::vector<Cx>& V, const std::vector<Cx>& S,
                   std::vector<double>& F) {
  const int npv = (int)g.pv.size(), npq = (int)g.pq.size();
  F.assign(npv + 2 * npq, 0.0);
  double err = 0.0;
  for (int id = 0; id < npv + npq; ++id) {
    const int bus = id < npv ? g.pv[id] : g.pq[id - npv];
    Cx c{0, 0};
    for (int k = y.ptr[bus]; k < y.ptr[bus + 1]; ++k) c = cadd(c, cmul(y.val[k], V[y.col[k]]));
    const Cx mis = csub(cmul(V[bus], cconj(c)), S[bus]);
    if (id < npv) {
      F[id] = mis.re;
      err = std::max(err, std::fabs(mis.re));
    } else {
      const int i = id - npv;
      F[npv + i] = mis.re;
      F[npv + npq + i] = mis.im;
      err = std::max(err, std::max(std::fabs(mis.re), std::fabs(mis.im)));
    }
  }
  return err;
}

struct CsrR {  // real CSR
  int n = 0;
  std::vector<int> ptr, col;
  std::vector<double> val;
};

// Jacobian pattern of newtonpf.h:215-310 (rows sorted by column inside a row)
CsrR jac_pattern(const Grid& g, const CsrC& y) {
  const int npv = (int)g.pv.size(), npq = (int)g.pq.size();
  const int n = npv + 2 * npq;
  std::vector<std::vector<int>> rows(n);
  for (int i = 0; i < g.nb; ++i) {
    const int ti = g.bus[i].type;
    if (ti != MPF_BUS_PV && ti != MPF_BUS_PQ) continue;
    for (int k = y.ptr[i]; k < y.ptr[i + 1]; ++k) {
      const int j = y.col[k];
      const int tj = g.bus[j].type;
      if (tj != MPF_BUS_PV && tj != MPF_BUS_PQ) continue;
      const int ri = g.idx[i], cj = g.idx[j];
      rows[ri].push_back(cj);
      if (tj == MPF_BUS_PQ) rows[ri].push_back(cj + npq);
      if (ti == MPF_BUS_PQ) {
        rows[ri + npq].push_back(cj);
        if (tj == MPF_BUS_PQ) rows[ri + npq].push_back(cj + npq);
      }
    }
  }
  CsrR J;
  J.n = n;
  J.ptr.assign(n + 1, 0);
  for (int r = 0; r < n; ++r) {
    std::sort(rows[r].begin(), rows[r].end());
    J.ptr[r + 1] = J.ptr[r] + (int)rows[r].size();
  }
  J.col.resize(J.ptr[n]);
  for (int r = 0; r < n; ++r) std::copy(rows[r].begin(), rows[r].end(), J.col.begin() + J.ptr[r]);
  J.val.assign(J.col.size(), 0.0);
  return J;
}

int var_bus(const Grid& g, int v) {
  const int npv = (int)g.pv.size(), npq = (int)g.pq.size();
  if (v < npv + npq) return v < npv ? g.pv[v] : g.pq[v - npv];
  return g.pq[v - npv - npq];
}

// newtonpf.h:97-186 (rectangular-component form of dS/dVa and dS/dVm)
void jac_values(const Grid& g, const CsrC& y, const std::vector<Cx>& V, const std::vector<Cx>& Ibus, CsrR& J) {
  const int len = (int)(g.pv.size() + g.pq.size());
  for (int r = 0; r < J.n; ++r) {
    const int ii = var_bus(g, r);
    for (int k = J.ptr[r]; k < J.ptr[r + 1]; ++k) {
      const int c = J.col[k];
      const int jj = var_bus(g, c);
      Cx a{0, 0};
      for (int q = y.ptr[ii]; q < y.ptr[ii + 1]; ++q)
        if (y.col[q] == jj) { a = y.val[q]; break; }
      const double ar = a.re, ai = a.im;
      const double mj = V[jj].re, aj = V[jj].im;  // real / imaginary parts
      const double ir = ii == jj ? Ibus[ii].re : 0.0, iim = ii == jj ? Ibus[ii].im : 0.0;
      const double mi = V[ii].re, ai_ = V[ii].im;
      double val;
      if (r < len) {
        if (c < len) {
          const double re = ar * mj - ai * aj, im = ar * aj + ai * mj;
          val = -ai_ * (ir - re) - mi * (-iim + im);
        } else {
          const double ab = std::sqrt(mj * mj + aj * aj);
          const double re = ar * mj / ab - ai * aj / ab, im = ar * aj / ab + ai * mj / ab;
          val = mi * re - ai_ * -im + ir * mj / ab + iim * aj / ab;
        }
      } else {
        if (c < len) {
          const double re = ar * mj - ai * aj, im = ar * aj + ai * mj;
          val = -ai_ * (-iim + im) + mi * (ir - re);
        } else {
          const double ab = std::sqrt(mj * mj + aj * aj);
          const double re = ar * mj / ab - ai * aj / ab, im = ar * aj / ab + ai * mj / ab;
          val = mi * -im + ai_ * re + ir * aj / ab + -iim * mj / ab;
        }
      }
      J.val[k] = val;
    }
  }
}

// ---------------------------------------------------------------- linear solvers
// Minimum degree on the pattern of A + A^T (ties: lowest index).
std::vector<int> min_degree(const CsrR& A) {
  const int n = A.n;
  std::vector<std::vector<int>> adj(n);
  for (int r = 0; r < n; ++r)
    for (int k = A.ptr[r]; k < A.ptr[r + 1]; ++k) {
      const int c = A.col[k];
      if (c == r) continue;
      adj[r].push_back(c);
      adj[c].push_back(r);
    }
  for (auto& a : adj) {
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end()), a.end());
  }
  std::set<std::pair<int, int>> heap;
  for (int v = 0; v < n; ++v) heap.insert({(int)adj[v].size(), v});
  std::vector<int> order;
  std::vector<int> merged;
  while (!heap.empty()) {
    const int v = heap.begin()->second;
    heap.erase(heap.begin());
    order.push_back(v);
    const std::vector<int> nv = adj[v];
    for (int a : nv) {
      heap.erase({(int)adj[a].size(), a});
      merged.clear();
      std::set_union(adj[a].begin(), adj[a].end(), nv.begin(), nv.end(), std::back_inserter(merged));
      adj[a].clear();
      for (int u : merged)
        if (u != a && u != v) adj[a].push_back(u);
      heap.insert({(int)adj[a].size(), a});
    }
    adj[v].clear();
  }
  return order;
}

// Left-looking sparse LU with partial pivoting (Gilbert-Peierls): P A Q = L U.
// Returns false when a column has no usable pivot.
struct SparseLUPP {
  int n = 0;
  std::vector<int> q;                      // column order
  std::vector<int> pinv;                   // row -> pivot step
  std::vector<std::vector<int>> Li, Ui;    // per column: row indices (L: original rows)
  std::vector<std::vector<double>> Lx, Ux; // L unit diagonal omitted; U diagonal last
  bool factor(const CsrR& A, const std::vector<int>& order) {
    n = A.n;
    q = order;
    // CSC of A
    std::vector<int> cp(n + 1, 0), ri(A.col.size());
    std::vector<double> vx(A.col.size());
    for (int r = 0; r < n; ++r)
      for (int k = A.ptr[r]; k < A.ptr[r + 1]; ++k) cp[A.col[k] + 1]++;
    for (int c = 0; c < n; ++c) cp[c + 1] += cp[c];
    {
      std::vector<int> f(cp.begin(), cp.end() - 1);
      for (int r = 0; r < n; ++r)
        for (int k = A.ptr[r]; k < A.ptr[r + 1]; ++k) {
          const int p = f[A.col[k]]++;
          ri[p] = r;
          vx[p] = A.val[k];
        }
    }
    pinv.assign(n, -1);
    Li.assign(n, {});
    Lx.assign(n, {});
    Ui.assign(n, {});
    Ux.assign(n, {});
    std::vector<double> x(n, 0.0);
    std::vector<int> mark(n, -1), stack, outstack, xi;
    std::vector<int> pstack(n);
    for (int k = 0; k < n; ++k) {
      const int col = q[k];
      // reach: DFS from the nonzeros of A(:,col) through columns of L already pivoted
      xi.clear();
      for (int p = cp[col]; p < cp[col + 1]; ++p) {
        const int r0 = ri[p];
        if (mark[r0] == k) continue;
        stack.assign(1, r0);
        mark[r0] = k;
        pstack[r0] = 0;
        while (!stack.empty()) {
          const int r = stack.back();
          const int j = pinv[r];
          bool pushed = false;
          if (j >= 0) {
            for (int& t = pstack[r]; t < (int)Li[j].size();) {
              const int rr = Li[j][t++];
              if (mark[rr] != k) {
                mark[rr] = k;
                pstack[rr] = 0;
                stack.push_back(rr);
                pushed = true;
                break;
              }
            }
          }
          if (!pushed) {
            stack.pop_back();
            xi.push_back(r);  // postorder
          }
        }
      }
      // numeric: x = L \ A(:,col) in topological order (reverse postorder)
      for (int r : xi) x[r] = 0.0;
      for (int p = cp[col]; p < cp[col + 1]; ++p) x[ri[p]] = vx[p];
      for (int t = (int)xi.size() - 1; t >= 0; --t) {
        const int r = xi[t];
        const int j = pinv[r];
        if (j < 0) continue;
        const double xr = x[r];
        for (size_t u = 0; u < Li[j].size(); ++u) x[Li[j][u]] -= Lx[j][u] * xr;
      }
      // pivot: largest |x| among rows not yet pivoted
      int piv = -1;
      double best = -1.0;
      for (int r : xi) {
        if (pinv[r] < 0 && std::fabs(x[r]) > best) {
          best = std::fabs(x[r]);
          piv = r;
        }
      }
      if (piv < 0 || !(best > 0.0) || !std::isfinite(best)) return false;
      const double pv = x[piv];
      for (int r : xi) {
        if (pinv[r] >= 0) {
          Ui[k].push_back(pinv[r]);
          Ux[k].push_back(x[r]);
        } else if (r != piv) {
          Li[k].push_back(r);
          Lx[k].push_back(x[r] / pv);
        }
      }
      Ui[k].push_back(k);
      Ux[k].push_back(pv);
      pinv[piv] = k;
    }
    return true;
  }
  // solves A x = b
  void solve(const std::vector<double>& b, std::vector<double>& xout) const {
    // A Q = Lt U with Lt = L in original-row numbering (unit entry at the pivot row).
    // Forward: Lt w = b, column by column; backward: U w' = w; x(q) = w'.
    std::vector<int> prow(n);
    for (int r = 0; r < n; ++r) prow[pinv[r]] = r;
    std::vector<double> z(b), w(n, 0.0);
    for (int k = 0; k < n; ++k) {
      const double zk = z[prow[k]];
      w[k] = zk;
      for (size_t u = 0; u < Li[k].size(); ++u) z[Li[k][u]] -= Lx[k][u] * zk;
    }
    for (int k = n - 1; k >= 0; --k) {
      w[k] /= Ux[k].back();
      const double wk = w[k];
      for (size_t u = 0; u + 1 < Ui[k].size(); ++u) w[Ui[k][u]] -= Ux[k][u] * wk;
    }
    xout.assign(n, 0.0);
    for (int k = 0; k < n; ++k) xout[q[k]] = w[k];
  }
};

struct Solver {
  int kind = ORACLE_SOLVER_GP;
  std::vector<int> order;  // cached column order for GP (pattern fixed per system)
#ifdef ORACLE_WITH_EIGEN
  // ORACLE_SOLVER_EIGEN_REUSE: the same SparseLU with its symbolic analysis (COLAMD
  // ordering, elimination tree) done on the first solve and reused, the pattern of the
  // system being fixed
  std::unique_ptr<Eigen::SparseLU<Eigen::SparseMatrix<double>, Eigen::COLAMDOrdering<int> > > reuse;
#endif
  bool solve(const CsrR& A, const std::vector<double>& b, std::vector<double>& x) {
#ifdef ORACLE_WITH_EIGEN
    if (kind == ORACLE_SOLVER_EIGEN_REUSE) {
      Eigen::SparseMatrix<double> M(A.n, A.n);
      for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) M.insert(i, A.col[k]) = A.val[k];
      M.makeCompressed();
      if (!reuse) {
        reuse.reset(new Eigen::SparseLU<Eigen::SparseMatrix<double>, Eigen::COLAMDOrdering<int> >());
        reuse->analyzePattern(M);
      }
      reuse->factorize(M);
      if (reuse->info() != Eigen::Success) return false;
      Eigen::VectorXd B(A.n);
      for (int i = 0; i < A.n; ++i) B(i) = b[i];
      Eigen::VectorXd X = reuse->solve(B);
      x.assign(A.n, 0.0);
      for (int i = 0; i < A.n; ++i) x[i] = X(i);
      return true;
    }
    if (kind == ORACLE_SOLVER_EIGEN) {
      // newtonpf.h:341-363: insert, makeCompressed, SparseLU<COLAMD>.compute, solve
      Eigen::SparseMatrix<double> M(A.n, A.n);
      for (int i = 0; i < A.n; ++i)
        for (int k = A.ptr[i]; k < A.ptr[i + 1]; ++k) M.insert(i, A.col[k]) = A.val[k];
      M.makeCompressed();
      Eigen::SparseLU<Eigen::SparseMatrix<double>, Eigen::COLAMDOrdering<int> > lu;
      lu.compute(M);
      if (lu.info() != Eigen::Success) return false;
      Eigen::VectorXd B(A.n);
      for (int i = 0; i < A.n; ++i) B(i) = b[i];
      Eigen::VectorXd X = lu.solve(B);
      x.assign(A.n, 0.0);
      for (int i = 0; i < A.n; ++i) x[i] = X(i);
      return true;
    }
#endif
    if (order.size() != (size_t)A.n) order = min_degree(A);
    SparseLUPP lu;
    if (!lu.factor(A, order)) return false;
    lu.solve(b, x);
    for (double v : x)
      if (!std::isfinite(v)) return false;
    return true;
  }
};

struct CaseResult {
  int iters = 0;
  int converged = 0;
  double err = 0.0;
  std::vector<Cx> V;
};

std::vector<Cx> start_point(const Grid& g) {  // runpf.h:211-226
  std::vector<Cx> V(g.nb);
  for (int i = 0; i < g.nb; ++i) {
    const mpf_bus& b = g.bus[i];
    V[i] = cmul(Cx{b.vm, 0}, cexpj(b.va));
    if (b.type == MPF_BUS_PV || b.type == MPF_BUS_SLACK) V[i] = cmul(Cx{b.vm / cabs_(V[i]), 0.0}, V[i]);
  }
  return V;
}

// newtonpf.h:188-213
void nr_update(const Grid& g, std::vector<Cx>& V, const std::vector<double>& dx, int angle_mode) {
  const int npv = (int)g.pv.size(), npq = (int)g.pq.size();
  for (int id = 0; id < npv + npq; ++id) {
    if (id < npv) {
      const int i = g.pv[id];
      V[i] = cmul(Cx{cabs_(V[i]), 0}, cexpj(angle_of(V[i], angle_mode) - dx[id]));
    } else {
      const int i = g.pq[id - npv];
      V[i] = cmul(Cx{cabs_(V[i]) - dx[npq + id], 0}, cexpj(angle_of(V[i], angle_mode) - dx[id]));
    }
  }
}

CaseResult run_nr(const Grid& g, const CsrC& y, const std::vector<Cx>& S, int max_it, double tol,
                  Solver& solver, int angle_mode, CsrR& J) {
  CaseResult res;
  res.V = start_point(g);
  std::vector<double> F, dx;
  double err = nr_mismatch(g, y, res.V, S, F);
  bool converged = err < tol;
  int iter = 0;
  std::vector<Cx> Ibus(g.nb);
  while (!converged && iter < max_it) {
    ++iter;
    for (int i = 0; i < g.nb; ++i) {  // newtonpf.h:73-95
      Cx c{0, 0};
      for (int k = y.ptr[i]; k < y.ptr[i + 1]; ++k) c = cadd(c, cmul(y.val[k], res.V[y.col[k]]));
      Ibus[i] = c;
    }
    jac_values(g, y, res.V, Ibus, J);
    if (!solver.solve(J, F, dx)) {
      err = NAN;
      break;
    }
    nr_update(g, res.V, dx, angle_mode);
    err = nr_mismatch(g, y, res.V, S, F);
    converged = err < tol;
  }
  res.iters = iter;
  res.converged = converged ? 1 : 0;
  res.err = err;
  return res;
}

// fdpf.h:369-414: P = Re(mis)/|V| over pvpq, Q = Im(mis)/|V| over pq
double fd_mismatch(const Grid& g, const CsrC& y, const std::vector<Cx>& V, const std::vector<Cx>& S,
                   std::vector<double>& P, std::vector<double>& Q) {
  const int npv = (int)g.pv.size(), npq = (int)g.pq.size();
  P.assign(npv + npq, 0.0);
  Q.assign(npq, 0.0);
  double errP = -1.0, errQ = -1.0;
  for (int id = 0; id < npv + npq; ++id) {
    const int bus = id < npv ? g.pv[id] : g.pq[id - npv];
    Cx c{0, 0};
    for (int k = y.ptr[bus]; k < y.ptr[bus + 1]; ++k) c = cadd(c, cmul(y.val[k], V[y.col[k]]));
    Cx mis = csub(cmul(V[bus], cconj(c)), S[bus]);
    const double a = cabs_(V[bus]);
    mis = Cx{mis.re / a, mis.im / a};
    if (id < npv) {
      P[id] = mis.re;
      errP = std::max(errP, std::fabs(P[id]));
    } else {
      const int i = id - npv;
      P[npv + i] = mis.re;
      errP = std::max(errP, std::fabs(P[npv + i]));
      Q[i] = mis.im;
      errQ = std::max(errQ, std::fabs(Q[i]));
    }
  }
  return std::max(errP, errQ);
}

// makeB.h:326-381: -Im(Ybus) restricted to the listed buses, in list order
CsrR restrict_b(const CsrC& y, const std::vector<int>& buses, int nb) {
  std::vector<int> pos(nb, -1);
  for (size_t k = 0; k < buses.size(); ++k) pos[buses[k]] = (int)k;
  CsrR B;
  B.n = (int)buses.size();
  B.ptr.assign(B.n + 1, 0);
  std::vector<std::pair<int, double>> row;
  for (int r = 0; r < B.n; ++r) {
    const int i = buses[r];
    row.clear();
    for (int k = y.ptr[i]; k < y.ptr[i + 1]; ++k)
      if (pos[y.col[k]] >= 0) row.push_back({pos[y.col[k]], -y.val[k].im});
    std::sort(row.begin(), row.end());
    for (auto& e : row) {
      B.col.push_back(e.first);
      B.val.push_back(e.second);
    }
    B.ptr[r + 1] = (int)B.col.size();
  }
  return B;
}

CaseResult run_fd(const Grid& g, const std::vector<mpf_branch>& br, const CsrC& y, const std::vector<Cx>& S,
                  int alg, int max_it, double tol, Solver& sp, Solver& spp, int angle_mode) {
  // makeB.h:392-501: B' from zeroed charging / taps / shunts (XB: R=0),
  // B'' from zeroed shifts (BX: R=0)
  std::vector<mpf_branch> b1(br), b2(br);
  std::vector<double> bsh0(g.nb, 0.0), bsh(g.nb);
  for (int i = 0; i < g.nb; ++i) bsh[i] = g.bus[i].bsh;
  for (auto& b : b1) {
    b.b = 0.0;
    b.tap = 0.0;
    if (alg == MPF_FDXB) b.r = 0.0;
  }
  for (auto& b : b2) {
    b.shift = 0.0;
    if (alg == MPF_FDBX) b.r = 0.0;
  }
  std::vector<int> pvpq(g.pv);
  pvpq.insert(pvpq.end(), g.pq.begin(), g.pq.end());
  const CsrR Bp = restrict_b(make_ybus(g, b1, bsh0), pvpq, g.nb);
  const CsrR Bpp = restrict_b(make_ybus(g, b2, bsh), g.pq, g.nb);

  CaseResult res;
  res.V = start_point(g);
  std::vector<double> P, Q, dVa, dVm;
  double err = fd_mismatch(g, y, res.V, S, P, Q);
  bool converged = err < tol;
  const int npv = (int)g.pv.size(), npq = (int)g.pq.size();
  int i = 0;
  while (!converged && i < max_it) {
    ++i;
    if (!sp.solve(Bp, P, dVa)) { err = NAN; break; }
    for (int id = 0; id < npv + npq; ++id) {  // fdpf.h:416-434
      const int b = id < npv ? g.pv[id] : g.pq[id - npv];
      res.V[b] = cmul(Cx{cabs_(res.V[b]), 0}, cexpj(angle_of(res.V[b], angle_mode) - dVa[id]));
    }
    err = fd_mismatch(g, y, res.V, S, P, Q);
    if (err < tol) { converged = true; break; }
    if (!spp.solve(Bpp, Q, dVm)) { err = NAN; break; }
    for (int id = 0; id < npq; ++id) {  // fdpf.h:436-448
      const int b = g.pq[id];
      res.V[b] = cmul(Cx{cabs_(res.V[b]) - dVm[id], 0}, cexpj(angle_of(res.V[b], angle_mode)));
    }
    err = fd_mismatch(g, y, res.V, S, P, Q);
    if (err < tol) converged = true;
  }
  res.iters = i;
  res.converged = converged ? 1 : 0;
  res.err = err;
  return res;
}

}  // namespace

extern "C" {

int oracle_abi_version(void) { return 1; }

int oracle_has_eigen(void) {
#ifdef ORACLE_WITH_EIGEN
  return 1;
#else
  return 0;
#endif
}

// Runs every case.  Outputs: v_out[case][nb][2], iters[case], converged[case],
// max_mis[case].  Returns 0, or -1 on bad input.
int oracle_runpf(const mpf_bus* buses, int nb, const mpf_branch* branches, int nbr, int alg,
                 int max_it, double tol, int solver, int angle_mode, int n_cases,
                 const int* outage_offsets, const int* outage_branches, const double* sbus,
                 double* v_out, int* iters, unsigned char* converged, double* max_mis,
                 int n_threads) {
  if (!buses || !branches || nb < 2 || nbr < 1 || n_cases < 0) return -1;
  if ((solver == ORACLE_SOLVER_EIGEN || solver == ORACLE_SOLVER_EIGEN_REUSE) && !oracle_has_eigen()) return -1;
  Grid g;
  g.nb = nb;
  g.nbr = nbr;
  g.bus.assign(buses, buses + nb);
  g.br.assign(branches, branches + nbr);
  classify(g);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads > 0 ? n_threads : 1) reduction(+ : bad)
  for (int c = 0; c < n_cases; ++c) {
    std::vector<mpf_branch> br(g.br);
    if (outage_offsets) {
      for (int k = outage_offsets[c]; k < outage_offsets[c + 1]; ++k) {
        const int e = outage_branches[k];
        if (e < 0 || e >= nbr) { bad++; continue; }
        br[e].status = 0;
      }
    }
    std::vector<Cx> S(nb);
    for (int i = 0; i < nb; ++i) {
      if (sbus) S[i] = Cx{sbus[((size_t)c * nb + i) * 2], sbus[((size_t)c * nb + i) * 2 + 1]};
      else S[i] = Cx{g.bus[i].p, g.bus[i].q};
    }
    std::vector<double> bsh(nb);
    for (int i = 0; i < nb; ++i) bsh[i] = g.bus[i].bsh;
    const CsrC y = make_ybus(g, br, bsh);
    CaseResult r;
    Solver s1, s2;
    s1.kind = s2.kind = solver;
    if (alg == MPF_NR) {
      CsrR J = jac_pattern(g, y);
      r = run_nr(g, y, S, max_it, tol, s1, angle_mode, J);
    } else {
      r = run_fd(g, br, y, S, alg, max_it, tol, s1, s2, angle_mode);
    }
    for (int i = 0; i < nb; ++i) {
      v_out[((size_t)c * nb + i) * 2] = r.V[i].re;
      v_out[((size_t)c * nb + i) * 2 + 1] = r.V[i].im;
    }
    iters[c] = r.iters;
    converged[c] = (unsigned char)r.converged;
    max_mis[c] = r.err;
  }
  return bad ? -1 : 0;
}

// Ybus of one case (outaged branches removed) as CSR; returns nnz.  With col/val
// NULL it only returns nnz.  val is (re, im) pairs.
int oracle_ybus(const mpf_bus* buses, int nb, const mpf_branch* branches, int nbr,
                const int* outages, int n_out, int* ptr, int* col, double* val) {
  Grid g;
  g.nb = nb;
  g.nbr = nbr;
  g.bus.assign(buses, buses + nb);
  g.br.assign(branches, branches + nbr);
  std::vector<mpf_branch> br(g.br);
  for (int k = 0; k < n_out; ++k) br[outages[k]].status = 0;
  std::vector<double> bsh(nb);
  for (int i = 0; i < nb; ++i) bsh[i] = g.bus[i].bsh;
  const CsrC y = make_ybus(g, br, bsh);
  if (ptr) std::copy(y.ptr.begin(), y.ptr.end(), ptr);
  if (col && val) {
    std::copy(y.col.begin(), y.col.end(), col);
    for (size_t k = 0; k < y.val.size(); ++k) {
      val[2 * k] = y.val[k].re;
      val[2 * k + 1] = y.val[k].im;
    }
  }
  return (int)y.col.size();
}

// Mismatch F (reference order) and Jacobian (CSR, reference order) at voltage V
// (nb complex) for one case; returns max |F|.  Any output may be NULL; jac_nnz
// receives nnz(J).
double oracle_nr_system(const mpf_bus* buses, int nb, const mpf_branch* branches, int nbr,
                        const int* outages, int n_out, const double* v, double* F, int* jptr,
                        int* jcol, double* jval, int* jac_nnz) {
  Grid g;
  g.nb = nb;
  g.nbr = nbr;
  g.bus.assign(buses, buses + nb);
  g.br.assign(branches, branches + nbr);
  classify(g);
  std::vector<mpf_branch> br(g.br);
  for (int k = 0; k < n_out; ++k) br[outages[k]].status = 0;
  std::vector<double> bsh(nb);
  for (int i = 0; i < nb; ++i) bsh[i] = g.bus[i].bsh;
  const CsrC y = make_ybus(g, br, bsh);
  std::vector<Cx> V(nb), S(nb), Ibus(nb);
  for (int i = 0; i < nb; ++i) {
    V[i] = Cx{v[2 * i], v[2 * i + 1]};
    S[i] = Cx{g.bus[i].p, g.bus[i].q};
  }
  std::vector<double> Fv;
  const double err = nr_mismatch(g, y, V, S, Fv);
  if (F) std::copy(Fv.begin(), Fv.end(), F);
  CsrR J = jac_pattern(g, y);
  if (jac_nnz) *jac_nnz = (int)J.col.size();
  if (jptr || jcol || jval) {
    for (int i = 0; i < nb; ++i) {
      Cx c{0, 0};
      for (int k = y.ptr[i]; k < y.ptr[i + 1]; ++k) c = cadd(c, cmul(y.val[k], V[y.col[k]]));
      Ibus[i] = c;
    }
    jac_values(g, y, V, Ibus, J);
    if (jptr) std::copy(J.ptr.begin(), J.ptr.end(), jptr);
    if (jcol) std::copy(J.col.begin(), J.col.end(), jcol);
    if (jval) std::copy(J.val.begin(), J.val.end(), jval);
  }
  return err;
}

// Total branch active loss at V (runpf.h:228-257) for one case.
double oracle_loss(const mpf_bus* buses, int nb, const mpf_branch* branches, int nbr,
                   const int* outages, int n_out, const double* v) {
  std::vector<mpf_branch> br(branches, branches + nbr);
  for (int k = 0; k < n_out; ++k) br[outages[k]].status = 0;
  double loss = 0.0;
  for (int k = 0; k < nbr; ++k) {
    const mpf_branch& b = br[k];
    const double stat = b.status ? 1.0 : 0.0;
    const Cx ys = cdiv(Cx{stat, 0}, Cx{b.r, b.x});
    Cx tap = Cx{b.tap != 0.0 ? b.tap : 1.0, 0.0};
    tap = cmul(tap, cexpj(M_PI / 180.0 * b.shift));
    const Cx ytt = cadd(ys, Cx{0, stat * b.b / 2});
    const Cx yff = cdiv(ytt, cmul(tap, cconj(tap)));
    const Cx yft = cdiv(Cx{-ys.re, -ys.im}, cconj(tap));
    const Cx ytf = cdiv(Cx{-ys.re, -ys.im}, tap);
    const Cx vf{v[2 * b.from], v[2 * b.from + 1]}, vt{v[2 * b.to], v[2 * b.to + 1]};
    const Cx If = cadd(cmul(yff, vf), cmul(yft, vt));
    const Cx It = cadd(cmul(ytf, vf), cmul(ytt, vt));
    loss += cadd(cmul(cconj(If), vf), cmul(cconj(It), vt)).re;
  }
  (void)buses;
  (void)nb;
  return loss;
}

}  // extern "C"

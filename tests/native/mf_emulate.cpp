// Host emulation of the multifrontal kernels' index arithmetic (one lane), used by
// tests/test_symbolic.py to check the symbolic layer (supernodes, arrowheads,
// extend-add maps, panel offsets) without a GPU: factor + forward + backward
// solve of a random diagonally dominant matrix on the Newton-system pattern of a
// synthetic grid, compared with a dense LU solve.  Prints the max relative error.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace mpf;

// fronts above this many rows take k_mf_factor_big's panel / trailing-block split
static const int kBigFront = 167;
static long big_fronts = 0, big_mismatch = 0;

static double solve_check(const LUSymbolic& L, const std::vector<int>& ah_ptr, const std::vector<int>& ah_loc,
                          const std::vector<int>& rows, const std::vector<int>& cols, const std::vector<int>& a_index,
                          Rng& rng, bool fused_forward) {
  const int n = L.n;
  const size_t m = rows.size();
  // values: random off-diagonal, dominant diagonal
  std::vector<double> val(m);
  std::vector<double> rowsum(n, 0.0);
  for (size_t e = 0; e < m; ++e)
    if (rows[e] != cols[e]) { val[e] = rng.uniform() - 0.5; rowsum[rows[e]] += std::fabs(val[e]); }
  for (size_t e = 0; e < m; ++e)
    if (rows[e] == cols[e]) val[e] = rowsum[rows[e]] + 1.0 + rng.uniform();
  std::vector<double> A(m);
  for (size_t e = 0; e < m; ++e) A[a_index[e]] = val[e];
  std::vector<double> b(n), x(n);
  for (int i = 0; i < n; ++i) b[i] = rng.uniform() - 0.5;
  x = b;
  std::vector<double> pan(L.nnz), cb(L.sum_cb), cbr(L.cbr_off.back());
  // factor (k_mf_factor with G = 1, SLOTS = 1), levels ascending
  for (int lv = 0; lv < L.nlevels; ++lv) {
    for (int k = L.lev_ptr[lv]; k < L.lev_ptr[lv + 1]; ++k) {
      const int s = L.lev_sn[k];
      const int w = L.sn_w[s], f = L.sn_f[s], f1 = (f + 1) | 1;
      const int* rw = L.sn_rows.data() + L.sn_rptr[s];
      std::vector<double> F((size_t)f * f1, 0.0);  // row stride (f + 1) | 1 as in the kernel
      for (int e = ah_ptr[s]; e < ah_ptr[s + 1]; ++e) {
        // an arrowhead entry lies in a pivot row or a pivot column (the panel of a
        // large front)
        if (ah_loc[e] / f1 >= w && ah_loc[e] % f1 >= w) { std::printf("arrowhead entry outside the panel\n"); std::exit(5); }
        F[ah_loc[e]] = A[e];
      }
      if (fused_forward)
        for (int p = 0; p < w; ++p) F[p * f1 + f] = x[rw[p]];
      for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
        const int ch = L.child_list[ci];
        const int mm = L.sn_f[ch] - L.sn_w[ch];
        const int* rel = L.relmap.data() + L.rel_ptr[ch];
        // a child's rows map in increasing order (k_mf_factor_big finds the rows that
        // fall in pivot rows, and in each trailing slab, as ranges of them)
        for (int a = 1; a < mm; ++a)
          if (rel[a] <= rel[a - 1]) { std::printf("relative map not increasing\n"); std::exit(6); }
        for (int idx = 0; idx < mm * mm; ++idx) F[rel[idx / mm] * f1 + rel[idx % mm]] += cb[L.cb_off[ch] + idx];
        if (fused_forward)
          for (int a = 0; a < mm; ++a) F[rel[a] * f1 + f] += cbr[L.cbr_off[ch] + a];
      }
      const int extra = fused_forward ? 1 : 0;
      // fronts above kFmaxAll: k_mf_factor_big's split of the same front into a panel
      // (pivot rows with the right-hand side, then the other rows' pivot columns) and a
      // trailing block updated after the panel's LU; its factors must equal the dense
      // loop's bit for bit
      std::vector<double> Fbig;
      if (f > kBigFront) {
        const int mm = f - w, ncols = f + extra;
        std::vector<double> P((size_t)w * (f + 1) + (size_t)mm * w, 0.0), C((size_t)mm * mm), R(mm);
        auto PE = [&](int r, int c) -> double& {
          if (r < 0 || r >= f || c < 0 || c > f || (r >= w && c >= w)) { std::printf("panel index %d %d\n", r, c); std::exit(4); }
          return r < w ? P[(size_t)r * (f + 1) + c] : P[(size_t)w * (f + 1) + (size_t)(r - w) * w + c];
        };
        for (int r = 0; r < f; ++r)
          for (int c = 0; c < f + 1; ++c) {
            const double v = F[r * f1 + c];  // the assembled front: arrowhead, children, right-hand side
            if (r < w || c < w) PE(r, c) = v;
            else if (c < f) C[(size_t)(r - w) * mm + (c - w)] = v;
            else R[r - w] = v;
          }
        for (int p = 0; p < w; ++p) {
          const double inv = 1.0 / PE(p, p);
          for (int i = p + 1; i < w; ++i)
            for (int q = p + 1; q < ncols; ++q) PE(i, q) = PE(i, q) - (PE(i, p) * inv) * PE(p, q);
          for (int i = w; i < f; ++i)
            for (int q = p + 1; q < w; ++q) PE(i, q) = PE(i, q) - (PE(i, p) * inv) * PE(p, q);
          for (int i = p + 1; i < f; ++i) PE(i, p) *= inv;
        }
        for (int a = 0; a < mm; ++a) {
          for (int b = 0; b < mm; ++b) {
            double c = C[(size_t)a * mm + b];
            for (int p = 0; p < w; ++p) c = c - PE(w + a, p) * PE(p, w + b);
            C[(size_t)a * mm + b] = c;
          }
          if (fused_forward) {
            double c = R[a];
            for (int p = 0; p < w; ++p) c = c - PE(w + a, p) * PE(p, f);
            R[a] = c;
          }
        }
        Fbig.assign(F.size(), 0.0);
        for (int r = 0; r < f; ++r)
          for (int c = 0; c < f + 1; ++c)
            Fbig[r * f1 + c] = (r < w || c < w) ? PE(r, c) : c < f ? C[(size_t)(r - w) * mm + (c - w)] : R[r - w];
        ++big_fronts;
      }
      for (int p = 0; p < w; ++p) {
        const double inv = 1.0 / F[p * f1 + p];
        for (int i = p + 1; i < f; ++i) F[i * f1 + p] *= inv;
        for (int i = p + 1; i < f; ++i)
          for (int q = p + 1; q < f + extra; ++q) F[i * f1 + q] -= F[i * f1 + p] * F[p * f1 + q];
      }
      if (!Fbig.empty())
        for (int r = 0; r < f; ++r)
          for (int c = 0; c < f + extra; ++c)
            if (std::memcmp(&Fbig[r * f1 + c], &F[r * f1 + c], sizeof(double)) != 0) ++big_mismatch;
      for (int idx = 0; idx < w * f; ++idx) pan[L.pan_off[s] + idx] = F[(idx / f) * f1 + idx % f];
      const int mm = f - w;
      for (int idx = 0; idx < mm * w; ++idx) pan[L.pan_off[s] + (long)w * f + idx] = F[(w + idx / w) * f1 + idx % w];
      if (fused_forward)
        for (int p = 0; p < w; ++p) x[rw[p]] = F[p * f1 + f];
      if (L.sn_parent[s] >= 0) {
        for (int idx = 0; idx < mm * mm; ++idx) cb[L.cb_off[s] + idx] = F[(w + idx / mm) * f1 + w + idx % mm];
        if (fused_forward)
          for (int a = 0; a < mm; ++a) cbr[L.cbr_off[s] + a] = F[(w + a) * f1 + f];
      }
    }
  }
  if (!fused_forward) {  // k_mf_fsolve
    for (int lv = 0; lv < L.nlevels; ++lv)
      for (int k = L.lev_ptr[lv]; k < L.lev_ptr[lv + 1]; ++k) {
        const int s = L.lev_sn[k];
        const int w = L.sn_w[s], f = L.sn_f[s];
        const int* rw = L.sn_rows.data() + L.sn_rptr[s];
        std::vector<double> bl(f, 0.0);
        for (int p = 0; p < w; ++p) bl[p] = x[rw[p]];
        for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
          const int ch = L.child_list[ci];
          const int mm = L.sn_f[ch] - L.sn_w[ch];
          const int* rel = L.relmap.data() + L.rel_ptr[ch];
          for (int a = 0; a < mm; ++a) bl[rel[a]] += cbr[L.cbr_off[ch] + a];
        }
        for (int p = 0; p < w; ++p) {
          for (int i = p + 1; i < w; ++i) bl[i] -= pan[L.pan_off[s] + (long)i * f + p] * bl[p];
          for (int i = w; i < f; ++i) bl[i] -= pan[L.pan_off[s] + (long)w * f + (long)(i - w) * w + p] * bl[p];
        }
        for (int p = 0; p < w; ++p) x[rw[p]] = bl[p];
        if (L.sn_parent[s] >= 0)
          for (int a = 0; a < f - w; ++a) cbr[L.cbr_off[s] + a] = bl[w + a];
      }
  }
  // k_mf_bsolve, levels descending
  for (int lv = L.nlevels - 1; lv >= 0; --lv)
    for (int k = L.lev_ptr[lv]; k < L.lev_ptr[lv + 1]; ++k) {
      const int s = L.lev_sn[k];
      const int w = L.sn_w[s], f = L.sn_f[s];
      const int* rw = L.sn_rows.data() + L.sn_rptr[s];
      for (int p = w - 1; p >= 0; --p) {
        double acc = x[rw[p]];
        for (int q = p + 1; q < f; ++q) acc -= pan[L.pan_off[s] + (long)p * f + q] * x[rw[q]];
        x[rw[p]] = acc / pan[L.pan_off[s] + (long)p * f + p];
      }
    }
  // residual check against the matrix: r = A x - b
  std::vector<double> r(n, 0.0);
  for (size_t e = 0; e < m; ++e) r[rows[e]] += val[e] * x[cols[e]];
  double err = 0.0, bn = 0.0;
  for (int i = 0; i < n; ++i) {
    err = std::fmax(err, std::fabs(r[i] - b[i]));
    bn = std::fmax(bn, std::fabs(b[i]));
  }
  return err / bn;
}

int main(int argc, char** argv) {
  const int nb = argc > 1 ? atoi(argv[1]) : 300;
  const int nbr = argc > 2 ? atoi(argv[2]) : 411;
  const int npv = argc > 3 ? atoi(argv[3]) : 69;
  const int ordering = argc > 4 ? atoi(argv[4]) : 0;  // MPF_ORDER_*
  const int topology = argc > 5 ? atoi(argv[5]) : 0;  // 1: uniform-random extra branches
  mpf_synth_params p;
  mpf_synth_default(&p);
  p.n_bus = nb;
  p.n_branch = nbr;
  p.n_pv = npv;
  p.tap_fraction = 0.1;
  p.topology = topology;
  std::vector<mpf_bus> b(nb);
  std::vector<mpf_branch> br(nbr);
  if (mpf_synth_grid(&p, b.data(), br.data()) != MPF_OK) return 2;
  GridSymbolic g;
  if (!build_symbolic(b.data(), nb, br.data(), nbr, g, nullptr, ordering).empty()) return 3;
  Rng rng(11);
  // Newton system pattern, as the J fill scatters it (jpos)
  std::vector<int> rows, cols, aidx;
  for (int i = 0; i < nb; ++i)
    for (int q = g.y_rowptr[i]; q < g.y_rowptr[i + 1]; ++q) {
      const int j = g.y_col[q];
      const int r4[4] = {g.var_va[i], g.var_va[i], g.var_vm[i], g.var_vm[i]};
      const int c4[4] = {g.var_va[j], g.var_vm[j], g.var_va[j], g.var_vm[j]};
      for (int k = 0; k < 4; ++k)
        if (g.jpos[4 * (size_t)q + k] >= 0) {
          rows.push_back(r4[k]);
          cols.push_back(c4[k]);
          aidx.push_back(g.jpos[4 * (size_t)q + k]);
        }
    }
  const double e1 = solve_check(g.jac, g.ah_ptr, g.ah_loc, rows, cols, aidx, rng, true);
  const double e2 = solve_check(g.jac, g.ah_ptr, g.ah_loc, rows, cols, aidx, rng, false);
  // B' pattern (XB variant): Ybus entries between PV/PQ buses, br_pos tells A-array indices of branch parts
  double e3 = 0.0;
  for (int v = 0; v < 2; ++v) {
    for (int which = 0; which < 2; ++which) {
      const GridSymbolic::FDSystem& fs = which == 0 ? g.bp[v] : g.bpp[v];
      std::vector<int> r2, c2, a2(fs.base.size(), -1), ai;
      // reconstruct (row, col) of each A-array entry from the front positions
      r2.resize(fs.base.size());
      c2.resize(fs.base.size());
      for (int s = 0; s < fs.lu.nsn; ++s) {
        const int f1 = (fs.lu.sn_f[s] + 1) | 1;
        const int* rw = fs.lu.sn_rows.data() + fs.lu.sn_rptr[s];
        for (int e = fs.ah_ptr[s]; e < fs.ah_ptr[s + 1]; ++e) {
          r2[e] = rw[fs.ah_loc[e] / f1];
          c2[e] = rw[fs.ah_loc[e] % f1];
        }
      }
      for (size_t e = 0; e < r2.size(); ++e) ai.push_back((int)e);
      e3 = std::fmax(e3, solve_check(fs.lu, fs.ah_ptr, fs.ah_loc, r2, c2, ai, rng, false));
    }
  }
  printf("%.3e %.3e %.3e\n", e1, e2, e3);
  // the split-front emulation of large fronts differs from the dense loop in this many
  // entries (must be 0); its fronts count goes to stderr
  std::fprintf(stderr, "big fronts %ld, mismatching entries %ld\n", big_fronts, big_mismatch);
  return (e1 < 1e-10 && e2 < 1e-10 && e3 < 1e-10 && big_mismatch == 0) ? 0 : 1;
}

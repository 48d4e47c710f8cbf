// Host-side internals shared by the library's translation units.
#ifndef MPF_INTERNAL_H_
#define MPF_INTERNAL_H_

#include <cstdint>
#include <string>
#include <vector>

#include "mpf.h"

namespace mpf {

uint64_t splitmix64(uint64_t& x);

// xoshiro256** seeded with splitmix64: identical streams on every machine.
struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed);
  uint64_t next();
  double uniform();            // [0, 1)
  uint64_t below(uint64_t n);  // [0, n)
  double normal();             // N(0, 1), Box-Muller
};

int find_bridges(const mpf_branch* br, int nbr, int nb, std::vector<uint8_t>& is_bridge);

// Branch pi-model admittances (complex as re/im pairs), makeYbus.h:40-107 (CPU)
// and :306-366 (GPU): Ys = stat/(R+jX), Bc = stat*jB, t = tap*e^{j*pi*shift/180}
// (tap 0 -> 1), Ytt = Ys + Bc/2, Yff = Ytt/|t|^2, Yft = -Ys/conj(t), Ytf = -Ys/t.
struct BranchY {
  double ff[2], ft[2], tf[2], tt[2];
};
BranchY branch_admittance(double r, double x, double b, double tap, double shift_deg, int stat);

// Multifrontal symbolic LU of a structurally symmetric n x n matrix factorised
// without pivoting (diagonal pivots) in a fixed elimination order.
//
// Supernode s owns w_s pivot variables and its front rows R_s =
// sn_rows[sn_rptr[s] .. sn_rptr[s+1]) (f_s of them, ascending; the first w_s are
// the pivots, every other row is a later variable).  Pivots of an amalgamated
// supernode need not be consecutive.  The front is the dense f x f matrix
// A(R_s, R_s) restricted to the arrowhead of the pivots plus the contribution
// blocks (CB) of the children; a partial LU of its first w pivots produces
//   U-panel  F(0:w, 0:f)          w*f entries, row-major (holds L of the diagonal
//                                 block below its diagonal, unit diagonal implied)
//   L-panel  F(w:f, 0:w)          (f-w)*w entries, row-major
//   CB       F(w:f, w:f)          (f-w)^2 entries, added into the parent's front
//   CB-RHS   b(w:f) - L y         (f-w) entries (forward solve carried upward)
// Panels of all supernodes are concatenated (pan_off) and hold exactly nnz(L+U)
// entries.
struct LUSymbolic {
  int n = 0;
  int64_t nnz = 0;                   // entries of L+U (= sum of panel sizes)
  std::vector<int> etree_parent;     // per variable, -1 for roots
  int nsn = 0;
  std::vector<int> sn_w;             // pivots
  std::vector<int> sn_f;             // front size
  std::vector<int> sn_rptr, sn_rows; // front rows
  std::vector<int> sn_parent;        // -1 for roots
  std::vector<int> sn_level;         // 0 for leaves, parent = 1 + max(children)
  int nlevels = 0;
  std::vector<int> lev_ptr, lev_sn;  // supernodes grouped by level, by front size within a level
  std::vector<int> child_ptr, child_list;
  std::vector<int64_t> pan_off;      // nsn+1, entries
  // offsets of each supernode's contribution block ((f-w)^2 entries) and carried
  // right-hand side (f-w); siblings adjacent; [nsn] = the totals
  std::vector<int64_t> cb_off;       // nsn+1
  std::vector<int64_t> cbr_off;      // nsn+1
  std::vector<int> rel_ptr, relmap;  // per supernode: CB index -> index in the parent's front
  std::vector<int> sn_of;            // per variable
  int max_front = 0;
  int64_t flops = 0;                 // 2 * multiply-adds of one factorisation
  int64_t sum_cb = 0;                // sum of (f-w)^2
  int64_t nnz_l = 0;                 // strictly lower entries

  int local(int s, int var) const;               // index of var in R_s or -1
  int64_t entry_pos(int row, int col) const;     // panel position of LU entry or -1
};

// Relaxed supernode amalgamation: a child joins its parent's front when the merged
// front has at most max_pivots pivots and max_front rows and gains at most
// max(max_zeros, max_zero_frac * size) explicit zeros.  max_pivots <= 1 disables it.
// Measured on the 9241-bus workload (1000 N-1 cases, mixed precision, solves/s):
// none 20.5k, zero-free merges only 21.3k, (4, 0.1) 21.9k, (16, 0.3) 20.4k,
// (32, 0.4) 18.3k, (64, 0.5) 16.7k: the kernels' per-task cost is now low enough
// that explicit zeros cost more than the tasks they save.  Again with the launch DAG
// and the two-pivot kernels: these defaults 29.7k; zeros (8, 0.15) 28.9k, (2, 0.05)
// 29.0k; 48 pivots / 100 rows 29.7k; 16 pivots 29.6k.
struct Relax {
  int max_pivots = 32;
  int max_front = 83;
  long long max_zeros = 4;
  double max_zero_frac = 0.1;
};

// Builds the symbolic LU of the pattern given as symmetric adjacency (no diagonal)
// in the already-permuted variable numbering.
void lu_symbolic(int n, const std::vector<std::vector<int>>& adj, LUSymbolic& s, const Relax& relax = Relax());

// Groups matrix entries (rows[e], cols[e]) by the supernode that owns min(row, col)
// (its arrowhead).  a_index[e] = position of entry e in the grouped ("A-array")
// order; supernode s owns A-array range [ah_ptr[s], ah_ptr[s+1]); ah_loc[k] is the
// flat position row * RS + col of A-array entry k inside the front, with the row
// stride RS = (f + 1) | 1 (the front carries a right-hand-side column f; the odd
// stride spreads consecutive rows over shared-memory banks).
void arrowhead_layout(const LUSymbolic& s, const std::vector<int>& rows,
                      const std::vector<int>& cols, std::vector<int>& a_index,
                      std::vector<int>& ah_ptr, std::vector<int>& ah_loc);

// Minimum-degree ordering of an undirected graph (adjacency lists without self
// loops).  Returns perm with perm[k] = vertex eliminated k-th.  Ties: lowest index.
std::vector<int> minimum_degree(int n, const std::vector<std::vector<int>>& adj);

// Minimum-deficiency (minimum fill-in) ordering: eliminates next the vertex whose
// elimination adds the fewest edges among its neighbours, each missing edge (a, b)
// counted weight[a] x weight[b] (weight null: 1).  Ties: smaller weighted degree,
// then lowest index.  Returns perm as minimum_degree, or an empty vector once the work
// of counting fill (which grows with it) passes max_work (0: no limit).
std::vector<int> minimum_fill(int n, const std::vector<std::vector<int>>& adj, const std::vector<int>* weight,
                              long long max_work = 0);

// Everything that does not depend on the case batch.
struct GridSymbolic {
  int nb = 0, nbr = 0, npv = 0, npq = 0, slack = -1, n_slack = 0;
  int n_islands = 0;                 // connected islands with a slack (grids of a multi-grid handle)
  std::vector<int> bus_island;       // per bus: island, -1 for buses of slack-less islands without equations
  std::vector<int> br_island;        // per branch: island of its buses
  std::vector<int> pv, pq;           // bus-index order (Topology.h:100-126)
  std::vector<int> bus_type;
  // Ybus superset pattern (every branch, in or out of service), CSR, columns sorted
  std::vector<int> y_rowptr, y_col;
  std::vector<double> y_val;         // base values, 2 per entry (re, im)
  std::vector<int> y_diag;           // position of (i, i)
  std::vector<int> br_pos;           // 4 per branch: ff, ft, tf, tt positions in Ybus
  std::vector<double> br_y;          // 8 per branch: ff, ft, tf, tt (re, im), with status
  std::vector<int> br_from, br_to, br_status;
  std::vector<double> sbus;          // 2 per bus
  std::vector<double> v0;            // 2 per bus: start point (runpf.h:211-226)

  // Newton system: variables = Va of every PV/PQ bus, Vm of every PQ bus
  std::vector<int> bus_order;        // elimination order of PV/PQ buses
  int ordering = 0;                  // the method that produced it (MPF_ORDER_*)
  std::vector<int> var_va, var_vm;   // per bus: LU variable index or -1
  LUSymbolic jac;
  int nnz_jac = 0;
  std::vector<int> jpos;             // 4 per Ybus entry: J-array index of the
                                     // (Va,Va), (Va,Vm), (Vm,Va), (Vm,Vm) block entries or -1
  std::vector<int> ah_ptr, ah_loc;   // arrowhead of supernode s: J-array range
                                     // [ah_ptr[s], ah_ptr[s+1]) and flat front positions
  std::vector<int> mis_rows;         // PV/PQ buses (rows of the mismatch)

  // Fast-decoupled systems (B': Va of PV/PQ buses; B'': Vm of PQ buses), for
  // XB (alg 1) and BX (alg 2) variants (makeB.h:311-501)
  struct FDSystem {
    LUSymbolic lu;
    std::vector<int> var;            // per bus: variable index or -1
    std::vector<double> base;        // arrowhead values of the base case (A-array order)
    std::vector<int> ah_ptr, ah_loc; // arrowhead of each supernode (as for the Newton system)
    std::vector<int> br_pos;         // 4 per branch: A-array index (ff, ft, tf, tt) or -1
    std::vector<double> br_val;      // 4 per branch: B contributions (ff, ft, tf, tt)
    std::vector<int> diag_pos;       // per bus: A-array index of its diagonal or -1
  };
  FDSystem bp[2], bpp[2];            // [0] = XB, [1] = BX
  std::vector<int> bpp_order;
};

// Validates the grid and fills g.  Returns empty string on success, else a message.
// vm_free (nullable): PV buses that also get a Vm variable and a Q equation (buses
// whose reactive limits may switch them to PQ).
// ordering: MPF_ORDER_* of the Newton system's bus elimination order (AUTO picks the
// candidate with the least estimated factorisation time).
std::string build_symbolic(const mpf_bus* buses, int nb, const mpf_branch* br, int nbr,
                           GridSymbolic& g, const std::vector<char>* vm_free = nullptr, int ordering = 0);

}  // namespace mpf

#endif  // MPF_INTERNAL_H_

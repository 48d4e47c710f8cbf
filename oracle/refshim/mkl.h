// mkl.h — in-project stand-in for the few Intel MKL routines that the reference's CPU
// power-flow path (the mkl_* functions of src/powerflow/{runpf,makeYbus,newtonpf,makeB,
// fdpf}.h) calls, so that those reference files compile here unmodified (MKL is not
// installed).  TEST INFRASTRUCTURE: only oracle/ref_pf.cu includes it, to build the
// reference's own code as a checker (oracle/_ref/librefpf.so).
//
// Each routine is written from MKL's published interface description:
//   MKL_malloc / MKL_free / MKL_Set_Num_Threads   aligned allocation, OpenMP thread count
//   mkl_?csrcoo (MKL_ZCSRCOO, MKL_DCSRCOO)        coordinate -> CSR (job[0] = 1, or 2 with the
//                                                 column indices of each row sorted), bases
//                                                 job[1] (CSR) and job[2] (COO); the value
//                                                 arrays may alias (newtonpf.h:305)
//   mkl_zcsrmultcsr (MKL_ZCSRMULTCSR)              C = A B, one-based, request 1 (row pointer
//                                                 only) / 2 (columns and values after 1) / 0
//                                                 (everything within nzmax); sort = 0 keeps
//                                                 each output row in order of first appearance
//   mkl_zcsradd (MKL_ZCSRADD)                      C = A + beta B, same conventions
//   DSS (direct sparse solver)                     create / define structure (CSR) / reorder /
//                                                 factor / solve / delete, with the LU done by
//                                                 the reference's vendored Eigen SparseLU
//                                                 (COLAMD ordering), i.e. the same solver as
//                                                 the reference's own Eigen_SparseLU option
// MKL's own DSS (PARDISO) is not reproduced: its pivoting and ordering differ, so results
// through this DSS agree with real MKL to rounding, not bit for bit.
#ifndef REFSHIM_MKL_H_
#define REFSHIM_MKL_H_

#include <omp.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <vector>

#include <Eigen/SparseLU>

#ifndef MKL_Complex16
#error "define MKL_Complex16 (the reference defines it as double2) before including mkl.h"
#endif

typedef int MKL_INT;

inline void* MKL_malloc(size_t bytes, int alignment) {
  void* p = nullptr;
  const size_t a = std::max<size_t>((size_t)alignment, sizeof(void*));
  if (posix_memalign(&p, a, bytes ? bytes : 1) != 0) return nullptr;
  return p;
}
inline void MKL_free(void* p) { std::free(p); }
inline void MKL_Set_Num_Threads(int n) { omp_set_num_threads(n); }

namespace refshim {

// ---------------------------------------------------------------- COO -> CSR
template <class V>
void csrcoo(const int* job, const int* n, V* acsr, int* ja, int* ia, const int* nnz, const V* acoo,
            const int* rowind, const int* colind, int* info) {
  *info = 0;
  if (job[0] != 1 && job[0] != 2) {  // only the COO -> CSR direction is used by the reference
    *info = 1;
    return;
  }
  const int rows = *n, nz = *nnz, bcsr = job[1], bcoo = job[2];
  std::vector<int> cnt(rows + 1, 0);
  for (int k = 0; k < nz; ++k) cnt[rowind[k] - bcoo + 1]++;
  for (int r = 0; r < rows; ++r) cnt[r + 1] += cnt[r];
  // stable placement by row, then (job[0] = 2) by column within each row
  std::vector<int> order(nz), fill(cnt.begin(), cnt.end() - 1);
  for (int k = 0; k < nz; ++k) order[fill[rowind[k] - bcoo]++] = k;
  if (job[0] == 2)
    for (int r = 0; r < rows; ++r)
      std::stable_sort(order.begin() + cnt[r], order.begin() + cnt[r + 1],
                       [&](int a, int b) { return colind[a] < colind[b]; });
  std::vector<V> vals(nz);
  std::vector<int> cols(nz);
  for (int p = 0; p < nz; ++p) {
    vals[p] = acoo[order[p]];
    cols[p] = colind[order[p]] - bcoo + bcsr;
  }
  for (int p = 0; p < nz; ++p) {  // acsr may be the same array as acoo
    acsr[p] = vals[p];
    ja[p] = cols[p];
  }
  for (int r = 0; r <= rows; ++r) ia[r] = cnt[r] + bcsr;
}

inline MKL_Complex16 cmul(MKL_Complex16 a, MKL_Complex16 b) {
  MKL_Complex16 c;
  c.x = a.x * b.x - a.y * b.y;
  c.y = a.x * b.y + a.y * b.x;
  return c;
}
inline MKL_Complex16 cadd(MKL_Complex16 a, MKL_Complex16 b) {
  MKL_Complex16 c;
  c.x = a.x + b.x;
  c.y = a.y + b.y;
  return c;
}

// One output row of a sparse product or sum: columns in order of first appearance,
// values accumulated in that order.  `mark` maps a column to its slot in the row.
struct RowAcc {
  std::vector<int> mark, cols;
  std::vector<MKL_Complex16> vals;
  explicit RowAcc(int ncols) : mark(ncols, -1) {}
  void add(int col, MKL_Complex16 v) {
    if (mark[col] < 0) {
      mark[col] = (int)cols.size();
      cols.push_back(col);
      vals.push_back(v);
    } else {
      vals[mark[col]] = cadd(vals[mark[col]], v);
    }
  }
  void reset() {
    for (int c : cols) mark[c] = -1;
    cols.clear();
    vals.clear();
  }
};

// Shared driver of the request protocol (one-based arrays, as MKL documents for
// mkl_?csrmultcsr and mkl_?csradd): request 1 fills ic only; request 2 fills jc and c
// (ic from request 1); request 0 fills all three, stopping with info = row (one-based)
// when nzmax entries do not suffice.
template <class RowFn>
void run_request(int request, int m, int ncols, const int* nzmax, MKL_Complex16* c, int* jc, int* ic, int* info,
                 RowFn row) {
  *info = 0;
  RowAcc acc(ncols);
  int pos = 0;
  if (request == 1 || request == 0) ic[0] = 1;
  for (int i = 0; i < m; ++i) {
    acc.reset();
    row(i, acc);
    const int len = (int)acc.cols.size();
    if (request == 1) {
      ic[i + 1] = ic[i] + len;
      continue;
    }
    if (request == 2) pos = ic[i] - 1;
    if (request == 0 && pos + len > *nzmax) {
      *info = i + 1;
      return;
    }
    for (int t = 0; t < len; ++t) {
      jc[pos + t] = acc.cols[t] + 1;
      c[pos + t] = acc.vals[t];
    }
    pos += len;
    if (request == 0) ic[i + 1] = pos + 1;
  }
}

}  // namespace refshim

inline void MKL_ZCSRCOO(const int* job, const int* n, MKL_Complex16* acsr, int* ja, int* ia, int* nnz,
                        MKL_Complex16* acoo, int* rowind, int* colind, int* info) {
  refshim::csrcoo<MKL_Complex16>(job, n, acsr, ja, ia, nnz, acoo, rowind, colind, info);
}
inline void MKL_DCSRCOO(const int* job, const int* n, double* acsr, int* ja, int* ia, int* nnz, double* acoo,
                        int* rowind, int* colind, int* info) {
  refshim::csrcoo<double>(job, n, acsr, ja, ia, nnz, acoo, rowind, colind, info);
}

// C (m x k) = A (m x n) B (n x k); transa 'N' only, sort ignored (no reordering)
inline void MKL_ZCSRMULTCSR(const char* transa, const int* request, const int* /*sort*/, const int* m, const int* n,
                            const int* k, MKL_Complex16* a, int* ja, int* ia, MKL_Complex16* b, int* jb, int* ib,
                            MKL_Complex16* c, int* jc, int* ic, const int* nzmax, int* info) {
  (void)n;
  if (*transa != 'N' && *transa != 'n') {
    *info = -1;
    return;
  }
  refshim::run_request(*request, *m, *k, nzmax, c, jc, ic, info, [&](int i, refshim::RowAcc& acc) {
    for (int p = ia[i] - 1; p < ia[i + 1] - 1; ++p) {
      const int r = ja[p] - 1;
      for (int q = ib[r] - 1; q < ib[r + 1] - 1; ++q) acc.add(jb[q] - 1, refshim::cmul(a[p], b[q]));
    }
  });
}

// C (m x n) = A + beta B; transa 'N' only, sort ignored (no reordering)
inline void MKL_ZCSRADD(const char* transa, const int* request, const int* /*sort*/, const int* m, const int* n,
                        MKL_Complex16* a, int* ja, int* ia, MKL_Complex16* beta, MKL_Complex16* b, int* jb, int* ib,
                        MKL_Complex16* c, int* jc, int* ic, const int* nzmax, int* info) {
  if (*transa != 'N' && *transa != 'n') {
    *info = -1;
    return;
  }
  const MKL_Complex16 be = *beta;
  refshim::run_request(*request, *m, *n, nzmax, c, jc, ic, info, [&](int i, refshim::RowAcc& acc) {
    for (int p = ia[i] - 1; p < ia[i + 1] - 1; ++p) acc.add(ja[p] - 1, a[p]);
    for (int q = ib[i] - 1; q < ib[i + 1] - 1; ++q) acc.add(jb[q] - 1, refshim::cmul(be, b[q]));
  });
}

// ---------------------------------------------------------------- DSS
#define MKL_DSS_SUCCESS 0
#define MKL_DSS_FAILURE (-1)
#define MKL_DSS_DEFAULTS 0
#define MKL_DSS_MSG_LVL_WARNING 0x1
#define MKL_DSS_TERM_LVL_ERROR 0x2
#define MKL_DSS_ZERO_BASED_INDEXING 0x4
#define MKL_DSS_NON_SYMMETRIC 0x8
#define MKL_DSS_AUTO_ORDER 0x10
#define MKL_DSS_GET_ORDER 0x20
#define MKL_DSS_POSITIVE_DEFINITE 0x40

typedef void* _MKL_DSS_HANDLE_t;
typedef void* MKL_DSS_HANDLE_t;

namespace refshim {
struct Dss {
  int base = 1, n = 0, nnz = 0;
  std::vector<int> rp, ci;
  Eigen::SparseLU<Eigen::SparseMatrix<double>, Eigen::COLAMDOrdering<int> > lu;
  long long solves = 0;
};
// solves per handle, in creation order, since the last reset (the driver reads how many
// P half-steps a fast-decoupled solve took from the first handle's count)
inline std::vector<long long>& dss_solve_log() {
  static std::vector<long long> log;
  return log;
}
inline std::vector<Dss*>& dss_live() {
  static std::vector<Dss*> live;
  return live;
}
}  // namespace refshim

inline int refshim_dss_create(_MKL_DSS_HANDLE_t* h, MKL_INT opt) {
  refshim::Dss* d = new refshim::Dss;
  d->base = (opt & MKL_DSS_ZERO_BASED_INDEXING) ? 0 : 1;
  refshim::dss_live().push_back(d);
  refshim::dss_solve_log().push_back(0);
  *h = d;
  return MKL_DSS_SUCCESS;
}
inline int refshim_dss_define_structure(_MKL_DSS_HANDLE_t h, MKL_INT /*opt*/, const int* rowIndex, int nRows, int nCols,
                                        const int* columns, int nNonZeros) {
  refshim::Dss* d = static_cast<refshim::Dss*>(h);
  if (nRows != nCols) return MKL_DSS_FAILURE;
  d->n = nRows;
  d->nnz = nNonZeros;
  d->rp.assign(rowIndex, rowIndex + nRows + 1);
  d->ci.assign(columns, columns + nNonZeros);
  return MKL_DSS_SUCCESS;
}
inline int refshim_dss_reorder(_MKL_DSS_HANDLE_t, MKL_INT, int*) { return MKL_DSS_SUCCESS; }  // ordered in factor
inline int refshim_dss_factor_real(_MKL_DSS_HANDLE_t h, MKL_INT /*opt*/, const double* values) {
  refshim::Dss* d = static_cast<refshim::Dss*>(h);
  Eigen::SparseMatrix<double> A(d->n, d->n);
  std::vector<Eigen::Triplet<double> > t;
  t.reserve(d->nnz);
  for (int i = 0; i < d->n; ++i)
    for (int p = d->rp[i] - d->base; p < d->rp[i + 1] - d->base; ++p)
      t.push_back(Eigen::Triplet<double>(i, d->ci[p] - d->base, values[p]));
  A.setFromTriplets(t.begin(), t.end());
  A.makeCompressed();
  d->lu.compute(A);
  return d->lu.info() == Eigen::Success ? MKL_DSS_SUCCESS : MKL_DSS_FAILURE;
}
inline int refshim_dss_solve_real(_MKL_DSS_HANDLE_t h, MKL_INT /*opt*/, const double* rhs, int nrhs, double* sol) {
  refshim::Dss* d = static_cast<refshim::Dss*>(h);
  auto& live = refshim::dss_live();
  const size_t idx = std::find(live.begin(), live.end(), d) - live.begin();
  for (int r = 0; r < nrhs; ++r) {
    Eigen::Map<const Eigen::VectorXd> b(rhs + (size_t)r * d->n, d->n);
    Eigen::VectorXd x = d->lu.solve(b);
    std::copy(x.data(), x.data() + d->n, sol + (size_t)r * d->n);
  }
  if (idx < refshim::dss_solve_log().size()) refshim::dss_solve_log()[idx]++;
  return MKL_DSS_SUCCESS;
}
inline int refshim_dss_delete(_MKL_DSS_HANDLE_t h, MKL_INT) {
  refshim::Dss* d = static_cast<refshim::Dss*>(h);
  auto& live = refshim::dss_live();
  auto it = std::find(live.begin(), live.end(), d);
  if (it != live.end()) *it = nullptr;  // keep creation order for the solve log
  delete d;
  return MKL_DSS_SUCCESS;
}

// the call forms of src/powerflow/newtonpf.h:318-338 and fdpf.h:468-561
#define DSS_CREATE(handle, opt) refshim_dss_create(&(handle), (opt))
#define DSS_DEFINE_STRUCTURE(handle, opt, rowIndex, nRows, nCols, columns, nNonZeros) \
  refshim_dss_define_structure((handle), (opt), (rowIndex), (nRows), (nCols), (columns), (nNonZeros))
#define DSS_REORDER(handle, opt, perm) refshim_dss_reorder((handle), (opt), (perm))
#define DSS_FACTOR_REAL(handle, opt, values) refshim_dss_factor_real((handle), (opt), (values))
#define DSS_SOLVE_REAL(handle, opt, rhs, nrhs, sol) refshim_dss_solve_real((handle), (opt), (rhs), (nrhs), (sol))
#define DSS_DELETE(handle, opt) refshim_dss_delete((handle), (opt))

#endif  // REFSHIM_MKL_H_

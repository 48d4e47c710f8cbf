// ref_pf.cu — builds the reference's own CPU power-flow code as a checker.  TEST
// INFRASTRUCTURE: only tests/ and bench.py's reference arm load the library made from it
// (oracle/_ref/librefpf.so), as the thing checked against or timed beside the product.
//
// The reference's src/powerflow/runpf.h (with makeYbus.h, newtonpf.h, makeB.h, fdpf.h,
// and the types of src/powersystem/ and src/pso/Particula.h) is compiled UNMODIFIED from
// the reference tree, the way its src/main.cu:1-105 sets it up (BASE_INDEX 1,
// MKL_Complex16 = double2, the timing table), with two in-project stand-ins for what is
// missing here: refshim/mkl.h (the MKL routines its CPU path calls, written from their
// documented semantics; DSS solves through the reference's vendored Eigen SparseLU) and
// refshim/cusparse_legacy.h (CUDA 12 removed some cuSPARSE routines its GPU path names;
// the CPU path never calls them).
//
// refpf_runpf solves each case with mkl_init / mkl_runpf / mkl_clean (runpf.h:359, 259,
// 452): a case is the base grid with its outaged branches' inservice flag cleared (the
// reference's own removal, makeYbus.h:69-73) and optionally its own bus injections.  The
// reference's CPU path reads every transformer's ratio from the particle
// (makeYbus.h:78: tap != 0 -> particula[indiceEstrutura]), so each tapped branch gets an
// OLTC structure holding its own ratio, as main.cu:232-262 binds them.
//
// Iteration counts are not returned by the reference (mkl_newtonpf's counter is local),
// so the timer the reference calls around each stage (util/timer.h's GetTimer) is
// replaced by a call counter: every timed stage then adds exactly 1 to its timing-table
// slot, and the slot of the voltage update counts Newton iterations.  Fast-decoupled
// iterations are the solves on the first DSS handle (B') that mkl_fdpf creates.
#define BASE_INDEX 1

#include <cfloat>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>

#include <fcntl.h>
#include <unistd.h>

#include <thrust/host_vector.h>
#include "Eigen/SparseLU"

using namespace std;
using namespace Eigen;

// stands in for util/timer.h (see above): consecutive calls differ by exactly 1
#define TIMER_H
static double g_timer_ticks = 0.0;
inline double GetTimer() { return g_timer_ticks += 1.0; }

double* timeTable;
enum TimeTableIndexes {
  TIME_MAIN = 0,
  TIME_INIT_STRUCT_PSO,
  TIME_ALLOC,
  TIME_PSO,
  TIME_RUNPF,
  TIME_COMPUTEVOLTAGE,
  TIME_MAKEYBUS,
  TIME_NEWTONPF,
  TIME_COMPUTEDIAGIBUS,
  TIME_COMPUTENNZJACOBIANMATRIX,
  TIME_COMPUTEJACOBIANMATRIX,
  TIME_D2H_MEM_COPY,
  TIME_SOLVER_MKL_DSS,
  TIME_H2D_MEM_COPY,
  TIME_UPDATEVOLTAGE,
  TIME_COMPUTE_POWER,
  TIME_CHECKCONVERGENCE,
  TIME_COMPUTELOSS,
  TIME_FREE,
  TIME_TABLE_SIZE
};
fstream logFile;

#include <pso/Particula.h>

#define MKL_Complex16 double2
#include "mkl.h"

#include <cublas_v2.h>
#include <cusparse_v2.h>
#include <cusolverSp.h>
#include <cusolverSp_LOWLEVEL_PREVIEW.h>
#include <cusolverRf.h>
#include "cusparse_legacy.h"
#include "util/helper_cuda.h"

#include "powersystem/Topology.h"
#include "powersystem/Bus.h"
#include "powersystem/Branch.h"
#include "powersystem/Generator.h"
#include "powerflow/runpf.h"

#include "mpf.h"

namespace {
// stdout of the reference's own progress prints ("DGM:: Entered ...") goes to /dev/null
struct QuietStdout {
  int saved = -1;
  QuietStdout() {
    fflush(stdout);
    saved = dup(1);
    const int nul = open("/dev/null", O_WRONLY);
    if (nul >= 0) {
      dup2(nul, 1);
      close(nul);
    }
  }
  ~QuietStdout() {
    fflush(stdout);
    if (saved >= 0) {
      dup2(saved, 1);
      close(saved);
    }
  }
};
}  // namespace

namespace {
// The reference's host data for one grid: Topology (Topology.h: PV/PQ lists and
// indicePVPQ computed by its constructor), the optimiser structures (one OLTC per
// tapped branch, holding the branch's own ratio) and the particle that carries them.
struct RefGrid {
  Topology topo;
  vector<pso::Particula::Estrutura> estrutura;
  pso::Particula particula;
  std::vector<mpf_branch> br_in;
  std::vector<mpf_bus> bus_in;
  std::vector<double> table;

  RefGrid(const mpf_bus* bus, int nb, const mpf_branch* br, int nbr)
      : br_in(br, br + nbr), bus_in(bus, bus + nb), table(TIME_TABLE_SIZE, 0.0) {
    timeTable = table.data();
    thrust::host_vector<unsigned int> ids(nb);
    thrust::host_vector<Bus> buses(nb);
    thrust::host_vector<Branch> branches(nbr);
    thrust::host_vector<Generator> gens(0);
    for (int i = 0; i < nb; ++i) {
      Bus b;
      b.id = i;
      b.type = (Bus::Type)bus[i].type;
      b.V = bus[i].vm;
      b.O = bus[i].va;
      b.P = bus[i].p;
      b.Q = bus[i].q;
      b.Gsh = bus[i].gsh;
      b.Bsh = bus[i].bsh;
      buses[i] = b;
      ids[i] = i;
    }
    for (int k = 0; k < nbr; ++k) {
      Branch r;
      r.from = br[k].from;
      r.to = br[k].to;
      r.inservice = br[k].status != 0;
      r.R = br[k].r;
      r.X = br[k].x;
      r.B = br[k].b;
      r.tap = br[k].tap;
      r.shift = br[k].shift;
      if (r.tap != 0) {
        r.indiceEstrutura = (int)estrutura.size();
        estrutura.push_back(pso::Particula::Estrutura::newOLTC(r.tap, r.tap, r.tap, 1, k));
        particula.X.push_back(r.tap);
      }
      branches[k] = r;
    }
    topo = Topology(1.0, ids, buses, branches, gens);
  }
  Branch* branch_data() { return thrust::raw_pointer_cast(topo.branches.data()); }
  Bus* bus_data() { return thrust::raw_pointer_cast(topo.buses.data()); }
  // case c: outaged branches out of service, optionally its own injections
  void apply_case(int n_out, const int* out, const double* sbus_c) {
    for (int p = 0; p < n_out; ++p) branch_data()[out[p]].inservice = false;
    if (sbus_c)
      for (size_t i = 0; i < bus_in.size(); ++i) {
        bus_data()[i].P = sbus_c[2 * i];
        bus_data()[i].Q = sbus_c[2 * i + 1];
      }
  }
  void restore_case(int n_out, const int* out, const double* sbus_c) {
    for (int p = 0; p < n_out; ++p) branch_data()[out[p]].inservice = br_in[out[p]].status != 0;
    if (sbus_c)
      for (size_t i = 0; i < bus_in.size(); ++i) {
        bus_data()[i].P = bus_in[i].p;
        bus_data()[i].Q = bus_in[i].q;
      }
  }
};

void copy_v(double* dst) {
  for (int i = 0; i < H_NBUS; ++i) {
    dst[2 * (size_t)i] = V[i].x;
    dst[2 * (size_t)i + 1] = V[i].y;
  }
}

// mkl_clean (runpf.h:452-521) frees the reference's global arrays without clearing the
// pointers, and some of them (the Jacobian's, the B' / B'' ones) are allocated lazily
// by the first solve rather than by mkl_init, so a second mkl_init / mkl_clean cycle in
// the same process would free them twice.  The reference runs one cycle per process;
// this driver runs several, so it clears every pointer mkl_clean releases.
void clean_reference() {
  mkl_clean();
  void** freed[] = {(void**)&V, (void**)&csrColIndYf, (void**)&csrColIndYt, (void**)&csrColIndYsh,
                    (void**)&csrColIndCt, (void**)&csrColIndCf, (void**)&cooColCt, (void**)&cooColCf,
                    (void**)&csrRowPtrYbus, (void**)&csrRowPtrYf, (void**)&csrRowPtrYt, (void**)&csrRowPtrYsh,
                    (void**)&csrRowPtrCt, (void**)&csrRowPtrCf, (void**)&cooRowCt, (void**)&cooRowCf,
                    (void**)&csrRowPtrCfYf, (void**)&csrRowPtrCtYt, (void**)&csrRowPtrCfYfCtYt, (void**)&csrValYf,
                    (void**)&csrValYt, (void**)&csrValYsh, (void**)&csrValCf, (void**)&csrValCt, (void**)&cooValCf,
                    (void**)&cooValCt, (void**)&pBuffer, (void**)&converged_test, (void**)&F, (void**)&dx,
                    (void**)&csrValJ, (void**)&csrRowPtrJ, (void**)&csrColIndJ, (void**)&diagIbus, (void**)&cooRowJ,
                    (void**)&h_csrColIndJ, (void**)&h_csrRowPtrJ, (void**)&cooBpRow, (void**)&cooBpCol,
                    (void**)&cooBpVal, (void**)&csrBpVal, (void**)&csrBpCol, (void**)&csrBpRow, (void**)&cooBppRow,
                    (void**)&cooBppCol, (void**)&cooBppVal, (void**)&csrBppVal, (void**)&csrBppCol,
                    (void**)&csrBppRow, (void**)&tmpBuses, (void**)&tmpBranches, (void**)&tmpCsrColIndYbus,
                    (void**)&tmpCsrColIndYf, (void**)&tmpCsrColIndYt, (void**)&tmpCsrRowPtrYbus,
                    (void**)&tmpCsrRowPtrYf, (void**)&tmpCsrRowPtrYt, (void**)&tmpCsrValYbus, (void**)&tmpCsrValYf,
                    (void**)&tmpCsrValYt, (void**)&P, (void**)&Q};
  for (void** q : freed) *q = nullptr;
  nnzJ = 0;
}
}  // namespace

// solver: 0 = MKL_DSS (through refshim's DSS), 5 = Eigen_SparseLU (runpf.h:20-27).
// Per case c: outages outage_branches[offs[c] .. offs[c+1]-1]; sbus (nullable)
// [n_cases][n_bus][2] net injections.  Outputs (each nullable): v [n_cases][n_bus][2],
// iterations, converged (1/0), loss (mkl_runpf's return: total active loss, DBL_MAX if
// not converged).
extern "C" int refpf_runpf(const mpf_bus* bus_in, int nb, const mpf_branch* br_in, int nbr, int alg, int solver,
                           int n_cases, const int* offs, const int* outages, const double* sbus, double* v_out,
                           int* iterations, unsigned char* converged, double* loss) {
  if (nb <= 0 || nbr <= 0 || n_cases < 0 || (alg != NR && alg != FDXB && alg != FDBX) ||
      (solver != MKL_DSS && solver != Eigen_SparseLU))
    return 1;
  RefGrid grid(bus_in, nb, br_in, nbr);
  QuietStdout quiet;
  H_LinearSolver = solver;
  mkl_init(grid.topo, 1, grid.estrutura, alg);
  for (int c = 0; c < n_cases; ++c) {
    const double* sb = sbus ? sbus + (size_t)c * nb * 2 : nullptr;
    grid.apply_case(offs[c + 1] - offs[c], outages + offs[c], sb);
    refshim::dss_live().clear();
    refshim::dss_solve_log().clear();
    const double it0 = timeTable[TIME_UPDATEVOLTAGE];
    const double l = mkl_runpf(grid.estrutura, grid.particula);
    if (loss) loss[c] = l;
    if (converged) converged[c] = l != DBL_MAX;
    if (iterations) {
      if (alg == NR)
        iterations[c] = (int)(timeTable[TIME_UPDATEVOLTAGE] - it0);
      else
        iterations[c] = refshim::dss_solve_log().empty() ? 0 : (int)refshim::dss_solve_log()[0];
    }
    if (v_out) copy_v(v_out + (size_t)c * nb * 2);
    grid.restore_case(offs[c + 1] - offs[c], outages + offs[c], sb);
  }
  clean_reference();
  return 0;
}

// The reference's Ybus (mkl_makeYbus, makeYbus.h:113-274) of the base grid with the
// given outages: one-based CSR as the reference keeps it.  Call with col/val NULL to get
// nnz (returned), then again with arrays of that size.
extern "C" int refpf_ybus(const mpf_bus* bus_in, int nb, const mpf_branch* br_in, int nbr, int n_out,
                          const int* outages, int* rowptr, int* col, double* val) {
  RefGrid grid(bus_in, nb, br_in, nbr);
  grid.apply_case(n_out, outages, nullptr);
  QuietStdout quiet;
  H_LinearSolver = Eigen_SparseLU;
  mkl_init(grid.topo, 1, grid.estrutura, NR);
  mkl_makeYbus(grid.estrutura, grid.particula, buses, branches);
  const int nnz = nnzYbus;
  if (rowptr) std::copy(csrRowPtrYbus, csrRowPtrYbus + nb + 1, rowptr);
  if (col && val)
    for (int p = 0; p < nnz; ++p) {
      col[p] = csrColIndYbus[p];
      val[2 * p] = csrValYbus[p].x;
      val[2 * p + 1] = csrValYbus[p].y;
    }
  MKL_free(csrColIndYbus);
  MKL_free(csrValYbus);
  clean_reference();
  return nnz;
}

// ---- Newton-Raphson one iteration at a time (the timed CPU arm of the benchmark) ----
// The same sequence of the reference's functions as mkl_runpf (runpf.h:259-352) and
// mkl_newtonpf (newtonpf.h:365-523), cut at iteration boundaries so that a caller can
// time a bounded slice of a large case and keep its state between slices:
//   a case starts with mkl_computeVoltage, mkl_makeYbus and the first
//   mkl_checkConvergence; each Newton iteration is mkl_computeDiagIbus,
//   (once per grid) mkl_computeNnzJacobianMatrix, mkl_compuateJacobianMatrix, the linear
//   solver of H_LinearSolver, mkl_updateVoltage and mkl_checkConvergence; a case ends when
//   max |F| < EPS or after MAX_IT_NR iterations, with mkl_computeLoss when converged.
// One grid per process (the reference keeps its state in globals).
namespace {
RefGrid* g_step_grid = nullptr;
struct StepCase {
  bool active = false;
  int iter = 0;
  std::vector<int> out;
} g_step;
}  // namespace

extern "C" int refpf_nr_open(const mpf_bus* bus_in, int nb, const mpf_branch* br_in, int nbr, int solver) {
  if (g_step_grid || (solver != MKL_DSS && solver != Eigen_SparseLU)) return 1;
  g_step_grid = new RefGrid(bus_in, nb, br_in, nbr);
  QuietStdout quiet;
  H_LinearSolver = solver;
  mkl_init(g_step_grid->topo, 1, g_step_grid->estrutura, NR);
  g_step = StepCase();
  return 0;
}

// Starts a case (outages) when none is active, then runs one Newton iteration.
// On return *done = 1 when the case finished in this call (converged or iteration
// limit); then *converged, *iterations and (nullable) v [n_bus][2] describe it.
extern "C" int refpf_nr_step(int n_out, const int* outages, int* done, int* converged, int* iterations, double* v) {
  if (!g_step_grid) return 1;
  QuietStdout quiet;
  *done = 0;
  bool conv = false;
  if (!g_step.active) {
    g_step.out.assign(outages, outages + n_out);
    g_step_grid->apply_case(n_out, outages, nullptr);
    mkl_computeVoltage(buses, V, g_step_grid->estrutura, g_step_grid->particula);
    mkl_makeYbus(g_step_grid->estrutura, g_step_grid->particula, buses, branches);
    const double err = mkl_checkConvergence(buses, pv, pq, nnzYbus, csrRowPtrYbus, csrColIndYbus, csrValYbus, V, F);
    g_step.active = true;
    g_step.iter = 0;
    conv = err < EPS;
  }
  if (!conv) {
    g_step.iter++;
    mkl_computeDiagIbus(nnzYbus, csrRowPtrYbus, csrColIndYbus, csrValYbus, V, diagIbus);
    if (nnzJ == 0) mkl_computeNnzJacobianMatrix();
    mkl_compuateJacobianMatrix(nnzJ, cooRowJ, csrRowPtrJ, csrColIndJ, csrValJ, pq, pv, nnzYbus, csrRowPtrYbus,
                               csrColIndYbus, csrValYbus, diagIbus, V);
    if (H_LinearSolver == MKL_DSS)
      mkl_solver_MKL_DSS();
    else
      eigen_sparseLU_solver();
    mkl_updateVoltage(pv, pq, V, dx);
    const double err = mkl_checkConvergence(buses, pv, pq, nnzYbus, csrRowPtrYbus, csrColIndYbus, csrValYbus, V, F);
    conv = err < EPS;
  }
  if (conv || g_step.iter >= MAX_IT_NR) {
    if (conv)
      mkl_computeLoss(branches, V, nnzYf, csrRowPtrYf, csrColIndYf, csrValYf, nnzYt, csrRowPtrYt, csrColIndYt,
                      csrValYt);
    *done = 1;
    *converged = conv ? 1 : 0;
    *iterations = g_step.iter;
    if (v) copy_v(v);
    MKL_free(csrColIndYbus);
    MKL_free(csrValYbus);
    g_step_grid->restore_case((int)g_step.out.size(), g_step.out.data(), nullptr);
    g_step.active = false;
  }
  return 0;
}

extern "C" int refpf_nr_close() {
  if (!g_step_grid) return 1;
  QuietStdout quiet;
  clean_reference();
  delete g_step_grid;
  g_step_grid = nullptr;
  return 0;
}

/*
 * mpf.h — C-ABI of the B200-native batched AC power-flow engine (libmpf.so).
 *
 * One handle = one grid (buses + branches) with its symbolic analysis done
 * once on the host, plus a batch of cases.  A case is the base grid with a
 * set of outaged branches (N-1, N-k) and, optionally, its own bus
 * injections (load scenarios).  mpf_solve runs Newton-Raphson or
 * fast-decoupled XB/BX over every case of the batch on one GPU.
 *
 * This replaces the reference's power-flow entry points:
 *   hybrid_init  (src/powerflow/runpf.h:795)  -> mpf_create + mpf_set_cases
 *   hybrid_runpf (src/powerflow/runpf.h:606)  -> mpf_solve (+ mpf_get_results)
 *   hybrid_free  (src/powerflow/runpf.h:984)  -> mpf_destroy
 *   mkl_runpf    (src/powerflow/runpf.h:259)  -> mpf_runpf_host (host buffers in/out)
 * and the algorithm constants NR/FDXB/FDBX (src/powerflow/runpf.h:16-18),
 * MAX_IT_NR/MAX_IT_FD/EPS (src/powerflow/runpf.h:45-47).
 *
 * Conventions follow the reference data model:
 *   bus.p, bus.q   net injection (generation - demand) in p.u.   (Bus.h:27-28,
 *                  files/loadMatpowerFormat.h:87-88,120-123)
 *   bus.va         voltage angle in radians                       (loadMatpowerFormat.h:87)
 *   branch.tap     off-nominal ratio, 0 means "no transformer" -> 1 (makeYbus.h:332)
 *   branch.shift   phase shift in degrees                         (makeYbus.h:333-335)
 *   J ordering     rows [P_pv, P_pq, Q_pq], cols [Va_pv, Va_pq, Vm_pq], PV and PQ
 *                  buses in bus-index order                       (Topology.h:100-126)
 *
 * Errors never exit or trap: every entry point returns an mpf_status and
 * mpf_last_error() gives a message.  Per-case outcomes are mpf_case_status.
 */
#ifndef MPF_H_
#define MPF_H_

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPF_ABI_VERSION 3

/* algorithms — same values as NR / FDXB / FDBX in src/powerflow/runpf.h:16-18 */
#define MPF_NR   0
#define MPF_FDXB 1
#define MPF_FDBX 2

/* precision of the LU factorisation and triangular solves (mismatch, update and
 * convergence test are always FP64) */
#define MPF_FP64  0
#define MPF_MIXED 1

/* defaults — MAX_IT_NR, MAX_IT_FD, EPS in src/powerflow/runpf.h:45-47 */
#define MPF_DEFAULT_MAX_IT_NR 10
#define MPF_DEFAULT_MAX_IT_FD 30
#define MPF_DEFAULT_TOL 1e-8

/* bus types — Bus::Type in src/powersystem/Bus.h:11-13 (MATPOWER codes) */
#define MPF_BUS_NONE     0
#define MPF_BUS_PQ       1
#define MPF_BUS_PV       2
#define MPF_BUS_SLACK    3
#define MPF_BUS_ISOLATED 4

typedef enum mpf_status {
  MPF_OK = 0,
  MPF_ERR_BAD_INPUT = 1,   /* invalid argument or grid */
  MPF_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  MPF_ERR_OOM = 3,         /* device or host allocation failed */
  MPF_ERR_STATE = 4,       /* call out of order (e.g. solve before set_cases) */
  MPF_ERR_TIMEOUT = 5,     /* a bounded device-side wait ran out */
  MPF_ERR_INTERNAL = 6,
  MPF_ERR_NO_DEVICE = 7    /* no CUDA device visible */
} mpf_status;

typedef enum mpf_case_status {
  MPF_CASE_RUNNING = 0,    /* not finished (only seen mid-solve) */
  MPF_CASE_CONVERGED = 1,  /* max |mismatch| < tol */
  MPF_CASE_MAX_ITER = 2,   /* iteration limit reached (the reference's "not converged") */
  MPF_CASE_DIVERGED = 3,   /* non-finite mismatch or voltage */
  MPF_CASE_SINGULAR = 4    /* zero / tiny pivot in the LU, or outages that cut PV / PQ
                              buses off from every slack (found by mpf_set_cases: the
                              Jacobian is structurally singular; such a case is not
                              iterated and reports 0 iterations and its start point) */
} mpf_case_status;

/* Bus record: the fields of Bus (src/powersystem/Bus.h:18-31) the power flow reads. */
typedef struct mpf_bus {
  int32_t type;   /* MPF_BUS_* */
  int32_t pad_;
  double vm;      /* voltage magnitude (p.u.); PV/slack: set-point */
  double va;      /* voltage angle (radians) */
  double p;       /* net active injection (p.u.) */
  double q;       /* net reactive injection (p.u.) */
  double gsh;     /* shunt conductance (p.u.) */
  double bsh;     /* shunt susceptance (p.u.) */
} mpf_bus;

/* Branch record: the fields of Branch (src/powersystem/Branch.h:18-26). */
typedef struct mpf_branch {
  int32_t from;   /* 0-based bus index */
  int32_t to;
  int32_t status; /* 1 in service, 0 out of service (Branch::inservice) */
  int32_t pad_;
  double r, x, b; /* series R, X and total line charging B (p.u.) */
  double tap;     /* ratio; 0 = no transformer (treated as 1) */
  double shift;   /* degrees */
} mpf_branch;

typedef struct mpf_options {
  int32_t max_it_nr;   /* default 10 */
  int32_t max_it_fd;   /* default 30 */
  double tol;          /* default 1e-8 p.u., strict '<' on max |F| */
  int32_t angle_mode;  /* 0: atan2 (default); 1: atan(y/x) as cuCangle in
                          src/util/complexUtils.h:21-23 (loses the quadrant) */
  int32_t device;      /* CUDA device ordinal, default 0 */
  int32_t use_graph;   /* 2: the whole Newton loop as one CUDA graph whose while node
                          tests "any case running" and the iteration count on the device
                          (one read-back per solve; mpf_timing then reports the loop in
                          other_ms) (default 2); 1: the Newton iteration as captured CUDA
                          graphs, the host reads one flag per iteration and mpf_timing
                          splits the solve by kernel family; 0: direct launches.  All
                          three give the same results bit for bit. */
  int32_t autotune;    /* 1: time the candidate kernels of every factorisation launch on
                          the first solve of a batch size and keep the fastest (default 1);
                          0: fixed heuristic */
  int32_t ordering;    /* fill-reducing bus order of the Newton system, MPF_ORDER_*:
                          0 automatic (default), 1 minimum degree, 2 minimum fill,
                          3 minimum fill weighted by variables per bus */
  int32_t reserved[3];
} mpf_options;

/* orderings (mpf_options.ordering).  Automatic: the candidate with the least estimated
 * factorisation time per case, flops + 53000 x elimination-tree levels (a level costs
 * about one launch of the level-synchronous factorisation and backward solve). */
#define MPF_ORDER_AUTO 0
#define MPF_ORDER_MIN_DEGREE 1
#define MPF_ORDER_MIN_FILL 2
#define MPF_ORDER_MIN_FILL_WEIGHTED 3

/* Per-kernel device time of the last mpf_solve (CUDA events on the solve stream),
 * milliseconds, summed over all launches of that kernel in the solve. */
typedef struct mpf_timing {
  double total_ms;
  double mismatch_ms, jacobian_ms, factor_ms, solve_ms, update_ms, other_ms;
  int32_t iterations_max;   /* max iterations over cases */
  int32_t launches;         /* kernels launched by the last solve */
} mpf_timing;

/* Symbolic statistics of the handle (for reports and tests). */
typedef struct mpf_stats {
  int32_t n_bus, n_branch, n_pv, n_pq, n_slack;
  int32_t nnz_ybus;
  int32_t n_jac, nnz_jac, nnz_lu, lu_levels;   /* Newton system */
  int64_t lu_flops;                            /* multiply-adds x2 per factorisation */
  int32_t n_bp, nnz_bp_lu, bp_levels;          /* B' system */
  int32_t n_bpp, nnz_bpp_lu, bpp_levels;       /* B'' system */
  int32_t n_cases, case_groups;
  int64_t device_bytes;                        /* device memory held by the handle */
  int64_t nnz_lu_upper;                        /* entries of the Newton system's U panels (the
                                                  pivot rows of each supernode: what a backward
                                                  substitution reads) */
  int32_t ordering;                            /* MPF_ORDER_* the Newton system uses */
  int32_t pad_;
} mpf_stats;

typedef struct mpf_handle mpf_handle;

/* ---- library ---------------------------------------------------------- */
int32_t mpf_abi_version(void);
void mpf_default_options(mpf_options* opt);
const char* mpf_status_string(int32_t status);

/* ---- handle lifecycle (replaces hybrid_init / hybrid_free) ------------- */
/* Validates the grid, builds the superset Ybus pattern, the Jacobian, B' and B''
 * patterns, their fill-reducing orderings and symbolic LU, and uploads the shared
 * (case-independent) arrays to the device.  Every connected island with PV/PQ
 * buses needs exactly one slack bus (one island per grid; several islands: see
 * mpf_set_cases_islands). */
int32_t mpf_create(const mpf_bus* buses, int32_t n_bus,
                   const mpf_branch* branches, int32_t n_branch,
                   const mpf_options* opt, mpf_handle** out);
int32_t mpf_destroy(mpf_handle* h);
const char* mpf_last_error(const mpf_handle* h);
int32_t mpf_get_stats(const mpf_handle* h, mpf_stats* st);

/* ---- cases ------------------------------------------------------------- */
/* Defines the batch.  Case c outages branches
 *   outage_branches[outage_offsets[c] .. outage_offsets[c+1]-1]
 * (outage_offsets has n_cases+1 entries; both may be NULL for n_cases base cases).
 * sbus (nullable): per-case net injections, [n_cases][n_bus][2] (p, q) in p.u.;
 * NULL means every case uses the grid's bus.p / bus.q.
 * All pointers are host pointers; the data is copied. */
int32_t mpf_set_cases(mpf_handle* h, int32_t n_cases,
                      const int32_t* outage_offsets, const int32_t* outage_branches,
                      const double* sbus);

/* Several grids in one batch.  A handle may hold several grids as the islands of
 * one grid (concatenate their buses and branches with index offsets; each island,
 * i.e. connected component, has exactly one slack bus; islands are numbered in the
 * order of their slack buses).  Every Newton / fast-decoupled stage then runs all
 * islands' cases in the same launches: the Jacobian is block-diagonal by island, each
 * case belongs to one island, and rows, branches and supernodes of other islands are
 * skipped.  mpf_set_cases takes a case's island from its outaged branches; this form
 * gives island_of_case[n_cases] explicitly (required for cases without outages on a
 * grid with several islands).  Results stay per case, over all buses / branches of
 * the handle (entries of other islands hold the start point / zero).  No counterpart
 * in the reference, which handles one grid per process (runpf.h:795). */
int32_t mpf_set_cases_islands(mpf_handle* h, int32_t n_cases, const int32_t* island_of_case,
                              const int32_t* outage_offsets, const int32_t* outage_branches,
                              const double* sbus);

/* Reactive-power limits of PV buses (PV -> PQ switching).  No counterpart in the
 * reference, which parses generator Q limits (src/files/loadMatpowerFormat.h:130-137)
 * and never enforces them.  qmin / qmax: per bus, limits of the net reactive injection
 * in p.u. (generators' Qmin / Qmax minus the reactive load); +-inf or NaN = no limit;
 * only PV buses with a finite limit are affected; NULL for both disables the limits.
 * The Newton system gets a Vm variable and a Q equation for every limited PV bus (one
 * pattern for all cases; while a bus is PV in a case its Q equation reads dVm = 0).
 * mpf_solve(MPF_NR) then runs Newton to convergence, switches every PV bus whose Q lies
 * outside its limits to PQ with Q held at the violated limit (all violators of a case
 * at once, as MATPOWER's runpf with ENFORCE_Q_LIMS = 1), solves those cases again from
 * their voltages, and repeats until no case has a new violation (at most 20 rounds);
 * iteration counts add up over the rounds.  Fast-decoupled solves are refused while
 * limits are set.  Rebuilds the Newton system: call before mpf_set_cases, which must
 * be called again afterwards. */
int32_t mpf_set_q_limits(mpf_handle* h, const double* qmin, const double* qmax);
/* Bus types after the last solve, [n_cases][n_bus] (host): the grid's types, with the
 * PV buses a case switched to PQ reading MPF_BUS_PQ. */
int32_t mpf_get_bus_types(mpf_handle* h, uint8_t* types);

/* Per-case control overrides: the optimiser's structures of
 * src/pso/Particula.h:26-60 (kinds keep the values of its enum Tipo), applied as
 * hybrid_computeVoltage (src/powerflow/runpf.h:524-541) and hybrid_computeYfYt
 * (src/powerflow/makeYbus.h:313-332) apply a particle:
 *   MPF_CTRL_AVR  index = PV or slack bus;      value = its |V| set-point (p.u.)
 *   MPF_CTRL_OLTC index = branch with tap != 0; value = its tap ratio (> 0)
 *   MPF_CTRL_SHC  index = bus;                  value = its shunt susceptance Bsh (p.u.)
 * values[c * n_controls + k] is control k's value in case c.  Replaces
 * hybrid_runpf's particle upload (runpf.h:606-624).  A tap or shunt change enters
 * the case's Ybus and B''; B' ignores both, as the reference builds it from zeroed
 * taps and shunts (makeB.h:311-324).  A tap control on a branch that the case
 * outages has no effect.  Must follow mpf_set_cases, which clears the controls;
 * n_controls = 0 clears them.  Each (kind, index) at most once. */
#define MPF_CTRL_AVR  1
#define MPF_CTRL_OLTC 2
#define MPF_CTRL_SHC  3
typedef struct mpf_control {
  int32_t kind;
  int32_t index;
} mpf_control;
int32_t mpf_set_controls(mpf_handle* h, int32_t n_controls, const mpf_control* controls,
                         const double* values);

/* ---- solve (replaces hybrid_runpf) ------------------------------------- */
/* Runs alg (MPF_NR / MPF_FDXB / MPF_FDBX) at precision (MPF_FP64 / MPF_MIXED) over
 * every case, from the reference's start point (runpf.h:211-226: V = vm e^{j va},
 * PV/slack magnitude = set-point).  stream is a cudaStream_t (NULL = the handle's
 * own stream).  Asynchronous with respect to the host except for the first call
 * per (alg, precision), which may synchronise.  Results stay on the device until
 * read with mpf_get_results / mpf_get_results_device. */
int32_t mpf_solve(mpf_handle* h, int32_t alg, int32_t precision, void* stream);

/* Blocking copy of the results of the last solve into host buffers (each may be NULL):
 *   v          [n_cases][n_bus][2]  rectangular voltage (re, im)
 *   iterations [n_cases]            NR iterations, or FD iterations (P half-steps)
 *   status     [n_cases]            mpf_case_status
 *   max_mis    [n_cases]            final max |F| (p.u.)                          */
int32_t mpf_get_results(mpf_handle* h, double* v, int32_t* iterations,
                        uint8_t* status, double* max_mis);

/* Same, into device buffers, enqueued on stream (no host synchronisation). */
int32_t mpf_get_results_device(mpf_handle* h, double* v, int32_t* iterations,
                               uint8_t* status, double* max_mis, void* stream);

/* One call end to end from host memory, as mkl_runpf / hybrid_runpf are used by
 * their caller: copies the case definition from host buffers, solves, and copies
 * the results back into host buffers (each output may be NULL).  Blocking. */
int32_t mpf_runpf_host(mpf_handle* h, int32_t alg, int32_t precision,
                       int32_t n_cases, const int32_t* outage_offsets,
                       const int32_t* outage_branches, const double* sbus,
                       double* v, int32_t* iterations, uint8_t* status,
                       double* max_mis);

/* Max |F| of each case of the batch at the given voltages, F = [Re mis_pv; Re mis_pq;
 * Im mis_pq] with each case's outages and injections: the batched counterpart of
 * hybrid_checkConvergence (src/powerflow/newtonpf.h:526-568) and the max |F| loop
 * that follows it (newtonpf.h:1241-1254).  v: device [n_cases][n_bus][2] (the
 * layout of mpf_get_results_device); max_mis: device [n_cases].  Enqueued on
 * stream; the first call allocates a small accumulator owned by the handle. */
int32_t mpf_mismatch(mpf_handle* h, const double* v, double* max_mis, void* stream);

/* Same result as mpf_mismatch, for callers that must not allocate device memory at
 * this point: real-time control loops that may not enter an allocator (cudaMalloc can
 * block and synchronise the device), or processes where another framework's caching
 * pool owns the GPU's memory, so a fresh cudaMalloc may fail or fragment it.  No
 * counterpart in the reference.  The call allocates nothing: its accumulator is a
 * fixed 512 KB device array built into the library (held on every GPU that loads it
 * until the process exits), so a batch may have at most 65536 cases
 * (MPF_ERR_BAD_INPUT beyond that).  The handle itself (mpf_create, mpf_set_cases)
 * must have been set up beforehand.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for the life of the
 * process; make that first call before any stream capture, and reload the library
 * after a cudaDeviceReset, which invalidates the kept address.  All calls share the
 * array and each clears its own slots first: calls that overlap on the GPU
 * (different streams, or different handles on the same device) race and must be
 * serialised. */
int32_t mpf_mismatch_noalloc(mpf_handle* h, const double* v, double* max_mis, void* stream);

/* Branch ratings (host array [n_branch], p.u. of apparent power; NULL clears them),
 * used by the overload term of mpf_branch_flows and by mpf_adjoint. */
int32_t mpf_set_ratings(mpf_handle* h, const double* rating);

/* Branch flows at the solved voltages of the last mpf_solve, every case:
 *   ploss    device [n_cases]: total active loss sum_k Re(Sf_k + St_k), the quantity
 *            mkl_computeLoss / hybrid_computeLoss + reduceLoss return per case
 *            (src/powerflow/runpf.h:228-257, 543-604)
 *   overload device [n_cases] or NULL: sum_k relu(|Sf_k| - 0.9 rating_k)^2 (needs ratings)
 *   sf, st   device [n_cases][n_branch][2] or NULL: from-/to-end complex power
 * Sf = Vf conj(Yff Vf + Yft Vt), St = Vt conj(Ytf Vf + Ytt Vt); an outaged branch
 * carries nothing.  The caller decides which cases count (the reference uses
 * DBL_MAX for cases that did not converge, runpf.h:782-789). */
int32_t mpf_branch_flows(mpf_handle* h, double* ploss, double* overload, double* sf, double* st, void* stream);

/* Adjoint gradients of each converged case's overload loss
 *   L = sum_k relu(|Sf_k| - 0.9 rating_k)^2        (needs mpf_set_ratings)
 * at the solved voltages of the last mpf_solve.  J is refactorised at the solution in
 * `precision` (MPF_FP64 or MPF_MIXED = FP32 factors) and J^T lambda = dL/dx is solved
 * with transposed substitutions on those factors; with FP32 factors the solution is
 * refined twice with FP64 residuals dL/dx - J^T lambda (J refilled in FP64, whose
 * buffer is allocated on first use), which brings it to FP64 accuracy.  Outputs (device, each nullable):
 *   grad_p, grad_q [n_cases][n_bus]     dL/dP, dL/dQ of the net injections (0 where the
 *                                       injection is not a Newton equation: slack, Q of PV)
 *   grad_g, grad_b [n_cases][n_branch]  dL/dg, dL/db of the series admittance g + jb =
 *                                       1/(r + jx) (0 for outaged branches)
 * Cases that did not converge get zero gradients.  No counterpart in the reference. */
int32_t mpf_adjoint(mpf_handle* h, int32_t precision, double* grad_p, double* grad_q, double* grad_g,
                    double* grad_b, void* stream);

/* Device time per kernel family of the last solve (synchronises the solve stream). */
int32_t mpf_get_timing(mpf_handle* h, mpf_timing* t);

/* ---- synthetic inputs (no counterpart in the reference; the reference reads
 *      MATPOWER files, src/files/loadMatpowerFormat.h:14) --------------------- */
typedef struct mpf_synth_params {
  int32_t n_bus;
  int32_t n_branch;       /* total branches: spanning tree + (n_branch - n_bus + 1) extras */
  int32_t n_pv;           /* PV buses (plus one slack) */
  int32_t topology;       /* 0: geometrically local extras; 1: uniform-random extras (stress) */
  double tap_fraction;    /* fraction of branches with a tap ratio */
  double tap_lo, tap_hi;  /* tap ~ U(tap_lo, tap_hi) */
  double r_lo, r_hi;      /* r ~ U(r_lo, r_hi) */
  double xr_lo, xr_hi;    /* x = r * U(xr_lo, xr_hi) */
  double b_hi;            /* b ~ U(0, b_hi) */
  double vset_lo, vset_hi;/* PV/slack |V| set-point ~ U(lo, hi) */
  double pload_hi;        /* PQ load P ~ U(0, pload_hi) */
  double qp_lo, qp_hi;    /* Q = P * U(qp_lo, qp_hi) */
  double gen_factor;      /* PV generation sums to gen_factor * total load */
  double loading;         /* loading level: drawn loads (P and Q) are multiplied by it */
  uint64_t seed;
} mpf_synth_params;

/* Fills params with the distributions shared by all synthetic workloads
 * (r ~ U(0.01,0.10), x = r U(2,6), b ~ U(0,0.05), |V|set ~ U(1.00,1.06),
 *  P ~ U(0,0.5), Q = P U(0.2,0.5), generation 1.02 x load, taps U(0.95,1.05))
 * and loading = 0.2: with these line impedances the unscaled loads leave the base
 * case without a power-flow solution (loadability 0.2-0.3 at 300+ buses). */
void mpf_synth_default(mpf_synth_params* p);

/* Deterministic (seeded) synthetic grid; buses[n_bus], branches[n_branch] are caller-owned. */
int32_t mpf_synth_grid(const mpf_synth_params* p, mpf_bus* buses, mpf_branch* branches);

/* Marks bridges (branches whose removal disconnects the in-service graph):
 * is_bridge[n_branch] = 1 / 0.  Out-of-service branches are never bridges. */
int32_t mpf_find_bridges(const mpf_branch* branches, int32_t n_branch, int32_t n_bus,
                         uint8_t* is_bridge);

/* Picks n_out distinct in-service non-bridge branches in a seeded random order. */
int32_t mpf_select_outages(const mpf_branch* branches, int32_t n_branch, int32_t n_bus,
                           int32_t n_out, uint64_t seed, int32_t* out);

/* Load scenarios: sbus[n_cases][n_bus][2] where every bus with a load (p < 0)
 * gets p, q scaled by (1 + N(0, sigma^2)) (fixed power factor); generation unchanged. */
int32_t mpf_synth_load_scenarios(const mpf_bus* buses, int32_t n_bus, int32_t n_cases,
                                 double sigma, uint64_t seed, double* sbus);

#ifdef __cplusplus
}
#endif

#endif /* MPF_H_ */

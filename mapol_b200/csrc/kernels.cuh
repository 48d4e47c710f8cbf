// Device kernels of the batched power flow (sm_100a).
//
// Batch layout: cases are lanes.  Every per-case array is stored as
// [group][entry][32]: case c lives in group c / 32, lane c % 32, so a warp that
// handles one entry (a bus, a Jacobian entry, a factor entry) for the 32 cases of a
// group reads or writes one contiguous 256-byte (FP64) or 128-byte (FP32) row.
// Index arrays (Ybus pattern, front structures) are shared by all lanes.
//
// Per Newton iteration (newtonpf.h:365-523 does the same steps for one case):
//   k_mismatch_nr   Ibus = Ybus V, mis = V conj(Ibus) - Sbus, F into the LU
//                   right-hand side, per-case max |F|       (newtonpf.h:18-95),
//                   and in the same pass the Jacobian entries straight into the
//                   factor input (A-array)                  (newtonpf.h:97-186)
//   k_check         per-case convergence / iteration-limit / divergence mask
//   k_mf_factor     multifrontal LU of all cases, level by level, forward
//                   substitution of F carried through the fronts
//   k_mf_bsolve     backward substitution, level by level (top down)
//   k_update_nr     polar voltage update V <- (|V| - dVm) e^{j(Va - dVa)}
//                                                           (newtonpf.h:188-213)
// Each case's Ybus is the superset base minus its outaged branches, applied on the
// fly where an entry is read (no per-case Ybus, no SpGEMM).
#pragma once

#include <cfloat>
#include <cstdint>

#include <cuda_runtime.h>

namespace mpfk {

constexpr int kMaxOut = 4;  // outaged branches per case

enum : int { ST_RUNNING = 0, ST_CONVERGED = 1, ST_MAX_ITER = 2, ST_DIVERGED = 3, ST_SINGULAR = 4 };

__device__ __forceinline__ size_t at32(int g, long long n, long long e, int lane) {
  return ((size_t)g * (size_t)n + (size_t)e) * 32 + lane;
}

struct DevGrid {
  int nb, nfree, ngroups, n_jac, nA_jac;
  int angle_mode;
  int nslot, noltc;         // per-case control slots / controlled taps (0: none)
  const int* y_rowptr;
  const int* y_col;
  const double2* y_val;
  const int* y_diag;        // [nb] position of (i, i)
  const int4* br_ypos;      // per branch: Ybus positions (ff, ft, tf, tt)
  const int2* br_ft;        // per branch: from, to buses
  const double2* br_y;      // per branch: 4 admittances
  const double2* sbus0;     // [nb]
  const double2* sbus_case; // [g][nb][32] or null
  const double2* v0;        // [nb]
  const int* mis_rows;      // [nfree] PV/PQ buses
  const int2* jvar;         // [nb] (Va var, Vm var) of the Newton system, -1 if none
  const int4* jpos;         // [nnzY] A-array index of the 4 Jacobian quadrants, -1 if none
  const int* out_br;        // [kMaxOut][ngroups*32] outaged branch or -1
  double2* V;               // [g][nb][32]
  double2* Ibus;            // [g][nb][32]
  int* status;              // [ngroups*32]
  int* iters;
  double* maxmis;
  unsigned long long* facc; // running max |F| (bits of a non-negative double)
  int* group_active;        // [ngroups]
  int* any_active;          // [1]
  int* it_ptr;              // [1] Newton iterations done (graph replays read it)
  // per-case controls (null when none are set)
  const int* y_slot;        // [nnzY] control slot of a Ybus position or -1
  const double2* ctl_dy;    // [g][nslot][32] change of the Ybus entry at each slot
  const int* br_ctl;        // [nbr] index among the controlled taps or -1
  const double2* ctl_bry;   // [g][4 noltc][32] admittances (ff, ft, tf, tt) of the controlled taps
  const double2* ctl_bdy;   // [g][4 noltc][32] their dY/dg (adjoint)
  // several islands (multi-grid handle; null for one): a group's lanes all belong to
  // one island, and rows, branches and supernodes of other islands are skipped
  const int* bus_island;    // [nb]
  const int* br_island;     // [nbr]
  const int* group_island;  // [ngroups]
  // case <-> lane when lanes are grouped by island and padded (null: lane = case)
  const int* lane_case;     // [ngroups*32] user case or -1 (padding)
  const int* case_lane;     // [ncases]
  // reactive limits (null when not enforced): PV buses with limits have a Vm variable
  // and a Q equation; while a bus is PV in a case its Q row is the identity, its Vm
  // column zero and its mismatch 0, so dVm = 0 exactly
  int nsw;                  // PV buses whose limits are enforced
  const int* sw_index;      // [nb] index among them or -1
  unsigned char* pv_on;     // [g][nsw][32] 1 while PV in that case, 0 once switched to PQ
  double* q_fix;            // [g][nsw][32] Q the switched bus holds (its violated limit)
  int* iter_base;           // [ngroups*32] Newton iterations of the case's earlier rounds
  // cases whose outages cut PV/PQ buses off from every slack (their Jacobian is
  // structurally singular): SINGULAR from the start, never iterated (null: none)
  const unsigned char* case_cut;  // [ngroups*32]
};

__device__ __forceinline__ bool row_here(const DevGrid& d, int i, int g) {
  return !d.group_island || d.bus_island[i] == d.group_island[g];
}
__device__ __forceinline__ bool branch_here(const DevGrid& d, int k, int g) {
  return !d.group_island || d.br_island[k] == d.group_island[g];
}
// index among the limited PV buses of bus i if it is still PV in this lane, else -1
__device__ __forceinline__ bool still_pv(const DevGrid& d, int i, int g, int lane) {
  if (!d.sw_index) return false;
  const int k = d.sw_index[i];
  return k >= 0 && d.pv_on[at32(g, d.nsw, k, lane)];
}
__device__ __forceinline__ int lane_of_case(const DevGrid& d, int c) { return d.case_lane ? d.case_lane[c] : c; }
__device__ __forceinline__ int case_of_lane(const DevGrid& d, int lane, int ncases) {
  return d.lane_case ? d.lane_case[lane] : (lane < ncases ? lane : -1);
}

// A child's contribution block as its parent reads it: offsets of the block and of
// its right-hand-side part, its size m (= f - w) and the start of its relative map.
struct ChildRef {
  long long cb_off, cbr_off;
  int m, rel_ptr;
};
// Everything a supernode assembles from its children: the children's contribution
// blocks (entries [cb, cb + ncb)) and carried right-hand sides ([cbr, cbr + ncbr)),
// adjacent in storage
struct CbIn {
  long long cb, cbr;
  int ncb, ncbr;
};

struct DevLU {
  int n, nsn, nA;
  long long nnz, sumcb, sumcbr;
  const int* sn_w;
  const int* sn_f;
  const int* sn_rptr;
  const int* sn_rows;
  const int* child_ptr;
  const int* child_list;
  const ChildRef* child_ref;  // per child_list position
  const CbIn* cb_in;          // per supernode
  const int* sn_parent;
  const int* rel_ptr;
  const int* relmap;
  const int* ah_ptr;
  const int* ah_loc;
  const long long* pan_off;
  const long long* cb_off;
  const long long* cbr_off;
  const int* sn_island;     // [nsn] island of each supernode (null: one island)
  const int* group_island;  // [ngroups]
};

__device__ __forceinline__ bool task_here(const DevLU& L, int s, int g) {
  return !L.sn_island || L.sn_island[s] == L.group_island[g];
}

// ---------------------------------------------------------------- helpers
// A zero or non-finite pivot ends a running case as SINGULAR.  The factorisation runs
// on whole groups of 32 lanes, so lanes whose case already finished (converged,
// diverged, or cut off at set-up) are factored too; their status stays as it is.
__device__ __forceinline__ void mark_singular(int* st) { atomicCAS(st, (int)ST_RUNNING, (int)ST_SINGULAR); }

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// A lane's outaged branches: their indices and end buses.  An outage only changes
// the Ybus rows of its two end buses, so a row whose bus is neither end reads the
// base Ybus unchanged.
struct LaneOut {
  int e[kMaxOut];
  int2 ft[kMaxOut];
};

__device__ __forceinline__ void load_outages(const DevGrid& d, int c, LaneOut& o) {
  const int stride = d.ngroups * 32;
#pragma unroll
  for (int k = 0; k < kMaxOut; ++k) {
    o.e[k] = d.out_br[k * stride + c];
    if (o.e[k] >= 0) {
      const int4 q = d.br_ypos[o.e[k]];
      // positions ff (diagonal of from) and tt (diagonal of to) identify the end
      // buses' rows; the row of a position is found by the caller's row index
      o.ft[k] = make_int2(q.x, q.w);
    } else {
      o.ft[k] = make_int2(-1, -1);
    }
  }
}

// True when row i (whose diagonal Ybus position is pdiag) belongs to an end bus of
// one of the lane's outaged branches.
__device__ __forceinline__ bool row_touched(const LaneOut& o, int pdiag) {
  bool t = false;
#pragma unroll
  for (int k = 0; k < kMaxOut; ++k) t |= (o.ft[k].x == pdiag) | (o.ft[k].y == pdiag);
  return t;
}

// Ybus entry p of this case: base value minus the outaged branches' parts
// (makeYbus.h:69-73 scales a branch by its status; status 0 removes it).
__device__ __forceinline__ double2 ycase(const DevGrid& d, const LaneOut& o, int p, double2 y) {
#pragma unroll
  for (int k = 0; k < kMaxOut; ++k) {
    if (o.e[k] < 0) continue;
    const int4 q = d.br_ypos[o.e[k]];
    const double2* by = d.br_y + 4 * o.e[k];
    if (p == q.x) { const double2 t = by[0]; y.x -= t.x; y.y -= t.y; }
    if (p == q.y) { const double2 t = by[1]; y.x -= t.x; y.y -= t.y; }
    if (p == q.z) { const double2 t = by[2]; y.x -= t.x; y.y -= t.y; }
    if (p == q.w) { const double2 t = by[3]; y.x -= t.x; y.y -= t.y; }
  }
  return y;
}

// Ybus entry p of this case: ycase() on rows an outage touches, plus the change a
// per-case control (tap or shunt susceptance) makes at p.
// CTL = false compiles the correction out (kernels whose register budget is tight
// have a variant per case; the others pass true and test d.y_slot).
template <bool CTL = true>
__device__ __forceinline__ double2 yentry(const DevGrid& d, const LaneOut& o, bool touched, int p, int g, int lane) {
  double2 y = touched ? ycase(d, o, p, d.y_val[p]) : d.y_val[p];
  if (CTL && d.y_slot) {
    const int s = d.y_slot[p];
    if (s >= 0) {
      const double2 t = d.ctl_dy[at32(g, d.nslot, s, lane)];
      y.x += t.x;
      y.y += t.y;
    }
  }
  return y;
}

// Branch k's four admittances (ff, ft, tf, tt) in this case: the base values, or the
// case's own when its tap is a per-case control.
__device__ __forceinline__ void branch_y(const DevGrid& d, int k, int g, int lane, double2 y[4]) {
  const int j = d.br_ctl ? d.br_ctl[k] : -1;
  if (j < 0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) y[q] = d.br_y[4 * k + q];
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) y[q] = d.ctl_bry[at32(g, 4 * d.noltc, 4 * j + q, lane)];
  }
}

__device__ __forceinline__ bool outaged(const LaneOut& o, int k) {
  bool out = false;
#pragma unroll
  for (int q = 0; q < kMaxOut; ++q) out |= (o.e[q] == k);
  return out;
}

__device__ __forceinline__ double vangle(double2 v, int mode) {
  return mode == 1 ? atan(v.y / v.x) : atan2(v.y, v.x);
}

__device__ __forceinline__ double finite_or_inf(double m) { return (m <= DBL_MAX) ? m : INFINITY; }

// block-wide per-lane max of 8 warps, then one atomicMax per lane
__device__ __forceinline__ void block_lane_max(double v, unsigned long long* dst, bool active) {
  __shared__ double red[8][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  red[warp][lane] = v;
  __syncthreads();
  if (warp == 0) {
    double m = red[0][lane];
#pragma unroll
    for (int k = 1; k < 8; ++k) m = fmax(m, red[k][lane]);
    if (active) atomicMax(dst, (unsigned long long)__double_as_longlong(m));
  }
}

// ---------------------------------------------------------------- init / check
__global__ void k_init(DevGrid d, int ncases) {
  const size_t total = (size_t)d.ngroups * d.nb * 32;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)((t >> 5) % d.nb);
    d.V[t] = d.v0[i];
  }
  const int nl = d.ngroups * 32;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < nl; c += gridDim.x * blockDim.x) {
    d.status[c] = case_of_lane(d, c, ncases) < 0 ? ST_CONVERGED : (d.case_cut && d.case_cut[c] ? ST_SINGULAR : ST_RUNNING);
    d.iters[c] = 0;
    d.maxmis[c] = 0.0;
    d.facc[c] = 0ull;
  }
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < d.ngroups; g += gridDim.x * blockDim.x)
    d.group_active[g] = 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) *d.it_ptr = 0;
}

// Condition of the device-side Newton loop (mpf_options.use_graph = 2), run before the
// loop's while node and at the end of each body: another iteration while a case is
// running and fewer than max_it iterations are done.  k_update_nr counts the
// iterations in *it_ptr, so the loop stops after max_it bodies whatever the cases do.
__global__ void k_loop_cond(cudaGraphConditionalHandle hc, const int* __restrict__ any_active,
                            const int* __restrict__ it_ptr, int max_it) {
  cudaGraphSetConditional(hc, (*any_active != 0 && *it_ptr < max_it) ? 1u : 0u);
}

// One thread per case (a warp = a group): decide convergence of the mismatch just
// evaluated.  it = iterations done so far (it_arg, or the device counter when
// it_arg < 0); the reference loop stops when max |F| < tol or it == max_it
// (newtonpf.h:394-398, 518).
__global__ void k_check(DevGrid d, int it_arg, int max_it, double tol) {
  const int it = it_arg >= 0 ? it_arg : *d.it_ptr;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nl = d.ngroups * 32;
  bool active = false;
  if (c < nl) {
    if (d.status[c] == ST_RUNNING) {
      const double m = __longlong_as_double((long long)d.facc[c]);
      d.maxmis[c] = m;
      d.iters[c] = it + (d.iter_base ? d.iter_base[c] : 0);
      if (!(m <= DBL_MAX)) d.status[c] = ST_DIVERGED;
      else if (m < tol) d.status[c] = ST_CONVERGED;
      else if (it >= max_it) d.status[c] = ST_MAX_ITER;
      else active = true;
    }
    d.facc[c] = 0ull;
  }
  const unsigned any = __ballot_sync(0xffffffffu, active);
  if ((threadIdx.x & 31) == 0 && c < nl) {
    d.group_active[c >> 5] = any != 0u;
    if (any) atomicAdd(d.any_active, 1);
  }
}

// ---------------------------------------------------------------- Newton mismatch
// grid (row blocks, groups); 8 warps per block; a warp = one bus row x 32 cases.
constexpr int kRowsPerBlock = 64;
constexpr int kYB = 2;  // Ybus entries per batch of loads in the mismatch row pass

// With JAC, the same warp then writes the Jacobian entries of its row, reusing the
// row's admittances, voltages and Ibus; the Jacobian of a case that converges on
// this mismatch is simply not used.
// J block entries of Ybus entry (i, j) in rectangular form (newtonpf.h:97-186):
//   V_i = a + jb, V_j = c + jd, yv = Y_ij V_j, w = yv / |V_j|, I = Ibus_i if i == j else 0
//   dP/dVa = -b (I_r - yv_r) - a (-I_i + yv_i)     dP/dVm = a w_r + b w_i + (I_r c + I_i d)/|V_j|
//   dQ/dVa = -b (-I_i + yv_i) + a (I_r - yv_r)     dQ/dVm = -a w_i + b w_r + (I_r d - I_i c)/|V_j|
// J entries of Ybus entry (i, j) of this lane's case, written at the arrowhead
// positions jp (-1: not a J entry).  I = Ibus_i on the diagonal, 0 elsewhere.
// qrow_off: row i's Q equation is inactive (bus i still PV); vmcol_off: column j's Vm
// is fixed (bus j still PV).  Inactive entries are 0, the (Q_i, Vm_i) diagonal 1.
// Jacobian entries of one Ybus entry.  The FP32 Jacobian of the mixed form is also
// computed in FP32 (from the FP64 voltages, admittance and Ibus rounded once): it only
// feeds the FP32 factorisation, whose rounding it matches, while the mismatch that
// steers the Newton iteration stays FP64.
__device__ __forceinline__ void jac_entry(const DevGrid& d, float* A, int g, int lane, int4 jp, double2 y2,
                                          double2 vj, double a2, double b2, double ir2, double ii2,
                                          bool qrow_off = false, bool vmcol_off = false, bool diag = false) {
  const float cc = (float)vj.x, dd = (float)vj.y, yr = (float)y2.x, yi = (float)y2.y;
  const float a = (float)a2, b = (float)b2, ir = (float)ir2, ii = (float)ii2;
  const float yvr = yr * cc - yi * dd, yvi = yr * dd + yi * cc;
  if (jp.x >= 0) A[at32(g, d.nA_jac, jp.x, lane)] = -b * (ir - yvr) - a * (-ii + yvi);
  if (jp.z >= 0) A[at32(g, d.nA_jac, jp.z, lane)] = qrow_off ? 0.0f : -b * (-ii + yvi) + a * (ir - yvr);
  if (jp.y >= 0 || jp.w >= 0) {
    const float inv = rsqrtf(cc * cc + dd * dd);  // 1 / |V_j|
    const float wr = yvr * inv, wi = yvi * inv;
    if (jp.y >= 0) A[at32(g, d.nA_jac, jp.y, lane)] = vmcol_off ? 0.0f : a * wr + b * wi + (ir * cc + ii * dd) * inv;
    if (jp.w >= 0)
      A[at32(g, d.nA_jac, jp.w, lane)] = (qrow_off || vmcol_off) ? (qrow_off && vmcol_off && diag ? 1.0f : 0.0f)
                                                                 : -a * wi + b * wr + (ir * dd - ii * cc) * inv;
  }
}

__device__ __forceinline__ void jac_entry(const DevGrid& d, double* A, int g, int lane, int4 jp, double2 y, double2 vj,
                                          double a, double b, double ir, double ii, bool qrow_off = false,
                                          bool vmcol_off = false, bool diag = false) {
  using T = double;
  const double cc = vj.x, dd = vj.y;
  const double yvr = y.x * cc - y.y * dd, yvi = y.x * dd + y.y * cc;
  if (jp.x >= 0) A[at32(g, d.nA_jac, jp.x, lane)] = (T)(-b * (ir - yvr) - a * (-ii + yvi));
  if (jp.z >= 0) A[at32(g, d.nA_jac, jp.z, lane)] = qrow_off ? (T)0 : (T)(-b * (-ii + yvi) + a * (ir - yvr));
  if (jp.y >= 0 || jp.w >= 0) {
    const double inv = 1.0 / sqrt(cc * cc + dd * dd);  // 1 / |V_j|
    const double wr = yvr * inv, wi = yvi * inv;
    if (jp.y >= 0) A[at32(g, d.nA_jac, jp.y, lane)] = vmcol_off ? (T)0 : (T)(a * wr + b * wi + (ir * cc + ii * dd) * inv);
    if (jp.w >= 0)
      A[at32(g, d.nA_jac, jp.w, lane)] = (qrow_off || vmcol_off) ? (T)(qrow_off && vmcol_off && diag ? 1 : 0)
                                                                 : (T)(-a * wi + b * wr + (ir * dd - ii * cc) * inv);
  }
}

// One pass over the row: the off-diagonal J entries need no Ibus and are written
// while Ibus accumulates; the diagonal entry follows once Ibus is complete.
template <typename T, bool JAC, bool CTL, bool QL>
__global__ void __launch_bounds__(256, 4) k_mismatch_nr(DevGrid d, T* x, T* A) {
  const int g = blockIdx.y;
  if (!d.group_active[g]) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = g * 32 + lane;
  LaneOut o;
  load_outages(d, c, o);
  double lmax = 0.0;
  const int r1 = min(d.nfree, (blockIdx.x + 1) * kRowsPerBlock);
  for (int r = blockIdx.x * kRowsPerBlock + warp; r < r1; r += 8) {
    const int i = d.mis_rows[r];
    if (!row_here(d, i, g)) continue;
    double2 ib = make_double2(0.0, 0.0);
    const int p0 = d.y_rowptr[i], p1 = d.y_rowptr[i + 1];
    const bool touched = row_touched(o, d.y_diag[i]);
    const double2 vi = d.V[at32(g, d.nb, i, lane)];
    const bool pvi = QL && still_pv(d, i, g, lane);
    // kYB entries at a time: their column indices, then their voltages, are loaded
    // before any of them is used, so the row's chain of dependent loads is one round
    // trip per kYB entries (padding entries point at the diagonal and load nothing);
    // Ibus accumulates in the row's order as before
    for (int p = p0; p < p1; p += kYB) {
      int jj[kYB];
      double2 vv[kYB];
#pragma unroll
      for (int u = 0; u < kYB; ++u) jj[u] = p + u < p1 ? d.y_col[p + u] : i;
#pragma unroll
      for (int u = 0; u < kYB; ++u) vv[u] = jj[u] == i ? vi : d.V[at32(g, d.nb, jj[u], lane)];
#pragma unroll
      for (int u = 0; u < kYB; ++u) {
        if (p + u >= p1) break;
        const int j = jj[u];
        const double2 y = yentry<CTL>(d, o, touched, p + u, g, lane);
        const double2 v = vv[u];
        ib.x += y.x * v.x - y.y * v.y;
        ib.y += y.x * v.y + y.y * v.x;
        if (JAC && j != i) {
          const int4 jp = d.jpos[p + u];
          if (jp.x >= 0 || jp.y >= 0 || jp.z >= 0 || jp.w >= 0)
            jac_entry(d, A, g, lane, jp, y, v, vi.x, vi.y, 0.0, 0.0, pvi, QL && still_pv(d, j, g, lane));
        }
      }
    }
    double2 s = d.sbus_case ? d.sbus_case[at32(g, d.nb, i, lane)] : d.sbus0[i];
    if (QL && !pvi && d.sw_index[i] >= 0) s.y = d.q_fix[at32(g, d.nsw, d.sw_index[i], lane)];
    // mis = V conj(Ibus) - S
    const double mr = vi.x * ib.x + vi.y * ib.y - s.x;
    const double mi = vi.y * ib.x - vi.x * ib.y - s.y;
    const int2 jv = d.jvar[i];
    x[at32(g, d.n_jac, jv.x, lane)] = (T)mr;
    double m = fabs(mr);
    if (jv.y >= 0 && pvi) {
      x[at32(g, d.n_jac, jv.y, lane)] = (T)0;  // Q of a PV bus is free: its row asks dVm = 0
    } else if (jv.y >= 0) {
      x[at32(g, d.n_jac, jv.y, lane)] = (T)mi;
      m = fmax(m, fabs(mi));
      if (mi != mi) m = INFINITY;
    }
    if (mr != mr) m = INFINITY;
    lmax = fmax(lmax, finite_or_inf(m));
    if (JAC) {
      const int pd = d.y_diag[i];
      const int4 jp = d.jpos[pd];
      jac_entry(d, A, g, lane, jp, yentry<CTL>(d, o, touched, pd, g, lane), vi, vi.x, vi.y, ib.x, ib.y, pvi, pvi,
                   true);
    } else {
      d.Ibus[at32(g, d.nb, i, lane)] = ib;
    }
  }
  block_lane_max(lmax, &d.facc[c], d.status[c] == ST_RUNNING);
}

// ---------------------------------------------------------------- Newton update
template <typename T>
__global__ void __launch_bounds__(256) k_update_nr(DevGrid d, const T* x) {
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(d.it_ptr, 1);  // one more iteration
  const int g = blockIdx.y;
  if (!d.group_active[g]) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = g * 32 + lane;
  if (d.status[c] != ST_RUNNING) return;
  const int r1 = min(d.nfree, (blockIdx.x + 1) * kRowsPerBlock);
  for (int r = blockIdx.x * kRowsPerBlock + warp; r < r1; r += 8) {
    const int i = d.mis_rows[r];
    if (!row_here(d, i, g)) continue;
    const int2 jv = d.jvar[i];
    const double dva = (double)x[at32(g, d.n_jac, jv.x, lane)];
    const double dvm = jv.y >= 0 ? (double)x[at32(g, d.n_jac, jv.y, lane)] : 0.0;
    const size_t k = at32(g, d.nb, i, lane);
    const double2 v = d.V[k];
    const double mag = sqrt(v.x * v.x + v.y * v.y) - dvm;
    const double ang = vangle(v, d.angle_mode) - dva;
    double sn, cs;
    sincos(ang, &sn, &cs);
    d.V[k] = make_double2(mag * cs, mag * sn);
  }
}

// ---------------------------------------------------------------- fast decoupled
struct DevFD {
  int n_bp, n_bpp;
  const int2* fdvar;   // [nb] (B' var, B'' var) or -1
};

// P = Re(mis)/|V| over PV/PQ, Q = Im(mis)/|V| over PQ (fdpf.h:369-414)
template <typename T>
__global__ void __launch_bounds__(256) k_mismatch_fd(DevGrid d, DevFD f, T* xp, T* xq) {
  const int g = blockIdx.y;
  if (!d.group_active[g]) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = g * 32 + lane;
  LaneOut o;
  load_outages(d, c, o);
  double lmax = 0.0;
  const int r1 = min(d.nfree, (blockIdx.x + 1) * kRowsPerBlock);
  for (int r = blockIdx.x * kRowsPerBlock + warp; r < r1; r += 8) {
    const int i = d.mis_rows[r];
    if (!row_here(d, i, g)) continue;
    double2 ib = make_double2(0.0, 0.0);
    const bool touched = row_touched(o, d.y_diag[i]);
    for (int p = d.y_rowptr[i]; p < d.y_rowptr[i + 1]; ++p) {
      const double2 y = yentry(d, o, touched, p, g, lane);
      const double2 v = d.V[at32(g, d.nb, d.y_col[p], lane)];
      ib.x += y.x * v.x - y.y * v.y;
      ib.y += y.x * v.y + y.y * v.x;
    }
    const double2 vi = d.V[at32(g, d.nb, i, lane)];
    const double2 s = d.sbus_case ? d.sbus_case[at32(g, d.nb, i, lane)] : d.sbus0[i];
    const double av = sqrt(vi.x * vi.x + vi.y * vi.y);
    const double mr = (vi.x * ib.x + vi.y * ib.y - s.x) / av;
    const double mi = (vi.y * ib.x - vi.x * ib.y - s.y) / av;
    const int2 fv = f.fdvar[i];
    xp[at32(g, f.n_bp, fv.x, lane)] = (T)mr;
    double m = fabs(mr);
    if (mr != mr) m = INFINITY;
    if (fv.y >= 0) {
      xq[at32(g, f.n_bpp, fv.y, lane)] = (T)mi;
      m = fmax(m, fabs(mi));
      if (mi != mi) m = INFINITY;
    }
    lmax = fmax(lmax, finite_or_inf(m));
  }
  block_lane_max(lmax, &d.facc[c], d.status[c] == ST_RUNNING);
}

// half updates (fdpf.h:416-448): Va -= dVa over PV/PQ (half 0), |V| -= dVm over PQ (half 1)
template <typename T>
__global__ void __launch_bounds__(256) k_update_fd(DevGrid d, DevFD f, const T* xp, const T* xq, int half) {
  const int g = blockIdx.y;
  if (!d.group_active[g]) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = g * 32 + lane;
  if (d.status[c] != ST_RUNNING) return;
  const int r1 = min(d.nfree, (blockIdx.x + 1) * kRowsPerBlock);
  for (int r = blockIdx.x * kRowsPerBlock + warp; r < r1; r += 8) {
    const int i = d.mis_rows[r];
    if (!row_here(d, i, g)) continue;
    const int2 fv = f.fdvar[i];
    if (half == 1 && fv.y < 0) continue;
    const size_t k = at32(g, d.nb, i, lane);
    const double2 v = d.V[k];
    double mag = sqrt(v.x * v.x + v.y * v.y);
    double ang = vangle(v, d.angle_mode);
    if (half == 0) ang -= (double)xp[at32(g, f.n_bp, fv.x, lane)];
    else mag -= (double)xq[at32(g, f.n_bpp, fv.y, lane)];
    double sn, cs;
    sincos(ang, &sn, &cs);
    d.V[k] = make_double2(mag * cs, mag * sn);
  }
}

// B'/B'' values of every case: base arrowhead values, then minus the outaged
// branches' contributions.  Thread per (entry, lane).
template <typename T>
__global__ void k_fd_base(int ngroups, int nA, const double* base, T* A) {
  const size_t total = (size_t)ngroups * nA * 32;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x)
    A[t] = (T)base[(t >> 5) % nA];
}

template <typename T>
__global__ void k_fd_outage(DevGrid d, int nA, const int4* br_apos, const double4* br_bval, T* A) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= d.ngroups * 32) return;
  const int g = c >> 5, lane = c & 31;
  const int stride = d.ngroups * 32;
  for (int k = 0; k < kMaxOut; ++k) {
    const int e = d.out_br[k * stride + c];
    if (e < 0) continue;
    const int4 p = br_apos[e];
    const double4 v = br_bval[e];
    const int ps[4] = {p.x, p.y, p.z, p.w};
    const double vs[4] = {v.x, v.y, v.z, v.w};
    for (int q = 0; q < 4; ++q) {
      if (ps[q] < 0) continue;
      const size_t idx = at32(g, nA, ps[q], lane);
      A[idx] = (T)((double)A[idx] - vs[q]);
    }
  }
}

// ---------------------------------------------------------------- multifrontal LU
// Task = (supernode s, lane chunk of G cases).  A team of TEAM threads holds the
// front F (f x (f+1), right-hand side in column f) in shared memory as
// F[(row * (f+1) + col) * G + lane]; SLOTS = TEAM / G threads share each lane.
//   1. F = 0; scatter the arrowhead (this supernode's J / B entries) and the
//      right-hand side of its pivot rows;
//   2. extend-add each child's contribution block (and carried right-hand side);
//   3. partial LU of the w pivots (no pivoting: diagonal pivots, the reference's
//      J is factorised in the same static order for every case);
//   4. store the U- and L-panels, the forward-substituted y of the pivots, and
//      the contribution block for the parent.
// A pivot that is zero, subnormal or the smallest normal value, infinite or NaN, tested
// in the pivot's own precision
__device__ __forceinline__ bool bad_pivot(float pk) { return !(fabsf(pk) > FLT_MIN) || !(fabsf(pk) <= FLT_MAX); }
__device__ __forceinline__ bool bad_pivot(double pk) { return !(fabs(pk) > DBL_MIN) || !(fabs(pk) <= DBL_MAX); }

// Advances task (q, r) by a stride of sq whole supernodes and sr lane chunks (r < nch)
__device__ __forceinline__ void next_task(int& q, int& r, int sq, int sr, int nch) {
  q += sq;
  r += sr;
  if (r >= nch) {
    r -= nch;
    ++q;
  }
}

// First index a < n with rel[a] >= v (rel increasing), or n
__device__ __forceinline__ int first_at_least(const int* rel, int n, int v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (rel[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if (TEAM == 32) __syncwarp();
  else __syncthreads();
}

// Row stride of a front in shared memory: f + 1 columns (right-hand side last),
// rounded up to odd so that slots working on consecutive rows hit distinct banks.
__host__ __device__ __forceinline__ int front_stride(int f) { return (f + 1) | 1; }

// V adjacent lanes of one entry, moved as one 16-byte (or narrower) access
template <typename T, int V>
struct alignas(sizeof(T) * V) Lanes {
  T v[V];
};
template <typename T, int V>
__device__ __forceinline__ Lanes<T, V> ld(const T* p) { return *reinterpret_cast<const Lanes<T, V>*>(p); }
template <typename T, int V>
__device__ __forceinline__ void st(T* p, const Lanes<T, V>& a) { *reinterpret_cast<Lanes<T, V>*>(p) = a; }
// Pivot inverses, one division per thread: every thread of a warp inverts the pivot of
// lane ml = (warp lane) % G of its task's G lanes (own_inverse; a bad pivot is replaced
// by 1 and marks its case SINGULAR, by the marker threads, one per lane), and the V
// inverses a thread carries (lanes lv .. lv + V - 1) reach it by shuffles from threads
// lv .. lv + V - 1, which inverted exactly those lanes (gather_lanes; all 32 threads of
// the warp call it together).  A warp thus runs one IEEE division per thread instead
// of V, with the same quotients.
template <typename T, int G>
__device__ __forceinline__ T own_inverse(T pk, bool marker, int* st_lane0) {
  if (bad_pivot(pk)) {
    if (marker) mark_singular(&st_lane0[(threadIdx.x & 31) % G]);
    pk = (T)1;
  }
  return (T)1 / pk;
}
template <typename T, int V>
__device__ __forceinline__ Lanes<T, V> gather_lanes(T own, int lv) {
  Lanes<T, V> r;
#pragma unroll
  for (int k = 0; k < V; ++k) r.v[k] = __shfl_sync(0xffffffffu, own, lv + k);
  return r;
}

// V adjacent lanes of one entry copied global -> shared asynchronously (cp.async, cache
// at all levels); both addresses aligned to the copy size; completes at the next
// cp.async.wait_all of the issuing thread
template <typename T, int V>
__device__ __forceinline__ void cp_async(T* dst_shared, const T* src_global) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst_shared);
  constexpr int B = V * (int)sizeof(T);
  static_assert(B == 4 || B == 8 || B == 16, "cp.async moves 4, 8 or 16 bytes");
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(sa), "l"(src_global), "n"(B) : "memory");
}

// Asks L2 to fetch [p, p + bytes) from DRAM (bulk prefetch: no completion, no data
// returned to the thread); p and bytes multiples of 16
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// Partial LU of a front held in registers (256 threads as 16 x 16; thread (r, c)
// owns entries (r + 16 a, c + 16 b), a, b < TT, of its V lanes).  Per pivot the
// owners publish column p (rows >= p) and row p (columns > p) to a shared buffer
// (two buffers alternate, so one barrier per pivot suffices: a thread can only
// reuse a buffer after passing the next pivot's barrier); every thread then
// updates its own entries from the buffers.  Shared-memory traffic per pivot is
// 2 TT values per thread for TT^2 multiply-adds, instead of a load and a store
// of every updated entry.  The pivots run in blocks of 16 (pivot block pt, unrolled):
// rows and columns of tiles a < pt or b < pt lie above or left of every pivot of the
// block, so those tiles are final and skipped, and the owner tests are resolved at
// compile time.  Same operations per live entry, in the same order, as the
// shared-memory loop of k_mf_factor.  F: the assembled front; on return it holds the
// factors (and the forward-substituted right-hand side column).
template <typename T, int V, int TT>
__device__ __forceinline__ void lu_registers(T* F, int RS, int f, int ncols, int w, T* cbuf, T* rbuf, int fcap,
                                             int* st_lanes, bool lead) {
  using LV = Lanes<T, V>;
  constexpr int G = V;
  const int r = threadIdx.x & 15, c = threadIdx.x >> 4;
  LV t[TT][TT];
#pragma unroll
  for (int a = 0; a < TT; ++a)
#pragma unroll
    for (int b = 0; b < TT; ++b) {
      const int i = r + 16 * a, j = c + 16 * b;
      if (i < f && j < ncols) t[a][b] = ld<T, V>(F + (i * RS + j) * G);
      else {
#pragma unroll
        for (int k = 0; k < V; ++k) t[a][b].v[k] = (T)0;
      }
    }
  int p = 0;
#pragma unroll
  for (int pt = 0; pt < TT; ++pt) {
    const int pe = min(w, 16 * (pt + 1));
    for (; p < pe; ++p) {
      T* cp = cbuf + (p & 1) * fcap * G;        // column p, indexed by row
      T* rp = rbuf + (p & 1) * (fcap + 1) * G;  // row p, indexed by column
      const int pr = p & 15;                    // owners: thread row / column pr
      if (c == pr) {
#pragma unroll
        for (int a = pt; a < TT; ++a) {
          const int i = r + 16 * a;
          if (i >= p && i < f) st<T, V>(cp + i * G, t[a][pt]);
        }
      }
      if (r == pr) {
#pragma unroll
        for (int b = pt; b < TT; ++b) {
          const int j = c + 16 * b;
          if (j > p && j < ncols) st<T, V>(rp + j * G, t[pt][b]);
        }
      }
      __syncthreads();
      // one thread per entry carries all G = V lanes (lv = 0)
      const LV inv = gather_lanes<T, V>(own_inverse<T, G>(cp[p * G + (threadIdx.x & 31) % G], threadIdx.x < G, st_lanes), 0);
      // row p's entries right of the pivot and the multipliers of the rows below it;
      // zero elsewhere, so that the update leaves every other entry as it is (x - 0)
      LV u[TT], l[TT];
#pragma unroll
      for (int b = pt; b < TT; ++b) {
        const int j = c + 16 * b;
        if (j > p && j < ncols) u[b] = ld<T, V>(rp + j * G);
        else {
#pragma unroll
          for (int k = 0; k < V; ++k) u[b].v[k] = (T)0;
        }
      }
#pragma unroll
      for (int a = pt; a < TT; ++a) {
        const int i = r + 16 * a;
        if (i > p && i < f) {
          l[a] = ld<T, V>(cp + i * G);
#pragma unroll
          for (int k = 0; k < V; ++k) l[a].v[k] *= inv.v[k];
        } else {
#pragma unroll
          for (int k = 0; k < V; ++k) l[a].v[k] = (T)0;
        }
      }
#pragma unroll
      for (int a = pt; a < TT; ++a)
#pragma unroll
        for (int b = pt; b < TT; ++b)
#pragma unroll
          for (int k = 0; k < V; ++k) t[a][b].v[k] = t[a][b].v[k] - l[a].v[k] * u[b].v[k];
      if (c == pr) {
#pragma unroll
        for (int a = pt; a < TT; ++a) {
          const int i = r + 16 * a;
          if (i > p && i < f) t[a][pt] = l[a];
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < TT; ++a)
#pragma unroll
    for (int b = 0; b < TT; ++b) {
      const int i = r + 16 * a, j = c + 16 * b;
      if (i < f && j < ncols) st<T, V>(F + (i * RS + j) * G, t[a][b]);
    }
  __syncthreads();
}

// TT > 0: the partial LU runs in registers (lu_registers; TEAM 256 with one thread
// per entry-lane group, i.e. G <= 16 bytes of lanes); TT = 0: in shared memory, one
// barrier per pivot; TT = -2: in shared memory, two pivots per barrier.
//
// Register budgets: warp teams are launched in blocks of at most 256 threads; their
// bound of 288 threads x 3 blocks gives them 72 registers (no spills; shared memory
// holds them to at most ~24 warps per SM anyway).  9241-bus workload, mixed solves/s
// at 64 / 72 / 80 registers: 34.7k / 35.7k / 35.8k (64 spills 48 bytes per thread).
template <typename T, int G, int TEAM, int TT = 0>
__global__ void __launch_bounds__(TEAM == 32 ? 288 : TEAM, TT > 0 ? 2 : (TEAM > 256 ? 1 : (TT < 0 ? 2 : (TEAM == 32 ? 3 : 4)))) k_mf_factor(
    DevLU L, const int* __restrict__ task_sn, int nsn_l, int ngroups, int fcap,
    const T* __restrict__ A, T* __restrict__ pan, T* __restrict__ cb, T* __restrict__ cbr,
    T* __restrict__ x, int* __restrict__ status, const int* __restrict__ group_active, int with_rhs) {
  // a thread carries V adjacent lanes (16 bytes), NV threads cover the G lanes of a task
  constexpr int V = (int)(16 / sizeof(T)) < G ? (int)(16 / sizeof(T)) : G;
  constexpr int NV = G / V;
  constexpr int SLOTS = TEAM / NV;
  constexpr int LPG = 32 / G;  // lane chunks per group
  // slots form RSL row slots x CG column groups: rows are dealt to the row slots,
  // and each column group takes a contiguous share of a row's columns (fronts have
  // fewer rows than a 256-thread team has slots)
  constexpr int RSL = SLOTS < 32 ? SLOTS : 32;
  constexpr int CG = SLOTS / RSL;
  constexpr int U = V * sizeof(T) >= 16 ? 4 : 8;  // entries loaded before the dependent shared-memory stores
  using LV = Lanes<T, V>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int teams = blockDim.x / TEAM;
  const int team = threadIdx.x / TEAM, tid = threadIdx.x % TEAM;
  const int slot = tid / NV, lv = (tid % NV) * V;
  const int rs = slot % RSL, cg = slot / RSL;
  T* F = reinterpret_cast<T*>(smem_raw) + (size_t)team * fcap * front_stride(fcap) * G + lv;
  // Task t = q * nch + r is lane chunk r of the launch's q-th supernode.  Teams stride
  // over t by gridDim.x * teams (< 2^31, as are nch and q); q and r advance by the
  // stride's quotient and remainder, so no task needs a 64-bit division.
  const int nch = ngroups * LPG;
  const int tstride = gridDim.x * teams;
  const int sq = tstride / nch, sr = tstride % nch;
  for (int q = (blockIdx.x * teams + team) / nch, r = (blockIdx.x * teams + team) % nch; q < nsn_l;
       next_task(q, r, sq, sr, nch)) {
    const int s = task_sn[q];
    const int ch = r;
    const int g = ch / LPG;
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int lane = (ch % LPG) * G + lv;  // first of this thread's V lanes
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    // the rest of the supernode's description, loaded here with the above (one round
    // trip) rather than after the barriers of the phases that use it
    const int ah0 = L.ah_ptr[s], ah1 = L.ah_ptr[s + 1];
    const int ci0 = L.child_ptr[s], ci1 = L.child_ptr[s + 1];
    const long long po = L.pan_off[s];
    const bool has_parent = L.sn_parent[s] >= 0;
    const long long cbo_s = L.cb_off[s], cbro_s = L.cbr_off[s];
    const int RS = front_stride(f);
    const int ncols = with_rhs ? f + 1 : f;
    // The task's global inputs are two or three contiguous blocks per group of 32 lanes:
    // its arrowhead values, its children's contribution blocks and their carried
    // right-hand sides (siblings are adjacent in storage).  Bulk L2 prefetches of these,
    // issued before the front is zeroed, start all of the task's DRAM reads at once; the
    // loads of the assembly then mostly wait on L2.  The other lane chunks of a group
    // ask for the same lines, which L2 merges.
    {
      const CbIn cin = L.cb_in[s];
      constexpr unsigned B32 = 32 * sizeof(T);  // one entry of a group
      if (tid == 0 && ah1 > ah0) prefetch_l2(A + at32(g, L.nA, ah0, 0), (unsigned)(ah1 - ah0) * B32);
      if (tid == 1 && cin.ncb > 0) prefetch_l2(cb + at32(g, L.sumcb, cin.cb, 0), (unsigned)cin.ncb * B32);
      if (tid == 2 && with_rhs && cin.ncbr > 0) prefetch_l2(cbr + at32(g, L.sumcbr, cin.cbr, 0), (unsigned)cin.ncbr * B32);
    }
    // the first child's reference and this thread's first arrowhead positions, loaded
    // before the front is zeroed so that their latency overlaps the zeroing (larger
    // teams: more slots per front and fewer registers, so fewer positions per thread)
    ChildRef next = ci0 < ci1 ? L.child_ref[ci0] : ChildRef{};
    constexpr int H = TEAM == 32 ? (sizeof(T) == 4 ? 8 : 4) : (TT > 0 ? 1 : 2);
    int loc0[H];
#pragma unroll
    for (int u = 0; u < H; ++u) {
      const int e = ah0 + slot + u * SLOTS;
      loc0[u] = e < ah1 ? L.ah_loc[e] : 0;
    }
    // F + (r * RS + c) * G: entry (r, c) of this thread's lanes
#define FP(r, c) (F + ((r) * RS + (c)) * G)
    {
      LV z;
#pragma unroll
      for (int k = 0; k < V; ++k) z.v[k] = (T)0;
      for (int idx = slot; idx < f * RS; idx += SLOTS) st<T, V>(F + idx * G, z);
    }
    team_sync<TEAM>();
    {
      // the arrowhead values (and the pivot rows' right-hand side) are assignments into
      // the zeroed front: asynchronous global-to-shared copies put all of a task's in
      // flight at once without holding registers, then one wait
      const T* a0 = A + at32(g, L.nA, 0, lane);
      const int e1 = ah1;
      int e = ah0 + slot;
#pragma unroll
      for (int u = 0; u < H; ++u)
        if (e + u * SLOTS < e1) cp_async<T, V>(F + loc0[u] * G, a0 + (size_t)(e + u * SLOTS) * 32);
      e += H * SLOTS;
      for (; e + 7 * SLOTS < e1; e += 8 * SLOTS) {
        int loc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) loc[u] = L.ah_loc[e + u * SLOTS];
#pragma unroll
        for (int u = 0; u < 8; ++u) cp_async<T, V>(F + loc[u] * G, a0 + (size_t)(e + u * SLOTS) * 32);
      }
      for (; e < e1; e += SLOTS) cp_async<T, V>(F + L.ah_loc[e] * G, a0 + (size_t)e * 32);
      if (with_rhs)
        for (int p = slot; p < w; p += SLOTS) cp_async<T, V>(FP(p, f), x + at32(g, L.n, rows[p], lane));
      asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    team_sync<TEAM>();
    for (int ci = ci0; ci < ci1; ++ci) {
      // the next child's reference is loaded while this one is added
      const ChildRef cr = next;
      if (ci + 1 < ci1) next = L.child_ref[ci + 1];
      const int m = cr.m;
      const int* rel = L.relmap + cr.rel_ptr;
      const long long cbo = cr.cb_off;
      const int b0 = (m * cg) / CG, b1 = (m * (cg + 1)) / CG;
      for (int a = rs; a < m; a += RSL) {
        T* dst = FP(rel[a], 0);
        const T* src = cb + at32(g, L.sumcb, cbo + (long long)a * m, lane);
        int b = b0;
        for (; b + U <= b1; b += U) {
          int rb[U];
          LV v[U], o[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            rb[u] = rel[b + u] * G;
            v[u] = ld<T, V>(src + (size_t)(b + u) * 32);
          }
          // rel is injective: the U destinations are distinct
#pragma unroll
          for (int u = 0; u < U; ++u) o[u] = ld<T, V>(dst + rb[u]);
#pragma unroll
          for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int k = 0; k < V; ++k) o[u].v[k] += v[u].v[k];
            st<T, V>(dst + rb[u], o[u]);
          }
        }
        for (; b < b1; ++b) {
          T* d = dst + rel[b] * G;
          LV o = ld<T, V>(d);
          const LV v = ld<T, V>(src + (size_t)b * 32);
#pragma unroll
          for (int k = 0; k < V; ++k) o.v[k] += v.v[k];
          st<T, V>(d, o);
        }
        if (with_rhs && cg == 0) {
          T* d = FP(rel[a], f);
          LV o = ld<T, V>(d);
          const LV v = ld<T, V>(cbr + at32(g, L.sumcbr, cr.cbr_off + a, lane));
#pragma unroll
          for (int k = 0; k < V; ++k) o.v[k] += v.v[k];
          st<T, V>(d, o);
        }
      }
      team_sync<TEAM>();
    }
    if constexpr (TT > 0) {
      static_assert(TEAM == 256 && NV == 1, "register LU: one 256-thread team, one thread per entry");
      T* bufs = reinterpret_cast<T*>(smem_raw) + (size_t)fcap * front_stride(fcap) * G;
      lu_registers<T, V, TT>(F, RS, f, ncols, w, bufs, bufs + 2 * (size_t)fcap * G, fcap, status + g * 32 + lane,
                             tid == 0);
    } else if constexpr (TT < 0) {
    // Right-looking partial LU, two pivots (p, p1 = p + 1) per team barrier.  Every
    // thread computes both pivots' inverses, u = F(p,p1) and l = F(p1,p) / F(p,p); rows
    // i > p1 then take both rank-1 updates at once on columns q > p1:
    //   l0 = F(i,p) / F(p,p);  x1 = F(i,p1) - l0 u;  l1 = x1 / F'(p1,p1)
    //   F(i,q) = (F(i,q) - l0 F(p,q)) - l1 (F(p1,q) - l F(p,q))
    // Row p1 (updated by pivot p) and columns p, p1 (scaled, and column p1 updated by
    // pivot p) are read by every thread during the step, so they are written at the
    // start of the next step (no thread reads them there) or after the last one.
    // Every entry sees the operations of the one-pivot loop in the same order, so the
    // factors are the same bit for bit.
    // lane ml of the task's chunk (the lane whose pivots this thread inverts) and the
    // threads that mark a bad pivot's case
    const T* Fl = F - lv;
    const int ml = (threadIdx.x & 31) % G;
    const bool marker = tid < G;
    int* st0 = status + g * 32 + (lane - lv);
    int pend = 0, pc = 0;  // deferred work of the last step: 1 = one pivot pc, 2 = pivots pc, pc + 1
    LV pinv0, pinv1, pu, pl;
    auto finish = [&]() {
      if (pend == 1) {
        for (int i = pc + 1 + slot; i < f; i += SLOTS) {
          LV c = ld<T, V>(FP(i, pc));
#pragma unroll
          for (int k = 0; k < V; ++k) c.v[k] *= pinv0.v[k];
          st<T, V>(FP(i, pc), c);
        }
      } else if (pend == 2) {
        const int p1 = pc + 1;
        for (int i = p1 + slot; i < f; i += SLOTS) {
          LV c0 = ld<T, V>(FP(i, pc));
#pragma unroll
          for (int k = 0; k < V; ++k) c0.v[k] *= pinv0.v[k];
          st<T, V>(FP(i, pc), c0);
          if (i > p1) {
            LV c1 = ld<T, V>(FP(i, p1));
#pragma unroll
            for (int k = 0; k < V; ++k) {
              c1.v[k] = c1.v[k] - c0.v[k] * pu.v[k];
              c1.v[k] *= pinv1.v[k];
            }
            st<T, V>(FP(i, p1), c1);
          }
        }
        for (int q = p1 + slot; q < ncols; q += SLOTS) {
          LV r1 = ld<T, V>(FP(p1, q));
          const LV r0 = ld<T, V>(FP(pc, q));
#pragma unroll
          for (int k = 0; k < V; ++k) r1.v[k] = r1.v[k] - pl.v[k] * r0.v[k];
          st<T, V>(FP(p1, q), r1);
        }
      }
      pend = 0;
    };
    for (int p = 0; p < w;) {
      const T i0 = own_inverse<T, G>(Fl[(p * RS + p) * G + ml], marker, st0);
      const LV inv0 = gather_lanes<T, V>(i0, lv);
      if (p + 1 < w) {
        const int p1 = p + 1;
        const LV u = ld<T, V>(FP(p, p1));
        LV l = ld<T, V>(FP(p1, p));
#pragma unroll
        for (int k = 0; k < V; ++k) l.v[k] *= inv0.v[k];
        // the second pivot of lane ml, updated by the first one: F(p1,p1) - l u
        const T lm = Fl[(p1 * RS + p) * G + ml] * i0;
        const T pk1 = Fl[(p1 * RS + p1) * G + ml] - lm * Fl[(p * RS + p1) * G + ml];
        const LV inv1 = gather_lanes<T, V>(own_inverse<T, G>(pk1, marker, st0), lv);
        finish();
        const int nq = ncols - (p1 + 1);
        const int q0 = p1 + 1 + (nq * cg) / CG, q1 = p1 + 1 + (nq * (cg + 1)) / CG;
        const T* rp0 = FP(p, 0);
        const T* rp1 = FP(p1, 0);
        for (int i = p1 + 1 + rs; i < f; i += RSL) {
          T* ri = FP(i, 0);
          const LV a0 = ld<T, V>(ri + p * G), a1 = ld<T, V>(ri + p1 * G);
          LV l0, l1;
#pragma unroll
          for (int k = 0; k < V; ++k) {
            l0.v[k] = a0.v[k] * inv0.v[k];
            const T x1 = a1.v[k] - l0.v[k] * u.v[k];
            l1.v[k] = x1 * inv1.v[k];
          }
          int q = q0;
          for (; q + 2 <= q1; q += 2) {
            LV r0[2], r1[2], b[2];
#pragma unroll
            for (int t = 0; t < 2; ++t) {
              r0[t] = ld<T, V>(rp0 + (q + t) * G);
              r1[t] = ld<T, V>(rp1 + (q + t) * G);
              b[t] = ld<T, V>(ri + (q + t) * G);
            }
#pragma unroll
            for (int t = 0; t < 2; ++t) {
#pragma unroll
              for (int k = 0; k < V; ++k) {
                const T u1 = r1[t].v[k] - l.v[k] * r0[t].v[k];
                b[t].v[k] = b[t].v[k] - l0.v[k] * r0[t].v[k];
                b[t].v[k] = b[t].v[k] - l1.v[k] * u1;
              }
              st<T, V>(ri + (q + t) * G, b[t]);
            }
          }
          for (; q < q1; ++q) {
            const LV r0 = ld<T, V>(rp0 + q * G), r1 = ld<T, V>(rp1 + q * G);
            LV b = ld<T, V>(ri + q * G);
#pragma unroll
            for (int k = 0; k < V; ++k) {
              const T u1 = r1.v[k] - l.v[k] * r0.v[k];
              b.v[k] = b.v[k] - l0.v[k] * r0.v[k];
              b.v[k] = b.v[k] - l1.v[k] * u1;
            }
            st<T, V>(ri + q * G, b);
          }
        }
        pend = 2;
        pc = p;
        pinv0 = inv0;
        pinv1 = inv1;
        pu = u;
        pl = l;
        p += 2;
      } else {
        finish();
        const int nq = ncols - (p + 1);
        const int q0 = p + 1 + (nq * cg) / CG, q1 = p + 1 + (nq * (cg + 1)) / CG;
        const T* rp = FP(p, 0);
        for (int i = p + 1 + rs; i < f; i += RSL) {
          T* ri = FP(i, 0);
          LV lip = ld<T, V>(ri + p * G);
#pragma unroll
          for (int k = 0; k < V; ++k) lip.v[k] *= inv0.v[k];
          for (int q = q0; q < q1; ++q) {
            const LV a = ld<T, V>(rp + q * G);
            LV b = ld<T, V>(ri + q * G);
#pragma unroll
            for (int k = 0; k < V; ++k) b.v[k] = b.v[k] - lip.v[k] * a.v[k];
            st<T, V>(ri + q * G, b);
          }
        }
        pend = 1;
        pc = p;
        pinv0 = inv0;
        p += 1;
      }
      team_sync<TEAM>();
    }
    finish();
    team_sync<TEAM>();
    } else {
    // Right-looking partial LU of the w pivots, one team barrier per pivot.  At
    // pivot p the threads of row i read the unscaled F(i,p) (l_ip = F(i,p) / F(p,p)).
    // With one column group (CG = 1: each row has one owner slot) the owner writes l_ip
    // back at once; otherwise the scaled values are written back one pivot later, when
    // no thread reads column p any more (and after the loop for the last pivot).
    LV inv_prev;
    for (int p = 0; p < w; ++p) {
      const LV inv = gather_lanes<T, V>(
          own_inverse<T, G>(F[(p * RS + p) * G - lv + (threadIdx.x & 31) % G], tid < G, status + g * 32 + (lane - lv)),
          lv);
      if (CG > 1 && p > 0 && cg == CG - 1)
        for (int i = p + rs; i < f; i += RSL) {
          LV c = ld<T, V>(FP(i, p - 1));
#pragma unroll
          for (int k = 0; k < V; ++k) c.v[k] *= inv_prev.v[k];
          st<T, V>(FP(i, p - 1), c);
        }
      const int nq = ncols - (p + 1);
      const int q0 = p + 1 + (nq * cg) / CG, q1 = p + 1 + (nq * (cg + 1)) / CG;
      const T* rp = FP(p, 0);
      for (int i = p + 1 + rs; i < f; i += RSL) {
        T* ri = FP(i, 0);
        LV lip = ld<T, V>(ri + p * G);
#pragma unroll
        for (int k = 0; k < V; ++k) lip.v[k] *= inv.v[k];
        if constexpr (CG == 1) st<T, V>(ri + p * G, lip);
        int q = q0;
        for (; q + U <= q1; q += U) {
          LV a[U], b[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            a[u] = ld<T, V>(rp + (q + u) * G);
            b[u] = ld<T, V>(ri + (q + u) * G);
          }
#pragma unroll
          for (int u = 0; u < U; ++u) {
#pragma unroll
            for (int k = 0; k < V; ++k) b[u].v[k] = b[u].v[k] - lip.v[k] * a[u].v[k];
            st<T, V>(ri + (q + u) * G, b[u]);
          }
        }
        for (; q < q1; ++q) {
          const LV a = ld<T, V>(rp + q * G);
          LV b = ld<T, V>(ri + q * G);
#pragma unroll
          for (int k = 0; k < V; ++k) b.v[k] = b.v[k] - lip.v[k] * a.v[k];
          st<T, V>(ri + q * G, b);
        }
      }
      inv_prev = inv;
      team_sync<TEAM>();
    }
    if (CG > 1 && w > 0) {
      if (cg == CG - 1)
        for (int i = w + rs; i < f; i += RSL) {
          LV c = ld<T, V>(FP(i, w - 1));
#pragma unroll
          for (int k = 0; k < V; ++k) c.v[k] *= inv_prev.v[k];
          st<T, V>(FP(i, w - 1), c);
        }
      team_sync<TEAM>();
    }
    }
    T* pbase = pan + at32(g, L.nnz, po, lane);
    // U-panel: rows 0..w-1, all f columns; L-panel: rows w..f-1, columns 0..w-1
    {
      const int c0 = (f * cg) / CG, c1 = (f * (cg + 1)) / CG;
      for (int p = rs; p < w; p += RSL) {
        T* dst = pbase + (size_t)p * f * 32;
        const T* src = FP(p, 0);
#pragma unroll 4
        for (int q = c0; q < c1; ++q) st<T, V>(dst + (size_t)q * 32, ld<T, V>(src + q * G));
      }
    }
    const int m = f - w;
    {
      const int c0 = (w * cg) / CG, c1 = (w * (cg + 1)) / CG;
      for (int i = rs; i < m; i += RSL) {
        T* dst = pbase + ((size_t)w * f + (size_t)i * w) * 32;
        const T* src = FP(w + i, 0);
#pragma unroll 4
        for (int q = c0; q < c1; ++q) st<T, V>(dst + (size_t)q * 32, ld<T, V>(src + q * G));
      }
    }
    if (with_rhs)
      for (int p = slot; p < w; p += SLOTS) st<T, V>(x + at32(g, L.n, rows[p], lane), ld<T, V>(FP(p, f)));
    if (has_parent) {
      T* cbase = cb + at32(g, L.sumcb, cbo_s, lane);
      const int c0 = (m * cg) / CG, c1 = (m * (cg + 1)) / CG;
      for (int a = rs; a < m; a += RSL) {
        T* dst = cbase + (size_t)a * m * 32;
        const T* src = FP(w + a, w);
#pragma unroll 4
        for (int b = c0; b < c1; ++b) st<T, V>(dst + (size_t)b * 32, ld<T, V>(src + b * G));
        if (with_rhs && cg == 0) st<T, V>(cbr + at32(g, L.sumcbr, cbro_s + a, lane), ld<T, V>(FP(w + a, f)));
      }
    }
#undef FP
    team_sync<TEAM>();
  }
}

// Fronts too large for a dense front in shared memory (densely meshed grids).  The
// panel stays in shared memory for the whole task: the w pivot rows with all f columns
// and the right-hand side (top part, w x (f + 1)) and the pivot columns of the other
// rows (left part, m x w, m = f - w), G lanes per entry.  The trailing m x m block
// follows in slabs of S rows (shared memory after the panel), each assembled from the
// children, updated by the Schur complement and written to the supernode's
// contribution block.  Every entry takes the same operations in the same order as in
// the one-pivot loop of k_mf_factor (assignment of the arrowhead value, the children's
// additions in child order, then x - l_ip u_pj for p = 0 .. w - 1), so the factors are
// the same bit for bit.  One 512-thread block per task (supernode, chunk of G lanes);
// thread = (entry slot, lane); dynamic shared memory: pcap panel entries (the launch's
// largest panel) and S (mcap + 1) slab entries (mcap: its largest m), G lanes each.
template <typename T, int G>
__global__ void __launch_bounds__(512, 1) k_mf_factor_big(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                       int ngroups, const T* __restrict__ A,
                                                       T* __restrict__ pan, T* __restrict__ cb,
                                                       T* __restrict__ cbr, T* __restrict__ x,
                                                       int* __restrict__ status,
                                                       const int* __restrict__ group_active, int with_rhs,
                                                       int pcap, int S) {
  constexpr int SLOTS = 512 / G, LPG = 32 / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* P = reinterpret_cast<T*>(smem_raw);
  const int slot = threadIdx.x / G, l = threadIdx.x % G;
  const int nch = ngroups * LPG;
  for (int q = blockIdx.x / nch, ch = blockIdx.x % nch; q < nsn_l;
       next_task(q, ch, (int)gridDim.x / nch, (int)gridDim.x % nch, nch)) {
    const int s = task_sn[q];
    const int g = ch / LPG;
    if (!group_active[g] || !task_here(L, s, g)) continue;  // uniform over the block
    const int lane = (ch % LPG) * G + l;
    const int w = L.sn_w[s], f = L.sn_f[s], m = f - w;
    const int* rows = L.sn_rows + L.sn_rptr[s];
    const int RS = front_stride(f);
    const int ncols = with_rhs ? f + 1 : f;
    const bool has_parent = L.sn_parent[s] >= 0;
    const long long cbo = L.cb_off[s], cbro = L.cbr_off[s];
    const int npan = w * (f + 1) + m * w;
    // panel entry (r, c), r < w or c < w: top part row-major, then the left part
    auto PE = [&](int r, int c) -> T& {
      return r < w ? P[((size_t)r * (f + 1) + c) * G + l] : P[((size_t)w * (f + 1) + (size_t)(r - w) * w + c) * G + l];
    };
    // trailing entry (a, b) of the contribution block, and the carried right-hand side
    auto CE = [&](int a, int b) -> T& { return cb[at32(g, L.sumcb, cbo + (long long)a * m + b, lane)]; };
    auto CR = [&](int a) -> T& { return cbr[at32(g, L.sumcbr, cbro + a, lane)]; };
    for (int e = slot; e < npan; e += SLOTS) P[(size_t)e * G + l] = (T)0;
    __syncthreads();
    // the arrowhead: pivot rows and pivot columns, all in the panel
    {
      const int e0 = L.ah_ptr[s], e1 = L.ah_ptr[s + 1];
      for (int e = e0 + slot; e < e1; e += SLOTS) {
        const int loc = L.ah_loc[e];
        PE(loc / RS, loc % RS) = A[at32(g, L.nA, e, lane)];
      }
      if (with_rhs)
        for (int p = slot; p < w; p += SLOTS) PE(p, f) = x[at32(g, L.n, rows[p], lane)];
    }
    __syncthreads();
    // The children's entries that fall in the panel, one child after the other
    // (siblings may add into the same entries; within a child the relative map is
    // injective).  A child's rows map in increasing order, so those landing in pivot
    // rows are its first aw rows, and its first aw columns land in pivot columns: the
    // panel takes rows a < aw (all columns) and, of the other rows, columns b < aw.  The
    // rest goes to the trailing block, slab by slab, after the panel's LU.
    for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
      const ChildRef cr = L.child_ref[ci];
      const int mc = cr.m;
      const int* rel = L.relmap + cr.rel_ptr;
      const int aw = first_at_least(rel, mc, w);
      const T* src = cb + at32(g, L.sumcb, cr.cb_off, lane);
      // entries (a_first + i, j), i rowlen + j < n, eight per thread at a time (their
      // loads before their stores); (i, j) advance by SLOTS without divisions
      auto add_panel = [&](int n, int a_first, int rowlen) {
        if (n <= 0) return;
        const int si = SLOTS / rowlen, sj = SLOTS % rowlen;
        int i = slot / rowlen, j = slot % rowlen;
        for (int e0 = slot; e0 < n; e0 += 8 * SLOTS) {
          int r[8], c[8];
          T v[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) {
            const bool ok = e0 + u * SLOTS < n;
            const int a = a_first + (ok ? i : 0), b = ok ? j : 0;
            r[u] = rel[a];
            c[u] = rel[b];
            v[u] = ok ? src[((size_t)a * mc + b) * 32] : (T)0;
            next_task(i, j, si, sj, rowlen);
          }
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (e0 + u * SLOTS < n) PE(r[u], c[u]) += v[u];
        }
      };
      add_panel(aw * mc, 0, mc);              // rows landing in pivot rows
      add_panel((mc - aw) * aw, aw, aw);      // the other rows' pivot columns
      if (with_rhs)
        for (int a = slot; a < aw; a += SLOTS) PE(rel[a], f) += cbr[at32(g, L.sumcbr, cr.cbr_off + a, lane)];
      __syncthreads();
    }
    // LU of the panel, one pivot per barrier: rows p < i < w over columns p < j < ncols
    // (top part) and rows i >= w over columns p < j < w (left part), each entry with
    // the unscaled l_ip = F(i,p) / F(p,p) of its row; column p is scaled one pivot later
    // (and after the loop for the last pivot), when no thread reads it any more
    T inv_prev = (T)1;
    for (int p = 0; p < w; ++p) {
      T pk = PE(p, p);
      if (bad_pivot(pk)) {
        if (slot == 0) mark_singular(&status[g * 32 + lane]);
        pk = (T)1;
      }
      const T inv = (T)1 / pk;
      if (p > 0)
        for (int i = p + slot; i < f; i += SLOTS) PE(i, p - 1) *= inv_prev;
      // four entries per thread at a time, loads before stores: the updated entries
      // (i > p, j > p) are distinct and none of them is in row p or column p, which the
      // updates read
      // rows of the part start at `base` (shared-memory index of column 0 of its first
      // row, row stride rstride entries); entry e = i rowlen + j' of the part is row i,
      // column p + 1 + j'; (i, j') advance by SLOTS without divisions
      auto update = [&](int n, int base, int rstride, int rowlen) {
        if (n <= 0) return;
        const int si = SLOTS / rowlen, sj = SLOTS % rowlen;
        int i = slot / rowlen, j = slot % rowlen;
        const T* prow = P + ((size_t)p * (f + 1) + p + 1) * G + l;  // u_pj, j > p
        for (int e0 = slot; e0 < n; e0 += 4 * SLOTS) {
          int at[4], jc[4];
          T lp[4], up[4], bv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const bool ok = e0 + u * SLOTS < n;
            const int row = base + (ok ? i : 0) * rstride;
            at[u] = row + p + 1 + (ok ? j : 0);
            jc[u] = ok ? j : 0;
            lp[u] = P[(size_t)(row + p) * G + l];
            up[u] = prow[(size_t)jc[u] * G];
            bv[u] = P[(size_t)at[u] * G + l];
            next_task(i, j, si, sj, rowlen);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (e0 + u * SLOTS < n) P[(size_t)at[u] * G + l] = bv[u] - (lp[u] * inv) * up[u];
        }
      };
      // top part: rows p+1 .. w-1, columns p+1 .. ncols-1
      update((w - 1 - p) * (ncols - 1 - p), (p + 1) * (f + 1), f + 1, ncols - 1 - p);
      // left part: rows w .. f-1, columns p+1 .. w-1
      update(m * (w - 1 - p), w * (f + 1), w, w - 1 - p);
      inv_prev = inv;
      __syncthreads();
    }
    if (w > 0) {
      for (int i = w + slot; i < f; i += SLOTS) PE(i, w - 1) *= inv_prev;
      __syncthreads();
    }
    // The trailing block (and the carried right-hand side as its column m), S rows at a
    // time in shared memory after the panel: zeroed, given the children's entries that
    // fall in those rows (a child's rows map in increasing order, so they are one range
    // of its rows), updated by the Schur complement x - l_ip u_pj in pivot order (4 x 4
    // register tiles: four l and four u values per pivot feed sixteen multiply-adds),
    // then written to the supernode's contribution block.  Every child entry is read
    // once and every trailing entry written once.
    if (has_parent && m > 0) {
      T* Sb = P + (size_t)pcap * G + l;  // slab entry (row, col) at Sb[(row * mcols + col) * G]
      const int mcols = m + 1;
      const int bc = with_rhs ? m + 1 : m;  // columns updated and written
      for (int a0 = 0; a0 < m; a0 += S) {
        const int sr = min(S, m - a0);
        for (int e = slot; e < sr * mcols; e += SLOTS) Sb[(size_t)e * G] = (T)0;
        __syncthreads();
        for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
          const ChildRef cr = L.child_ref[ci];
          const int mc = cr.m;
          const int* rel = L.relmap + cr.rel_ptr;
          const int aw = first_at_least(rel, mc, w);
          const int lo = first_at_least(rel, mc, w + a0), hi = first_at_least(rel, mc, w + a0 + sr);
          const int rowlen = mc - aw, n = (hi - lo) * rowlen;
          const T* src = cb + at32(g, L.sumcb, cr.cb_off, lane);
          if (n > 0) {
            const int si = SLOTS / rowlen, sj = SLOTS % rowlen;
            int i = slot / rowlen, j = slot % rowlen;
            for (int e0 = slot; e0 < n; e0 += 8 * SLOTS) {
              int at[8];
              T v[8], t[8];
#pragma unroll
              for (int u = 0; u < 8; ++u) {
                const bool ok = e0 + u * SLOTS < n;
                const int a = lo + (ok ? i : 0), b = aw + (ok ? j : 0);
                at[u] = (rel[a] - w - a0) * mcols + (rel[b] - w);
                v[u] = ok ? src[((size_t)a * mc + b) * 32] : (T)0;
                t[u] = Sb[(size_t)at[u] * G];
                next_task(i, j, si, sj, rowlen);
              }
#pragma unroll
              for (int u = 0; u < 8; ++u)
                if (e0 + u * SLOTS < n) Sb[(size_t)at[u] * G] = t[u] + v[u];
            }
          }
          if (with_rhs)
            for (int a = lo + slot; a < hi; a += SLOTS)
              Sb[((size_t)(rel[a] - w - a0) * mcols + m) * G] += cbr[at32(g, L.sumcbr, cr.cbr_off + a, lane)];
          __syncthreads();
        }
        const int nta = (sr + 3) / 4, ntb = (bc + 3) / 4;
        for (int tt = slot; tt < nta * ntb; tt += SLOTS) {
          const int ra = (tt / ntb) * 4, b0 = (tt % ntb) * 4;
          T acc[4][4];
#pragma unroll
          for (int ii = 0; ii < 4; ++ii)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
              acc[ii][jj] = (ra + ii < sr && b0 + jj < bc) ? Sb[((size_t)(ra + ii) * mcols + b0 + jj) * G] : (T)0;
          // l of trailing rows a0 + ra + ii (left part, stride w); u of columns w + b0 + jj
          // (top part; column w + m is the right-hand side f)
          const T* lb = P + ((size_t)w * (f + 1) + (size_t)(a0 + ra) * w) * G + l;
          const T* ub = P + (size_t)(w + b0) * G + l;
          for (int p = 0; p < w; ++p) {
            T lv[4], uv[4];
#pragma unroll
            for (int ii = 0; ii < 4; ++ii) lv[ii] = ra + ii < sr ? lb[((size_t)ii * w + p) * G] : (T)0;
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) uv[jj] = b0 + jj < bc ? ub[((size_t)p * (f + 1) + jj) * G] : (T)0;
#pragma unroll
            for (int ii = 0; ii < 4; ++ii)
#pragma unroll
              for (int jj = 0; jj < 4; ++jj) acc[ii][jj] = acc[ii][jj] - lv[ii] * uv[jj];
          }
#pragma unroll
          for (int ii = 0; ii < 4; ++ii)
#pragma unroll
            for (int jj = 0; jj < 4; ++jj)
              if (ra + ii < sr && b0 + jj < bc) Sb[((size_t)(ra + ii) * mcols + b0 + jj) * G] = acc[ii][jj];
        }
        __syncthreads();
        {
          const int si = SLOTS / m, sj = SLOTS % m;
          int i = slot / m, j = slot % m;
          for (int e = slot; e < sr * m; e += SLOTS) {
            CE(a0 + i, j) = Sb[((size_t)i * mcols + j) * G];
            next_task(i, j, si, sj, m);
          }
          if (with_rhs)
            for (int a = slot; a < sr; a += SLOTS) CR(a0 + a) = Sb[((size_t)a * mcols + m) * G];
        }
        __syncthreads();
      }
    }
    // U panel (rows 0 .. w-1, all f columns), L panel (rows w .. f-1, columns 0 .. w-1)
    T* pb = pan + at32(g, L.nnz, L.pan_off[s], lane);
    for (int e = slot; e < w * f; e += SLOTS) pb[(size_t)e * 32] = PE(e / f, e % f);
    for (int e = slot; e < m * w; e += SLOTS) pb[((size_t)w * f + e) * 32] = PE(w + e / w, e % w);
    if (with_rhs)
      for (int p = slot; p < w; p += SLOTS) x[at32(g, L.n, rows[p], lane)] = PE(p, f);
    __syncthreads();
  }
}

// The same factorisation with the trailing block kept in global memory (the
// supernode's contribution block, zeroed, the children's entries added into it, the
// Schur complement applied there after the panel's LU): only the panel takes shared
// memory, so more lanes fit per task; a tuning candidate beside k_mf_factor_big, whose
// slabs get short when the panel leaves little shared memory (FP64).  Same operations
// in the same order, so the same factors bit for bit.
template <typename T, int G>
__global__ void __launch_bounds__(512, 1) k_mf_factor_big_gt(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                       int ngroups, const T* __restrict__ A,
                                                       T* __restrict__ pan, T* __restrict__ cb,
                                                       T* __restrict__ cbr, T* __restrict__ x,
                                                       int* __restrict__ status,
                                                       const int* __restrict__ group_active, int with_rhs) {
  constexpr int SLOTS = 512 / G, LPG = 32 / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* P = reinterpret_cast<T*>(smem_raw);
  const int slot = threadIdx.x / G, l = threadIdx.x % G;
  const int nch = ngroups * LPG;
  for (int q = blockIdx.x / nch, ch = blockIdx.x % nch; q < nsn_l;
       next_task(q, ch, (int)gridDim.x / nch, (int)gridDim.x % nch, nch)) {
    const int s = task_sn[q];
    const int g = ch / LPG;
    if (!group_active[g] || !task_here(L, s, g)) continue;  // uniform over the block
    const int lane = (ch % LPG) * G + l;
    const int w = L.sn_w[s], f = L.sn_f[s], m = f - w;
    const int* rows = L.sn_rows + L.sn_rptr[s];
    const int RS = front_stride(f);
    const int ncols = with_rhs ? f + 1 : f;
    const bool has_parent = L.sn_parent[s] >= 0;
    const long long cbo = L.cb_off[s], cbro = L.cbr_off[s];
    const int npan = w * (f + 1) + m * w;
    // panel entry (r, c), r < w or c < w: top part row-major, then the left part
    auto PE = [&](int r, int c) -> T& {
      return r < w ? P[((size_t)r * (f + 1) + c) * G + l] : P[((size_t)w * (f + 1) + (size_t)(r - w) * w + c) * G + l];
    };
    // trailing entry (a, b) of the contribution block, and the carried right-hand side
    auto CE = [&](int a, int b) -> T& { return cb[at32(g, L.sumcb, cbo + (long long)a * m + b, lane)]; };
    auto CR = [&](int a) -> T& { return cbr[at32(g, L.sumcbr, cbro + a, lane)]; };
    const bool trail = has_parent && m > 0;
    for (int e = slot; e < npan; e += SLOTS) P[(size_t)e * G + l] = (T)0;
    if (trail) {
      for (int e = slot; e < m * m; e += SLOTS) CE(e / m, e % m) = (T)0;
      if (with_rhs)
        for (int a = slot; a < m; a += SLOTS) CR(a) = (T)0;
    }
    __syncthreads();
    // the arrowhead: pivot rows and pivot columns, all in the panel
    {
      const int e0 = L.ah_ptr[s], e1 = L.ah_ptr[s + 1];
      for (int e = e0 + slot; e < e1; e += SLOTS) {
        const int loc = L.ah_loc[e];
        PE(loc / RS, loc % RS) = A[at32(g, L.nA, e, lane)];
      }
      if (with_rhs)
        for (int p = slot; p < w; p += SLOTS) PE(p, f) = x[at32(g, L.n, rows[p], lane)];
    }
    __syncthreads();
    // the children's contribution blocks, one child after the other (siblings may add
    // into the same entries; within a child the relative map is injective)
    for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
      const ChildRef cr = L.child_ref[ci];
      const int mc = cr.m;
      const int* rel = L.relmap + cr.rel_ptr;
      // eight entries per thread at a time: all their loads (the child's values and the
      // trailing entries they add to, distinct within a child) before any store
      constexpr int B = 8;
      // entry e = a mc + b of the child's block; (a, b) advance by SLOTS without divisions
      const int sa = SLOTS / mc, sb = SLOTS % mc;
      int a = slot / mc, b = slot % mc;
      const T* src = cb + at32(g, L.sumcb, cr.cb_off, lane);
      for (int e0 = slot; e0 < mc * mc; e0 += B * SLOTS) {
        int r[B], c[B];
        T v[B], t[B];
#pragma unroll
        for (int u = 0; u < B; ++u) {
          const int e = e0 + u * SLOTS;
          r[u] = e < mc * mc ? rel[a] : 0;
          c[u] = e < mc * mc ? rel[b] : 0;
          v[u] = e < mc * mc ? src[(size_t)e * 32] : (T)0;
          next_task(a, b, sa, sb, mc);
        }
#pragma unroll
        for (int u = 0; u < B; ++u)
          t[u] = (e0 + u * SLOTS < mc * mc && r[u] >= w && c[u] >= w && trail) ? CE(r[u] - w, c[u] - w) : (T)0;
#pragma unroll
        for (int u = 0; u < B; ++u) {
          if (e0 + u * SLOTS >= mc * mc) break;
          if (r[u] < w || c[u] < w) PE(r[u], c[u]) += v[u];
          else if (trail) CE(r[u] - w, c[u] - w) = t[u] + v[u];
        }
      }
      if (with_rhs)
        for (int a = slot; a < mc; a += SLOTS) {
          const int r = rel[a];
          const T v = cbr[at32(g, L.sumcbr, cr.cbr_off + a, lane)];
          if (r < w) PE(r, f) += v;
          else if (trail) CR(r - w) += v;
        }
      __syncthreads();
    }
    // LU of the panel, one pivot per barrier: rows p < i < w over columns p < j < ncols
    // (top part) and rows i >= w over columns p < j < w (left part), each entry with
    // the unscaled l_ip = F(i,p) / F(p,p) of its row; column p is scaled one pivot later
    // (and after the loop for the last pivot), when no thread reads it any more
    T inv_prev = (T)1;
    for (int p = 0; p < w; ++p) {
      T pk = PE(p, p);
      if (bad_pivot(pk)) {
        if (slot == 0) mark_singular(&status[g * 32 + lane]);
        pk = (T)1;
      }
      const T inv = (T)1 / pk;
      if (p > 0)
        for (int i = p + slot; i < f; i += SLOTS) PE(i, p - 1) *= inv_prev;
      // four entries per thread at a time, loads before stores: the updated entries
      // (i > p, j > p) are distinct and none of them is in row p or column p, which the
      // updates read
      // rows of the part start at `base` (shared-memory index of column 0 of its first
      // row, row stride rstride entries); entry e = i rowlen + j' of the part is row i,
      // column p + 1 + j'; (i, j') advance by SLOTS without divisions
      auto update = [&](int n, int base, int rstride, int rowlen) {
        if (n <= 0) return;
        const int si = SLOTS / rowlen, sj = SLOTS % rowlen;
        int i = slot / rowlen, j = slot % rowlen;
        const T* prow = P + ((size_t)p * (f + 1) + p + 1) * G + l;  // u_pj, j > p
        for (int e0 = slot; e0 < n; e0 += 4 * SLOTS) {
          int at[4], jc[4];
          T lp[4], up[4], bv[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const bool ok = e0 + u * SLOTS < n;
            const int row = base + (ok ? i : 0) * rstride;
            at[u] = row + p + 1 + (ok ? j : 0);
            jc[u] = ok ? j : 0;
            lp[u] = P[(size_t)(row + p) * G + l];
            up[u] = prow[(size_t)jc[u] * G];
            bv[u] = P[(size_t)at[u] * G + l];
            next_task(i, j, si, sj, rowlen);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (e0 + u * SLOTS < n) P[(size_t)at[u] * G + l] = bv[u] - (lp[u] * inv) * up[u];
        }
      };
      // top part: rows p+1 .. w-1, columns p+1 .. ncols-1
      update((w - 1 - p) * (ncols - 1 - p), (p + 1) * (f + 1), f + 1, ncols - 1 - p);
      // left part: rows w .. f-1, columns p+1 .. w-1
      update(m * (w - 1 - p), w * (f + 1), w, w - 1 - p);
      inv_prev = inv;
      __syncthreads();
    }
    if (w > 0) {
      for (int i = w + slot; i < f; i += SLOTS) PE(i, w - 1) *= inv_prev;
      __syncthreads();
    }
    // the Schur complement on the trailing block (and the carried right-hand side):
    // x - l_ip u_pj in pivot order
    if (trail) {
      // 4 x 4 tiles of the trailing block per thread: per pivot, four l and four u
      // values from shared memory feed sixteen multiply-adds
      const int nt = (m + 3) / 4;
      for (int t = slot; t < nt * nt; t += SLOTS) {
        const int a0 = (t / nt) * 4, b0 = (t % nt) * 4;
        T acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = (a0 + i < m && b0 + j < m) ? CE(a0 + i, b0 + j) : (T)0;
        // l of rows w + a0 + i (left part, stride w) and u of columns w + b0 + j (top part)
        const T* lb = P + ((size_t)w * (f + 1) + (size_t)a0 * w) * G + l;
        const T* ub = P + (size_t)(w + b0) * G + l;
        for (int p = 0; p < w; ++p) {
          T lv[4], uv[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) lv[i] = a0 + i < m ? lb[((size_t)i * w + p) * G] : (T)0;
#pragma unroll
          for (int j = 0; j < 4; ++j) uv[j] = b0 + j < m ? ub[((size_t)p * (f + 1) + j) * G] : (T)0;
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = acc[i][j] - lv[i] * uv[j];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            if (a0 + i < m && b0 + j < m) CE(a0 + i, b0 + j) = acc[i][j];
      }
      if (with_rhs)
        for (int a = slot; a < m; a += SLOTS) {
          T c = CR(a);
          for (int p = 0; p < w; ++p) c = c - PE(w + a, p) * PE(p, f);
          CR(a) = c;
        }
    }
    // U panel (rows 0 .. w-1, all f columns), L panel (rows w .. f-1, columns 0 .. w-1)
    T* pb = pan + at32(g, L.nnz, L.pan_off[s], lane);
    for (int e = slot; e < w * f; e += SLOTS) pb[(size_t)e * 32] = PE(e / f, e % f);
    for (int e = slot; e < m * w; e += SLOTS) pb[((size_t)w * f + e) * 32] = PE(w + e / w, e % w);
    if (with_rhs)
      for (int p = slot; p < w; p += SLOTS) x[at32(g, L.n, rows[p], lane)] = PE(p, f);
    __syncthreads();
  }
}

// Forward substitution with stored factors (fast-decoupled solves): thread per
// case, warp per (supernode, group).  b accumulates in shared memory.
template <typename T>
__global__ void __launch_bounds__(128) k_mf_fsolve(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                   int ngroups, int fcap, const T* __restrict__ pan,
                                                   T* __restrict__ cbr, T* __restrict__ x,
                                                   const int* __restrict__ group_active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  T* b = reinterpret_cast<T*>(smem_raw) + (size_t)warp * fcap * 32;
  const long long ntasks = (long long)nsn_l * ngroups;
  for (long long t = (long long)blockIdx.x * warps + warp; t < ntasks; t += (long long)gridDim.x * warps) {
    const int s = task_sn[t / ngroups];
    const int g = (int)(t % ngroups);
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    for (int i = 0; i < f; ++i) b[i * 32 + lane] = (T)0;
    for (int p = 0; p < w; ++p) b[p * 32 + lane] = x[at32(g, L.n, rows[p], lane)];
    for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
      const int ch = L.child_list[ci];
      const int m = L.sn_f[ch] - L.sn_w[ch];
      const int* rel = L.relmap + L.rel_ptr[ch];
      for (int a = 0; a < m; ++a) b[rel[a] * 32 + lane] += cbr[at32(g, L.sumcbr, L.cbr_off[ch] + a, lane)];
    }
    const long long po = L.pan_off[s];
    for (int p = 0; p < w; ++p) {
      const T yp = b[p * 32 + lane];
      for (int i = p + 1; i < w; ++i) b[i * 32 + lane] -= pan[at32(g, L.nnz, po + (long long)i * f + p, lane)] * yp;
      for (int i = w; i < f; ++i)
        b[i * 32 + lane] -= pan[at32(g, L.nnz, po + (long long)w * f + (long long)(i - w) * w + p, lane)] * yp;
    }
    for (int p = 0; p < w; ++p) x[at32(g, L.n, rows[p], lane)] = b[p * 32 + lane];
    if (L.sn_parent[s] >= 0)
      for (int a = 0; a < f - w; ++a) cbr[at32(g, L.sumcbr, L.cbr_off[s] + a, lane)] = b[(w + a) * 32 + lane];
    __syncwarp();
  }
}

// Backward substitution: thread per case, warp per (supernode, group).  The
// supernode's front values of x (ancestors' solutions, final after the previous
// launches, and its own forward-substituted y) are staged in shared memory first,
// so the dependent chain over the w pivots runs on shared memory while the
// U-panel rows stream from global memory.
template <typename T>
__global__ void __launch_bounds__(128) k_mf_bsolve(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                   int ngroups, int fcap, const T* __restrict__ pan,
                                                   T* __restrict__ x, const int* __restrict__ group_active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  T* xs = reinterpret_cast<T*>(smem_raw) + (size_t)warp * fcap * 32;
  const long long ntasks = (long long)nsn_l * ngroups;
  for (long long t = (long long)blockIdx.x * warps + warp; t < ntasks; t += (long long)gridDim.x * warps) {
    const int s = task_sn[t / ngroups];
    const int g = (int)(t % ngroups);
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    const long long po = L.pan_off[s];
    // the supernode's U panel (w x f entries of the group) is read pivot row by pivot
    // row, each row after the last one's solve: one bulk L2 prefetch requests it all
    if (lane == 0) prefetch_l2(pan + at32(g, L.nnz, po, 0), (unsigned)(w * f) * (32 * sizeof(T)));
    for (int q = 0; q < f; ++q) xs[q * 32 + lane] = x[at32(g, L.n, rows[q], lane)];
    for (int p = w - 1; p >= 0; --p) {
      const T* urow = pan + at32(g, L.nnz, po + (long long)p * f, lane);
      T acc = xs[p * 32 + lane];
      T acc2 = (T)0;
      int q = p + 1;
      for (; q + 1 < f; q += 2) {
        acc -= urow[(size_t)q * 32] * xs[q * 32 + lane];
        acc2 -= urow[(size_t)(q + 1) * 32] * xs[(q + 1) * 32 + lane];
      }
      if (q < f) acc -= urow[(size_t)q * 32] * xs[q * 32 + lane];
      xs[p * 32 + lane] = (acc + acc2) / urow[(size_t)p * 32];
    }
    for (int p = 0; p < w; ++p) x[at32(g, L.n, rows[p], lane)] = xs[p * 32 + lane];
    __syncwarp();
  }
}

// Backward substitution for large fronts: warp per (supernode, chunk of G lanes);
// SLOTS = 32 / G threads per lane split each pivot row's dot product and fold it
// with shuffles, so a big supernode's chain of w pivots runs on 8x (FP64) or 4x
// (FP32) more warps than the thread-per-case kernel.
template <typename T, int G>
__global__ void __launch_bounds__(128) k_mf_bsolve_chunk(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                         int ngroups, int fcap, const T* __restrict__ pan,
                                                         T* __restrict__ x, const int* __restrict__ group_active) {
  constexpr int SLOTS = 32 / G, LPG = 32 / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const int slot = tid / G, l = tid % G;
  T* xs = reinterpret_cast<T*>(smem_raw) + (size_t)warp * fcap * G;
  const long long nchunks = (long long)ngroups * LPG;
  const long long ntasks = (long long)nsn_l * nchunks;
  for (long long t = (long long)blockIdx.x * warps + warp; t < ntasks; t += (long long)gridDim.x * warps) {
    const int s = task_sn[t / nchunks];
    const int ch = (int)(t % nchunks);
    const int g = ch / LPG;
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int lane = (ch % LPG) * G + l;
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    const long long po = L.pan_off[s];
    // the U panel of the group, requested from DRAM at once (the chunks of a group share it)
    if (tid == 0) prefetch_l2(pan + at32(g, L.nnz, po, 0), (unsigned)(w * f) * (32 * sizeof(T)));
    for (int q = slot; q < f; q += SLOTS) xs[q * G + l] = x[at32(g, L.n, rows[q], lane)];
    __syncwarp();
    for (int p = w - 1; p >= 0; --p) {
      const T* urow = pan + at32(g, L.nnz, po + (long long)p * f, lane);
      T part = (T)0;
      for (int q = p + 1 + slot; q < f; q += SLOTS) part += urow[(size_t)q * 32] * xs[q * G + l];
#pragma unroll
      for (int o = 16; o >= G; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
      if (slot == 0) xs[p * G + l] = (xs[p * G + l] - part) / urow[(size_t)p * 32];
      __syncwarp();
    }
    for (int p = slot; p < w; p += SLOTS) x[at32(g, L.n, rows[p], lane)] = xs[p * G + l];
    __syncwarp();
  }
}

// Backward substitution of the levels nearest the root in one launch.  A block per
// chunk of G lanes walks those levels from the root down; the block's warps take the
// supernodes of a level (as k_mf_bsolve_chunk: 32 / G slots per lane split each pivot
// row's dot product, folded with shuffles), and a block barrier separates the levels,
// so every parent is solved before its children read its x.  Lanes are independent:
// blocks never wait on each other, and one launch replaces the launches of those
// levels (each of which had too few supernodes to fill the GPU) and the gaps between
// them.  32 warps per block: a level's supernodes (at most 24) take one round.
// top_sn: the supernodes of those levels in descending level order, lev_ptr[l]
// .. lev_ptr[l + 1] the ones of the l-th level from the top; fcap: their largest front.
template <typename T, int G>
__global__ void __launch_bounds__(1024) k_mf_bsolve_top(DevLU L, const int* __restrict__ top_sn,
                                                       const int* __restrict__ lev_ptr, int nlev, int ngroups, int fcap,
                                                       const T* __restrict__ pan, T* __restrict__ x,
                                                       const int* __restrict__ group_active) {
  constexpr int SLOTS = 32 / G, LPG = 32 / G;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  const int slot = tid / G, l = tid % G;
  T* xs = reinterpret_cast<T*>(smem_raw) + (size_t)warp * fcap * G;
  const int ch = blockIdx.x;
  const int g = ch / LPG;
  if (g >= ngroups || !group_active[g]) return;  // uniform over the block, before any barrier
  const int lane = (ch % LPG) * G + l;
  for (int lv = 0; lv < nlev; ++lv) {
    for (int k = lev_ptr[lv] + warp; k < lev_ptr[lv + 1]; k += warps) {
      const int s = top_sn[k];
      if (!task_here(L, s, g)) continue;
      const int w = L.sn_w[s], f = L.sn_f[s];
      const int* rows = L.sn_rows + L.sn_rptr[s];
      const long long po = L.pan_off[s];
      if (tid == 0) prefetch_l2(pan + at32(g, L.nnz, po, 0), (unsigned)(w * f) * (32 * sizeof(T)));
      for (int q = slot; q < f; q += SLOTS) xs[q * G + l] = x[at32(g, L.n, rows[q], lane)];
      __syncwarp();
      for (int p = w - 1; p >= 0; --p) {
        const T* urow = pan + at32(g, L.nnz, po + (long long)p * f, lane);
        T part = (T)0;
        for (int q = p + 1 + slot; q < f; q += SLOTS) part += urow[(size_t)q * 32] * xs[q * G + l];
#pragma unroll
        for (int o = 16; o >= G; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (slot == 0) xs[p * G + l] = (xs[p * G + l] - part) / urow[(size_t)p * 32];
        __syncwarp();
      }
      for (int p = slot; p < w; p += SLOTS) x[at32(g, L.n, rows[p], lane)] = xs[p * G + l];
      __syncwarp();
    }
    __syncthreads();
  }
}

// Backward substitution with the U panel staged in shared memory: one warp per
// (supernode, chunk of G lanes) copies the supernode's whole U panel (w x f entries
// of its G lanes) and the front's x values into shared memory with asynchronous
// copies that are all in flight together, then solves row-oriented: SLOTS = 32 / G
// threads per lane, pivot row r owned by slot r % SLOTS.
//   1. every pivot row subtracts the columns q >= w (x already known) at once;
//   2. pivots p = w-1 .. 0: the owner divides row p by U(p,p), and after a warp
//      barrier every owner subtracts U(r,p) x_p from its rows r < p.
// Per pivot the dependent chain is one division, one barrier and one multiply-add,
// instead of a dot product.  Shared memory: (wfmax + fcap) * G values (wfmax =
// largest w * f of the level).
template <typename T, int G>
__global__ void __launch_bounds__(32) k_mf_bsolve_staged(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                         int ngroups, int wfmax, const T* __restrict__ pan,
                                                         T* __restrict__ x, const int* __restrict__ group_active) {
  constexpr int SLOTS = 32 / G, LPG = 32 / G;
  constexpr int V = (int)(16 / sizeof(T)) < G ? (int)(16 / sizeof(T)) : G;  // lanes per copy
  constexpr int NV = G / V;                                                  // copies per entry
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int tid = threadIdx.x & 31;
  const int slot = tid / G, l = tid % G;
  T* us = reinterpret_cast<T*>(smem_raw);  // [w * f][G]
  T* xs = us + (size_t)wfmax * G;          // [f][G]
  const long long nchunks = (long long)ngroups * LPG;
  const long long ntasks = (long long)nsn_l * nchunks;
  for (long long t = blockIdx.x; t < ntasks; t += gridDim.x) {
    const int s = task_sn[t / nchunks];
    const int ch = (int)(t % nchunks);
    const int g = ch / LPG;
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int lane0 = (ch % LPG) * G;
    const int lane = lane0 + l;
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    const T* src = pan + at32(g, L.nnz, L.pan_off[s], lane0);
    const int ncopy = w * f * NV;
    for (int k = tid; k < ncopy; k += 32) {
      const int e = k / NV, part = (k % NV) * V;
      const unsigned sa = (unsigned)__cvta_generic_to_shared(us + (size_t)e * G + part);
      const T* ga = src + (size_t)e * 32 + part;
      if constexpr (V * sizeof(T) == 16)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(ga) : "memory");
      else if constexpr (V * sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(ga) : "memory");
      else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(ga) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    for (int q = slot; q < f; q += SLOTS) xs[q * G + l] = x[at32(g, L.n, rows[q], lane)];
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    // 1. the known columns: two rows at a time for independent chains
    int r = slot;
    for (; r + SLOTS < w; r += 2 * SLOTS) {
      const T* u0 = us + (size_t)r * f * G + l;
      const T* u1 = u0 + (size_t)SLOTS * f * G;
      T a0 = xs[r * G + l], a1 = xs[(r + SLOTS) * G + l];
      for (int q = w; q < f; ++q) {
        const T xq = xs[q * G + l];
        a0 -= u0[q * G] * xq;
        a1 -= u1[q * G] * xq;
      }
      xs[r * G + l] = a0;
      xs[(r + SLOTS) * G + l] = a1;
    }
    if (r < w) {
      const T* u0 = us + (size_t)r * f * G + l;
      T a0 = xs[r * G + l];
      for (int q = w; q < f; ++q) a0 -= u0[q * G] * xs[q * G + l];
      xs[r * G + l] = a0;
    }
    // 2. the triangle, pivot by pivot (each row is only touched by its owner)
    for (int p = w - 1; p >= 0; --p) {
      if (p % SLOTS == slot) xs[p * G + l] /= us[((size_t)p * f + p) * G + l];
      __syncwarp();
      const T xp = xs[p * G + l];
      for (int rr = slot; rr < p; rr += SLOTS) xs[rr * G + l] -= us[((size_t)rr * f + p) * G + l] * xp;
    }
    __syncwarp();
    for (int p = slot; p < w; p += SLOTS) x[at32(g, L.n, rows[p], lane)] = xs[p * G + l];
    __syncwarp();
  }
}

// ---------------------------------------------------------------- mismatch of given voltages
// max |F| per case for voltages given case-major (v[c][i], the layout results use),
// F = [Re mis_pv; Re mis_pq; Im mis_pq] as newtonpf.h:18-71 (hybrid_checkConvergence,
// newtonpf.h:526-568, plus the host max loop of newtonpf.h:1241-1254).
// Grid (row blocks of 256, cases); a warp covers 32 mismatch rows of one case and
// folds them with shuffles, then one atomicMax per warp into acc[c].
__global__ void __launch_bounds__(256) k_mismatch_eval(DevGrid d, const double2* __restrict__ v, int ncases,
                                                       unsigned long long* __restrict__ acc) {
  // cases stride over gridDim.y (at most 65535), so any batch size launches
  for (int c = blockIdx.y; c < ncases; c += gridDim.y) {  // the user's case; its lane is ln
    const int ln = lane_of_case(d, c);
    LaneOut o;
    load_outages(d, ln, o);
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    double m = 0.0;
    if (r < d.nfree && row_here(d, d.mis_rows[r], ln >> 5)) {
      const double2* vc = v + (size_t)c * d.nb;
      const int i = d.mis_rows[r];
      double2 ib = make_double2(0.0, 0.0);
      const bool touched = row_touched(o, d.y_diag[i]);
      for (int p = d.y_rowptr[i]; p < d.y_rowptr[i + 1]; ++p) {
        const double2 y = yentry(d, o, touched, p, ln >> 5, ln & 31);
        const double2 vj = vc[d.y_col[p]];
        ib.x += y.x * vj.x - y.y * vj.y;
        ib.y += y.x * vj.y + y.y * vj.x;
      }
      const double2 vi = vc[i];
      double2 s = d.sbus_case ? d.sbus_case[at32(ln >> 5, d.nb, i, ln & 31)] : d.sbus0[i];
      const bool pvi = still_pv(d, i, ln >> 5, ln & 31);
      if (d.sw_index && !pvi && d.sw_index[i] >= 0) s.y = d.q_fix[at32(ln >> 5, d.nsw, d.sw_index[i], ln & 31)];
      const double mr = vi.x * ib.x + vi.y * ib.y - s.x;
      const double mi = vi.y * ib.x - vi.x * ib.y - s.y;
      m = fabs(mr);
      if (mr != mr) m = INFINITY;
      if (d.jvar[i].y >= 0 && !pvi) {
        m = fmax(m, fabs(mi));
        if (mi != mi) m = INFINITY;
      }
      m = finite_or_inf(m);
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, k));
    if ((threadIdx.x & 31) == 0) atomicMax(&acc[c], (unsigned long long)__double_as_longlong(m));
  }
}

// acc (bits of non-negative doubles) -> out, and acc back to zero for the next call
__global__ void k_acc_drain(unsigned long long* __restrict__ acc, double* __restrict__ out, int n) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  out[c] = __longlong_as_double((long long)acc[c]);
  acc[c] = 0ull;
}

// ---------------------------------------------------------------- branch flows
// Per case and branch: Sf = Vf conj(Yff Vf + Yft Vt), St = Vt conj(Ytf Vf + Ytt Vt)
// (an outaged branch carries nothing).  Per case sums: active loss sum(Re Sf + Re St)
// as mkl_computeLoss / hybrid_computeLoss + reduceLoss (runpf.h:228-257, 543-604),
// and, with ratings, the overload loss sum(relu(|Sf| - 0.9 rating)^2).
// Grid (branch blocks of 256, groups); thread = (branch, lane).
__global__ void __launch_bounds__(256) k_branch_flow(DevGrid d, int nbr, int ncases, const double* __restrict__ rating,
                                                     double* __restrict__ ploss, double* __restrict__ overload,
                                                     double2* __restrict__ sf_out, double2* __restrict__ st_out) {
  const int g = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = g * 32 + lane;
  const int uc = case_of_lane(d, c, ncases);  // the user's case in this lane, -1 for padding
  LaneOut o;
  load_outages(d, c, o);
  double lsum = 0.0, osum = 0.0;
  const int k0 = blockIdx.x * 64;
  const int k1 = min(nbr, k0 + 64);
  for (int k = k0 + warp; k < k1; k += 8) {
    double2 sf = make_double2(0.0, 0.0), stt = make_double2(0.0, 0.0);
    const bool here = branch_here(d, k, g);
    if (here && !outaged(o, k)) {
      const int2 ft = d.br_ft[k];
      double2 y[4];
      branch_y(d, k, g, lane, y);
      const double2 vf = d.V[at32(g, d.nb, ft.x, lane)], vt = d.V[at32(g, d.nb, ft.y, lane)];
      const double2 i_f = make_double2(y[0].x * vf.x - y[0].y * vf.y + y[1].x * vt.x - y[1].y * vt.y,
                                       y[0].x * vf.y + y[0].y * vf.x + y[1].x * vt.y + y[1].y * vt.x);
      const double2 i_t = make_double2(y[2].x * vf.x - y[2].y * vf.y + y[3].x * vt.x - y[3].y * vt.y,
                                       y[2].x * vf.y + y[2].y * vf.x + y[3].x * vt.y + y[3].y * vt.x);
      sf = make_double2(vf.x * i_f.x + vf.y * i_f.y, vf.y * i_f.x - vf.x * i_f.y);
      stt = make_double2(vt.x * i_t.x + vt.y * i_t.y, vt.y * i_t.x - vt.x * i_t.y);
    }
    lsum += sf.x + stt.x;
    if (rating && here) {
      const double ex = sqrt(sf.x * sf.x + sf.y * sf.y) - 0.9 * rating[k];
      if (ex > 0.0) osum += ex * ex;
    }
    if (uc >= 0) {
      if (sf_out) sf_out[(size_t)uc * nbr + k] = sf;
      if (st_out) st_out[(size_t)uc * nbr + k] = stt;
    }
  }
  __shared__ double red[2][8][32];
  red[0][warp][lane] = lsum;
  red[1][warp][lane] = osum;
  __syncthreads();
  if (warp == 0 && uc >= 0) {
    double a = 0.0, b = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      a += red[0][w][lane];
      b += red[1][w][lane];
    }
    atomicAdd(&ploss[uc], a);
    if (overload) atomicAdd(&overload[uc], b);
  }
}

// ---------------------------------------------------------------- adjoint
// Gradient of the per-case overload loss L = sum_k relu(|Sf_k| - 0.9 r_k)^2 w.r.t.
// bus injections and branch series admittance g + jb, through J^T lambda = dL/dx
// (x = [Va of PV/PQ buses, Vm of PQ buses], the Newton variables).
//
// With Sf = |Vf|^2 conj(Yff) + W, W = Vf conj(Yft Vt), E = |Sf| - 0.9 r > 0 and
// c = 2E/|Sf|:  dL/dVa_f = -c Im(conj(Sf) W),  dL/dVa_t = +c Im(conj(Sf) W),
//               dL/dVm_f = c Re(conj(Sf) (2|Vf| conj(Yff) + W/|Vf|)),
//               dL/dVm_t = c Re(conj(Sf) W) / |Vt|.
// Thread per (branch, lane), scattered into g (the right-hand side of J^T) with atomics.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_dldx(DevGrid d, int nbr, const double* __restrict__ rating, T* __restrict__ g) {
  const int grp = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = grp * 32 + lane;
  if (d.status[c] != ST_CONVERGED) return;
  LaneOut o;
  load_outages(d, c, o);
  const int k1 = min(nbr, (int)(blockIdx.x + 1) * 64);
  for (int k = blockIdx.x * 64 + warp; k < k1; k += 8) {
    if (!branch_here(d, k, grp) || outaged(o, k)) continue;
    const int2 ft = d.br_ft[k];
    double2 y[4];
    branch_y(d, k, grp, lane, y);
    const double2 vf = d.V[at32(grp, d.nb, ft.x, lane)], vt = d.V[at32(grp, d.nb, ft.y, lane)];
    // W = Vf conj(Yft Vt)
    const double2 yv = make_double2(y[1].x * vt.x - y[1].y * vt.y, y[1].x * vt.y + y[1].y * vt.x);
    const double2 W = make_double2(vf.x * yv.x + vf.y * yv.y, vf.y * yv.x - vf.x * yv.y);
    const double mf2 = vf.x * vf.x + vf.y * vf.y;
    const double2 S = make_double2(mf2 * y[0].x + W.x, -mf2 * y[0].y + W.y);
    const double aS = sqrt(S.x * S.x + S.y * S.y);
    const double E = aS - 0.9 * rating[k];
    if (!(E > 0.0)) continue;
    const double cc = 2.0 * E / aS;
    // conj(S) W
    const double swr = S.x * W.x + S.y * W.y, swi = S.x * W.y - S.y * W.x;
    const double mf = sqrt(mf2), mt = sqrt(vt.x * vt.x + vt.y * vt.y);
    // conj(S) (2|Vf| conj(Yff) + W/|Vf|), real part
    const double dvm_f = cc * (2.0 * mf * (S.x * y[0].x - S.y * y[0].y) + swr / mf);
    const int2 vfv = d.jvar[ft.x], vtv = d.jvar[ft.y];
    if (vfv.x >= 0) atomicAdd(&g[at32(grp, d.n_jac, vfv.x, lane)], (T)(-cc * swi));
    if (vtv.x >= 0) atomicAdd(&g[at32(grp, d.n_jac, vtv.x, lane)], (T)(cc * swi));
    if (vfv.y >= 0 && !still_pv(d, ft.x, grp, lane)) atomicAdd(&g[at32(grp, d.n_jac, vfv.y, lane)], (T)dvm_f);
    if (vtv.y >= 0 && !still_pv(d, ft.y, grp, lane)) atomicAdd(&g[at32(grp, d.n_jac, vtv.y, lane)], (T)(cc * swr / mt));
  }
}

// Iterative refinement of the adjoint solved with FP32 factors: the residual
// r = b - J^T lam is formed in FP64 with the Jacobian refilled in FP64 at the same
// point, solved again with the FP32 factors and added to lam (FP64), so the FP32 LU
// only has to reduce the error by its own accuracy at each step.  Column c of J^T lam
// gathers the J entries of variable c: col_ptr / col_ent list, per column, the
// A-array position and the row (equation) of each entry.  Warp = column x 32 lanes.
template <typename T>
__global__ void __launch_bounds__(256) k_adj_residual(int n, int ngroups, int nA, const int* __restrict__ col_ptr,
                                                      const int2* __restrict__ col_ent, const double* __restrict__ A,
                                                      const double* __restrict__ lam, const double* __restrict__ b,
                                                      T* __restrict__ r) {
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * 8 + (threadIdx.x >> 5);
  const int g = blockIdx.y;
  if (col >= n || g >= ngroups) return;
  double s = b[at32(g, n, col, lane)];
  for (int q = col_ptr[col]; q < col_ptr[col + 1]; ++q) {
    const int2 e = col_ent[q];  // (A-array position, row)
    s -= A[at32(g, nA, e.x, lane)] * lam[at32(g, n, e.y, lane)];
  }
  r[at32(g, n, col, lane)] = (T)s;
}

// lam (FP64) = or += the FP32 correction x; n_total entries
template <typename T>
__global__ void k_adj_accumulate(size_t n_total, const T* __restrict__ x, double* __restrict__ lam, int add) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n_total; t += (size_t)gridDim.x * blockDim.x)
    lam[t] = (add ? lam[t] : 0.0) + (double)x[t];
}

// x (T) = b (FP64)
template <typename T>
__global__ void k_adj_cast(size_t n_total, const double* __restrict__ b, T* __restrict__ x) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n_total; t += (size_t)gridDim.x * blockDim.x)
    x[t] = (T)b[t];
}

// U^T z = g, supernodes bottom-up (thread per case, warp per (supernode, group)):
// pivots in order, each pushes U(p, i) z_p into the later rows of its front; the
// non-pivot rows travel to the parent as a carried vector (as k_mf_fsolve).
template <typename T>
__global__ void __launch_bounds__(128) k_mf_fsolve_t(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                     int ngroups, int fcap, const T* __restrict__ pan,
                                                     T* __restrict__ cbr, T* __restrict__ x,
                                                     const int* __restrict__ group_active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  T* b = reinterpret_cast<T*>(smem_raw) + (size_t)warp * fcap * 32;
  const long long ntasks = (long long)nsn_l * ngroups;
  for (long long t = (long long)blockIdx.x * warps + warp; t < ntasks; t += (long long)gridDim.x * warps) {
    const int s = task_sn[t / ngroups];
    const int g = (int)(t % ngroups);
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    for (int i = 0; i < f; ++i) b[i * 32 + lane] = (T)0;
    for (int p = 0; p < w; ++p) b[p * 32 + lane] = x[at32(g, L.n, rows[p], lane)];
    for (int ci = L.child_ptr[s]; ci < L.child_ptr[s + 1]; ++ci) {
      const int ch = L.child_list[ci];
      const int m = L.sn_f[ch] - L.sn_w[ch];
      const int* rel = L.relmap + L.rel_ptr[ch];
      for (int a = 0; a < m; ++a) b[rel[a] * 32 + lane] += cbr[at32(g, L.sumcbr, L.cbr_off[ch] + a, lane)];
    }
    const long long po = L.pan_off[s];
    for (int p = 0; p < w; ++p) {
      const T* urow = pan + at32(g, L.nnz, po + (long long)p * f, lane);
      const T zp = b[p * 32 + lane] / urow[(size_t)p * 32];
      b[p * 32 + lane] = zp;
      for (int i = p + 1; i < f; ++i) b[i * 32 + lane] -= urow[(size_t)i * 32] * zp;
    }
    for (int p = 0; p < w; ++p) x[at32(g, L.n, rows[p], lane)] = b[p * 32 + lane];
    if (L.sn_parent[s] >= 0)
      for (int a = 0; a < f - w; ++a) cbr[at32(g, L.sumcbr, L.cbr_off[s] + a, lane)] = b[(w + a) * 32 + lane];
    __syncwarp();
  }
}

// L^T lambda = z, supernodes top-down (thread per case): the ancestors' lambda are
// final; lambda_p = z_p - sum_{i > p} L(i, p) lambda_i (unit diagonal), with L(i, p)
// in the U-panel below the diagonal block's diagonal (i < w) or in the L-panel.
template <typename T>
__global__ void __launch_bounds__(128) k_mf_bsolve_t(DevLU L, const int* __restrict__ task_sn, int nsn_l,
                                                     int ngroups, int fcap, const T* __restrict__ pan,
                                                     T* __restrict__ x, const int* __restrict__ group_active) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
  T* xs = reinterpret_cast<T*>(smem_raw) + (size_t)warp * fcap * 32;
  const long long ntasks = (long long)nsn_l * ngroups;
  for (long long t = (long long)blockIdx.x * warps + warp; t < ntasks; t += (long long)gridDim.x * warps) {
    const int s = task_sn[t / ngroups];
    const int g = (int)(t % ngroups);
    if (!group_active[g] || !task_here(L, s, g)) continue;
    const int w = L.sn_w[s], f = L.sn_f[s];
    const int* rows = L.sn_rows + L.sn_rptr[s];
    const long long po = L.pan_off[s];
    // the supernode's panels (U: w x f, L: (f - w) x w entries of the group) are read
    // column by column, each after the last one's solve: one bulk L2 prefetch for all
    if (lane == 0) prefetch_l2(pan + at32(g, L.nnz, po, 0), (unsigned)(w * f + (f - w) * w) * (32 * sizeof(T)));
    for (int q = 0; q < f; ++q) xs[q * 32 + lane] = x[at32(g, L.n, rows[q], lane)];
    for (int p = w - 1; p >= 0; --p) {
      T acc = xs[p * 32 + lane];
      for (int i = p + 1; i < w; ++i) acc -= pan[at32(g, L.nnz, po + (long long)i * f + p, lane)] * xs[i * 32 + lane];
      for (int i = w; i < f; ++i)
        acc -= pan[at32(g, L.nnz, po + (long long)w * f + (long long)(i - w) * w + p, lane)] * xs[i * 32 + lane];
      xs[p * 32 + lane] = acc;
    }
    for (int p = 0; p < w; ++p) x[at32(g, L.n, rows[p], lane)] = xs[p * 32 + lane];
    __syncwarp();
  }
}

// dL/dP_i = lambda(P_i row), dL/dQ_i = lambda(Q_i row): F = S(V) - Sbus, so
// dF/dSbus = -I and dL/dtheta = dL/dtheta|explicit - lambda^T dF/dtheta.
template <typename T>
__global__ void k_adj_grad_bus(DevGrid d, int ncases, const T* __restrict__ lam, double* __restrict__ gp,
                               double* __restrict__ gq) {
  const size_t total = (size_t)ncases * d.nb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int uc = (int)(t / d.nb), i = (int)(t % d.nb);
    const int c = lane_of_case(d, uc);
    const int2 jv = d.jvar[i];
    const bool ok = d.status[c] == ST_CONVERGED && row_here(d, i, c >> 5);
    if (gp) gp[t] = (ok && jv.x >= 0) ? (double)lam[at32(c >> 5, d.n_jac, jv.x, c & 31)] : 0.0;
    if (gq) gq[t] = (ok && jv.y >= 0 && !still_pv(d, i, c >> 5, c & 31)) ? (double)lam[at32(c >> 5, d.n_jac, jv.y, c & 31)] : 0.0;
  }
}

// Branch series admittance y = g + jb.  dY/dg for (ff, ft, tf, tt) = a = (1/|t|^2,
// -1/conj(t), -1/t, 1) (br_dy), dY/db = j a.  With Df = Vf conj(a_ff Vf + a_ft Vt),
// Dt = Vt conj(a_tf Vf + a_tt Vt) (the branch's injections' derivative w.r.t. g):
//   dL/dg = c Re(conj(Sf) Df) - [lam_Pf Re Df + lam_Qf Im Df + lam_Pt Re Dt + lam_Qt Im Dt]
//   dL/db = c Im(conj(Sf) Df) - [lam_Pf Im Df - lam_Qf Re Df + lam_Pt Im Dt - lam_Qt Re Dt]
// (first terms only when the branch is overloaded).  Thread per (branch, lane).
template <typename T>
__global__ void __launch_bounds__(256) k_adj_grad_branch(DevGrid d, int nbr, int ncases, const double* __restrict__ rating,
                                                         const double2* __restrict__ br_dy, const T* __restrict__ lam,
                                                         double* __restrict__ gg, double* __restrict__ gb) {
  const int grp = blockIdx.y;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int c = grp * 32 + lane;
  LaneOut o;
  load_outages(d, c, o);
  const int uc = case_of_lane(d, c, ncases);  // the user's case in this lane, -1 for padding
  const bool ok = uc >= 0 && d.status[c] == ST_CONVERGED;
  const int k1 = min(nbr, (int)(blockIdx.x + 1) * 64);
  for (int k = blockIdx.x * 64 + warp; k < k1; k += 8) {
    if (uc < 0) continue;
    double rg = 0.0, rb = 0.0;
    if (ok && branch_here(d, k, grp) && !outaged(o, k)) {
      const int2 ft = d.br_ft[k];
      double2 y[4], a[4];
      branch_y(d, k, grp, lane, y);
      const int jc = d.br_ctl ? d.br_ctl[k] : -1;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        a[q] = jc < 0 ? br_dy[4 * k + q] : d.ctl_bdy[at32(grp, 4 * d.noltc, 4 * jc + q, lane)];
      const double2 vf = d.V[at32(grp, d.nb, ft.x, lane)], vt = d.V[at32(grp, d.nb, ft.y, lane)];
      // Df = Vf conj(a_ff Vf + a_ft Vt), Dt = Vt conj(a_tf Vf + a_tt Vt)
      const double2 u = make_double2(a[0].x * vf.x - a[0].y * vf.y + a[1].x * vt.x - a[1].y * vt.y,
                                     a[0].x * vf.y + a[0].y * vf.x + a[1].x * vt.y + a[1].y * vt.x);
      const double2 Df = make_double2(vf.x * u.x + vf.y * u.y, vf.y * u.x - vf.x * u.y);
      const double2 u2 = make_double2(a[2].x * vf.x - a[2].y * vf.y + a[3].x * vt.x - a[3].y * vt.y,
                                      a[2].x * vf.y + a[2].y * vf.x + a[3].x * vt.y + a[3].y * vt.x);
      const double2 Dt = make_double2(vt.x * u2.x + vt.y * u2.y, vt.y * u2.x - vt.x * u2.y);
      // explicit part through this branch's own Sf
      const double2 yv = make_double2(y[0].x * vf.x - y[0].y * vf.y + y[1].x * vt.x - y[1].y * vt.y,
                                      y[0].x * vf.y + y[0].y * vf.x + y[1].x * vt.y + y[1].y * vt.x);
      const double2 S = make_double2(vf.x * yv.x + vf.y * yv.y, vf.y * yv.x - vf.x * yv.y);
      const double aS = sqrt(S.x * S.x + S.y * S.y);
      const double E = aS - 0.9 * rating[k];
      if (E > 0.0) {
        const double cc = 2.0 * E / aS;
        rg += cc * (S.x * Df.x + S.y * Df.y);
        rb += cc * (S.x * Df.y - S.y * Df.x);
      }
      const int2 vfv = d.jvar[ft.x], vtv = d.jvar[ft.y];
      const double lPf = vfv.x >= 0 ? (double)lam[at32(grp, d.n_jac, vfv.x, lane)] : 0.0;
      const double lQf = vfv.y >= 0 ? (double)lam[at32(grp, d.n_jac, vfv.y, lane)] : 0.0;
      const double lPt = vtv.x >= 0 ? (double)lam[at32(grp, d.n_jac, vtv.x, lane)] : 0.0;
      const double lQt = vtv.y >= 0 ? (double)lam[at32(grp, d.n_jac, vtv.y, lane)] : 0.0;
      rg -= lPf * Df.x + lQf * Df.y + lPt * Dt.x + lQt * Dt.y;
      rb -= lPf * Df.y - lQf * Df.x + lPt * Dt.y - lQt * Dt.x;
    }
    if (gg) gg[(size_t)uc * nbr + k] = rg;
    if (gb) gb[(size_t)uc * nbr + k] = rb;
  }
}

// ---------------------------------------------------------------- per-case controls
// The optimiser's structures (pso/Particula.h:26-60): AVR = |V| set-point of a PV or
// slack bus (runpf.h:524-541), OLTC = tap ratio of a branch and ShC = shunt
// susceptance of a bus (makeYbus.h:313-332).  values[g][k][32] holds control k of
// every case; a tap or shunt changes the Ybus entries at its slots, which yentry()
// adds to the base value.
struct DevCtl {
  int nc, navr, noltc, nshc, nslot;
  const double* val;        // [g][nc][32]
  const int2* avr;          // (bus, value column)
  const int2* oltc;         // (branch, value column)
  const double* oltc_par;   // 8 per tap: Ys (re, im), b/2, cos, sin of the shift, Ys with r = 0 (re, im), 0
  const int2* shc;          // (bus, value column)
  const double* shc_base;   // base Bsh of each controlled shunt
  const int* slot_ptr;      // [nslot + 1]
  const int2* slot_ent;     // (q, j): q < 3 entry q (ff, ft, tf) of tap j; q == 3 shunt j
};

// Admittances and dY/dg of every controlled tap in every case (branch_admittance with
// the case's tap; all zero for a branch out of service).  Thread per (tap, lane).
__global__ void k_ctl_branch(DevCtl t, int ngroups, double2* __restrict__ bry, double2* __restrict__ bdy) {
  const size_t total = (size_t)ngroups * t.noltc * 32;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < total; id += (size_t)gridDim.x * blockDim.x) {
    const int lane = (int)(id & 31);
    const size_t rest = id >> 5;
    const int j = (int)(rest % t.noltc), g = (int)(rest / t.noltc);
    const double tap = t.val[at32(g, t.nc, t.oltc[j].y, lane)];
    const double* pr = t.oltc_par + 8 * j;
    const double ysr = pr[0], ysi = pr[1], bc2 = pr[2];
    const double tr = tap * pr[3], ti = tap * pr[4];
    const double t2 = tr * tr + ti * ti;
    const double ytr = ysr, yti = ysi + bc2;
    const bool on = ysr != 0.0 || ysi != 0.0 || bc2 != 0.0;
    double2 y[4], a[4];
    y[0] = make_double2(ytr / t2, yti / t2);
    y[1] = make_double2(-(ysr * tr - ysi * ti) / t2, -(ysr * ti + ysi * tr) / t2);
    y[2] = make_double2(-(ysr * tr + ysi * ti) / t2, -(ysi * tr - ysr * ti) / t2);
    y[3] = make_double2(ytr, yti);
    a[0] = make_double2(1.0 / t2, 0.0);
    a[1] = make_double2(-tr / t2, -ti / t2);
    a[2] = make_double2(-tr / t2, ti / t2);
    a[3] = make_double2(1.0, 0.0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const size_t k = at32(g, 4 * t.noltc, 4 * j + q, lane);
      bry[k] = y[q];
      bdy[k] = on ? a[q] : make_double2(0.0, 0.0);
    }
  }
}

// Per case and slot: the sum of the changes the controls make at that Ybus position
// (a tap whose branch the case outages contributes nothing: ycase() removes the
// branch's base admittance).  Thread per (slot, lane).
__global__ void k_ctl_ydelta(DevGrid d, DevCtl t, const double2* __restrict__ bry, double2* __restrict__ dy) {
  const size_t total = (size_t)d.ngroups * t.nslot * 32;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < total; id += (size_t)gridDim.x * blockDim.x) {
    const int lane = (int)(id & 31);
    const size_t rest = id >> 5;
    const int s = (int)(rest % t.nslot), g = (int)(rest / t.nslot);
    LaneOut o;
    load_outages(d, g * 32 + lane, o);
    double2 acc = make_double2(0.0, 0.0);
    for (int e = t.slot_ptr[s]; e < t.slot_ptr[s + 1]; ++e) {
      const int2 en = t.slot_ent[e];
      if (en.x < 3) {
        const int k = t.oltc[en.y].x;
        if (outaged(o, k)) continue;
        const double2 nv = bry[at32(g, 4 * t.noltc, 4 * en.y + en.x, lane)];
        const double2 bv = d.br_y[4 * k + en.x];
        acc.x += nv.x - bv.x;
        acc.y += nv.y - bv.y;
      } else {
        acc.y += t.val[at32(g, t.nc, t.shc[en.y].y, lane)] - t.shc_base[en.y];
      }
    }
    dy[at32(g, t.nslot, s, lane)] = acc;
  }
}

// AVR set-points: V_i = value e^{j Va_i} (runpf.h:524-541).  Thread per (AVR, lane),
// after k_init.
__global__ void k_ctl_vm(DevGrid d, DevCtl t) {
  const size_t total = (size_t)d.ngroups * t.navr * 32;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < total; id += (size_t)gridDim.x * blockDim.x) {
    const int lane = (int)(id & 31);
    const size_t rest = id >> 5;
    const int j = (int)(rest % t.navr), g = (int)(rest / t.navr);
    const int2 a = t.avr[j];
    const double2 v0 = d.v0[a.x];
    double sn, cs;
    sincos(atan2(v0.y, v0.x), &sn, &cs);
    const double vm = t.val[at32(g, t.nc, a.y, lane)];
    d.V[at32(g, d.nb, a.x, lane)] = make_double2(vm * cs, vm * sn);
  }
}

// B'' of every case with its controls (B' has taps and shunts zeroed, makeB.h:311-324,
// so it has none): at each slot inside B'' (pos >= 0), the change of -Im(Y'') that the
// case's taps (phase shift 0; r = 0 in BX) and shunts make.  Thread per (slot, lane).
template <typename T>
__global__ void k_fd_ctl(DevGrid d, DevCtl t, int variant, int nA, const int* __restrict__ slot_pos,
                         const double4* __restrict__ br_bval, T* __restrict__ A) {
  const size_t total = (size_t)d.ngroups * t.nslot * 32;
  for (size_t id = blockIdx.x * (size_t)blockDim.x + threadIdx.x; id < total; id += (size_t)gridDim.x * blockDim.x) {
    const int lane = (int)(id & 31);
    const size_t rest = id >> 5;
    const int s = (int)(rest % t.nslot), g = (int)(rest / t.nslot);
    const int pos = slot_pos[s];
    if (pos < 0) continue;
    LaneOut o;
    load_outages(d, g * 32 + lane, o);
    double acc = 0.0;
    for (int e = t.slot_ptr[s]; e < t.slot_ptr[s + 1]; ++e) {
      const int2 en = t.slot_ent[e];
      if (en.x < 3) {
        const int k = t.oltc[en.y].x;
        if (outaged(o, k)) continue;
        const double* pr = t.oltc_par + 8 * en.y;
        const double ysi = variant == 1 ? pr[6] : pr[1];
        const double tap = t.val[at32(g, t.nc, t.oltc[en.y].y, lane)];
        const double nv = en.x == 0 ? -(ysi + pr[2]) / (tap * tap) : ysi / tap;
        const double4 bv = br_bval[k];
        acc += nv - (en.x == 0 ? bv.x : en.x == 1 ? bv.y : bv.z);
      } else {
        acc -= t.val[at32(g, t.nc, t.shc[en.y].y, lane)] - t.shc_base[en.y];
      }
    }
    const size_t idx = at32(g, nA, pos, lane);
    A[idx] = (T)((double)A[idx] + acc);
  }
}

// ---------------------------------------------------------------- reactive limits
// Start of a solve: every limited bus is PV in every case, no earlier rounds.
__global__ void k_qlim_reset(DevGrid d) {
  const size_t total = (size_t)d.ngroups * 32 * d.nsw;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x)
    d.pv_on[t] = 1;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.ngroups * 32; c += gridDim.x * blockDim.x)
    d.iter_base[c] = 0;
}

// After a Newton run: for every converged case and every bus still PV there, the net
// reactive injection Q = Im(V_i conj(Ibus_i)); outside [qmin, qmax] the bus becomes PQ
// holding the violated limit (all violators of a case at once, as MATPOWER's runpf with
// ENFORCE_Q_LIMS = 1) and the case is flagged for another run.  Thread per (bus, lane).
__global__ void k_qlim_check(DevGrid d, const int* __restrict__ sw_bus, const double2* __restrict__ q_lim,
                             int* __restrict__ flag) {
  const size_t total = (size_t)d.ngroups * d.nsw * 32;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int lane = (int)(t & 31);
    const size_t rest = t >> 5;
    const int k = (int)(rest % d.nsw), g = (int)(rest / d.nsw);
    const int c = g * 32 + lane;
    const size_t sk = at32(g, d.nsw, k, lane);
    const int i = sw_bus[k];
    if (d.status[c] != ST_CONVERGED || !d.pv_on[sk] || !row_here(d, i, g)) continue;
    LaneOut o;
    load_outages(d, c, o);
    const bool touched = row_touched(o, d.y_diag[i]);
    double2 ib = make_double2(0.0, 0.0);
    for (int p = d.y_rowptr[i]; p < d.y_rowptr[i + 1]; ++p) {
      const double2 y = yentry(d, o, touched, p, g, lane);
      const double2 v = d.V[at32(g, d.nb, d.y_col[p], lane)];
      ib.x += y.x * v.x - y.y * v.y;
      ib.y += y.x * v.y + y.y * v.x;
    }
    const double2 vi = d.V[at32(g, d.nb, i, lane)];
    const double q = vi.y * ib.x - vi.x * ib.y;
    const double2 lim = q_lim[k];
    if (q > lim.y || q < lim.x) {
      d.pv_on[sk] = 0;
      d.q_fix[sk] = q > lim.y ? lim.y : lim.x;
      flag[c] = 1;
    }
  }
}

// Flagged cases run Newton again from their voltages; the others keep their status.
__global__ void k_qlim_restart(DevGrid d, int* __restrict__ flag) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nl = d.ngroups * 32;
  bool again = false;
  if (c < nl && flag[c]) {
    flag[c] = 0;
    d.iter_base[c] = d.iters[c];
    d.status[c] = ST_RUNNING;
    again = true;
  }
  const unsigned any = __ballot_sync(0xffffffffu, again);
  if ((threadIdx.x & 31) == 0 && c < nl) {
    d.group_active[c >> 5] = any != 0u;
    if (any) atomicAdd(d.any_active, 1);
  }
}

// [group][..][32] bus types after the limits: a switched PV bus reads PQ.
__global__ void k_gather_types(DevGrid d, int ncases, const unsigned char* __restrict__ base_type,
                               unsigned char* __restrict__ out) {
  const size_t total = (size_t)ncases * d.nb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int uc = (int)(t / d.nb), i = (int)(t % d.nb);
    const int c = lane_of_case(d, uc);
    unsigned char ty = base_type[i];
    if (d.sw_index && d.sw_index[i] >= 0 && !d.pv_on[at32(c >> 5, d.nsw, d.sw_index[i], c & 31)]) ty = 1;
    out[t] = ty;
  }
}

__global__ void k_fill_int(int* p, int n, int v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// ---------------------------------------------------------------- results
// [group][bus][32] -> [case][bus]
// case_lane (nullable): lane of each case when lanes are grouped by island
__global__ void k_gather_v(int nb, int ncases, const int* case_lane, const double2* V, double2* out) {
  const size_t total = (size_t)ncases * nb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
    const int uc = (int)(t / nb), i = (int)(t % nb);
    const int c = case_lane ? case_lane[uc] : uc;
    out[t] = V[at32(c >> 5, nb, i, c & 31)];
  }
}

__global__ void k_gather_small(int ncases, const int* case_lane, const int* status, const int* iters,
                               const double* maxmis, uint8_t* st_out, int* it_out, double* mm_out) {
  const int uc = blockIdx.x * blockDim.x + threadIdx.x;
  if (uc >= ncases) return;
  const int c = case_lane ? case_lane[uc] : uc;
  if (st_out) st_out[uc] = (uint8_t)status[c];
  if (it_out) it_out[uc] = iters[c];
  if (mm_out) mm_out[uc] = maxmis[c];
}

}  // namespace mpfk

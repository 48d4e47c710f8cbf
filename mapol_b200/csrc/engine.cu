// Host side of libmpf: the handle, device uploads, level schedules, the Newton and
// fast-decoupled solve loops, and the C-ABI declared in include/mpf.h.
//
// Reference counterparts: hybrid_init (src/powerflow/runpf.h:795-982) allocates
// per-case copies of every sparse structure and creates one CUDA stream per case;
// hybrid_runpf (runpf.h:606-793) launches one small kernel per case per stage and
// solves the Newton systems on the host with MKL DSS (newtonpf.h:1086-1158).  Here
// one handle owns all device memory, every stage is one launch over all cases, and
// the linear systems are factorised on the device by k_mf_factor.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <array>
#include <climits>
#include <mutex>
#include <set>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include <cuda_runtime.h>

#include "internal.h"
#include "kernels.cuh"
#include "mpf.h"

using namespace mpf;
using namespace mpfk;

namespace {

// ------------------------------------------------------------------ errors
struct MpfError {
  int code;
  std::string msg;
};

#define CUDA_TRY(expr)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (expr);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      throw MpfError{e_ == cudaErrorMemoryAllocation ? MPF_ERR_OOM : MPF_ERR_CUDA,        \
                     std::string(#expr) + ": " + cudaGetErrorString(e_)};                  \
    }                                                                                      \
  } while (0)

// ------------------------------------------------------------------ device buffers
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  void alloc(size_t b) {
    release();
    if (b == 0) b = 16;
    CUDA_TRY(cudaMalloc(&p, b));
    bytes = b;
  }
  template <class T>
  T* as() const { return reinterpret_cast<T*>(p); }
};

// Copies v to the device, reusing b's allocation when it is large enough.
template <class T>
void upload(DevBuf& b, const std::vector<T>& v) {
  const size_t need = v.size() * sizeof(T);
  if (!b.p || b.bytes < need) b.alloc(need);
  if (!v.empty()) CUDA_TRY(cudaMemcpy(b.p, v.data(), need, cudaMemcpyHostToDevice));
}

// ------------------------------------------------------------------ LU system
enum TaskClass { CLS_S = 0, CLS_M = 1, CLS_L = 2, CLS_M1 = 3, CLS_BIG = 4 };
// fronts up to kFmaxS: one case per thread; up to kFmaxM: a warp per 32-byte lane
// chunk; larger: a 256-thread block per lane chunk, with fewer lanes per task when a
// 32-byte chunk would not fit in shared memory (kSmemMax)
constexpr int kFmaxS = 8, kFmaxM1 = 16, kFmaxM = 24;
constexpr size_t kSmemMax = 227 * 1024;
// rounds of PV -> PQ switching per solve (each switches at least one bus of a case)
constexpr int kMaxQRounds = 20;
// largest dense front in shared memory: one FP64 lane, f * ((f + 1) | 1) * 8 bytes.
// Larger fronts (CLS_BIG, densely meshed grids) keep only their panel, w (2f - w + 1)
// entries, in shared memory (k_mf_factor_big) and their trailing block in global memory
constexpr int kFmaxAll = 167;
inline size_t big_panel(int w, int f) { return (size_t)w * (2 * f - w + 1); }
// The fronts' limits: every panel of one FP64 lane and one warp's slice of x in the
// thread-per-case substitutions (f entries of 32 FP64 lanes) fit in shared memory
inline std::string front_limits(const LUSymbolic& L, const char* what) {
  for (int s = 0; s < L.nsn; ++s) {
    const int w = L.sn_w[s], f = L.sn_f[s];
    if (f > kFmaxAll && (big_panel(w, f) + (f - w + 1)) * 8 > kSmemMax)
      return std::string(what) + ": a front of " + std::to_string(f) + " rows with " + std::to_string(w) +
             " pivots needs a " + std::to_string((big_panel(w, f) + (f - w + 1)) * 8 / 1024) +
             " KB panel and trailing row, above the " +
             std::to_string(kSmemMax / 1024) + " KB of shared memory (grid too densely meshed)";
    if ((size_t)f * 32 * 8 > kSmemMax)
      return std::string(what) + ": a front of " + std::to_string(f) + " rows exceeds " +
             std::to_string(kSmemMax / 256) + " (grid too densely meshed)";
  }
  return {};
}
// warps per block of the substitution kernels that hold a warp's slice of x (fcap
// entries of `lanes` lanes) in shared memory: four, or fewer for large fronts
template <typename T>
int solve_warps(int fcap, int lanes) {
  const size_t per = (size_t)std::max(fcap, 1) * lanes * sizeof(T);
  return (int)std::max<size_t>(1, std::min<size_t>(4, kSmemMax / per));
}
// backward solve: levels nearest the root with at most this many supernodes can run as
// one k_mf_bsolve_top launch (an autotuner choice); codes kTopCode + G in the tuned
// per-launch choices mark the launches it replaces
constexpr int kTopLevelSn = 24;
constexpr int kTopCode = 100;
// factorisation launches split by front size (LUSystem::split_factor_launches; a ratio
// of at most 1 keeps one launch per level and task class).  9241-bus workload, mixed /
// FP64 solves/s: no split 35.7k / 22.5k, 1.35 with 64 supernodes 36.7k / 23.4k, 1.6
// with 128 35.9k / 22.6k
constexpr double kSplitRatio = 1.35;
constexpr int kSplitMinSn = 64;

struct Launch {
  int offset, count, cls, fcap;  // range of lev_sn, task class, max front in range
  int wfmax = 0;                 // largest w * f in range (U-panel entries)
  int level = 0;                 // elimination-tree level
  size_t pcap = 0;               // CLS_BIG: largest panel in range, w (2f - w + 1) entries
  int mcap = 0;                  // CLS_BIG: largest trailing block in range, m = f - w rows
};

// Side streams of one LU system, created on first use.  The factorisation's launches
// form a DAG (a launch needs the launches that hold its supernodes' children); each task
// class keeps its launches in order on one stream (class 0 on the caller's), and a
// launch waits by event only for the latest launch it needs on each other stream, so
// independent chains (small fronts near the leaves beside large fronts) run side by
// side; captured in a graph these are parallel branches.
struct SideStreams {
  static constexpr int kN = 3;
  cudaStream_t s[kN] = {};
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> done;  // per factorisation launch
  SideStreams() = default;
  SideStreams(const SideStreams&) = delete;
  SideStreams& operator=(const SideStreams&) = delete;
  ~SideStreams() {
    for (int i = 0; i < kN; ++i)
      if (s[i]) cudaStreamDestroy(s[i]);
    for (cudaEvent_t e : done) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
  }
  void ensure(size_t nlaunch) {
    if (!fork) {
      for (int i = 0; i < kN; ++i) CUDA_TRY(cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking));
      CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    }
    while (done.size() < nlaunch) {
      cudaEvent_t e;
      CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      done.push_back(e);
    }
  }
};

// Where each factorisation launch runs and what it waits for (see SideStreams).
struct LaunchDeps {
  int stream = 0;                 // 0 = the caller's, 1..3 = side streams
  std::vector<int> wait;          // launches on other streams to wait for (latest per stream)
  bool record = false;            // a later launch on another stream waits for this one
};

// FNV-1a over the structure that decides the launches and their work
inline uint64_t structure_fingerprint(const LUSymbolic& s) {
  uint64_t h = 1469598103934665603ull;
  auto mix = [&](int64_t v) {
    for (int b = 0; b < 8; ++b) {
      h ^= (uint64_t)((v >> (8 * b)) & 0xff);
      h *= 1099511628211ull;
    }
  };
  mix(s.n);
  mix(s.nnz);
  mix(s.nsn);
  for (int v : s.sn_w) mix(v);
  for (int v : s.sn_f) mix(v);
  for (int v : s.lev_ptr) mix(v);
  for (int v : s.lev_sn) mix(v);
  return h;
}

// Kernel of one factorisation launch: kind 0 = warp teams (k_mf_factor<T, ge, 32>,
// tpb teams per block), 1 = 256-thread teams with the LU in shared memory, 2 = the
// same with the LU in registers (TT x TT tile per thread), 3 = 512- or 1024-thread
// teams (tpb = threads / 256) with the LU in shared memory, 5 = 256- or 512-thread teams
// (tpb = threads / 256) taking two pivots per barrier
struct FactorChoice {
  int kind, ge, tt, tpb;
};

struct LUSystem {
  LUSymbolic sym;
  DevBuf sn_w, sn_f, sn_rptr, sn_rows, child_ptr, child_list, sn_parent, rel_ptr, relmap, ah_ptr, ah_loc;
  DevBuf pan_off, cb_off, cbr_off, lev_sn, child_ref, cb_in;
  DevBuf sn_island;                  // multi-island handles only
  const int* group_island = nullptr; // the handle's current per-group islands (or null)
  std::vector<Launch> factor_sched;  // ascending levels
  std::vector<LaunchDeps> factor_deps;
  // the backward substitution: the factorisation's launches (one per level and task
  // class), run from the root down; a launch waits for the launches holding its
  // supernodes' parents
  std::vector<Launch> bsolve_sched;
  std::vector<LaunchDeps> bsolve_deps;
  // the levels nearest the root, which k_mf_bsolve_top can solve in one launch:
  // bsolve_sched[bs_top_from ..] are their launches; top_sn / top_lev_ptr list their
  // supernodes from the root down, level by level
  int bs_top_from = 0, top_nlev = 0, top_fcap = 0;
  DevBuf top_sn, top_lev_ptr;
  std::unique_ptr<SideStreams> side = std::make_unique<SideStreams>();
  // autotuned kernel of every factor_sched launch, per (precision, case groups)
  uint64_t fingerprint = 0;          // of the symbolic structure (process-wide tuning cache key)
  std::map<std::pair<int, int>, std::vector<FactorChoice>> tuned;
  // autotuned lane count of every backward-solve level launch (0 = one case per thread)
  std::map<std::pair<int, int>, std::vector<int>> tuned_bs;
  std::vector<Launch> level_sched;   // one launch per level (fast-decoupled forward and adjoint solves), ascending
  std::vector<int> ah_host;          // arrowhead ranges (host copy of ah_ptr)
  int nA = 0;
  // values per precision [0] = FP64, [1] = FP32
  DevBuf A[2], pan[2], cb[2], cbr[2], x[2];
  int ngroups_alloc[2] = {0, 0};

  DevLU dev() const {
    DevLU d;
    d.n = sym.n;
    d.nsn = sym.nsn;
    d.nA = nA;
    d.nnz = sym.nnz;
    d.sumcb = sym.sum_cb;
    d.sumcbr = sym.cbr_off.empty() ? 0 : sym.cbr_off.back();
    d.sn_w = sn_w.as<int>();
    d.sn_f = sn_f.as<int>();
    d.sn_rptr = sn_rptr.as<int>();
    d.sn_rows = sn_rows.as<int>();
    d.child_ptr = child_ptr.as<int>();
    d.child_list = child_list.as<int>();
    d.sn_parent = sn_parent.as<int>();
    d.rel_ptr = rel_ptr.as<int>();
    d.relmap = relmap.as<int>();
    d.ah_ptr = ah_ptr.as<int>();
    d.ah_loc = ah_loc.as<int>();
    d.pan_off = pan_off.as<long long>();
    d.cb_off = cb_off.as<long long>();
    d.cbr_off = cbr_off.as<long long>();
    d.child_ref = child_ref.as<ChildRef>();
    d.cb_in = cb_in.as<CbIn>();
    d.sn_island = group_island ? sn_island.as<int>() : nullptr;
    d.group_island = group_island;
    return d;
  }

  // var_island (multi-island handles): island of each variable; a supernode's
  // variables all belong to one island (the matrix is block-diagonal by island)
  void setup(const LUSymbolic& s, const std::vector<int>& ahp, const std::vector<int>& ahl, int nA_,
             const std::vector<int>* var_island = nullptr) {
    sym = s;
    nA = nA_;
    if (var_island) {
      std::vector<int> si(s.nsn);
      for (int k = 0; k < s.nsn; ++k) {
        si[k] = (*var_island)[s.sn_rows[s.sn_rptr[k]]];
        for (int q = s.sn_rptr[k]; q < s.sn_rptr[k] + s.sn_w[k]; ++q)
          if ((*var_island)[s.sn_rows[q]] != si[k]) throw MpfError{MPF_ERR_INTERNAL, "supernode spans two islands"};
      }
      upload(sn_island, si);
    }
    upload(sn_w, s.sn_w);
    upload(sn_f, s.sn_f);
    upload(sn_rptr, s.sn_rptr);
    upload(sn_rows, s.sn_rows);
    upload(child_ptr, s.child_ptr);
    upload(child_list, s.child_list);
    upload(sn_parent, s.sn_parent);
    upload(rel_ptr, s.rel_ptr);
    upload(relmap, s.relmap);
    upload(ah_ptr, ahp);
    upload(ah_loc, ahl);
    ah_host = ahp;
    std::vector<long long> po(s.pan_off.begin(), s.pan_off.end()), co(s.cb_off.begin(), s.cb_off.end()),
        ro(s.cbr_off.begin(), s.cbr_off.end());
    upload(pan_off, po);
    upload(cb_off, co);
    upload(cbr_off, ro);
    upload(lev_sn, s.lev_sn);
    std::vector<ChildRef> cr(s.child_list.size());
    for (size_t q = 0; q < s.child_list.size(); ++q) {
      const int c = s.child_list[q];
      cr[q] = ChildRef{s.cb_off[c], s.cbr_off[c], s.sn_f[c] - s.sn_w[c], s.rel_ptr[c]};
    }
    upload(child_ref, cr);
    std::vector<CbIn> ci(s.nsn, CbIn{0, 0, 0, 0});
    for (int q = 0; q < s.nsn; ++q) {
      if (s.child_ptr[q] == s.child_ptr[q + 1]) continue;
      const int c0 = s.child_list[s.child_ptr[q]];
      ci[q].cb = s.cb_off[c0];
      ci[q].cbr = s.cbr_off[c0];
      for (int c = s.child_ptr[q]; c < s.child_ptr[q + 1]; ++c) {
        const int ch = s.child_list[c], m = s.sn_f[ch] - s.sn_w[ch];
        if (s.cb_off[ch] != ci[q].cb + ci[q].ncb || s.cbr_off[ch] != ci[q].cbr + ci[q].ncbr)
          throw MpfError{MPF_ERR_INTERNAL, "contribution blocks of siblings are not adjacent"};
        ci[q].ncb += m * m;
        ci[q].ncbr += m;
      }
    }
    upload(cb_in, ci);
    fingerprint = structure_fingerprint(s);
    factor_sched.clear();
    level_sched.clear();
    for (int l = 0; l < s.nlevels; ++l) {
      const int b = s.lev_ptr[l], e = s.lev_ptr[l + 1];
      int fmax_all = 0, wf = 0;
      for (int k = b; k < e; ++k) {
        fmax_all = std::max(fmax_all, s.sn_f[s.lev_sn[k]]);
        wf = std::max(wf, s.sn_w[s.lev_sn[k]] * s.sn_f[s.lev_sn[k]]);
      }
      level_sched.push_back({b, e - b, 0, fmax_all, wf});
      int k = b;
      while (k < e) {
        auto cls_of = [](int f) {
          return f <= kFmaxS ? CLS_S : f <= kFmaxM1 ? CLS_M1 : f <= kFmaxM ? CLS_M : f <= kFmaxAll ? CLS_L : CLS_BIG;
        };
        const int cls = cls_of(s.sn_f[s.lev_sn[k]]);
        int k2 = k, fcap = 0;
        while (k2 < e) {
          const int f = s.sn_f[s.lev_sn[k2]];
          const int c2 = cls_of(f);
          if (c2 != cls) break;
          fcap = std::max(fcap, f);
          ++k2;
        }
        factor_sched.push_back({k, k2 - k, cls, fcap, 0, l});
        k = k2;
      }
    }
    // the backward substitution's launches and their DAG (top-down: parents first)
    bsolve_sched = factor_sched;
    split_factor_launches(s);
    for (Launch& ln : factor_sched)
      if (ln.cls == CLS_BIG)
        for (int t = ln.offset; t < ln.offset + ln.count; ++t)
        {
          ln.pcap = std::max(ln.pcap, big_panel(s.sn_w[s.lev_sn[t]], s.sn_f[s.lev_sn[t]]));
          ln.mcap = std::max(ln.mcap, s.sn_f[s.lev_sn[t]] - s.sn_w[s.lev_sn[t]]);
        }
    for (const Launch& ln : factor_sched) {
      fingerprint = (fingerprint ^ (uint64_t)ln.offset) * 1099511628211ull;
      fingerprint = (fingerprint ^ (uint64_t)ln.count) * 1099511628211ull;
    }
    for (Launch& ln : bsolve_sched)
      for (int t = ln.offset; t < ln.offset + ln.count; ++t)
        ln.wfmax = std::max(ln.wfmax, s.sn_w[s.lev_sn[t]] * s.sn_f[s.lev_sn[t]]);
    {
      // near-root levels: from the root down while a level holds at most kTopLevelSn
      // supernodes (too few to fill the GPU as a launch of its own)
      int lcut = s.nlevels;
      while (lcut > 0 && s.lev_ptr[lcut] - s.lev_ptr[lcut - 1] <= kTopLevelSn) --lcut;
      bs_top_from = (int)bsolve_sched.size();
      while (bs_top_from > 0 && bsolve_sched[bs_top_from - 1].level >= lcut) --bs_top_from;
      std::vector<int> tsn, tlp{0};
      top_fcap = 0;
      for (int l = s.nlevels - 1; l >= lcut; --l) {
        for (int k = s.lev_ptr[l]; k < s.lev_ptr[l + 1]; ++k) {
          tsn.push_back(s.lev_sn[k]);
          top_fcap = std::max(top_fcap, s.sn_f[s.lev_sn[k]]);
        }
        tlp.push_back((int)tsn.size());
      }
      top_nlev = s.nlevels - lcut;
      if (top_nlev > 0) {
        upload(top_sn, tsn);
        upload(top_lev_ptr, tlp);
      }
    }
    bsolve_deps.assign(bsolve_sched.size(), LaunchDeps{});
    {
      std::vector<int> launch_of(s.nsn, -1);
      for (int q = (int)bsolve_sched.size() - 1; q >= 0; --q) {
        const Launch& ln = bsolve_sched[q];
        bsolve_deps[q].stream = ln.cls == CLS_S ? 0 : ln.cls == CLS_M1 ? 1 : ln.cls == CLS_M ? 2 : 3;
        int latest[4] = {INT_MAX, INT_MAX, INT_MAX, INT_MAX};  // launches run in descending order
        for (int t = ln.offset; t < ln.offset + ln.count; ++t) {
          const int sn = s.lev_sn[t];
          launch_of[sn] = q;
          const int par = s.sn_parent[sn];
          if (par < 0) continue;
          const int j = launch_of[par];
          const int js = bsolve_deps[j].stream;
          if (js != bsolve_deps[q].stream) latest[js] = std::min(latest[js], j);
        }
        for (int js = 0; js < 4; ++js)
          if (latest[js] != INT_MAX) {
            bsolve_deps[q].wait.push_back(latest[js]);
            bsolve_deps[latest[js]].record = true;
          }
      }
    }
    // the launch DAG: streams by task class, waits for the children's launches
    factor_deps.assign(factor_sched.size(), LaunchDeps{});
    {
      std::vector<int> launch_of(s.nsn, -1);
      for (size_t q = 0; q < factor_sched.size(); ++q) {
        const Launch& ln = factor_sched[q];
        factor_deps[q].stream = ln.cls == CLS_S ? 0 : ln.cls == CLS_M1 ? 1 : ln.cls == CLS_M ? 2 : 3;
        int latest[4] = {-1, -1, -1, -1};
        for (int t = ln.offset; t < ln.offset + ln.count; ++t) {
          const int sn = s.lev_sn[t];
          launch_of[sn] = (int)q;
          for (int c = s.child_ptr[sn]; c < s.child_ptr[sn + 1]; ++c) {
            const int j = launch_of[s.child_list[c]];
            const int js = factor_deps[j].stream;
            if (js != factor_deps[q].stream) latest[js] = std::max(latest[js], j);
          }
        }
        for (int js = 0; js < 4; ++js)
          if (latest[js] >= 0) {
            factor_deps[q].wait.push_back(latest[js]);
            factor_deps[latest[js]].record = true;
          }
      }
    }
  }

  // A launch's shared memory per team is set by its largest front, while its fronts'
  // sizes spread (a level's supernodes are sorted by front size): a run of fronts
  // 9..16 reserves 16 x 17 entries per lane for fronts averaging 12 x 13.  Shared
  // memory bounds the resident teams, and the teams in flight bound these
  // latency-bound launches, so a run splits where the next front would need more
  // than kSplitRatio times the shared memory of the run's first front, as long as both
  // parts keep at least kSplitMinSn supernodes (enough tasks to fill the GPU).
  void split_factor_launches(const LUSymbolic& s) {
    double ratio = kSplitRatio;
    int min_sn = kSplitMinSn;
    if (const char* e = std::getenv("MPF_FSPLIT")) ratio = std::atof(e);
    if (const char* e = std::getenv("MPF_FSPLIT_MIN")) min_sn = std::max(1, std::atoi(e));
    if (!(ratio > 1.0)) return;
    auto area = [](int f) { return (double)f * front_stride(f); };
    std::vector<Launch> out;
    for (const Launch& ln : factor_sched) {
      int k = ln.offset;
      const int end = ln.offset + ln.count;
      while (k < end) {
        const int f0 = s.sn_f[s.lev_sn[k]];
        int k2 = k + 1;
        while (k2 < end && (area(s.sn_f[s.lev_sn[k2]]) <= ratio * area(f0) || k2 - k < min_sn)) ++k2;
        if (end - k2 < min_sn) k2 = end;  // a short remainder joins this part
        Launch p = ln;
        p.offset = k;
        p.count = k2 - k;
        p.fcap = 0;
        for (int q = k; q < k2; ++q) p.fcap = std::max(p.fcap, s.sn_f[s.lev_sn[q]]);
        out.push_back(p);
        k = k2;
      }
    }
    factor_sched = out;
  }

  // Values one factorisation launch moves per case: arrowhead reads, children's
  // contribution blocks read, panels and its own contribution block written.
  int64_t launch_entries(const Launch& ln) const {
    int64_t e = 0;
    for (int k = ln.offset; k < ln.offset + ln.count; ++k) {
      const int sn = sym.lev_sn[k];
      const int64_t m = sym.sn_f[sn] - sym.sn_w[sn];
      e += (ah_host[sn + 1] - ah_host[sn]) + (sym.pan_off[sn + 1] - sym.pan_off[sn]);
      if (sym.sn_parent[sn] >= 0) e += m * m;
      for (int c = sym.child_ptr[sn]; c < sym.child_ptr[sn + 1]; ++c) {
        const int64_t mc = sym.sn_f[sym.child_list[c]] - sym.sn_w[sym.child_list[c]];
        e += mc * mc;
      }
    }
    return e;
  }

  void ensure_values(int prec, int ngroups) {
    if (ngroups_alloc[prec] == ngroups && x[prec].p) return;
    const size_t w = prec ? 4 : 8;
    const size_t lanes = (size_t)ngroups * 32;
    A[prec].alloc(lanes * w * (size_t)nA);
    pan[prec].alloc(lanes * w * (size_t)sym.nnz);
    cb[prec].alloc(lanes * w * (size_t)sym.sum_cb);
    cbr[prec].alloc(lanes * w * (size_t)(sym.cbr_off.empty() ? 0 : sym.cbr_off.back()));
    x[prec].alloc(lanes * w * (size_t)sym.n);
    ngroups_alloc[prec] = ngroups;
  }

  void release_values() {
    for (int p = 0; p < 2; ++p) {
      A[p].release();
      pan[p].release();
      cb[p].release();
      cbr[p].release();
      x[p].release();
      ngroups_alloc[p] = 0;
    }
  }
};

struct FDData {
  DevBuf base, br_apos, br_bval;
};

// ------------------------------------------------------------------ kernel launchers
template <typename T>
struct Prec;
template <>
struct Prec<double> { static constexpr int idx = 0; static constexpr int G = 4; };
template <>
struct Prec<float> { static constexpr int idx = 1; static constexpr int G = 8; };

// Opt every kernel that may take more than 48 KB of dynamic shared memory into the
// full 227 KB, once per device and value type, before any launch or graph capture.
template <typename T, int G>
void set_reg_attrs(int smax) {
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, G, 256, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, G, 256, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, G, 256, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  if constexpr (G * sizeof(T) <= 8) {
    CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, G, 256, 5>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
    CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, G, 256, 6>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  }
}

template <typename T>
void ensure_attrs(int device) {
  static std::mutex mu;
  static bool done[64] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return;
  const int smax = (int)kSmemMax;
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 32, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 32, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G / 2, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 16, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 16, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_chunk<T, 16>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_staged<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_staged<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_staged<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_staged<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G, 256, -2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G, 512, -2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G / 2, 256, -2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G / 2, 512, -2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G / 2, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, Prec<T>::G / 2, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 8, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 4, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 2, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor<T, 1, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  set_reg_attrs<T, 1>(smax);
  set_reg_attrs<T, 2>(smax);
  if constexpr (sizeof(T) == 4) set_reg_attrs<T, 4>(smax);
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_chunk<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_chunk<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_chunk<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_chunk<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_fsolve<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_fsolve_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_t<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor_big<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor_big<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor_big<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor_big_gt<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor_big_gt<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_factor_big_gt<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_top<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_top<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_top<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  CUDA_TRY(cudaFuncSetAttribute(k_mf_bsolve_top<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smax));
  done[device] = true;
}

// dynamic shared memory of a factor launch: the fronts, plus the pivot column/row
// buffers of the register LU
template <typename T, int G, int TT>
size_t factor_smem(int fcap, int teams_per_block) {
  size_t b = (size_t)fcap * front_stride(fcap) * G * sizeof(T) * teams_per_block;
  if (TT > 0) b += (size_t)(2 * fcap + 2 * (fcap + 1)) * G * sizeof(T);
  return b;
}

template <typename T, int G, int TEAM, int TT = 0>
void launch_factor_one(const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan, T* cb, T* cbr, T* x,
                       int* status, const int* group_active, int with_rhs, cudaStream_t st, int teams_per_block) {
  const size_t smem = factor_smem<T, G, TT>(ln.fcap, teams_per_block);
  const long long ntasks = (long long)ln.count * ngroups * (32 / G);
  long long blocks = (ntasks + teams_per_block - 1) / teams_per_block;
  blocks = std::min<long long>(blocks, 148LL * 32);
  k_mf_factor<T, G, TEAM, TT><<<(unsigned)blocks, TEAM * teams_per_block, smem, st>>>(
      sys.dev(), sys.lev_sn.as<int>() + ln.offset, ln.count, ngroups, ln.fcap, A, pan, cb, cbr, x, status,
      group_active, with_rhs);
  CUDA_TRY(cudaGetLastError());
}

// Fronts too large for a dense front in shared memory: k_mf_factor_big, a 512-thread
// block per (supernode, chunk of ge lanes); shared memory holds the launch's largest
// panel and a slab of S trailing rows of its largest trailing block
template <typename T>
void launch_factor_big(int ge, int S, const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan, T* cb,
                       T* cbr, T* x, int* status, const int* group_active, int with_rhs, cudaStream_t st) {
  const size_t smem = (ln.pcap + (size_t)S * (ln.mcap + 1)) * ge * sizeof(T);
  if (ln.pcap == 0 || S < 1 || smem > kSmemMax) throw MpfError{MPF_ERR_INTERNAL, "big-front panel does not fit"};
  const long long ntasks = (long long)ln.count * ngroups * (32 / ge);
  const unsigned blocks = (unsigned)std::min<long long>(ntasks, 148LL * 32);
  const DevLU dl = sys.dev();
  const int* ts = sys.lev_sn.as<int>() + ln.offset;
  switch (ge) {
    case 4: k_mf_factor_big<T, 4><<<blocks, 512, smem, st>>>(dl, ts, ln.count, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, (int)ln.pcap, S); break;
    case 2: k_mf_factor_big<T, 2><<<blocks, 512, smem, st>>>(dl, ts, ln.count, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, (int)ln.pcap, S); break;
    case 1: k_mf_factor_big<T, 1><<<blocks, 512, smem, st>>>(dl, ts, ln.count, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, (int)ln.pcap, S); break;
    default: throw MpfError{MPF_ERR_INTERNAL, "no big-front kernel for this lane count"};
  }
  CUDA_TRY(cudaGetLastError());
}

// The large-front variant with the trailing block in global memory (kind 7): only the
// launch's largest panel in shared memory
template <typename T>
void launch_factor_big_gt(int ge, const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan, T* cb,
                          T* cbr, T* x, int* status, const int* group_active, int with_rhs, cudaStream_t st) {
  const size_t smem = ln.pcap * ge * sizeof(T);
  if (ln.pcap == 0 || smem > kSmemMax) throw MpfError{MPF_ERR_INTERNAL, "big-front panel does not fit"};
  const long long ntasks = (long long)ln.count * ngroups * (32 / ge);
  const unsigned blocks = (unsigned)std::min<long long>(ntasks, 148LL * 32);
  const DevLU dl = sys.dev();
  const int* ts = sys.lev_sn.as<int>() + ln.offset;
  switch (ge) {
    case 4: k_mf_factor_big_gt<T, 4><<<blocks, 512, smem, st>>>(dl, ts, ln.count, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs); break;
    case 2: k_mf_factor_big_gt<T, 2><<<blocks, 512, smem, st>>>(dl, ts, ln.count, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs); break;
    case 1: k_mf_factor_big_gt<T, 1><<<blocks, 512, smem, st>>>(dl, ts, ln.count, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs); break;
    default: throw MpfError{MPF_ERR_INTERNAL, "no big-front kernel for this lane count"};
  }
  CUDA_TRY(cudaGetLastError());
}

// Warp teams need enough tasks to fill the GPU; a launch with fewer tasks gives
// each front a 256-thread team instead (8x the threads on the same chain of pivots).
constexpr long long kMinWarpTasks = 148LL * 24;
// block teams: aim for at least four resident blocks' worth of tasks per SM
constexpr long long kMinBlockTasks = 148LL * 4;

template <typename T>
void launch_factor_ge(int ge, const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan, T* cb, T* cbr,
                      T* x, int* status, const int* group_active, int with_rhs, cudaStream_t st) {
  switch (ge) {
    case 16: launch_factor_one<T, 16, 256>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    case 8: launch_factor_one<T, 8, 256>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    case 4: launch_factor_one<T, 4, 256>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    case 2: launch_factor_one<T, 2, 256>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    default: launch_factor_one<T, 1, 256>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
  }
}

// Register-LU tiles: TT x TT entries per thread covers fronts with f + 1 <= 16 TT
// (right-hand side column included).  Lane chunks: up to 16 bytes (one thread
// per entry); 4 FP32 lanes only up to TT = 4, 2 FP64 lanes up to TT = 4, to keep
// the tile within about 128 registers.
constexpr int kRegTTMax = 6;
inline int reg_tt(int fcap) { return std::max(2, (fcap + 1 + 15) / 16); }
template <typename T>
int reg_lanes_max(int tt) {
  if (sizeof(T) == 4) return tt <= 4 ? 4 : 2;
  return tt <= 4 ? 2 : 1;
}

template <typename T, int G>
void launch_factor_reg_g(int tt, const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan, T* cb,
                         T* cbr, T* x, int* status, const int* group_active, int with_rhs, cudaStream_t st) {
  switch (tt) {
    case 2: launch_factor_one<T, G, 256, 2>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    case 3: launch_factor_one<T, G, 256, 3>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    case 4: launch_factor_one<T, G, 256, 4>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1); break;
    case 5:
    case 6:
      if constexpr (G * sizeof(T) <= 8) {
        if (tt == 5) launch_factor_one<T, G, 256, 5>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
        else launch_factor_one<T, G, 256, 6>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
        break;
      }
      [[fallthrough]];
    default:
      throw MpfError{MPF_ERR_INTERNAL, "no register-LU kernel for this tile and lane count"};
  }
}

template <typename T>
void launch_factor_reg(int ge, int tt, const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan, T* cb,
                       T* cbr, T* x, int* status, const int* group_active, int with_rhs, cudaStream_t st) {
  if (ge >= 4) {
    if constexpr (sizeof(T) == 4)
      launch_factor_reg_g<T, 4>(tt, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
    else
      throw MpfError{MPF_ERR_INTERNAL, "no register-LU kernel for this lane count"};
  } else if (ge == 2) {
    launch_factor_reg_g<T, 2>(tt, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
  } else {
    launch_factor_reg_g<T, 1>(tt, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
  }
}

inline size_t factor_smem_rt(int fcap, int ge, int teams, int tt, size_t wsize) {
  size_t b = (size_t)fcap * front_stride(fcap) * ge * wsize * teams;
  if (tt > 0) b += (size_t)(4 * fcap + 2) * ge * wsize;
  return b;
}

// Rows of the trailing block a large-front task of ge lanes holds in shared memory
// beside the launch's largest panel (0: the panel alone does not fit)
template <typename T>
int big_slab_rows(const Launch& ln, int ge) {
  const size_t cap = kSmemMax / (ge * sizeof(T));
  if (cap <= ln.pcap) return 0;
  return (int)std::min<size_t>((cap - ln.pcap) / ((size_t)ln.mcap + 1), (size_t)std::max(ln.mcap, 1));
}

// The fixed rule (used without autotuning, and as the first candidate): thread per
// case for fronts up to 8, warp teams up to 24, 256-thread teams above (register
// LU up to 16 kRegTTMax - 1 rows); lane chunks shrink while a level has too few
// tasks to fill the GPU or the front would not fit in shared memory.
template <typename T>
FactorChoice heuristic_choice(const Launch& ln, int ngroups) {
  constexpr int G = Prec<T>::G;
  const long long lanes_tasks = (long long)ln.count * ngroups;
  if (ln.cls == CLS_BIG) {
    // the panel and a slab of S trailing rows in shared memory: as many lanes per task
    // as leave room for slabs of 12 rows (or the whole trailing block), else one lane
    // with the largest slab that fits (S in the tile field)
    for (int ge = std::min(G, 4); ge >= 1; ge /= 2) {
      const int S = big_slab_rows<T>(ln, ge);
      if (S >= std::min(ln.mcap, 12) && S >= 1) return {6, ge, S, 1};
      if (ge == 1) {
        if (S < 1) throw MpfError{MPF_ERR_INTERNAL, "a large front's panel and one trailing row exceed shared memory"};
        return {6, 1, S, 1};
      }
    }
    throw MpfError{MPF_ERR_INTERNAL, "a large front's panel exceeds shared memory"};
  }
  if (ln.cls == CLS_S && lanes_tasks < kMinWarpTasks) return {1, 32, 0, 1};
  if ((ln.cls == CLS_M1 || ln.cls == CLS_M) && lanes_tasks * (32 / G) < kMinWarpTasks) {
    int ge = G;
    while (ge > 1 && lanes_tasks * (32 / ge) < kMinBlockTasks) ge /= 2;
    return {1, ge, 0, 1};
  }
  if (ln.cls == CLS_S) return {0, 32, 0, sizeof(T) == 8 ? 4 : 8};
  if (ln.cls == CLS_M1) return {0, G, 0, 8};
  if (ln.cls == CLS_M) return {0, G, 0, 4};
  const size_t per_lane = (size_t)ln.fcap * front_stride(ln.fcap) * sizeof(T);
  int ge = G;
  while (ge > 1 && (per_lane * ge > kSmemMax || lanes_tasks * (32 / ge) < kMinBlockTasks)) ge /= 2;
  return {1, ge, 0, 1};
}

// Every kernel that can run the launch: warp teams (2 to 8 teams per block), the
// 256-thread shared-memory LU at each lane chunk, and the register LU at each
// lane chunk its tile allows, as long as the fronts fit in shared memory.
template <typename T>
std::vector<FactorChoice> factor_candidates(const Launch& ln, int ngroups) {
  constexpr int G = Prec<T>::G;
  const size_t ws = sizeof(T);
  std::vector<FactorChoice> c{heuristic_choice<T>(ln, ngroups)};
  if (ln.cls == CLS_BIG) {
    // the large-front kernel at each lane count whose panel and a trailing row fit,
    // with the largest slab beside the panel
    for (int ge = std::min(Prec<T>::G, 4); ge >= 1; ge /= 2) {
      const int S = big_slab_rows<T>(ln, ge);
      if (S >= 1) {
        const FactorChoice x{6, ge, S, 1};
        bool dup = false;
        for (const auto& y : c) dup = dup || (y.kind == x.kind && y.ge == x.ge && y.tt == x.tt);
        if (!dup) c.push_back(x);
      }
      // the trailing block in global memory instead: only the panel in shared memory
      if (ln.pcap * ge * sizeof(T) <= kSmemMax) c.push_back({7, ge, 0, 1});
    }
    return c;
  }
  auto add = [&](FactorChoice x) {
    for (const auto& y : c)
      if (y.kind == x.kind && y.ge == x.ge && y.tt == x.tt && y.tpb == x.tpb) return;
    c.push_back(x);
  };
  if (ln.fcap <= kFmaxS) {
    for (int tpb : {8, 4})
      if (factor_smem_rt(ln.fcap, 32, tpb, 0, ws) <= kSmemMax) add({0, 32, 0, tpb});
    add({1, 32, 0, 1});
  }
  for (int tpb : {8, 4, 2})
    if (factor_smem_rt(ln.fcap, G, tpb, 0, ws) <= kSmemMax) add({0, G, 0, tpb});
  // half-width lane chunks: half the shared memory per warp, twice the resident warps;
  // 16 lanes: wider contiguous accesses, fewer resident teams
  if (ln.fcap <= kFmaxM) {
    for (int tpb : {8, 4})
      if (factor_smem_rt(ln.fcap, G / 2, tpb, 0, ws) <= kSmemMax) add({0, G / 2, 0, tpb});
    if (G != 16)
      for (int tpb : {4, 2})
        if (factor_smem_rt(ln.fcap, 16, tpb, 0, ws) <= kSmemMax) add({0, 16, 0, tpb});
  }
  for (int ge = 16; ge >= 1; ge /= 2)
    if (factor_smem_rt(ln.fcap, ge, 1, 0, ws) <= kSmemMax) add({1, ge, 0, 1});
  // wider teams for large fronts: more threads per pivot step when few tasks run;
  // two pivots per barrier
  if (ln.fcap > kFmaxM)
    for (int ge : {G, G / 2})
      if (factor_smem_rt(ln.fcap, ge, 1, 0, ws) <= kSmemMax) {
        for (int tpb : {2, 4}) add({3, ge, 0, tpb});
        for (int tpb : {1, 2}) add({5, ge, 0, tpb});
      }
  const int tt = reg_tt(ln.fcap);
  if (ln.fcap > kFmaxS && tt <= kRegTTMax)
    for (int ge = reg_lanes_max<T>(tt); ge >= 1; ge /= 2)
      if (factor_smem_rt(ln.fcap, ge, 1, tt, ws) <= kSmemMax) add({2, ge, tt, 1});
  return c;
}

template <typename T>
void launch_choice(const FactorChoice& ch, const LUSystem& sys, const Launch& ln, int ngroups, const T* A, T* pan,
                   T* cb, T* cbr, T* x, int* status, const int* group_active, int with_rhs, cudaStream_t st) {
  constexpr int G = Prec<T>::G;
  if (ch.kind == 0) {
    if (ch.ge == 32)
      launch_factor_one<T, 32, 32>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, ch.tpb);
    else if (ch.ge == G)
      launch_factor_one<T, G, 32>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, ch.tpb);
    else if (ch.ge == G / 2)
      launch_factor_one<T, G / 2, 32>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st,
                                      ch.tpb);
    else if (ch.ge == 16)
      launch_factor_one<T, 16, 32>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, ch.tpb);
    else
      throw MpfError{MPF_ERR_INTERNAL, "no warp-team kernel for this lane count"};
  } else if (ch.kind == 1) {
    if (ch.ge == 32)
      launch_factor_one<T, 32, 256>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else
      launch_factor_ge<T>(ch.ge, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
  } else if (ch.kind == 2) {
    launch_factor_reg<T>(ch.ge, ch.tt, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
  } else if (ch.kind == 6) {
    launch_factor_big<T>(ch.ge, ch.tt, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
  } else if (ch.kind == 7) {
    launch_factor_big_gt<T>(ch.ge, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st);
  } else if (ch.kind == 5) {
    const bool wide = ch.tpb == 2;
    if (ch.ge == G && wide)
      launch_factor_one<T, G, 512, -2>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else if (ch.ge == G)
      launch_factor_one<T, G, 256, -2>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else if (ch.ge == G / 2 && wide)
      launch_factor_one<T, G / 2, 512, -2>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st,
                                           1);
    else if (ch.ge == G / 2)
      launch_factor_one<T, G / 2, 256, -2>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st,
                                           1);
    else
      throw MpfError{MPF_ERR_INTERNAL, "no two-pivot kernel for this lane count"};
  } else {
    const bool big = ch.tpb == 4;
    if (ch.ge == G && big)
      launch_factor_one<T, G, 1024>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else if (ch.ge == G)
      launch_factor_one<T, G, 512>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else if (ch.ge == G / 2 && big)
      launch_factor_one<T, G / 2, 1024>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else if (ch.ge == G / 2)
      launch_factor_one<T, G / 2, 512>(sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, st, 1);
    else
      throw MpfError{MPF_ERR_INTERNAL, "no wide-team kernel for this lane count"};
  }
}

template <typename T>
void launch_factor(const LUSystem& sys, int ngroups, const T* A, T* pan, T* cb, T* cbr, T* x, int* status,
                   const int* group_active, int with_rhs, cudaStream_t st, int* nlaunch) {
  const auto it = sys.tuned.find({Prec<T>::idx, ngroups});
  const std::vector<FactorChoice>* tuned = it != sys.tuned.end() ? &it->second : nullptr;
  const size_t n = sys.factor_sched.size();
  // MPF_FACTOR_KIND=k runs every launch that has a kernel of kind k with that kernel
  // (the first such candidate), to check that all kinds compute the same factors
  const char* fk_env = std::getenv("MPF_FACTOR_KIND");
  const int fk = fk_env ? std::atoi(fk_env) : -1;
  auto one = [&](size_t k, cudaStream_t s) {
    const Launch& ln = sys.factor_sched[k];
    FactorChoice ch = tuned ? (*tuned)[k] : heuristic_choice<T>(ln, ngroups);
    if (fk >= 0)
      for (const FactorChoice& c : factor_candidates<T>(ln, ngroups))
        if (c.kind == fk) {
          ch = c;
          break;
        }
    launch_choice<T>(ch, sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, with_rhs, s);
    ++*nlaunch;
  };
  // the launch DAG over the caller's stream and three side streams (see SideStreams)
  SideStreams& ss = *sys.side;
  ss.ensure(n);
  cudaStream_t streams[4] = {st, ss.s[0], ss.s[1], ss.s[2]};
  int last[4] = {-1, -1, -1, -1};  // latest launch on each stream
  CUDA_TRY(cudaEventRecord(ss.fork, st));
  bool forked[4] = {true, false, false, false};
  for (size_t k = 0; k < n; ++k) {
    const LaunchDeps& dp = sys.factor_deps[k];
    cudaStream_t s = streams[dp.stream];
    if (!forked[dp.stream]) {
      CUDA_TRY(cudaStreamWaitEvent(s, ss.fork, 0));
      forked[dp.stream] = true;
    }
    for (int j : dp.wait) CUDA_TRY(cudaStreamWaitEvent(s, ss.done[j], 0));
    one(k, s);
    if (dp.record || dp.stream != 0) CUDA_TRY(cudaEventRecord(ss.done[k], s));
    last[dp.stream] = (int)k;
  }
  // join: the caller's stream waits for the last launch of every side stream
  for (int q = 1; q < 4; ++q)
    if (last[q] >= 0) CUDA_TRY(cudaStreamWaitEvent(st, ss.done[last[q]], 0));
}

inline std::string hex64(uint64_t v) {
  char b[24];
  std::snprintf(b, sizeof b, "%llx", (unsigned long long)v);
  return b;
}
// Process-wide tuning results, keyed by (structure fingerprint, precision, groups): every
// handle of the same grid and batch size in a process runs the same kernels, so their
// results agree bit for bit (kernels that split a dot product differently round
// differently).
//
// MPF_TUNE_FILE names a text file that carries these results from one process to the
// next: entries found there are used instead of tuning (each choice is first checked
// against the launch's candidates; an entry that fails is tuned again), and new
// results are appended.  Lines:
//   factor <fingerprint, hex> <precision> <groups> <launches> kind,lanes,tile,teams ...
//   bsolve <fingerprint, hex> <precision> <groups> <levels> lanes ...
struct TuneCache {
  std::mutex mu;
  bool file_read = false;
  std::map<std::tuple<uint64_t, int, int>, std::vector<FactorChoice>> factor;
  std::map<std::tuple<uint64_t, int, int>, std::vector<int>> bsolve;
};
// the cache, with the tuning file's entries read on first use (caller holds no lock)
inline TuneCache& tune_cache() {
  static TuneCache c;
  std::lock_guard<std::mutex> lock(c.mu);
  if (!c.file_read) {
    c.file_read = true;
    const char* path = std::getenv("MPF_TUNE_FILE");
    if (std::FILE* fp = path ? std::fopen(path, "r") : nullptr) {
      char kind[16];
      unsigned long long fpr;
      int prec, ng, n;
      while (std::fscanf(fp, "%15s %llx %d %d %d", kind, &fpr, &prec, &ng, &n) == 5 && n >= 0 && n <= 1000000) {
        const auto key = std::make_tuple((uint64_t)fpr, prec, ng);
        bool ok = true;
        if (std::strcmp(kind, "factor") == 0) {
          std::vector<FactorChoice> v(n);
          for (auto& ch : v) ok = ok && std::fscanf(fp, " %d,%d,%d,%d", &ch.kind, &ch.ge, &ch.tt, &ch.tpb) == 4;
          if (ok) c.factor[key] = v;
        } else if (std::strcmp(kind, "bsolve") == 0) {
          std::vector<int> v(n);
          for (int& x : v) ok = ok && std::fscanf(fp, " %d", &x) == 1;
          if (ok) c.bsolve[key] = v;
        } else {
          ok = false;
        }
        if (!ok) break;
      }
      std::fclose(fp);
    }
  }
  return c;
}
inline void append_tune_file(const std::string& line) {
  const char* path = std::getenv("MPF_TUNE_FILE");
  if (std::FILE* fp = path ? std::fopen(path, "a") : nullptr) {
    std::fputs(line.c_str(), fp);
    std::fclose(fp);
  }
}

// Autotuner: for each launch, level by level, run every candidate twice (the
// first run loads the kernel) and keep the one with the shortest second run
// (CUDA events).  Runs without the right-hand side, so x is not touched; every
// candidate computes the same panels and contribution blocks, which the next
// level reads.  Called outside stream capture, once per (precision, groups).
template <typename T>
void tune_factor(LUSystem& sys, int ngroups, const T* A, T* pan, T* cb, T* cbr, T* x, int* status,
                 const int* group_active, cudaStream_t st) {
  if (sys.tuned.count({Prec<T>::idx, ngroups})) return;
  const auto key = std::make_tuple(sys.fingerprint, Prec<T>::idx, ngroups);
  {
    TuneCache& tc = tune_cache();
    std::lock_guard<std::mutex> lock(tc.mu);
    const auto it = tc.factor.find(key);
    if (it != tc.factor.end()) {
      // every choice must be one of its launch's candidates (entries may come from a file)
      bool ok = it->second.size() == sys.factor_sched.size();
      for (size_t k = 0; ok && k < it->second.size(); ++k) {
        const FactorChoice& c = it->second[k];
        bool found = false;
        for (const FactorChoice& y : factor_candidates<T>(sys.factor_sched[k], ngroups))
          found = found || (y.kind == c.kind && y.ge == c.ge && y.tt == c.tt && y.tpb == c.tpb);
        ok = found;
      }
      if (ok) {
        sys.tuned[{Prec<T>::idx, ngroups}] = it->second;
        return;
      }
      tc.factor.erase(it);
    }
  }
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  std::vector<FactorChoice> best;
  const bool log = std::getenv("MPF_TUNE_LOG") != nullptr;
  double sum_best = 0.0, sum_heur = 0.0;
  try {
    for (const Launch& ln : sys.factor_sched) {
      const std::vector<FactorChoice> cands = factor_candidates<T>(ln, ngroups);
      FactorChoice bc = cands[0];
      float bt = 0.0f, ht = 0.0f;
      for (size_t i = 0; i < cands.size(); ++i) {
        launch_choice<T>(cands[i], sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, 0, st);
        CUDA_TRY(cudaEventRecord(e0, st));
        launch_choice<T>(cands[i], sys, ln, ngroups, A, pan, cb, cbr, x, status, group_active, 0, st);
        CUDA_TRY(cudaEventRecord(e1, st));
        CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (i == 0) ht = ms;
        if (log && std::getenv("MPF_TUNE_LOG")[0] == '2')
          std::fprintf(stderr, "mpf tune:   cand kind %d lanes %d tile %d teams %d: %.1f us\n", cands[i].kind,
                       cands[i].ge, cands[i].tt, cands[i].tpb, ms * 1e3);
        if (i == 0 || ms < bt) {
          bt = ms;
          bc = cands[i];
        }
      }
      best.push_back(bc);
      sum_best += bt;
      sum_heur += ht;
      if (log) {
        const double bytes = (double)sys.launch_entries(ln) * sizeof(T) * 32.0 * ngroups;
        std::fprintf(stderr, "mpf tune: n %d fp%d groups %d launch sn %d cls %d fcap %d: %zu candidates, "
                     "heuristic %.1f us, best %.1f us (kind %d lanes %d tile %d teams %d), %.1f MB, %.0f GB/s\n",
                     sys.sym.n, (int)sizeof(T) * 8, ngroups, ln.count, ln.cls, ln.fcap, cands.size(), ht * 1e3,
                     bt * 1e3, bc.kind, bc.ge, bc.tt, bc.tpb, bytes * 1e-6, bytes / (bt * 1e-3) * 1e-9);
      }
    }
    if (log)
      std::fprintf(stderr, "mpf tune: n %d fp%d groups %d total heuristic %.3f ms, tuned %.3f ms\n", sys.sym.n,
                   (int)sizeof(T) * 8, ngroups, sum_heur, sum_best);
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  sys.tuned[{Prec<T>::idx, ngroups}] = best;
  std::string line = "factor " + hex64(sys.fingerprint) + " " + std::to_string(Prec<T>::idx) + " " +
                     std::to_string(ngroups) + " " + std::to_string(best.size());
  for (const FactorChoice& c : best)
    line += " " + std::to_string(c.kind) + "," + std::to_string(c.ge) + "," + std::to_string(c.tt) + "," +
            std::to_string(c.tpb);
  TuneCache& tc = tune_cache();
  std::lock_guard<std::mutex> lock(tc.mu);
  if (tc.factor.emplace(key, best).second) append_tune_file(line + "\n");
}

// Shared memory of k_mf_bsolve_staged for a level: its largest U panel and front of
// ge lanes.
inline size_t bsolve_staged_smem(const Launch& ln, int ge, size_t wsize) {
  return (size_t)(ln.wfmax + ln.fcap) * ge * wsize;
}

// Backward substitution of one level: ge = 0 one case per thread (k_mf_bsolve), ge > 0
// warps over chunks of ge lanes (k_mf_bsolve_chunk), ge < 0 the same with the U panel
// staged in shared memory first (k_mf_bsolve_staged, chunks of -ge lanes).
template <typename T>
void launch_bsolve_one(int ge, const LUSystem& sys, const Launch& ln, int ngroups, const T* pan, T* x,
                       const int* group_active, cudaStream_t st) {
  const DevLU dl = sys.dev();
  const int* ts = sys.lev_sn.as<int>() + ln.offset;
  if (ge < 0) {
    // staged U panel: a one-warp block per task
    const int gs = -ge;
    const long long ntasks = (long long)ln.count * ngroups * (32 / gs);
    const unsigned blocks = (unsigned)std::min<long long>(ntasks, 148LL * 32);
    const size_t smem = bsolve_staged_smem(ln, gs, sizeof(T));
    switch (gs) {
      case 8: k_mf_bsolve_staged<T, 8><<<blocks, 32, smem, st>>>(dl, ts, ln.count, ngroups, ln.wfmax, pan, x, group_active); break;
      case 4: k_mf_bsolve_staged<T, 4><<<blocks, 32, smem, st>>>(dl, ts, ln.count, ngroups, ln.wfmax, pan, x, group_active); break;
      case 2: k_mf_bsolve_staged<T, 2><<<blocks, 32, smem, st>>>(dl, ts, ln.count, ngroups, ln.wfmax, pan, x, group_active); break;
      case 1: k_mf_bsolve_staged<T, 1><<<blocks, 32, smem, st>>>(dl, ts, ln.count, ngroups, ln.wfmax, pan, x, group_active); break;
      default: throw MpfError{MPF_ERR_INTERNAL, "no staged backward-solve kernel for this lane count"};
    }
    CUDA_TRY(cudaGetLastError());
    return;
  }
  const long long ntasks = (long long)ln.count * ngroups * (ge ? 32 / ge : 1);
  const int wpb = solve_warps<T>(ln.fcap, ge ? ge : 32);
  const long long blocks = std::min<long long>((ntasks + wpb - 1) / wpb, 148LL * 32);
  const size_t smem = (size_t)wpb * ln.fcap * (ge ? ge : 32) * sizeof(T);
  const unsigned nt = 32 * wpb;
  switch (ge) {
    case 0: k_mf_bsolve<T><<<(unsigned)blocks, nt, smem, st>>>(dl, ts, ln.count, ngroups, ln.fcap, pan, x, group_active); break;
    case 16: k_mf_bsolve_chunk<T, 16><<<(unsigned)blocks, nt, smem, st>>>(dl, ts, ln.count, ngroups, ln.fcap, pan, x, group_active); break;
    case 8: k_mf_bsolve_chunk<T, 8><<<(unsigned)blocks, nt, smem, st>>>(dl, ts, ln.count, ngroups, ln.fcap, pan, x, group_active); break;
    case 4: k_mf_bsolve_chunk<T, 4><<<(unsigned)blocks, nt, smem, st>>>(dl, ts, ln.count, ngroups, ln.fcap, pan, x, group_active); break;
    case 2: k_mf_bsolve_chunk<T, 2><<<(unsigned)blocks, nt, smem, st>>>(dl, ts, ln.count, ngroups, ln.fcap, pan, x, group_active); break;
    case 1: k_mf_bsolve_chunk<T, 1><<<(unsigned)blocks, nt, smem, st>>>(dl, ts, ln.count, ngroups, ln.fcap, pan, x, group_active); break;
    default: throw MpfError{MPF_ERR_INTERNAL, "no backward-solve kernel for this lane count"};
  }
  CUDA_TRY(cudaGetLastError());
}

// the near-root levels in one launch (k_mf_bsolve_top), a block per chunk of ge lanes
template <typename T>
void launch_bsolve_top(int ge, const LUSystem& sys, int ngroups, const T* pan, T* x, const int* group_active,
                       cudaStream_t st) {
  const DevLU dl = sys.dev();
  const unsigned blocks = (unsigned)(ngroups * (32 / ge));
  const size_t smem = (size_t)32 * sys.top_fcap * ge * sizeof(T);
  const int* ts = sys.top_sn.as<int>();
  const int* lp = sys.top_lev_ptr.as<int>();
  switch (ge) {
    case 8: k_mf_bsolve_top<T, 8><<<blocks, 1024, smem, st>>>(dl, ts, lp, sys.top_nlev, ngroups, sys.top_fcap, pan, x, group_active); break;
    case 4: k_mf_bsolve_top<T, 4><<<blocks, 1024, smem, st>>>(dl, ts, lp, sys.top_nlev, ngroups, sys.top_fcap, pan, x, group_active); break;
    case 2: k_mf_bsolve_top<T, 2><<<blocks, 1024, smem, st>>>(dl, ts, lp, sys.top_nlev, ngroups, sys.top_fcap, pan, x, group_active); break;
    case 1: k_mf_bsolve_top<T, 1><<<blocks, 1024, smem, st>>>(dl, ts, lp, sys.top_nlev, ngroups, sys.top_fcap, pan, x, group_active); break;
    default: throw MpfError{MPF_ERR_INTERNAL, "no near-root backward-solve kernel for this lane count"};
  }
  CUDA_TRY(cudaGetLastError());
}

// the fixed rule: one case per thread for small fronts; on levels with few
// supernodes, fewer lanes per warp (more warps, more slots per lane)
template <typename T>
int bsolve_heuristic(const Launch& ln, int ngroups) {
  if (ln.fcap <= kFmaxM1) return 0;
  int ge = Prec<T>::G;
  while (ge > 1 && (long long)ln.count * ngroups * (32 / ge) < 148LL * 16) ge /= 2;
  return ge;
}

template <typename T>
void launch_bsolve(const LUSystem& sys, int ngroups, const T* pan, T* x, const int* group_active, cudaStream_t st,
                   int* nlaunch) {
  const auto it = sys.tuned_bs.find({Prec<T>::idx, ngroups});
  // MPF_BSOLVE_LANES (testing, tuning): every level runs this kernel instead: 0, a lane
  // count G of k_mf_bsolve_chunk (16, 8, 4, 2, 1), or -G for k_mf_bsolve_staged (8, 4,
  // 2, 1) on the levels where its shared memory fits
  int force = INT_MIN;
  if (const char* e = std::getenv("MPF_BSOLVE_LANES")) {
    const int v = std::atoi(e);
    for (int ok : {0, 16, 8, 4, 2, 1, -8, -4, -2, -1})
      if (v == ok) force = v;
  }
  // the launch DAG from the root down over the caller's stream and the side streams
  const int n = (int)sys.bsolve_sched.size();
  SideStreams& ss = *sys.side;
  ss.ensure(n);
  cudaStream_t streams[4] = {st, ss.s[0], ss.s[1], ss.s[2]};
  int last[4] = {-1, -1, -1, -1};
  bool forked[4] = {true, false, false, false};
  // the near-root levels as one launch when the tuner chose it (and no kernel is forced):
  // it runs first on the caller's stream, and the events of the launches it replaces are
  // recorded after it, so launches waiting for them wait for it
  // MPF_BSOLVE_TOP (testing): run the near-root levels as one launch with this lane
  // count (8, 4, 2, 1) whatever the tuner chose
  int top_ge = 0;
  if (it != sys.tuned_bs.end() && force == INT_MIN && sys.bs_top_from < n && it->second[n - 1] >= kTopCode)
    top_ge = it->second[n - 1] - kTopCode;
  if (const char* e = std::getenv("MPF_BSOLVE_TOP")) {
    const int v = std::atoi(e);
    if ((v == 8 || v == 4 || v == 2 || v == 1) && sys.top_nlev > 0) top_ge = v;
  }
  int kfrom = n - 1;
  if (top_ge > 0) {
    launch_bsolve_top<T>(top_ge, sys, ngroups, pan, x, group_active, st);
    ++*nlaunch;
    for (int k = sys.bs_top_from; k < n; ++k) CUDA_TRY(cudaEventRecord(ss.done[k], st));
    kfrom = sys.bs_top_from - 1;
  }
  CUDA_TRY(cudaEventRecord(ss.fork, st));
  for (int k = kfrom; k >= 0; --k) {
    const Launch& ln = sys.bsolve_sched[k];
    const LaunchDeps& dp = sys.bsolve_deps[k];
    cudaStream_t s = streams[dp.stream];
    if (!forked[dp.stream]) {
      CUDA_TRY(cudaStreamWaitEvent(s, ss.fork, 0));
      forked[dp.stream] = true;
    }
    for (int j : dp.wait) CUDA_TRY(cudaStreamWaitEvent(s, ss.done[j], 0));
    int ge = it != sys.tuned_bs.end() ? it->second[k] : bsolve_heuristic<T>(ln, ngroups);
    if (ge >= kTopCode) ge -= kTopCode;  // a fused launch's level run on its own: the same chunk solve
    if (force != INT_MIN && (force >= 0 || bsolve_staged_smem(ln, -force, sizeof(T)) <= kSmemMax)) ge = force;
    launch_bsolve_one<T>(ge, sys, ln, ngroups, pan, x, group_active, s);
    ++*nlaunch;
    if (dp.record || dp.stream != 0) CUDA_TRY(cudaEventRecord(ss.done[k], s));
    last[dp.stream] = k;
  }
  for (int q = 1; q < 4; ++q)
    if (last[q] >= 0) CUDA_TRY(cudaStreamWaitEvent(st, ss.done[last[q]], 0));
}

// Autotuner of the backward solve: per level, each lane count runs twice and the
// faster second run is kept.  The runs overwrite x, whose values do not change the
// timing; x is saved first and restored after.  Outside stream capture, once per
// (precision, groups).
template <typename T>
void tune_bsolve(LUSystem& sys, int ngroups, const T* pan, T* x, const int* group_active, cudaStream_t st) {
  if (sys.tuned_bs.count({Prec<T>::idx, ngroups})) return;
  const auto key = std::make_tuple(sys.fingerprint, Prec<T>::idx, ngroups);
  {
    TuneCache& tc = tune_cache();
    std::lock_guard<std::mutex> lock(tc.mu);
    const auto it = tc.bsolve.find(key);
    if (it != tc.bsolve.end()) {
      bool ok = it->second.size() == sys.bsolve_sched.size();
      for (size_t k = 0; ok && k < it->second.size(); ++k) {
        const int ge = it->second[k];
        ok = ge == 0 || ge == 16 || ge == 8 || ge == 4 || ge == 2 || ge == 1 ||
             ((ge == -8 || ge == -4 || ge == -2 || ge == -1) &&
              bsolve_staged_smem(sys.bsolve_sched[k], -ge, sizeof(T)) <= kSmemMax) ||
             // the fused near-root launch: the same code on every launch it replaces
             ((ge == kTopCode + 8 || ge == kTopCode + 4 || ge == kTopCode + 2 || ge == kTopCode + 1) &&
              (int)k >= sys.bs_top_from && ge == it->second.back());
        if ((int)k >= sys.bs_top_from && (it->second.back() >= kTopCode) != (ge >= kTopCode)) ok = false;
      }
      if (ok) {
        sys.tuned_bs[{Prec<T>::idx, ngroups}] = it->second;
        return;
      }
      tc.bsolve.erase(it);
    }
  }
  const size_t xbytes = (size_t)ngroups * 32 * sys.sym.n * sizeof(T);
  DevBuf saved;
  saved.alloc(xbytes);
  CUDA_TRY(cudaMemcpyAsync(saved.p, x, xbytes, cudaMemcpyDeviceToDevice, st));
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  std::vector<int> best(sys.bsolve_sched.size(), 0);
  const bool log = std::getenv("MPF_TUNE_LOG") != nullptr;
  double sum_best = 0.0, sum_heur = 0.0;
  try {
    for (int k = (int)sys.bsolve_sched.size() - 1; k >= 0; --k) {
      const Launch& ln = sys.bsolve_sched[k];
      const int h0 = bsolve_heuristic<T>(ln, ngroups);
      std::vector<int> cands{h0};
      for (int ge : {0, 16, 8, 4, 2, 1})
        if (ge != h0) cands.push_back(ge);
      // staged U panels (negative lane counts) where they fit in shared memory
      for (int gs : {8, 4, 2, 1})
        if (bsolve_staged_smem(ln, gs, sizeof(T)) <= kSmemMax) cands.push_back(-gs);
      float bt = 0.0f, ht = 0.0f;
      for (size_t i = 0; i < cands.size(); ++i) {
        launch_bsolve_one<T>(cands[i], sys, ln, ngroups, pan, x, group_active, st);
        CUDA_TRY(cudaEventRecord(e0, st));
        launch_bsolve_one<T>(cands[i], sys, ln, ngroups, pan, x, group_active, st);
        CUDA_TRY(cudaEventRecord(e1, st));
        CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        if (i == 0) ht = ms;
        if (i == 0 || ms < bt) {
          bt = ms;
          best[k] = cands[i];
        }
      }
      sum_best += bt;
      sum_heur += ht;
      if (log && std::getenv("MPF_TUNE_LOG")[0] == '2') {
        // U-panel rows and the front's x values read, the pivots' x written
        int64_t e = 0;
        for (int q = ln.offset; q < ln.offset + ln.count; ++q) {
          const int sn = sys.sym.lev_sn[q];
          e += (int64_t)sys.sym.sn_w[sn] * sys.sym.sn_f[sn] + sys.sym.sn_f[sn] + sys.sym.sn_w[sn];
        }
        const double bytes = (double)e * sizeof(T) * 32.0 * ngroups;
        std::fprintf(stderr, "mpf tune: n %d fp%d groups %d bsolve launch %d sn %d fcap %d: heuristic %.1f us, "
                     "best %.1f us (lanes %d), %.1f MB, %.0f GB/s\n", sys.sym.n, (int)sizeof(T) * 8, ngroups, k,
                     ln.count, ln.fcap, ht * 1e3, bt * 1e3, best[k], bytes * 1e-6, bytes / (bt * 1e-3) * 1e-9);
      }
    }
    // the near-root levels in one launch, against their tuned launches: the whole
    // backward solve (launch DAG included, where those launches overlap) timed both ways
    if (sys.top_nlev > 1 && (size_t)sys.top_fcap * 32 * 8 * sizeof(T) <= kSmemMax) {
      const auto key2 = std::make_pair(Prec<T>::idx, ngroups);
      auto whole = [&](const std::vector<int>& choice) {
        sys.tuned_bs[key2] = choice;
        int nl = 0;
        float best_ms = 0.0f;
        for (int rep = 0; rep < 3; ++rep) {
          CUDA_TRY(cudaEventRecord(e0, st));
          launch_bsolve<T>(sys, ngroups, pan, x, group_active, st, &nl);
          CUDA_TRY(cudaEventRecord(e1, st));
          CUDA_TRY(cudaEventSynchronize(e1));
          float ms = 0.0f;
          CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
          if (rep == 1 || (rep > 1 && ms < best_ms)) best_ms = ms;
        }
        return best_ms;
      };
      const float t_dag = whole(best);
      int best_ge = 0;
      float best_t = t_dag;
      for (int ge : {8, 4, 2, 1}) {
        std::vector<int> c = best;
        for (int k = sys.bs_top_from; k < (int)c.size(); ++k) c[k] = kTopCode + ge;
        const float t = whole(c);
        if (t < best_t) {
          best_t = t;
          best_ge = ge;
        }
      }
      sys.tuned_bs.erase(key2);
      if (log)
        std::fprintf(stderr, "mpf tune: n %d fp%d groups %d backward solve %.3f ms with %d near-root levels as %d "
                     "launches, %.3f ms as one launch (lanes %d)\n", sys.sym.n, (int)sizeof(T) * 8, ngroups, t_dag,
                     sys.top_nlev, (int)sys.bsolve_sched.size() - sys.bs_top_from, best_t, best_ge);
      if (best_ge > 0)
        for (int k = sys.bs_top_from; k < (int)sys.bsolve_sched.size(); ++k) best[k] = kTopCode + best_ge;
    }
    if (log)
      std::fprintf(stderr, "mpf tune: n %d fp%d groups %d backward solve heuristic %.3f ms, tuned %.3f ms\n",
                   sys.sym.n, (int)sizeof(T) * 8, ngroups, sum_heur, sum_best);
  } catch (...) {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    throw;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CUDA_TRY(cudaMemcpyAsync(x, saved.p, xbytes, cudaMemcpyDeviceToDevice, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  sys.tuned_bs[{Prec<T>::idx, ngroups}] = best;
  std::string line = "bsolve " + hex64(sys.fingerprint) + " " + std::to_string(Prec<T>::idx) + " " +
                     std::to_string(ngroups) + " " + std::to_string(best.size());
  for (int ge : best) line += " " + std::to_string(ge);
  TuneCache& tc = tune_cache();
  std::lock_guard<std::mutex> lock(tc.mu);
  if (tc.bsolve.emplace(key, best).second) append_tune_file(line + "\n");
}

template <typename T>
void launch_fsolve(const LUSystem& sys, int ngroups, const T* pan, T* cbr, T* x, const int* group_active,
                   cudaStream_t st, int* nlaunch) {
  for (const Launch& ln : sys.level_sched) {
    const long long ntasks = (long long)ln.count * ngroups;
    const int wpb = solve_warps<T>(ln.fcap, 32);
    long long blocks = std::min<long long>((ntasks + wpb - 1) / wpb, 148LL * 32);
    const size_t smem = (size_t)wpb * ln.fcap * 32 * sizeof(T);
    k_mf_fsolve<T><<<(unsigned)blocks, 32 * wpb, smem, st>>>(sys.dev(), sys.lev_sn.as<int>() + ln.offset, ln.count, ngroups,
                                                        ln.fcap, pan, cbr, x, group_active);
    CUDA_TRY(cudaGetLastError());
    ++*nlaunch;
  }
}

// ------------------------------------------------------------------ timing
enum Family { FAM_MIS = 0, FAM_JAC, FAM_FACT, FAM_SOLVE, FAM_UPD, FAM_OTHER, FAM_N };

struct EventTimer {
  std::vector<cudaEvent_t> pool;
  std::vector<std::pair<int, int>> marks;  // (family, event index of start); end = start + 1
  size_t used = 0;
  cudaStream_t st = nullptr;
  ~EventTimer() {
    for (auto e : pool) cudaEventDestroy(e);
  }
  void reset(cudaStream_t s) {
    st = s;
    used = 0;
    marks.clear();
  }
  cudaEvent_t next() {
    if (used == pool.size()) {
      cudaEvent_t e;
      CUDA_TRY(cudaEventCreate(&e));
      pool.push_back(e);
    }
    return pool[used++];
  }
  int begin(int fam) {
    const int i = (int)used;
    CUDA_TRY(cudaEventRecord(next(), st));
    next();
    marks.push_back({fam, i});
    return i;
  }
  void end(int i) { CUDA_TRY(cudaEventRecord(pool[i + 1], st)); }
  void collect(double* ms) {
    for (int f = 0; f < FAM_N; ++f) ms[f] = 0.0;
    for (auto& m : marks) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, pool[m.second], pool[m.second + 1]) == cudaSuccess) ms[m.first] += t;
    }
  }
};

}  // namespace

// ------------------------------------------------------------------ handle
struct mpf_handle {
  std::string err;
  mpf_options opt;
  int device = 0;
  cudaStream_t own_stream = nullptr;
  GridSymbolic g;
  // shared device arrays
  DevBuf y_rowptr, y_col, y_val, y_diag, br_ft, rating, br_ypos, br_y, sbus0, v0, mis_rows, jvar, jpos;
  LUSystem jac;
  LUSystem bp[2], bpp[2];
  FDData fdp[2], fdpp[2];
  DevBuf fdvar;
  bool fd_ready[2] = {false, false};
  // cases
  int ncases = 0, ngroups = 0, maxk = 0;
  DevBuf out_br, sbus_case, V, Ibus, status, iters, maxmis, facc, group_active, any_active, it_ctr;
  DevBuf vout, small_out;
  DevBuf eval_acc;  // mpf_mismatch accumulator, allocated on first use
  DevBuf br_dy;     // per branch dY/dg for (ff, ft, tf, tt), adjoint
  // adjoint refinement (FP32 factors): J^T by column (A-array position, row), the FP64
  // right-hand side and solution, allocated on the first mixed-precision adjoint
  DevBuf adj_colptr, adj_colent, adj_b64, adj_lam64;
  DevBuf adj_status;  // statuses the adjoint's refactorisation may write (kept apart)
  // several islands (grids) in one handle: per-bus / per-branch islands, and per
  // batch the island of each group and the case <-> lane maps
  DevBuf bus_island, br_island, group_island, lane_case, case_lane;
  std::vector<int> h_lane_case;
  // cases whose outages island PV/PQ buses (no path to a slack): per lane, uploaded
  // only when the batch has one; the grid's bridges make the single-outage check O(1)
  DevBuf case_cut;
  std::vector<uint8_t> is_bridge;
  // reactive limits: PV buses with limits (a Vm variable each), their limits, and per
  // batch the PV / switched state of each case
  int nsw = 0;
  std::vector<char> vm_free;         // per bus: PV bus with limits
  DevBuf sw_index, sw_bus, q_lim, base_type, pv_on, q_fix, q_flag, iter_base;
  std::vector<mpf_bus> buses;        // the grid as given (controls read base values)
  std::vector<mpf_branch> branches;
  // per-case controls of the current cases (mpf_set_controls)
  struct Controls {
    int nc = 0, navr = 0, noltc = 0, nshc = 0, nslot = 0;
    DevBuf val, avr, oltc, oltc_par, shc, shc_base, slot_ptr, slot_ent, y_slot, br_ctl, dy, bry, bdy, fdpos[2];
    void clear() { nc = navr = noltc = nshc = nslot = 0; }
    size_t bytes() const {
      const DevBuf* all[] = {&val, &avr, &oltc, &oltc_par, &shc, &shc_base, &slot_ptr, &slot_ent,
                             &y_slot, &br_ctl, &dy, &bry, &bdy, &fdpos[0], &fdpos[1]};
      size_t b = 0;
      for (auto p : all) b += p->bytes;
      return b;
    }
  } ctl;
  bool have_cases = false, have_results = false;
  int last_alg = -1, last_prec = -1;
  cudaStream_t last_stream = nullptr;  // stream of the last solve / result copy
  int* h_any = nullptr;  // pinned
  EventTimer timer;
  mpf_timing timing;
  // captured Newton iteration per precision [FP64, FP32]
  struct IterGraph {
    cudaGraph_t graph[4] = {};
    cudaGraphExec_t exec[4] = {};
    const void* key[4] = {nullptr, nullptr, nullptr, nullptr};
    DevGrid dkey;  // the grid descriptor the kernels were captured with
    int ngroups = 0, launches[4] = {0, 0, 0, 0};
    // use_graph = 2: the whole Newton loop as one graph (a condition kernel, then a
    // while node whose body is the four parts and the condition kernel again)
    cudaGraph_t loop_graph = nullptr;
    cudaGraphExec_t loop_exec = nullptr;
    int loop_launches = 0;  // launches per body run
    bool captured(bool dev_loop) const { return dev_loop ? loop_exec != nullptr : exec[0] != nullptr; }
    void release() {
      for (int k = 0; k < 4; ++k) {
        if (exec[k]) cudaGraphExecDestroy(exec[k]);
        if (graph[k]) cudaGraphDestroy(graph[k]);
        exec[k] = nullptr;
        graph[k] = nullptr;
      }
      if (loop_exec) cudaGraphExecDestroy(loop_exec);
      if (loop_graph) cudaGraphDestroy(loop_graph);  // also frees the while node's body
      loop_exec = nullptr;
      loop_graph = nullptr;
      ngroups = 0;
    }
  } nr_graph[2];
  cudaEvent_t t0 = nullptr, t1 = nullptr;

  DevGrid dev() const {
    DevGrid d;
    std::memset(&d, 0, sizeof(d));  // byte-comparable (graph key)
    d.nb = g.nb;
    d.nfree = (int)g.mis_rows.size();
    d.ngroups = ngroups;
    d.n_jac = jac.sym.n;
    d.nA_jac = jac.nA;
    d.angle_mode = opt.angle_mode;
    d.y_rowptr = y_rowptr.as<int>();
    d.y_col = y_col.as<int>();
    d.y_val = y_val.as<double2>();
    d.y_diag = y_diag.as<int>();
    d.br_ypos = br_ypos.as<int4>();
    d.br_ft = br_ft.as<int2>();
    d.br_y = br_y.as<double2>();
    d.sbus0 = sbus0.as<double2>();
    d.sbus_case = sbus_case.p ? sbus_case.as<double2>() : nullptr;
    d.v0 = v0.as<double2>();
    d.mis_rows = mis_rows.as<int>();
    d.jvar = jvar.as<int2>();
    d.jpos = jpos.as<int4>();
    d.out_br = out_br.as<int>();
    d.V = V.as<double2>();
    d.Ibus = Ibus.as<double2>();
    d.status = status.as<int>();
    d.iters = iters.as<int>();
    d.maxmis = maxmis.as<double>();
    d.facc = facc.as<unsigned long long>();
    d.group_active = group_active.as<int>();
    d.any_active = any_active.as<int>();
    d.it_ptr = it_ctr.as<int>();
    if (g.n_islands > 1 && group_island.p) {
      d.bus_island = bus_island.as<int>();
      d.br_island = br_island.as<int>();
      d.group_island = group_island.as<int>();
      d.lane_case = lane_case.as<int>();
      d.case_lane = case_lane.as<int>();
    }
    if (nsw > 0 && pv_on.p) {
      d.nsw = nsw;
      d.sw_index = sw_index.as<int>();
      d.pv_on = pv_on.as<unsigned char>();
      d.q_fix = q_fix.as<double>();
      d.iter_base = iter_base.as<int>();
    }
    if (case_cut.p) d.case_cut = case_cut.as<unsigned char>();
    if (ctl.nc > 0) {
      d.nslot = ctl.nslot;
      d.noltc = ctl.noltc;
      if (ctl.nslot > 0) {
        d.y_slot = ctl.y_slot.as<int>();
        d.ctl_dy = ctl.dy.as<double2>();
      }
      if (ctl.noltc > 0) {
        d.br_ctl = ctl.br_ctl.as<int>();
        d.ctl_bry = ctl.bry.as<double2>();
        d.ctl_bdy = ctl.bdy.as<double2>();
      }
    }
    return d;
  }

  DevCtl devctl() const {
    DevCtl t;
    std::memset(&t, 0, sizeof(t));
    t.nc = ctl.nc;
    t.navr = ctl.navr;
    t.noltc = ctl.noltc;
    t.nshc = ctl.nshc;
    t.nslot = ctl.nslot;
    t.val = ctl.val.as<double>();
    t.avr = ctl.avr.as<int2>();
    t.oltc = ctl.oltc.as<int2>();
    t.oltc_par = ctl.oltc_par.as<double>();
    t.shc = ctl.shc.as<int2>();
    t.shc_base = ctl.shc_base.as<double>();
    t.slot_ptr = ctl.slot_ptr.as<int>();
    t.slot_ent = ctl.slot_ent.as<int2>();
    return t;
  }

  size_t device_bytes() const {
    size_t b = 0;
    const DevBuf* all[] = {&y_rowptr, &y_col, &y_val, &y_diag, &br_ft, &rating, &br_ypos, &br_y, &sbus0, &v0, &mis_rows, &jvar, &jpos,
                           &out_br, &sbus_case, &V, &Ibus, &status, &iters, &maxmis, &facc, &group_active,
                           &any_active, &vout, &small_out, &fdvar, &eval_acc, &it_ctr, &br_dy,
                           &adj_status, &bus_island, &br_island, &group_island, &lane_case, &case_lane,
                           &sw_index, &sw_bus, &q_lim, &base_type, &pv_on, &q_fix, &q_flag, &iter_base, &case_cut,
                           &adj_colptr, &adj_colent, &adj_b64, &adj_lam64};
    for (auto p : all) b += p->bytes;
    b += ctl.bytes();
    const LUSystem* systems[] = {&jac, &bp[0], &bp[1], &bpp[0], &bpp[1]};
    for (auto s : systems) {
      for (int p = 0; p < 2; ++p) b += s->A[p].bytes + s->pan[p].bytes + s->cb[p].bytes + s->cbr[p].bytes + s->x[p].bytes;
      const DevBuf* idx[] = {&s->sn_w, &s->sn_f, &s->sn_rptr, &s->sn_rows, &s->child_ptr, &s->child_list,
                             &s->sn_parent, &s->rel_ptr, &s->relmap, &s->ah_ptr, &s->ah_loc, &s->pan_off,
                             &s->cb_off, &s->cbr_off, &s->lev_sn, &s->top_sn, &s->top_lev_ptr,
                             &s->child_ref, &s->cb_in};
      for (auto q : idx) b += q->bytes;
    }
    for (int v = 0; v < 2; ++v) b += fdp[v].base.bytes + fdp[v].br_apos.bytes + fdp[v].br_bval.bytes +
                                     fdpp[v].base.bytes + fdpp[v].br_apos.bytes + fdpp[v].br_bval.bytes;
    return b;
  }
};

namespace {

// The Newton system's device arrays: variable map, Jacobian positions, the LU system.
void upload_newton(mpf_handle* h) {
  const GridSymbolic& g = h->g;
  std::vector<int2> jv(g.nb);
  for (int i = 0; i < g.nb; ++i) jv[i] = make_int2(g.var_va[i], g.var_vm[i]);
  upload(h->jvar, jv);
  std::vector<int4> jp(g.y_col.size());
  for (size_t p = 0; p < jp.size(); ++p)
    jp[p] = make_int4(g.jpos[4 * p], g.jpos[4 * p + 1], g.jpos[4 * p + 2], g.jpos[4 * p + 3]);
  upload(h->jpos, jp);
  {
    // J^T by column for the adjoint refinement: entry (row, col) of each A-array slot
    // (jac_entry's quadrants: (P_i, Va_j), (P_i, Vm_j), (Q_i, Va_j), (Q_i, Vm_j))
    std::vector<std::array<int, 3>> ent;  // (col, row, A-array position)
    for (int i = 0; i < g.nb; ++i)
      for (int p = g.y_rowptr[i]; p < g.y_rowptr[i + 1]; ++p) {
        const int j = g.y_col[p];
        const int rows[4] = {g.var_va[i], g.var_va[i], g.var_vm[i], g.var_vm[i]};
        const int cols[4] = {g.var_va[j], g.var_vm[j], g.var_va[j], g.var_vm[j]};
        for (int q = 0; q < 4; ++q)
          if (g.jpos[4 * p + q] >= 0) ent.push_back({cols[q], rows[q], g.jpos[4 * p + q]});
      }
    std::sort(ent.begin(), ent.end());
    std::vector<int> cp(g.jac.n + 1, 0);
    std::vector<int2> ce(ent.size());
    for (size_t e = 0; e < ent.size(); ++e) {
      ++cp[ent[e][0] + 1];
      ce[e] = make_int2(ent[e][2], ent[e][1]);
    }
    for (int c = 0; c < g.jac.n; ++c) cp[c + 1] += cp[c];
    upload(h->adj_colptr, cp);
    upload(h->adj_colent, ce);
  }
  if (g.n_islands > 1) {
    std::vector<int> vi(g.jac.n, -1);
    for (int i = 0; i < g.nb; ++i) {
      if (g.var_va[i] >= 0) vi[g.var_va[i]] = g.bus_island[i];
      if (g.var_vm[i] >= 0) vi[g.var_vm[i]] = g.bus_island[i];
    }
    h->jac.setup(g.jac, g.ah_ptr, g.ah_loc, g.nnz_jac, &vi);
  } else {
    h->jac.setup(g.jac, g.ah_ptr, g.ah_loc, g.nnz_jac);
  }
}

int fail(mpf_handle* h, int code, const std::string& msg) {
  if (h) h->err = msg;
  return code;
}

template <class F>
int guarded(mpf_handle* h, F&& f) {
  try {
    return f();
  } catch (const MpfError& e) {
    return fail(h, e.code, e.msg);
  } catch (const std::bad_alloc&) {
    return fail(h, MPF_ERR_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(h, MPF_ERR_INTERNAL, e.what());
  }
}

void upload_fd(mpf_handle* h, int variant) {
  if (h->fd_ready[variant]) return;
  const GridSymbolic& g = h->g;
  auto setup_one = [&](const GridSymbolic::FDSystem& fs, LUSystem& sys, FDData& fd) {
    std::vector<int> vi;
    if (g.n_islands > 1) {
      vi.assign(fs.lu.n, -1);
      for (int i = 0; i < g.nb; ++i)
        if (fs.var[i] >= 0) vi[fs.var[i]] = g.bus_island[i];
    }
    sys.setup(fs.lu, fs.ah_ptr, fs.ah_loc, (int)fs.base.size(), g.n_islands > 1 ? &vi : nullptr);
    sys.group_island = h->jac.group_island;
    upload(fd.base, fs.base);
    std::vector<int4> pos(g.nbr);
    std::vector<double4> val(g.nbr);
    for (int e = 0; e < g.nbr; ++e) {
      pos[e] = make_int4(fs.br_pos[4 * e], fs.br_pos[4 * e + 1], fs.br_pos[4 * e + 2], fs.br_pos[4 * e + 3]);
      val[e] = make_double4(fs.br_val[4 * e], fs.br_val[4 * e + 1], fs.br_val[4 * e + 2], fs.br_val[4 * e + 3]);
    }
    upload(fd.br_apos, pos);
    upload(fd.br_bval, val);
  };
  setup_one(g.bp[variant], h->bp[variant], h->fdp[variant]);
  setup_one(g.bpp[variant], h->bpp[variant], h->fdpp[variant]);
  if (!h->fdvar.p) {
    std::vector<int2> fv(g.nb);
    for (int i = 0; i < g.nb; ++i) fv[i] = make_int2(g.bp[0].var[i], g.bpp[0].var[i]);
    upload(h->fdvar, fv);
  }
  h->fd_ready[variant] = true;
}

dim3 row_grid(const mpf_handle* h) {
  const int nfree = (int)h->g.mis_rows.size();
  return dim3((unsigned)((nfree + kRowsPerBlock - 1) / kRowsPerBlock), (unsigned)h->ngroups);
}

bool any_active(mpf_handle* h, cudaStream_t st) {
  CUDA_TRY(cudaMemcpyAsync(h->h_any, h->any_active.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return *h->h_any != 0;
}

template <typename T, bool QL>
void launch_mismatch_nr_q(const DevGrid& d, dim3 rg, cudaStream_t st, T* x, T* A, bool jac) {
  const bool ctl = d.y_slot != nullptr;
  if (jac && ctl) k_mismatch_nr<T, true, true, QL><<<rg, 256, 0, st>>>(d, x, A);
  else if (jac) k_mismatch_nr<T, true, false, QL><<<rg, 256, 0, st>>>(d, x, A);
  else if (ctl) k_mismatch_nr<T, false, true, QL><<<rg, 256, 0, st>>>(d, x, A);
  else k_mismatch_nr<T, false, false, QL><<<rg, 256, 0, st>>>(d, x, A);
  CUDA_TRY(cudaGetLastError());
}

// Newton mismatch (with the Jacobian when jac), in its variant with or without
// per-case Ybus controls and reactive limits
template <typename T>
void launch_mismatch_nr(const DevGrid& d, dim3 rg, cudaStream_t st, T* x, T* A, bool jac) {
  if (d.sw_index) launch_mismatch_nr_q<T, true>(d, rg, st, x, A, jac);
  else launch_mismatch_nr_q<T, false>(d, rg, st, x, A, jac);
}

// AVR controls: the set-points of the current cases into V (after k_init)
int apply_avr(mpf_handle* h, cudaStream_t st) {
  if (h->ctl.nc == 0 || h->ctl.navr == 0) return 0;
  const size_t tot = (size_t)h->ngroups * h->ctl.navr * 32;
  k_ctl_vm<<<(unsigned)std::min<size_t>(148 * 8, tot / 256 + 1), 256, 0, st>>>(h->dev(), h->devctl());
  CUDA_TRY(cudaGetLastError());
  return 1;
}

void check(mpf_handle* h, cudaStream_t st, int it, int max_it, int* nl) {
  CUDA_TRY(cudaMemsetAsync(h->any_active.p, 0, sizeof(int), st));
  const int nl_lanes = h->ngroups * 32;
  k_check<<<(nl_lanes + 255) / 256, 256, 0, st>>>(h->dev(), it, max_it, h->opt.tol);
  CUDA_TRY(cudaGetLastError());
  ++*nl;
}

// One Newton iteration after a check that left cases running, in four parts:
//   0 factorisation with the forward substitution fused
//   1 backward substitution
//   2 voltage update
//   3 the next mismatch (with the Jacobian of the new point) and its check
template <typename T>
int enqueue_nr_part(mpf_handle* h, int part, cudaStream_t st, T* A, T* pan, T* cb, T* cbr, T* x) {
  LUSystem& J = h->jac;
  const DevGrid d = h->dev();
  const dim3 rg = row_grid(h);
  int nl = 0;
  if (part == 0) {
    launch_factor<T>(J, h->ngroups, A, pan, cb, cbr, x, d.status, d.group_active, 1, st, &nl);
  } else if (part == 1) {
    launch_bsolve<T>(J, h->ngroups, pan, x, d.group_active, st, &nl);
  } else if (part == 2) {
    k_update_nr<T><<<rg, 256, 0, st>>>(d, x);
    CUDA_TRY(cudaGetLastError());
    ++nl;
  } else {
    launch_mismatch_nr<T>(d, rg, st, x, A, true);
    CUDA_TRY(cudaMemsetAsync(h->any_active.p, 0, sizeof(int), st));
    const int nl_lanes = h->ngroups * 32;
    k_check<<<(nl_lanes + 255) / 256, 256, 0, st>>>(d, -1, h->opt.max_it_nr, h->opt.tol);
    CUDA_TRY(cudaGetLastError());
    nl += 2;
  }
  return nl;
}

template <typename T>
void solve_nr(mpf_handle* h, cudaStream_t st) {
  constexpr int P = Prec<T>::idx;
  LUSystem& J = h->jac;
  J.ensure_values(P, h->ngroups);
  T* A = J.A[P].as<T>();
  T* pan = J.pan[P].as<T>();
  T* cb = J.cb[P].as<T>();
  T* cbr = J.cbr[P].as<T>();
  T* x = J.x[P].as<T>();
  const DevGrid d = h->dev();
  const dim3 rg = row_grid(h);
  int nl = 0;
  EventTimer& tm = h->timer;
  int ev = tm.begin(FAM_OTHER);
  k_init<<<std::min(148 * 8, (int)((size_t)h->ngroups * h->g.nb * 32 / 256 + 1)), 256, 0, st>>>(d, h->ncases);
  CUDA_TRY(cudaGetLastError());
  ++nl;
  nl += apply_avr(h, st);
  if (h->nsw > 0) {
    const size_t tot = (size_t)h->ngroups * 32 * h->nsw;
    k_qlim_reset<<<(unsigned)std::min<size_t>(148 * 8, tot / 256 + 1), 256, 0, st>>>(d);
    CUDA_TRY(cudaGetLastError());
    ++nl;
  }
  tm.end(ev);
  const int max_it = h->opt.max_it_nr;
  static const int kFam[4] = {FAM_FACT, FAM_SOLVE, FAM_UPD, FAM_MIS};
  int it_total = 0;
  auto& gph = h->nr_graph[P];
  // one Newton run over the running cases: mismatch at the current voltages, check,
  // then iterations until no case is running (first: also tune and capture)
  auto run_newton = [&](bool first) {
  if (!first) CUDA_TRY(cudaMemsetAsync(h->it_ctr.p, 0, sizeof(int), st));
  ev = tm.begin(FAM_MIS);
  launch_mismatch_nr<T>(d, rg, st, x, A, max_it > 0);
  ++nl;
  tm.end(ev);
  ev = tm.begin(FAM_OTHER);
  check(h, st, 0, max_it, &nl);
  tm.end(ev);
  int it = 0;
  // pick the factorisation kernels of this batch size (first solve only), before
  // the iteration is captured
  if (first && h->opt.autotune && max_it > 0 && any_active(h, st)) {
    tune_factor<T>(J, h->ngroups, A, pan, cb, cbr, x, d.status, d.group_active, st);
    tune_bsolve<T>(J, h->ngroups, pan, x, d.group_active, st);
  }
  const bool dev_loop = h->opt.use_graph == 2;
  if (h->opt.use_graph) {
    // the captured kernels hold every device pointer of d by value: capture again
    // when any of them (or the LU buffers) changed since
    const void* key[4] = {A, pan, cb, x};
    if ((gph.exec[0] || gph.loop_exec) &&
        (gph.ngroups != h->ngroups || std::memcmp(gph.key, key, sizeof(key)) != 0 ||
         std::memcmp(&gph.dkey, &d, sizeof(d)) != 0))
      gph.release();
    if (!gph.captured(dev_loop)) {
      // capture on a private stream (the caller's may be the legacy one)
      cudaStream_t cs;
      CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      if (!dev_loop) {
        for (int part = 0; part < 4; ++part) {
          CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
          gph.launches[part] = enqueue_nr_part<T>(h, part, cs, A, pan, cb, cbr, x);
          CUDA_TRY(cudaStreamEndCapture(cs, &gph.graph[part]));
          CUDA_TRY(cudaGraphInstantiate(&gph.exec[part], gph.graph[part], 0));
        }
      } else {
        // head: the condition at entry; then a while node running the four parts and
        // the condition again.  The update kernel counts iterations on the device, so
        // the loop ends after at most max_it bodies whatever the cases do.
        CUDA_TRY(cudaGraphCreate(&gph.loop_graph, 0));
        cudaGraphConditionalHandle hc;
        CUDA_TRY(cudaGraphConditionalHandleCreate(&hc, gph.loop_graph, 0, 0));
        CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, gph.loop_graph, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
        k_loop_cond<<<1, 1, 0, cs>>>(hc, h->any_active.as<int>(), d.it_ptr, max_it);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamEndCapture(cs, &gph.loop_graph));
        cudaGraphNode_t head;
        size_t nn = 1;
        CUDA_TRY(cudaGraphGetNodes(gph.loop_graph, &head, &nn));
        if (nn != 1) throw MpfError{MPF_ERR_CUDA, "device loop: the head graph should hold one kernel"};
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = hc;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t loop;
        CUDA_TRY(cudaGraphAddNode(&loop, gph.loop_graph, &head, 1, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
        int nlb = 0;
        for (int part = 0; part < 4; ++part) nlb += enqueue_nr_part<T>(h, part, cs, A, pan, cb, cbr, x);
        k_loop_cond<<<1, 1, 0, cs>>>(hc, h->any_active.as<int>(), d.it_ptr, max_it);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaStreamEndCapture(cs, &body));
        CUDA_TRY(cudaGraphInstantiate(&gph.loop_exec, gph.loop_graph, 0));
        gph.loop_launches = nlb + 1;
      }
      CUDA_TRY(cudaStreamDestroy(cs));
      std::memcpy(gph.key, key, sizeof(key));
      std::memcpy(&gph.dkey, &d, sizeof(d));
      gph.ngroups = h->ngroups;
    }
  }
  if (dev_loop) {
    // one launch for all iterations; their count is read back once
    const int e = tm.begin(FAM_OTHER);
    CUDA_TRY(cudaGraphLaunch(gph.loop_exec, st));
    tm.end(e);
    CUDA_TRY(cudaMemcpyAsync(h->h_any, d.it_ptr, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    it = *h->h_any;
    nl += 1 + it * gph.loop_launches;
  }
  while (!dev_loop && it < max_it && any_active(h, st)) {
    int e[4];
    for (int part = 0; part < 4; ++part) {
      e[part] = tm.begin(kFam[part]);
      if (h->opt.use_graph) {
        CUDA_TRY(cudaGraphLaunch(gph.exec[part], st));
        nl += gph.launches[part];
      } else {
        nl += enqueue_nr_part<T>(h, part, st, A, pan, cb, cbr, x);
      }
      tm.end(e[part]);
    }
    ++it;
  }
  it_total += it;
  };
  run_newton(true);
  // reactive limits: switch the violating PV buses of converged cases to PQ and run
  // those cases again from their voltages, until no case has a new violation
  if (h->nsw > 0 && max_it > 0) {
    const size_t tot = (size_t)h->ngroups * h->nsw * 32;
    const int lanes = h->ngroups * 32;
    for (int round = 0; round < kMaxQRounds; ++round) {
      CUDA_TRY(cudaMemsetAsync(h->any_active.p, 0, sizeof(int), st));
      k_qlim_check<<<(unsigned)std::min<size_t>(148 * 8, tot / 256 + 1), 256, 0, st>>>(
          d, h->sw_bus.as<int>(), h->q_lim.as<double2>(), h->q_flag.as<int>());
      k_qlim_restart<<<(lanes + 255) / 256, 256, 0, st>>>(d, h->q_flag.as<int>());
      CUDA_TRY(cudaGetLastError());
      nl += 2;
      if (!any_active(h, st)) break;
      run_newton(false);
    }
  }
  h->timing.launches = nl;
  h->timing.iterations_max = it_total;
}

template <typename T>
void solve_fd(mpf_handle* h, cudaStream_t st, int variant) {
  constexpr int P = Prec<T>::idx;
  upload_fd(h, variant);
  LUSystem& Bp = h->bp[variant];
  LUSystem& Bpp = h->bpp[variant];
  Bp.ensure_values(P, h->ngroups);
  Bpp.ensure_values(P, h->ngroups);
  const DevGrid d = h->dev();
  DevFD fdd;
  fdd.n_bp = Bp.sym.n;
  fdd.n_bpp = Bpp.sym.n;
  fdd.fdvar = h->fdvar.as<int2>();
  const dim3 rg = row_grid(h);
  int nl = 0;
  EventTimer& tm = h->timer;
  int ev = tm.begin(FAM_OTHER);
  k_init<<<std::min(148 * 8, (int)((size_t)h->ngroups * h->g.nb * 32 / 256 + 1)), 256, 0, st>>>(d, h->ncases);
  CUDA_TRY(cudaGetLastError());
  ++nl;
  nl += apply_avr(h, st);
  tm.end(ev);
  // B' and B'' of every case, factorised once and reused by all iterations
  ev = tm.begin(FAM_JAC);
  LUSystem* systems[2] = {&Bp, &Bpp};
  FDData* fds[2] = {&h->fdp[variant], &h->fdpp[variant]};
  for (int k = 0; k < 2; ++k) {
    LUSystem& S = *systems[k];
    const size_t total = (size_t)h->ngroups * S.nA * 32;
    k_fd_base<T><<<(unsigned)std::min<size_t>(148 * 16, total / 256 + 1), 256, 0, st>>>(
        h->ngroups, S.nA, fds[k]->base.as<double>(), S.A[P].as<T>());
    CUDA_TRY(cudaGetLastError());
    k_fd_outage<T><<<(h->ngroups * 32 + 127) / 128, 128, 0, st>>>(d, S.nA, fds[k]->br_apos.as<int4>(),
                                                                    fds[k]->br_bval.as<double4>(), S.A[P].as<T>());
    CUDA_TRY(cudaGetLastError());
    nl += 2;
    if (k == 1 && h->ctl.nc > 0 && h->ctl.nslot > 0) {
      const size_t tot = (size_t)h->ngroups * h->ctl.nslot * 32;
      k_fd_ctl<T><<<(unsigned)std::min<size_t>(148 * 8, tot / 256 + 1), 256, 0, st>>>(
          d, h->devctl(), variant, S.nA, h->ctl.fdpos[variant].as<int>(), fds[k]->br_bval.as<double4>(), S.A[P].as<T>());
      CUDA_TRY(cudaGetLastError());
      ++nl;
    }
  }
  tm.end(ev);
  if (h->opt.autotune)
    for (int k = 0; k < 2; ++k) {
      LUSystem& S = *systems[k];
      tune_factor<T>(S, h->ngroups, S.A[P].as<T>(), S.pan[P].as<T>(), S.cb[P].as<T>(), S.cbr[P].as<T>(),
                     S.x[P].as<T>(), d.status, d.group_active, st);
    }
  ev = tm.begin(FAM_FACT);
  for (int k = 0; k < 2; ++k) {
    LUSystem& S = *systems[k];
    launch_factor<T>(S, h->ngroups, S.A[P].as<T>(), S.pan[P].as<T>(), S.cb[P].as<T>(), S.cbr[P].as<T>(),
                     S.x[P].as<T>(), d.status, d.group_active, 0, st, &nl);
  }
  tm.end(ev);
  if (h->opt.autotune)
    for (int k = 0; k < 2; ++k) {
      LUSystem& S = *systems[k];
      tune_bsolve<T>(S, h->ngroups, S.pan[P].as<T>(), S.x[P].as<T>(), d.group_active, st);
    }
  T* xp = Bp.x[P].as<T>();
  T* xq = Bpp.x[P].as<T>();
  const int max_it = h->opt.max_it_fd;
  auto mismatch = [&]() {
    int e2 = tm.begin(FAM_MIS);
    k_mismatch_fd<T><<<rg, 256, 0, st>>>(d, fdd, xp, xq);
    CUDA_TRY(cudaGetLastError());
    ++nl;
    tm.end(e2);
  };
  mismatch();
  ev = tm.begin(FAM_OTHER);
  check(h, st, 0, max_it, &nl);
  tm.end(ev);
  int i = 0;
  if (any_active(h, st)) {
    while (i < max_it) {
      ++i;
      for (int half = 0; half < 2; ++half) {
        LUSystem& S = half == 0 ? Bp : Bpp;
        ev = tm.begin(FAM_SOLVE);
        launch_fsolve<T>(S, h->ngroups, S.pan[P].as<T>(), S.cbr[P].as<T>(), S.x[P].as<T>(), d.group_active, st, &nl);
        launch_bsolve<T>(S, h->ngroups, S.pan[P].as<T>(), S.x[P].as<T>(), d.group_active, st, &nl);
        tm.end(ev);
        ev = tm.begin(FAM_UPD);
        k_update_fd<T><<<rg, 256, 0, st>>>(d, fdd, xp, xq, half);
        CUDA_TRY(cudaGetLastError());
        ++nl;
        tm.end(ev);
        mismatch();
        ev = tm.begin(FAM_OTHER);
        // after the P half only convergence retires a case (fdpf.h:529-540); the
        // iteration limit is tested after the Q half
        check(h, st, i, half == 0 ? INT32_MAX : max_it, &nl);
        tm.end(ev);
        if (!any_active(h, st)) break;
      }
      if (*h->h_any == 0) break;
    }
  }
  h->timing.launches = nl;
  h->timing.iterations_max = i;
}

}  // namespace

// ------------------------------------------------------------------ fixed-scratch mismatch
// mpf_mismatch_noalloc keeps its per-case accumulator in this file-scope device array
// instead of handle-owned memory, so the call never reaches an allocator.  The array
// exists on every GPU that loads the library (512 KB each) until the process exits.
// Host code may not use g_noalloc_acc as an address (it names a host-side shadow);
// the device address comes from cudaGetSymbolAddress, once per device.
constexpr int kNoAllocMaxCases = 65536;
static __device__ __align__(256) unsigned long long g_noalloc_acc[kNoAllocMaxCases];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_acc on the current device (which must be `device`).
cudaError_t noalloc_scratch(int device, unsigned long long** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[device]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_acc);
    if (e != cudaSuccess) return e;
    g_noalloc_ptr[device] = static_cast<unsigned long long*>(p);
  }
  *out = g_noalloc_ptr[device];
  return cudaSuccess;
}
}  // namespace

// ------------------------------------------------------------------ adjoint
template <typename T>
void launch_fsolve_t(const LUSystem& sys, int ngroups, const T* pan, T* cbr, T* x, const int* group_active,
                     cudaStream_t st) {
  for (const Launch& ln : sys.level_sched) {
    const long long ntasks = (long long)ln.count * ngroups;
    const int wpb = solve_warps<T>(ln.fcap, 32);
    const long long blocks = std::min<long long>((ntasks + wpb - 1) / wpb, 148LL * 32);
    const size_t smem = (size_t)wpb * ln.fcap * 32 * sizeof(T);
    k_mf_fsolve_t<T><<<(unsigned)blocks, 32 * wpb, smem, st>>>(sys.dev(), sys.lev_sn.as<int>() + ln.offset, ln.count,
                                                          ngroups, ln.fcap, pan, cbr, x, group_active);
    CUDA_TRY(cudaGetLastError());
  }
}

template <typename T>
void launch_bsolve_t(const LUSystem& sys, int ngroups, const T* pan, T* x, const int* group_active, cudaStream_t st) {
  for (int k = (int)sys.level_sched.size() - 1; k >= 0; --k) {
    const Launch& ln = sys.level_sched[k];
    const long long ntasks = (long long)ln.count * ngroups;
    const int wpb = solve_warps<T>(ln.fcap, 32);
    const long long blocks = std::min<long long>((ntasks + wpb - 1) / wpb, 148LL * 32);
    const size_t smem = (size_t)wpb * ln.fcap * 32 * sizeof(T);
    k_mf_bsolve_t<T><<<(unsigned)blocks, 32 * wpb, smem, st>>>(sys.dev(), sys.lev_sn.as<int>() + ln.offset, ln.count,
                                                          ngroups, ln.fcap, pan, x, group_active);
    CUDA_TRY(cudaGetLastError());
  }
}

// Refinement steps of the adjoint solved with FP32 factors (each reduces the error by
// about the FP32 LU's own accuracy, ~1e-4 relative on the 1354-bus grid).
constexpr int kAdjRefine = 2;

// J of the solved point refactorised in T, then J^T lambda = dL/dx by U^T (bottom-up)
// and L^T (top-down) substitutions, then the bus and branch gradients.
template <typename T>
void adjoint_impl(mpf_handle* h, cudaStream_t st, double* gp, double* gq, double* gg, double* gb) {
  constexpr int P = Prec<T>::idx;
  LUSystem& J = h->jac;
  J.ensure_values(P, h->ngroups);
  T* A = J.A[P].as<T>();
  T* pan = J.pan[P].as<T>();
  T* x = J.x[P].as<T>();
  const int lanes = h->ngroups * 32;
  if (!h->adj_status.p || h->adj_status.bytes < lanes * sizeof(int)) h->adj_status.alloc(lanes * sizeof(int));
  CUDA_TRY(cudaMemsetAsync(h->adj_status.p, 0, lanes * sizeof(int), st));  // all RUNNING: a sink for bad pivots
  DevGrid d = h->dev();
  k_fill_int<<<(h->ngroups + 255) / 256, 256, 0, st>>>(d.group_active, h->ngroups, 1);
  CUDA_TRY(cudaGetLastError());
  const dim3 rg = row_grid(h);
  launch_mismatch_nr<T>(d, rg, st, x, A, true);
  int nl = 0;
  launch_factor<T>(J, h->ngroups, A, pan, J.cb[P].as<T>(), J.cbr[P].as<T>(), x, h->adj_status.as<int>(),
                   d.group_active, 0, st, &nl);
  const size_t nx = (size_t)lanes * J.sym.n;
  const dim3 bg((unsigned)((h->g.nbr + 63) / 64), (unsigned)h->ngroups);
  auto gradients = [&](const auto* lam) {
    using L = std::remove_cv_t<std::remove_pointer_t<decltype(lam)>>;
    if (gp || gq) {
      const size_t total = (size_t)h->ncases * h->g.nb;
      k_adj_grad_bus<L><<<(unsigned)std::min<size_t>(148 * 16, total / 256 + 1), 256, 0, st>>>(d, h->ncases, lam, gp,
                                                                                                 gq);
      CUDA_TRY(cudaGetLastError());
    }
    if (gg || gb) {
      k_adj_grad_branch<L><<<bg, 256, 0, st>>>(d, h->g.nbr, h->ncases, h->rating.as<double>(),
                                               h->br_dy.as<double2>(), lam, gg, gb);
      CUDA_TRY(cudaGetLastError());
    }
  };
  if constexpr (std::is_same<T, double>::value) {
    CUDA_TRY(cudaMemsetAsync(x, 0, nx * sizeof(T), st));
    k_adj_dldx<T><<<bg, 256, 0, st>>>(d, h->g.nbr, h->rating.as<double>(), x);
    CUDA_TRY(cudaGetLastError());
    launch_fsolve_t<T>(J, h->ngroups, pan, J.cbr[P].as<T>(), x, d.group_active, st);
    launch_bsolve_t<T>(J, h->ngroups, pan, x, d.group_active, st);
    gradients(x);
  } else {
    // FP32 factors: solve, then refine with FP64 residuals of the FP64 Jacobian
    J.ensure_values(0, h->ngroups);
    double* A64 = J.A[0].as<double>();
    if (!h->adj_b64.p || h->adj_b64.bytes < nx * sizeof(double)) {
      h->adj_b64.alloc(nx * sizeof(double));
      h->adj_lam64.alloc(nx * sizeof(double));
    }
    double* b64 = h->adj_b64.as<double>();
    double* lam64 = h->adj_lam64.as<double>();
    // entries of other islands are never filled: start from zeros so they stay finite
    CUDA_TRY(cudaMemsetAsync(A64, 0, (size_t)lanes * J.nA * sizeof(double), st));
    launch_mismatch_nr<double>(d, rg, st, J.x[0].as<double>(), A64, true);
    CUDA_TRY(cudaMemsetAsync(b64, 0, nx * sizeof(double), st));
    k_adj_dldx<double><<<bg, 256, 0, st>>>(d, h->g.nbr, h->rating.as<double>(), b64);
    CUDA_TRY(cudaGetLastError());
    const unsigned eb = (unsigned)std::min<size_t>(148 * 16, nx / 256 + 1);
    k_adj_cast<T><<<eb, 256, 0, st>>>(nx, b64, x);
    CUDA_TRY(cudaGetLastError());
    const dim3 cgrid((unsigned)((J.sym.n + 7) / 8), (unsigned)h->ngroups);
    for (int r = 0; r <= kAdjRefine; ++r) {
      if (r > 0) {
        k_adj_residual<T><<<cgrid, 256, 0, st>>>(J.sym.n, h->ngroups, J.nA, h->adj_colptr.as<int>(),
                                                 h->adj_colent.as<int2>(), A64, lam64, b64, x);
        CUDA_TRY(cudaGetLastError());
      }
      launch_fsolve_t<T>(J, h->ngroups, pan, J.cbr[P].as<T>(), x, d.group_active, st);
      launch_bsolve_t<T>(J, h->ngroups, pan, x, d.group_active, st);
      k_adj_accumulate<T><<<eb, 256, 0, st>>>(nx, x, lam64, r > 0);
      CUDA_TRY(cudaGetLastError());
    }
    gradients(lam64);
  }
}

// ====================================================================== C-ABI
extern "C" {

int32_t mpf_abi_version(void) { return MPF_ABI_VERSION; }

void mpf_default_options(mpf_options* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->max_it_nr = MPF_DEFAULT_MAX_IT_NR;
  opt->max_it_fd = MPF_DEFAULT_MAX_IT_FD;
  opt->tol = MPF_DEFAULT_TOL;
  opt->angle_mode = 0;
  opt->device = 0;
  opt->use_graph = 2;
  opt->autotune = 1;
}

const char* mpf_status_string(int32_t status) {
  switch (status) {
    case MPF_OK: return "ok";
    case MPF_ERR_BAD_INPUT: return "bad input";
    case MPF_ERR_CUDA: return "CUDA error";
    case MPF_ERR_OOM: return "out of memory";
    case MPF_ERR_STATE: return "call out of order";
    case MPF_ERR_TIMEOUT: return "device wait timed out";
    case MPF_ERR_INTERNAL: return "internal error";
    case MPF_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
  }
}

const char* mpf_last_error(const mpf_handle* h) { return h ? h->err.c_str() : "null handle"; }

int32_t mpf_create(const mpf_bus* buses, int32_t n_bus, const mpf_branch* branches, int32_t n_branch,
                   const mpf_options* opt, mpf_handle** out) {
  if (!out) return MPF_ERR_BAD_INPUT;
  *out = nullptr;
  if (!buses || !branches || n_bus < 2 || n_branch < 1) return MPF_ERR_BAD_INPUT;
  std::unique_ptr<mpf_handle> h(new (std::nothrow) mpf_handle());
  if (!h) return MPF_ERR_OOM;
  mpf_default_options(&h->opt);
  if (opt) h->opt = *opt;
  if (h->opt.max_it_nr < 0 || h->opt.max_it_fd < 0 || !(h->opt.tol > 0.0) ||
      (h->opt.angle_mode != 0 && h->opt.angle_mode != 1) || h->opt.ordering < MPF_ORDER_AUTO ||
      h->opt.ordering > MPF_ORDER_MIN_FILL_WEIGHTED) {
    h->err = "invalid options";
    *out = h.release();
    return MPF_ERR_BAD_INPUT;
  }
  int rc = guarded(h.get(), [&]() -> int {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(h.get(), MPF_ERR_NO_DEVICE, "no CUDA device visible");
    if (h->opt.device < 0 || h->opt.device >= ndev) return fail(h.get(), MPF_ERR_BAD_INPUT, "device ordinal out of range");
    h->device = h->opt.device;
    CUDA_TRY(cudaSetDevice(h->device));
    const std::string msg = build_symbolic(buses, n_bus, branches, n_branch, h->g, nullptr, h->opt.ordering);
    if (!msg.empty()) return fail(h.get(), MPF_ERR_BAD_INPUT, msg);
    h->buses.assign(buses, buses + n_bus);
    h->branches.assign(branches, branches + n_branch);
    if (find_bridges(branches, n_branch, n_bus, h->is_bridge) != 0)
      return fail(h.get(), MPF_ERR_BAD_INPUT, "bridge search failed");
    const GridSymbolic& g = h->g;
    {
      std::string lim = front_limits(g.jac, "Newton system");
      for (int v = 0; v < 2 && lim.empty(); ++v) {
        lim = front_limits(g.bp[v].lu, "B'");
        if (lim.empty()) lim = front_limits(g.bpp[v].lu, "B''");
      }
      if (!lim.empty()) return fail(h.get(), MPF_ERR_BAD_INPUT, lim);
    }
    CUDA_TRY(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaMallocHost(&h->h_any, sizeof(int)));
    CUDA_TRY(cudaEventCreate(&h->t0));
    CUDA_TRY(cudaEventCreate(&h->t1));
    upload(h->y_rowptr, g.y_rowptr);
    upload(h->y_col, g.y_col);
    upload(h->y_diag, g.y_diag);
    {
      std::vector<double2> yv(g.y_val.size() / 2);
      for (size_t k = 0; k < yv.size(); ++k) yv[k] = make_double2(g.y_val[2 * k], g.y_val[2 * k + 1]);
      upload(h->y_val, yv);
      std::vector<int4> bp(g.nbr);
      std::vector<double2> by(4 * (size_t)g.nbr);
      for (int e = 0; e < g.nbr; ++e) {
        bp[e] = make_int4(g.br_pos[4 * e], g.br_pos[4 * e + 1], g.br_pos[4 * e + 2], g.br_pos[4 * e + 3]);
        for (int q = 0; q < 4; ++q) by[4 * e + q] = make_double2(g.br_y[8 * e + 2 * q], g.br_y[8 * e + 2 * q + 1]);
      }
      upload(h->br_ypos, bp);
      std::vector<int2> ft(g.nbr);
      for (int e = 0; e < g.nbr; ++e) ft[e] = make_int2(g.br_from[e], g.br_to[e]);
      upload(h->br_ft, ft);
      // dY/dg of each branch's four entries (series admittance g + jb): 1/|t|^2,
      // -1/conj(t), -1/t, 1 with t = tap e^{j shift} (tap 0 -> 1); 0 when out of service
      std::vector<double2> dy(4 * (size_t)g.nbr, make_double2(0.0, 0.0));
      for (int e = 0; e < g.nbr; ++e) {
        if (!branches[e].status) continue;
        const double a = branches[e].tap != 0.0 ? branches[e].tap : 1.0;
        const double ang = M_PI / 180.0 * branches[e].shift;
        const double tr = a * std::cos(ang), ti = a * std::sin(ang), t2 = tr * tr + ti * ti;
        dy[4 * e + 0] = make_double2(1.0 / t2, 0.0);
        dy[4 * e + 1] = make_double2(-tr / t2, -ti / t2);  // -1/conj(t) = -t/|t|^2
        dy[4 * e + 2] = make_double2(-tr / t2, ti / t2);   // -1/t = -conj(t)/|t|^2
        dy[4 * e + 3] = make_double2(1.0, 0.0);
      }
      upload(h->br_dy, dy);
      upload(h->br_y, by);
      std::vector<double2> sb(g.nb), v0(g.nb);
      for (int i = 0; i < g.nb; ++i) {
        sb[i] = make_double2(g.sbus[2 * i], g.sbus[2 * i + 1]);
        v0[i] = make_double2(g.v0[2 * i], g.v0[2 * i + 1]);
      }
      upload(h->sbus0, sb);
      upload(h->v0, v0);
      upload(h->mis_rows, g.mis_rows);
    }
    if (g.n_islands > 1) {
      upload(h->bus_island, g.bus_island);
      upload(h->br_island, g.br_island);
    }
    upload_newton(h.get());
    h->any_active.alloc(sizeof(int));
    h->it_ctr.alloc(sizeof(int));
    return MPF_OK;
  });
  *out = h.release();
  return rc;
}

int32_t mpf_destroy(mpf_handle* h) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (h->own_stream) {
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->own_stream);
    cudaStreamDestroy(h->own_stream);
  }
  for (auto& gph : h->nr_graph) gph.release();
  if (h->h_any) cudaFreeHost(h->h_any);
  if (h->t0) cudaEventDestroy(h->t0);
  if (h->t1) cudaEventDestroy(h->t1);
  delete h;
  return MPF_OK;
}

int32_t mpf_get_stats(const mpf_handle* h, mpf_stats* st) {
  if (!h || !st) return MPF_ERR_BAD_INPUT;
  std::memset(st, 0, sizeof(*st));
  const GridSymbolic& g = h->g;
  st->n_bus = g.nb;
  st->n_branch = g.nbr;
  st->n_pv = g.npv;
  st->n_pq = g.npq;
  st->n_slack = g.n_slack;
  st->nnz_ybus = g.y_rowptr.empty() ? 0 : g.y_rowptr.back();
  st->n_jac = g.jac.n;
  st->nnz_jac = g.nnz_jac;
  st->nnz_lu = (int32_t)g.jac.nnz;
  st->lu_levels = g.jac.nlevels;
  st->lu_flops = g.jac.flops;
  st->n_bp = g.bp[0].lu.n;
  st->nnz_bp_lu = (int32_t)g.bp[0].lu.nnz;
  st->bp_levels = g.bp[0].lu.nlevels;
  st->n_bpp = g.bpp[0].lu.n;
  st->nnz_bpp_lu = (int32_t)g.bpp[0].lu.nnz;
  st->bpp_levels = g.bpp[0].lu.nlevels;
  st->n_cases = h->ncases;
  st->case_groups = h->ngroups;
  st->device_bytes = (int64_t)h->device_bytes();
  for (int s = 0; s < g.jac.nsn; ++s) st->nnz_lu_upper += (int64_t)g.jac.sn_w[s] * g.jac.sn_f[s];
  st->ordering = g.ordering;
  return MPF_OK;
}

namespace {
int set_cases_impl(mpf_handle* h, int32_t n_cases, const int32_t* island_of_case, const int32_t* outage_offsets,
                   const int32_t* outage_branches, const double* sbus);
}  // namespace

int32_t mpf_set_cases(mpf_handle* h, int32_t n_cases, const int32_t* outage_offsets, const int32_t* outage_branches,
                      const double* sbus) {
  return set_cases_impl(h, n_cases, nullptr, outage_offsets, outage_branches, sbus);
}

int32_t mpf_set_cases_islands(mpf_handle* h, int32_t n_cases, const int32_t* island_of_case,
                              const int32_t* outage_offsets, const int32_t* outage_branches, const double* sbus) {
  if (h && !island_of_case) return fail(h, MPF_ERR_BAD_INPUT, "island_of_case is required");
  return set_cases_impl(h, n_cases, island_of_case, outage_offsets, outage_branches, sbus);
}

namespace {
int set_cases_impl(mpf_handle* h, int32_t n_cases, const int32_t* island_of_case, const int32_t* outage_offsets,
                   const int32_t* outage_branches, const double* sbus) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (n_cases < 1) return fail(h, MPF_ERR_BAD_INPUT, "n_cases must be >= 1");
  if ((outage_offsets == nullptr) != (outage_branches == nullptr) && outage_offsets && outage_offsets[n_cases] > 0)
    return fail(h, MPF_ERR_BAD_INPUT, "outage_offsets given without outage_branches");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    // the case buffers are rewritten below: wait for work that may still read them
    CUDA_TRY(cudaStreamSynchronize(h->own_stream));
    if (h->last_stream) CUDA_TRY(cudaStreamSynchronize(h->last_stream));
    const GridSymbolic& g = h->g;
    const bool multi = g.n_islands > 1;
    if (outage_offsets && outage_offsets[0] != 0) return fail(h, MPF_ERR_BAD_INPUT, "outage_offsets[0] must be 0");
    // island of each case; lanes grouped by island, each island padded to whole groups
    std::vector<int> island(n_cases, 0);
    for (int c = 0; c < n_cases; ++c) {
      const bool has_out = outage_offsets && outage_offsets[c + 1] > outage_offsets[c];
      if (island_of_case) {
        if (island_of_case[c] < 0 || island_of_case[c] >= g.n_islands)
          return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + ": island out of range");
        island[c] = island_of_case[c];
      } else if (multi) {
        if (!has_out)
          return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + " has no outage to tell its island: "
                                            "use mpf_set_cases_islands on a grid with several islands");
        const int br = outage_branches[outage_offsets[c]];
        if (br < 0 || br >= g.nbr)
          return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + ": outaged branch index out of range");
        island[c] = g.br_island[br];
      }
    }
    std::vector<int> case_lane(n_cases), lane_case, group_island;
    int ngroups = 0;
    if (multi) {
      std::vector<int> count(g.n_islands, 0), next(g.n_islands, 0);
      for (int c = 0; c < n_cases; ++c) ++count[island[c]];
      for (int k = 0; k < g.n_islands; ++k) {
        next[k] = ngroups * 32;
        const int gk = (count[k] + 31) / 32;
        for (int q = 0; q < gk; ++q) group_island.push_back(k);
        ngroups += gk;
      }
      lane_case.assign((size_t)ngroups * 32, -1);
      for (int c = 0; c < n_cases; ++c) {
        case_lane[c] = next[island[c]]++;
        lane_case[case_lane[c]] = c;
      }
    } else {
      ngroups = (n_cases + 31) / 32;
      for (int c = 0; c < n_cases; ++c) case_lane[c] = c;
    }
    const int lanes = ngroups * 32;
    std::vector<int> outs((size_t)kMaxOut * lanes, -1);
    int maxk = 0;
    if (outage_offsets) {
      for (int c = 0; c < n_cases; ++c) {
        const int b = outage_offsets[c], e = outage_offsets[c + 1];
        if (e < b) return fail(h, MPF_ERR_BAD_INPUT, "outage_offsets must be non-decreasing");
        if (e - b > kMaxOut)
          return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + " outages more than " +
                                                std::to_string(kMaxOut) + " branches");
        for (int k = b; k < e; ++k) {
          const int br = outage_branches[k];
          if (br < 0 || br >= g.nbr)
            return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + ": outaged branch index out of range");
          for (int k2 = b; k2 < k; ++k2)
            if (outage_branches[k2] == br)
              return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + " lists a branch twice");
          if (multi && g.br_island[br] != island[c])
            return fail(h, MPF_ERR_BAD_INPUT, "case " + std::to_string(c) + " outages a branch of another island");
          outs[(size_t)(k - b) * lanes + case_lane[c]] = br;
        }
        maxk = std::max(maxk, e - b);
      }
    }
    // cases whose outages cut PV/PQ buses off from every slack: a non-bridge single
    // outage never does; otherwise search from the slacks over the remaining branches
    std::vector<unsigned char> cut(lanes, 0);
    bool any_cut = false;
    if (outage_offsets) {
      std::vector<std::vector<int>> adj;  // built on first need
      std::vector<int> seen(g.nb, -1), stack;
      for (int c = 0; c < n_cases; ++c) {
        const int b = outage_offsets[c], e = outage_offsets[c + 1];
        if (e == b || (e - b == 1 && !h->is_bridge[outage_branches[b]])) continue;
        if (adj.empty()) {
          adj.resize(g.nb);
          for (int k = 0; k < g.nbr; ++k)
            if (h->branches[k].status != 0) {
              adj[h->branches[k].from].push_back(k);
              adj[h->branches[k].to].push_back(k);
            }
        }
        auto out_here = [&](int k) {
          for (int q = b; q < e; ++q)
            if (outage_branches[q] == k) return true;
          return false;
        };
        stack.clear();
        for (int i = 0; i < g.nb; ++i)
          if (g.bus_type[i] == MPF_BUS_SLACK) {
            seen[i] = c;
            stack.push_back(i);
          }
        while (!stack.empty()) {
          const int i = stack.back();
          stack.pop_back();
          for (int k : adj[i]) {
            if (out_here(k)) continue;
            const int j = h->branches[k].from == i ? h->branches[k].to : h->branches[k].from;
            if (seen[j] != c) {
              seen[j] = c;
              stack.push_back(j);
            }
          }
        }
        for (int i = 0; i < g.nb; ++i)
          if (seen[i] != c && (g.bus_type[i] == MPF_BUS_PV || g.bus_type[i] == MPF_BUS_PQ)) {
            cut[case_lane[c]] = 1;
            any_cut = true;
            break;
          }
      }
    }
    std::vector<double2> sb;
    if (sbus) {
      sb.assign((size_t)ngroups * g.nb * 32, make_double2(0.0, 0.0));
      for (int c = 0; c < n_cases; ++c)
        for (int i = 0; i < g.nb; ++i) {
          const double p = sbus[((size_t)c * g.nb + i) * 2], q = sbus[((size_t)c * g.nb + i) * 2 + 1];
          if (!std::isfinite(p) || !std::isfinite(q))
            return fail(h, MPF_ERR_BAD_INPUT, "sbus has a non-finite value");
          const int ln = case_lane[c];
          sb[((size_t)(ln >> 5) * g.nb + i) * 32 + (ln & 31)] = make_double2(p, q);
        }
    }
    if (ngroups != h->ngroups) {
      const size_t per_bus = (size_t)ngroups * g.nb * 32 * sizeof(double2);
      h->V.alloc(per_bus);
      h->Ibus.alloc(per_bus);
      h->status.alloc(lanes * sizeof(int));
      h->iters.alloc(lanes * sizeof(int));
      h->maxmis.alloc(lanes * sizeof(double));
      h->facc.alloc(lanes * sizeof(unsigned long long));
      h->group_active.alloc(ngroups * sizeof(int));
      h->vout.release();
      h->small_out.release();
      h->jac.release_values();
      for (int v = 0; v < 2; ++v) {
        h->bp[v].release_values();
        h->bpp[v].release_values();
      }
    }
    upload(h->out_br, outs);
    if (any_cut) upload(h->case_cut, cut);
    else h->case_cut.release();
    if (sbus) upload(h->sbus_case, sb);
    else h->sbus_case.release();
    if (multi) {
      upload(h->group_island, group_island);
      upload(h->lane_case, lane_case);
      upload(h->case_lane, case_lane);
    }
    h->h_lane_case = lane_case;
    const int* gi = multi ? h->group_island.as<int>() : nullptr;
    h->jac.group_island = gi;
    for (int v = 0; v < 2; ++v) {
      h->bp[v].group_island = gi;
      h->bpp[v].group_island = gi;
    }
    if (h->nsw > 0) {
      // every limited bus starts as PV in every case
      const size_t n = (size_t)lanes * h->nsw;
      h->pv_on.alloc(n);
      h->q_fix.alloc(n * sizeof(double));
      h->q_flag.alloc((size_t)lanes * sizeof(int));
      h->iter_base.alloc((size_t)lanes * sizeof(int));
      CUDA_TRY(cudaMemset(h->pv_on.p, 1, n));
      CUDA_TRY(cudaMemset(h->q_fix.p, 0, n * sizeof(double)));
      CUDA_TRY(cudaMemset(h->q_flag.p, 0, (size_t)lanes * sizeof(int)));
      CUDA_TRY(cudaMemset(h->iter_base.p, 0, (size_t)lanes * sizeof(int)));
    }
    h->ncases = n_cases;
    h->ngroups = ngroups;
    h->maxk = maxk;
    h->ctl.clear();
    h->have_cases = true;
    h->have_results = false;
    return MPF_OK;
  });
}
}  // namespace

int32_t mpf_set_controls(mpf_handle* h, int32_t n_controls, const mpf_control* controls, const double* values) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_cases) return fail(h, MPF_ERR_STATE, "mpf_set_cases must be called before mpf_set_controls");
  if (n_controls < 0) return fail(h, MPF_ERR_BAD_INPUT, "n_controls must be >= 0");
  if (n_controls > 0 && (!controls || !values)) return fail(h, MPF_ERR_BAD_INPUT, "controls and values are required");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    // the control buffers are rewritten below: wait for work that may still read them
    CUDA_TRY(cudaStreamSynchronize(h->own_stream));
    if (h->last_stream) CUDA_TRY(cudaStreamSynchronize(h->last_stream));
    auto& C = h->ctl;
    C.clear();
    h->have_results = false;
    if (n_controls == 0) return MPF_OK;
    const GridSymbolic& g = h->g;
    const int nc = n_controls, ncases = h->ncases, lanes = h->ngroups * 32;
    std::vector<int2> avr, oltc, shc;
    std::vector<double> base(nc);
    std::set<std::pair<int, int>> seen;
    for (int k = 0; k < nc; ++k) {
      const int kind = controls[k].kind, idx = controls[k].index;
      const std::string who = "control " + std::to_string(k);
      if (!seen.insert({kind, idx}).second) return fail(h, MPF_ERR_BAD_INPUT, who + " repeats a (kind, index)");
      if (kind == MPF_CTRL_AVR || kind == MPF_CTRL_SHC) {
        if (idx < 0 || idx >= g.nb) return fail(h, MPF_ERR_BAD_INPUT, who + ": bus index out of range");
        if (kind == MPF_CTRL_AVR) {
          if (g.bus_type[idx] != MPF_BUS_PV && g.bus_type[idx] != MPF_BUS_SLACK)
            return fail(h, MPF_ERR_BAD_INPUT, who + ": AVR on a bus that is neither PV nor slack");
          avr.push_back(make_int2(idx, k));
          base[k] = h->buses[idx].vm;
        } else {
          shc.push_back(make_int2(idx, k));
          base[k] = h->buses[idx].bsh;
        }
      } else if (kind == MPF_CTRL_OLTC) {
        if (idx < 0 || idx >= g.nbr) return fail(h, MPF_ERR_BAD_INPUT, who + ": branch index out of range");
        if (h->branches[idx].tap == 0.0)
          return fail(h, MPF_ERR_BAD_INPUT, who + ": OLTC on a branch without a tap (tap 0)");
        oltc.push_back(make_int2(idx, k));
        base[k] = h->branches[idx].tap;
      } else {
        return fail(h, MPF_ERR_BAD_INPUT, who + ": unknown kind");
      }
    }
    // values, lane-interleaved; padding lanes hold the base values
    std::vector<double> val((size_t)h->ngroups * nc * 32);
    for (int c = 0; c < lanes; ++c)
      for (int k = 0; k < nc; ++k) {
        const int uc = h->h_lane_case.empty() ? (c < ncases ? c : -1) : h->h_lane_case[c];
        const double v = uc >= 0 ? values[(size_t)uc * nc + k] : base[k];
        if (!std::isfinite(v)) return fail(h, MPF_ERR_BAD_INPUT, "control values must be finite");
        if (controls[k].kind != MPF_CTRL_SHC && !(v > 0.0))
          return fail(h, MPF_ERR_BAD_INPUT, "AVR and OLTC values must be > 0");
        val[((size_t)(c >> 5) * nc + k) * 32 + (c & 31)] = v;
      }
    // tap parameters: Ys, b/2, cos / sin of the shift, Ys with r = 0 (BX's B'')
    std::vector<double> par(8 * oltc.size(), 0.0);
    std::vector<int> br_ctl(g.nbr, -1);
    for (size_t j = 0; j < oltc.size(); ++j) {
      const mpf_branch& b = h->branches[oltc[j].x];
      br_ctl[oltc[j].x] = (int)j;
      if (!b.status) continue;
      const double den = b.r * b.r + b.x * b.x;
      const double ang = M_PI / 180.0 * b.shift;
      double* p = &par[8 * j];
      p[0] = b.r / den;
      p[1] = -b.x / den;
      p[2] = 0.5 * b.b;
      p[3] = std::cos(ang);
      p[4] = std::sin(ang);
      p[5] = 0.0;
      p[6] = -1.0 / b.x;
    }
    // slots: the distinct Ybus positions the taps (ff, ft, tf) and shunts (ii) change
    std::vector<int> y_slot(g.y_col.size(), -1), slot_pos;
    std::vector<std::vector<int2>> ents;
    auto slot_of = [&](int p) {
      if (y_slot[p] < 0) {
        y_slot[p] = (int)slot_pos.size();
        slot_pos.push_back(p);
        ents.emplace_back();
      }
      return y_slot[p];
    };
    for (size_t j = 0; j < oltc.size(); ++j)
      for (int q = 0; q < 3; ++q) ents[slot_of(g.br_pos[4 * oltc[j].x + q])].push_back(make_int2(q, (int)j));
    for (size_t j = 0; j < shc.size(); ++j) ents[slot_of(g.y_diag[shc[j].x])].push_back(make_int2(3, (int)j));
    std::vector<int> slot_ptr(1, 0);
    std::vector<int2> slot_ent;
    for (auto& e : ents) {
      slot_ent.insert(slot_ent.end(), e.begin(), e.end());
      slot_ptr.push_back((int)slot_ent.size());
    }
    // B'' array position of each slot, per fast-decoupled variant
    std::vector<int> fdpos[2];
    for (int v = 0; v < 2; ++v) {
      const auto& fs = g.bpp[v];
      fdpos[v].assign(slot_pos.size(), -1);
      for (size_t s = 0; s < slot_pos.size(); ++s) {
        const int2 e = ents[s][0];
        fdpos[v][s] = e.x < 3 ? fs.br_pos[4 * oltc[e.y].x + e.x] : fs.diag_pos[shc[e.y].x];
      }
    }
    std::vector<double> shc_base(shc.size());
    for (size_t j = 0; j < shc.size(); ++j) shc_base[j] = h->buses[shc[j].x].bsh;
    upload(C.val, val);
    upload(C.avr, avr);
    upload(C.oltc, oltc);
    upload(C.oltc_par, par);
    upload(C.shc, shc);
    upload(C.shc_base, shc_base);
    upload(C.slot_ptr, slot_ptr);
    upload(C.slot_ent, slot_ent);
    upload(C.y_slot, y_slot);
    upload(C.br_ctl, br_ctl);
    upload(C.fdpos[0], fdpos[0]);
    upload(C.fdpos[1], fdpos[1]);
    const size_t nbry = (size_t)h->ngroups * 4 * std::max<size_t>(oltc.size(), 1) * 32 * sizeof(double2);
    if (!C.bry.p || C.bry.bytes < nbry) C.bry.alloc(nbry);
    if (!C.bdy.p || C.bdy.bytes < nbry) C.bdy.alloc(nbry);
    const size_t ndy = (size_t)h->ngroups * std::max<size_t>(slot_pos.size(), 1) * 32 * sizeof(double2);
    if (!C.dy.p || C.dy.bytes < ndy) C.dy.alloc(ndy);
    C.nc = nc;
    C.navr = (int)avr.size();
    C.noltc = (int)oltc.size();
    C.nshc = (int)shc.size();
    C.nslot = (int)slot_pos.size();
    cudaStream_t st = h->own_stream;
    const DevCtl t = h->devctl();
    if (C.noltc > 0) {
      const size_t tot = (size_t)h->ngroups * C.noltc * 32;
      k_ctl_branch<<<(unsigned)std::min<size_t>(148 * 8, tot / 256 + 1), 256, 0, st>>>(t, h->ngroups, C.bry.as<double2>(),
                                                                                       C.bdy.as<double2>());
      CUDA_TRY(cudaGetLastError());
    }
    if (C.nslot > 0) {
      const size_t tot = (size_t)h->ngroups * C.nslot * 32;
      k_ctl_ydelta<<<(unsigned)std::min<size_t>(148 * 8, tot / 256 + 1), 256, 0, st>>>(h->dev(), t, C.bry.as<double2>(),
                                                                                       C.dy.as<double2>());
      CUDA_TRY(cudaGetLastError());
    }
    CUDA_TRY(cudaStreamSynchronize(st));
    return MPF_OK;
  });
}

int32_t mpf_set_q_limits(mpf_handle* h, const double* qmin, const double* qmax) {
  if (!h) return MPF_ERR_BAD_INPUT;
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(h->own_stream));
    if (h->last_stream) CUDA_TRY(cudaStreamSynchronize(h->last_stream));
    const int nb = h->g.nb;
    std::vector<char> vf(nb, 0);
    std::vector<int> swi(nb, -1), swb;
    std::vector<double2> lim;
    for (int i = 0; i < nb && (qmin || qmax); ++i) {
      if (h->g.bus_type[i] != MPF_BUS_PV) continue;
      double lo = qmin ? qmin[i] : -INFINITY, hi = qmax ? qmax[i] : INFINITY;
      if (lo != lo) lo = -INFINITY;
      if (hi != hi) hi = INFINITY;
      if (lo > hi) return fail(h, MPF_ERR_BAD_INPUT, "bus " + std::to_string(i) + ": qmin > qmax");
      if (!std::isfinite(lo) && !std::isfinite(hi)) continue;
      vf[i] = 1;
      swi[i] = (int)swb.size();
      swb.push_back(i);
      lim.push_back(make_double2(lo, hi));
    }
    // the Newton system with a Vm variable and a Q equation for every limited PV bus
    GridSymbolic g2;
    const std::string msg = build_symbolic(h->buses.data(), nb, h->branches.data(), (int)h->branches.size(), g2,
                                           swb.empty() ? nullptr : &vf, h->opt.ordering);
    if (!msg.empty()) return fail(h, MPF_ERR_BAD_INPUT, msg);
    {
      const std::string lim = front_limits(g2.jac, "Newton system with the limited PV buses");
      if (!lim.empty()) return fail(h, MPF_ERR_BAD_INPUT, lim);
    }
    for (int p = 0; p < 2; ++p) h->nr_graph[p].release();
    h->jac.release_values();
    h->jac.tuned.clear();
    h->jac.tuned_bs.clear();
    h->g = std::move(g2);
    h->vm_free = vf;
    h->nsw = (int)swb.size();
    upload_newton(h);
    if (h->nsw > 0) {
      upload(h->sw_index, swi);
      upload(h->sw_bus, swb);
      upload(h->q_lim, lim);
    }
    // the batch must be defined again for the new system
    h->have_cases = false;
    h->have_results = false;
    h->ngroups = 0;
    h->ctl.clear();
    return MPF_OK;
  });
}

int32_t mpf_get_bus_types(mpf_handle* h, uint8_t* types) {
  if (!h || !types) return MPF_ERR_BAD_INPUT;
  if (!h->have_results) return fail(h, MPF_ERR_STATE, "no results: call mpf_solve first");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = h->own_stream;
    CUDA_TRY(cudaStreamWaitEvent(st, h->t1, 0));
    if (!h->base_type.p) {
      std::vector<uint8_t> bt(h->g.nb);
      for (int i = 0; i < h->g.nb; ++i) bt[i] = (uint8_t)h->g.bus_type[i];
      upload(h->base_type, bt);
    }
    const size_t total = (size_t)h->ncases * h->g.nb;
    DevBuf out;
    out.alloc(total);
    k_gather_types<<<(unsigned)std::min<size_t>(148 * 16, total / 256 + 1), 256, 0, st>>>(
        h->dev(), h->ncases, h->base_type.as<unsigned char>(), out.as<unsigned char>());
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(types, out.p, total, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return MPF_OK;
  });
}

int32_t mpf_solve(mpf_handle* h, int32_t alg, int32_t precision, void* stream) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_cases) return fail(h, MPF_ERR_STATE, "mpf_set_cases must be called before mpf_solve");
  if (alg != MPF_NR && alg != MPF_FDXB && alg != MPF_FDBX) return fail(h, MPF_ERR_BAD_INPUT, "unknown algorithm");
  if (alg != MPF_NR && h->nsw > 0)
    return fail(h, MPF_ERR_BAD_INPUT, "reactive limits are enforced with Newton-Raphson only");
  if (precision != MPF_FP64 && precision != MPF_MIXED) return fail(h, MPF_ERR_BAD_INPUT, "unknown precision");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    h->last_stream = st;
    std::memset(&h->timing, 0, sizeof(h->timing));
    h->timer.reset(st);
    CUDA_TRY(cudaEventRecord(h->t0, st));
    ensure_attrs<double>(h->device);
    ensure_attrs<float>(h->device);
    if (alg == MPF_NR) {
      if (precision == MPF_FP64) solve_nr<double>(h, st);
      else solve_nr<float>(h, st);
    } else {
      const int variant = alg == MPF_FDXB ? 0 : 1;
      if (precision == MPF_FP64) solve_fd<double>(h, st, variant);
      else solve_fd<float>(h, st, variant);
    }
    CUDA_TRY(cudaEventRecord(h->t1, st));
    CUDA_TRY(cudaGetLastError());
    h->have_results = true;
    h->last_alg = alg;
    h->last_prec = precision;
    return MPF_OK;
  });
}

int32_t mpf_get_timing(mpf_handle* h, mpf_timing* t) {
  if (!h || !t) return MPF_ERR_BAD_INPUT;
  if (!h->have_results) return fail(h, MPF_ERR_STATE, "no solve to report");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaEventSynchronize(h->t1));
    double ms[FAM_N];
    h->timer.collect(ms);
    float tot = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&tot, h->t0, h->t1));
    h->timing.total_ms = tot;
    h->timing.mismatch_ms = ms[FAM_MIS];
    h->timing.jacobian_ms = ms[FAM_JAC];
    h->timing.factor_ms = ms[FAM_FACT];
    h->timing.solve_ms = ms[FAM_SOLVE];
    h->timing.update_ms = ms[FAM_UPD];
    h->timing.other_ms = ms[FAM_OTHER];
    *t = h->timing;
    return MPF_OK;
  });
}

int32_t mpf_get_results_device(mpf_handle* h, double* v, int32_t* iterations, uint8_t* status, double* max_mis,
                               void* stream) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_results) return fail(h, MPF_ERR_STATE, "no results: call mpf_solve first");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    if (v) {
      const size_t total = (size_t)h->ncases * h->g.nb;
      k_gather_v<<<(unsigned)std::min<size_t>(148 * 16, total / 256 + 1), 256, 0, st>>>(
          h->g.nb, h->ncases, h->dev().case_lane, h->V.as<double2>(), reinterpret_cast<double2*>(v));
      CUDA_TRY(cudaGetLastError());
    }
    if (iterations || status || max_mis) {
      k_gather_small<<<(h->ncases + 255) / 256, 256, 0, st>>>(h->ncases, h->dev().case_lane, h->status.as<int>(),
                                                             h->iters.as<int>(), h->maxmis.as<double>(), status,
                                                             iterations, max_mis);
      CUDA_TRY(cudaGetLastError());
    }
    return MPF_OK;
  });
}

int32_t mpf_get_results(mpf_handle* h, double* v, int32_t* iterations, uint8_t* status, double* max_mis) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_results) return fail(h, MPF_ERR_STATE, "no results: call mpf_solve first");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = h->own_stream;
    const size_t vbytes = (size_t)h->ncases * h->g.nb * sizeof(double2);
    const size_t sbytes = (size_t)h->ncases * (sizeof(int) + sizeof(double) + 1) + 64;
    if (h->vout.bytes < vbytes) h->vout.alloc(vbytes);
    if (h->small_out.bytes < sbytes) h->small_out.alloc(sbytes);
    int32_t* d_it = h->small_out.as<int32_t>();
    double* d_mm = reinterpret_cast<double*>(reinterpret_cast<char*>(h->small_out.p) + ((h->ncases * sizeof(int) + 15) / 16) * 16);
    uint8_t* d_st = reinterpret_cast<uint8_t*>(d_mm + h->ncases);
    // the solve may have run on a caller stream: order after it
    CUDA_TRY(cudaStreamWaitEvent(st, h->t1, 0));
    int rc = mpf_get_results_device(h, v ? h->vout.as<double>() : nullptr, d_it, d_st, d_mm, st);
    if (rc != MPF_OK) return rc;
    if (v) CUDA_TRY(cudaMemcpyAsync(v, h->vout.p, vbytes, cudaMemcpyDeviceToHost, st));
    if (iterations) CUDA_TRY(cudaMemcpyAsync(iterations, d_it, h->ncases * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    if (max_mis) CUDA_TRY(cudaMemcpyAsync(max_mis, d_mm, h->ncases * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (status) CUDA_TRY(cudaMemcpyAsync(status, d_st, h->ncases, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return MPF_OK;
  });
}

int32_t mpf_mismatch(mpf_handle* h, const double* v, double* max_mis, void* stream) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_cases) return fail(h, MPF_ERR_STATE, "mpf_set_cases must be called before mpf_mismatch");
  if (!v || !max_mis) return fail(h, MPF_ERR_BAD_INPUT, "v and max_mis must be device pointers");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    const size_t need = (size_t)h->ncases * sizeof(unsigned long long);
    if (!h->eval_acc.p || h->eval_acc.bytes < need) {
      h->eval_acc.alloc(need);
      CUDA_TRY(cudaMemset(h->eval_acc.p, 0, need));
    }
    const int nfree = (int)h->g.mis_rows.size();
    k_mismatch_eval<<<dim3((unsigned)((nfree + 255) / 256), (unsigned)std::min(h->ncases, 65535)), 256, 0, st>>>(
        h->dev(), reinterpret_cast<const double2*>(v), h->ncases, h->eval_acc.as<unsigned long long>());
    CUDA_TRY(cudaGetLastError());
    k_acc_drain<<<(h->ncases + 255) / 256, 256, 0, st>>>(h->eval_acc.as<unsigned long long>(), max_mis, h->ncases);
    CUDA_TRY(cudaGetLastError());
    h->last_stream = st;
    return MPF_OK;
  });
}

int32_t mpf_mismatch_noalloc(mpf_handle* h, const double* v, double* max_mis, void* stream) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_cases) return fail(h, MPF_ERR_STATE, "mpf_set_cases must be called before mpf_mismatch_noalloc");
  if (!v || !max_mis) return fail(h, MPF_ERR_BAD_INPUT, "v and max_mis must be device pointers");
  if (h->ncases > kNoAllocMaxCases)
    return fail(h, MPF_ERR_BAD_INPUT,
                "mpf_mismatch_noalloc handles at most " + std::to_string(kNoAllocMaxCases) + " cases per call (batch has " +
                    std::to_string(h->ncases) + ")");
  if (h->device < 0 || h->device >= kMaxDevices) return fail(h, MPF_ERR_BAD_INPUT, "device ordinal too large");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    unsigned long long* acc = nullptr;
    CUDA_TRY(noalloc_scratch(h->device, &acc));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    // the array keeps whatever the previous call left: clear this call's slots
    CUDA_TRY(cudaMemsetAsync(acc, 0, (size_t)h->ncases * sizeof(unsigned long long), st));
    const int nfree = (int)h->g.mis_rows.size();
    k_mismatch_eval<<<dim3((unsigned)((nfree + 255) / 256), (unsigned)std::min(h->ncases, 65535)), 256, 0, st>>>(
        h->dev(), reinterpret_cast<const double2*>(v), h->ncases, acc);
    CUDA_TRY(cudaGetLastError());
    k_acc_drain<<<(h->ncases + 255) / 256, 256, 0, st>>>(acc, max_mis, h->ncases);
    CUDA_TRY(cudaGetLastError());
    h->last_stream = st;  // later set_cases / set_controls wait for these reads
    return MPF_OK;
  });
}

int32_t mpf_set_ratings(mpf_handle* h, const double* rating) {
  if (!h) return MPF_ERR_BAD_INPUT;
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    if (!rating) {
      h->rating.release();
      return MPF_OK;
    }
    std::vector<double> r(rating, rating + h->g.nbr);
    for (double v : r)
      if (!std::isfinite(v) || v < 0.0) return fail(h, MPF_ERR_BAD_INPUT, "ratings must be finite and >= 0");
    CUDA_TRY(cudaStreamSynchronize(h->own_stream));
    upload(h->rating, r);
    return MPF_OK;
  });
}

int32_t mpf_branch_flows(mpf_handle* h, double* ploss, double* overload, double* sf, double* st, void* stream) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_results) return fail(h, MPF_ERR_STATE, "no solved voltages: call mpf_solve first");
  if (!ploss) return fail(h, MPF_ERR_BAD_INPUT, "ploss must be a device pointer");
  if (overload && !h->rating.p) return fail(h, MPF_ERR_STATE, "overload needs ratings: call mpf_set_ratings");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st_ = stream ? (cudaStream_t)stream : h->own_stream;
    CUDA_TRY(cudaStreamWaitEvent(st_, h->t1, 0));
    CUDA_TRY(cudaMemsetAsync(ploss, 0, (size_t)h->ncases * sizeof(double), st_));
    if (overload) CUDA_TRY(cudaMemsetAsync(overload, 0, (size_t)h->ncases * sizeof(double), st_));
    const dim3 grid((unsigned)((h->g.nbr + 63) / 64), (unsigned)h->ngroups);
    k_branch_flow<<<grid, 256, 0, st_>>>(h->dev(), h->g.nbr, h->ncases, overload ? h->rating.as<double>() : nullptr,
                                         ploss, overload, reinterpret_cast<double2*>(sf), reinterpret_cast<double2*>(st));
    CUDA_TRY(cudaGetLastError());
    h->last_stream = st_;
    return MPF_OK;
  });
}

int32_t mpf_adjoint(mpf_handle* h, int32_t precision, double* grad_p, double* grad_q, double* grad_g,
                    double* grad_b, void* stream) {
  if (!h) return MPF_ERR_BAD_INPUT;
  if (!h->have_results) return fail(h, MPF_ERR_STATE, "no solved voltages: call mpf_solve first");
  if (!h->rating.p) return fail(h, MPF_ERR_STATE, "the adjoint's loss needs ratings: call mpf_set_ratings");
  if (precision != MPF_FP64 && precision != MPF_MIXED) return fail(h, MPF_ERR_BAD_INPUT, "unknown precision");
  return guarded(h, [&]() -> int {
    CUDA_TRY(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t)stream : h->own_stream;
    CUDA_TRY(cudaStreamWaitEvent(st, h->t1, 0));
    ensure_attrs<double>(h->device);
    ensure_attrs<float>(h->device);
    if (precision == MPF_FP64) adjoint_impl<double>(h, st, grad_p, grad_q, grad_g, grad_b);
    else adjoint_impl<float>(h, st, grad_p, grad_q, grad_g, grad_b);
    h->last_stream = st;
    return MPF_OK;
  });
}

int32_t mpf_runpf_host(mpf_handle* h, int32_t alg, int32_t precision, int32_t n_cases, const int32_t* outage_offsets,
                       const int32_t* outage_branches, const double* sbus, double* v, int32_t* iterations,
                       uint8_t* status, double* max_mis) {
  int rc = mpf_set_cases(h, n_cases, outage_offsets, outage_branches, sbus);
  if (rc != MPF_OK) return rc;
  rc = mpf_solve(h, alg, precision, nullptr);
  if (rc != MPF_OK) return rc;
  return mpf_get_results(h, v, iterations, status, max_mis);
}

}  // extern "C"
